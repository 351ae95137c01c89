/*
 * nn_oracle.c -- CPU restatement of RTDL's neighbor-row semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA backend:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  The product path (librtdl_b200.so) never links or calls it.
 *
 * Semantics followed (reference file:line, paths within rubaolee/rtdl):
 *   - distance:   src/rtdsl/reference.py:882-890  _point_distance_sq
 *                 dx = right.x - left.x (search minus query), the sum is
 *                 ((dx*dx + dy*dy) + dz*dz) with every product and sum rounded
 *                 to double separately; 2D points use z = 0.0.
 *   - FRN:        src/rtdsl/reference.py:349-376  fixed_radius_neighbors_cpu
 *                 keep d2 <= radius*radius (inclusive), sort the candidates by
 *                 (sqrt(d2), neighbor_id) with Python's stable sort (equal keys
 *                 keep search-input order), keep the first k_max.
 *   - KNN:        src/rtdsl/reference.py:379-403  knn_rows_cpu
 *                 all search points, same sort key, first k, rank 1..k.
 *   - bounded:    src/rtdsl/reference.py:406-434  bounded_knn_rows_cpu
 *                 FRN plus rank 1..k_max.
 *   - row order:  every function ends with a stable sort on query_id, so rows
 *                 are grouped by (query_id, query-input index).
 *
 * Compile with -ffp-contract=off: a fused multiply-add would round d2 once
 * instead of three times and break bit-exactness with the Python reference.
 * Work is split over query ranges with pthreads (rows are per-query
 * independent, reference.py:358-375), which is how the CPU baseline uses the
 * host cores.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint32_t id; double x, y; } OPoint2;         /* RtdlPoint   */
typedef struct { uint32_t id; double x, y, z; } OPoint3;      /* RtdlPoint3D */
typedef struct { uint32_t query_id, neighbor_id; double distance; } OFrnRow;
typedef struct { uint32_t query_id, neighbor_id; double distance; uint32_t neighbor_rank; } OKnnRow;

/* A candidate carries the full Python sort key: (distance, neighbor_id, search index). */
typedef struct { double dist; uint32_t id; uint32_t index; } Cand;

static int cand_cmp(const void* a, const void* b) {
  const Cand* l = (const Cand*)a;
  const Cand* r = (const Cand*)b;
  if (l->dist < r->dist) return -1;
  if (l->dist > r->dist) return 1;
  if (l->id < r->id) return -1;
  if (l->id > r->id) return 1;
  return (l->index < r->index) ? -1 : (l->index > r->index);
}

static inline int cand_less(const Cand* l, const Cand* r) { return cand_cmp(l, r) < 0; }

/* Points are passed as separate coordinate columns so 2D and 3D share code. */
typedef struct {
  const uint32_t* qid; const double* qx; const double* qy; const double* qz;
  const uint32_t* sid; const double* sx; const double* sy; const double* sz;
  size_t nq, ns;
} Sets;

static inline double dist_sq(const Sets* s, size_t qi, size_t si) {
  double dx = s->sx[si] - s->qx[qi];
  double dy = s->sy[si] - s->qy[qi];
  double qz = s->qz ? s->qz[qi] : 0.0;
  double sz = s->sz ? s->sz[si] : 0.0;
  double dz = sz - qz;
  return (dx * dx + dy * dy) + dz * dz;
}

/* Per-query result block produced by a worker. */
typedef struct { Cand* c; uint32_t n; uint32_t total; } QBlock;

typedef struct {
  const Sets* sets;
  int mode;            /* 0 = FRN/bounded, 1 = KNN */
  double radius_sq;
  uint32_t k;          /* k_max or k */
  size_t q_begin, q_end;
  QBlock* blocks;
  int failed;
} Work;

static void* worker(void* arg) {
  Work* w = (Work*)arg;
  const Sets* s = w->sets;
  size_t cap = 64;
  Cand* scratch = (Cand*)malloc(sizeof(Cand) * cap);
  if (!scratch) { w->failed = 1; return NULL; }
  for (size_t qi = w->q_begin; qi < w->q_end; ++qi) {
    uint32_t n = 0, total = 0;
    if (w->mode == 0) {
      for (size_t si = 0; si < s->ns; ++si) {
        double d2 = dist_sq(s, qi, si);
        if (d2 > w->radius_sq) continue;  /* reference.py:362: skip only when strictly greater */
        if (n == cap) {
          cap *= 2;
          Cand* grown = (Cand*)realloc(scratch, sizeof(Cand) * cap);
          if (!grown) { w->failed = 1; free(scratch); return NULL; }
          scratch = grown;
        }
        scratch[n].dist = sqrt(d2);
        scratch[n].id = s->sid[si];
        scratch[n].index = (uint32_t)si;
        ++n;
      }
      total = n;
      qsort(scratch, n, sizeof(Cand), cand_cmp);
      if (n > w->k) n = w->k;
    } else {
      /* Bounded insertion keeps the k best by the full key; identical to a
       * full stable sort followed by truncation. */
      uint32_t k = w->k;
      if (cap < (size_t)k + 1) {
        Cand* grown = (Cand*)realloc(scratch, sizeof(Cand) * ((size_t)k + 1));
        if (!grown) { w->failed = 1; free(scratch); return NULL; }
        scratch = grown;
        cap = (size_t)k + 1;
      }
      for (size_t si = 0; si < s->ns; ++si) {
        Cand c;
        c.dist = sqrt(dist_sq(s, qi, si));
        c.id = s->sid[si];
        c.index = (uint32_t)si;
        if (n == k && !cand_less(&c, &scratch[n - 1])) continue;
        uint32_t pos = (n < k) ? n++ : k - 1;
        while (pos > 0 && cand_less(&c, &scratch[pos - 1])) {
          scratch[pos] = scratch[pos - 1];
          --pos;
        }
        scratch[pos] = c;
      }
      total = (uint32_t)s->ns;
    }
    w->blocks[qi].n = n;
    w->blocks[qi].total = total;
    w->blocks[qi].c = NULL;
    if (n) {
      w->blocks[qi].c = (Cand*)malloc(sizeof(Cand) * n);
      if (!w->blocks[qi].c) { w->failed = 1; free(scratch); return NULL; }
      memcpy(w->blocks[qi].c, scratch, sizeof(Cand) * n);
    }
  }
  free(scratch);
  return NULL;
}

typedef struct { uint32_t qid; uint32_t index; } QOrder;

static int qorder_cmp(const void* a, const void* b) {
  const QOrder* l = (const QOrder*)a;
  const QOrder* r = (const QOrder*)b;
  if (l->qid != r->qid) return (l->qid < r->qid) ? -1 : 1;
  return (l->index < r->index) ? -1 : (l->index > r->index);
}

/* Runs the per-query work on `threads` threads and returns the blocks in
 * output order (stable by query_id).  Returns 0 on success. */
static int run_blocks(const Sets* s, int mode, double radius, uint32_t k, int threads,
                      QBlock** blocks_out, QOrder** order_out) {
  *blocks_out = NULL;
  *order_out = NULL;
  QBlock* blocks = (QBlock*)calloc(s->nq ? s->nq : 1, sizeof(QBlock));
  QOrder* order = (QOrder*)malloc(sizeof(QOrder) * (s->nq ? s->nq : 1));
  if (!blocks || !order) { free(blocks); free(order); return 1; }
  if (threads < 1) threads = 1;
  if ((size_t)threads > s->nq) threads = s->nq ? (int)s->nq : 1;
  Work* works = (Work*)calloc((size_t)threads, sizeof(Work));
  pthread_t* tids = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  if (!works || !tids) { free(blocks); free(order); free(works); free(tids); return 1; }
  size_t per = (s->nq + (size_t)threads - 1) / (size_t)threads;
  int failed = 0;
  for (int t = 0; t < threads; ++t) {
    works[t].sets = s;
    works[t].mode = mode;
    works[t].radius_sq = radius * radius;
    works[t].k = k;
    works[t].q_begin = (size_t)t * per < s->nq ? (size_t)t * per : s->nq;
    works[t].q_end = (size_t)(t + 1) * per < s->nq ? (size_t)(t + 1) * per : s->nq;
    works[t].blocks = blocks;
    if (threads == 1) {
      worker(&works[t]);
    } else if (pthread_create(&tids[t], NULL, worker, &works[t]) != 0) {
      worker(&works[t]);
      tids[t] = 0;
    }
  }
  if (threads > 1)
    for (int t = 0; t < threads; ++t)
      if (tids[t]) pthread_join(tids[t], NULL);
  for (int t = 0; t < threads; ++t) failed |= works[t].failed;
  free(works);
  free(tids);
  for (size_t i = 0; i < s->nq; ++i) { order[i].qid = s->qid[i]; order[i].index = (uint32_t)i; }
  qsort(order, s->nq, sizeof(QOrder), qorder_cmp);
  *blocks_out = blocks;
  *order_out = order;
  return failed;
}

static void free_blocks(QBlock* blocks, size_t n) {
  if (!blocks) return;
  for (size_t i = 0; i < n; ++i) free(blocks[i].c);
  free(blocks);
}

/* Public entry points.  `qz`/`sz` may be NULL for 2D.  Rows are malloc'd and
 * released with nn_oracle_free.  `ranked` selects RtdlKnnNeighborRow output
 * (bounded_knn_rows / knn_rows); otherwise RtdlFixedRadiusNeighborRow.
 * `counts_out` (optional, nq entries, query-input order) receives the
 * uncapped in-radius count per query for FRN, or ns for KNN. */
int nn_oracle_rows(const uint32_t* qid, const double* qx, const double* qy, const double* qz, size_t nq,
                   const uint32_t* sid, const double* sx, const double* sy, const double* sz, size_t ns,
                   int mode, double radius, uint32_t k, int ranked, int threads,
                   void** rows_out, size_t* row_count_out, uint32_t* counts_out) {
  *rows_out = NULL;
  *row_count_out = 0;
  Sets s = {qid, qx, qy, qz, sid, sx, sy, sz, nq, ns};
  QBlock* blocks = NULL;
  QOrder* order = NULL;
  if (nq == 0) return 0;
  if (run_blocks(&s, mode, radius, k, threads, &blocks, &order)) {
    free_blocks(blocks, nq);
    free(order);
    return 1;
  }
  size_t total = 0;
  for (size_t i = 0; i < nq; ++i) total += blocks[i].n;
  size_t row_size = ranked ? sizeof(OKnnRow) : sizeof(OFrnRow);
  char* rows = (char*)calloc(total ? total : 1, row_size);  /* zeroed: RtdlKnnNeighborRow has 4 padding bytes */
  if (!rows) { free_blocks(blocks, nq); free(order); return 1; }
  size_t r = 0;
  for (size_t j = 0; j < nq; ++j) {
    const QBlock* b = &blocks[order[j].index];
    for (uint32_t i = 0; i < b->n; ++i, ++r) {
      if (ranked) {
        OKnnRow* row = (OKnnRow*)(rows + r * row_size);
        row->query_id = order[j].qid;
        row->neighbor_id = b->c[i].id;
        row->distance = b->c[i].dist;
        row->neighbor_rank = i + 1;
      } else {
        OFrnRow* row = (OFrnRow*)(rows + r * row_size);
        row->query_id = order[j].qid;
        row->neighbor_id = b->c[i].id;
        row->distance = b->c[i].dist;
      }
    }
  }
  if (counts_out)
    for (size_t i = 0; i < nq; ++i) counts_out[i] = blocks[i].total;
  free_blocks(blocks, nq);
  free(order);
  *rows_out = rows;
  *row_count_out = total;
  return 0;
}

/* Directed nearest distances for Hausdorff: per query (input order) the
 * nearest (distance, neighbor_id) by the knn_rows(k=1) key.  The directed
 * Hausdorff witness is then max over queries of (distance, -query_id,
 * -neighbor_id), following
 * examples/v2_0/research_benchmarks/hausdorff_xhd/rtdl_hausdorff_distance_app.py:108-130. */
int nn_oracle_nearest(const uint32_t* qid, const double* qx, const double* qy, const double* qz, size_t nq,
                      const uint32_t* sid, const double* sx, const double* sy, const double* sz, size_t ns,
                      int threads, double* dist_out, uint32_t* nid_out) {
  Sets s = {qid, qx, qy, qz, sid, sx, sy, sz, nq, ns};
  QBlock* blocks = NULL;
  QOrder* order = NULL;
  if (nq == 0) return 0;
  if (ns == 0) return 1;
  if (run_blocks(&s, 1, 0.0, 1, threads, &blocks, &order)) {
    free_blocks(blocks, nq);
    free(order);
    return 1;
  }
  for (size_t i = 0; i < nq; ++i) {
    dist_out[i] = blocks[i].c[0].dist;
    nid_out[i] = blocks[i].c[0].id;
  }
  free_blocks(blocks, nq);
  free(order);
  return 0;
}

void nn_oracle_free(void* p) { free(p); }
