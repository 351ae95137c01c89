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

/* ---- optional uniform grid over the search set ------------------------------
 * Only a candidate generator: every point it yields is tested with the same
 * FP64 dist_sq and kept or ranked by the same key as the brute-force loop, so
 * the rows are identical whenever the grid's candidates include every point
 * the brute-force loop would keep.  That holds because (fixed radius) the cells
 * scanned cover [q - r, q + r] widened by one whole cell on each side, which
 * absorbs the rounding of dx, and (k nearest) the rings stop only when the
 * k-th kept distance is below the distance to any unscanned cell by a relative
 * margin far above the rounding of sqrt(d2).  It makes the full-size sets of
 * the benchmark checkable on a CPU in minutes. */
typedef struct {
  int dim;
  double lo[3], cell;
  double scale;          /* largest |coordinate| of the grid's box: bounds the rounding of cell assignment */
  int64_t n[3];          /* cells per axis */
  uint32_t* start;       /* n[0]*n[1]*n[2] + 1 offsets into pts */
  uint32_t* pts;         /* search indices grouped by cell */
} Grid;

static inline int64_t grid_axis(const Grid* g, int a, double v) {
  double c = floor((v - g->lo[a]) / g->cell);
  if (c < 0) return 0;
  if (c >= (double)g->n[a]) return g->n[a] - 1;
  return (int64_t)c;
}

static inline double axis_value(const Sets* s, int a, size_t i, int query) {
  if (a == 0) return query ? s->qx[i] : s->sx[i];
  if (a == 1) return query ? s->qy[i] : s->sy[i];
  const double* z = query ? s->qz : s->sz;
  return z ? z[i] : 0.0;
}

static void grid_free(Grid* g) {
  if (!g) return;
  free(g->start);
  free(g->pts);
  free(g);
}

/* cell: the desired cell size (widened until the grid has at most 2^26 cells). */
static Grid* grid_build(const Sets* s, double cell) {
  Grid* g = (Grid*)calloc(1, sizeof(Grid));
  if (!g) return NULL;
  g->dim = (s->sz || s->qz) ? 3 : 2;
  double hi[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) { g->lo[a] = 0.0; hi[a] = 0.0; }
  for (int a = 0; a < g->dim; ++a) {
    double lo = INFINITY, h = -INFINITY;
    for (size_t i = 0; i < s->ns; ++i) {
      double v = axis_value(s, a, i, 0);
      if (v < lo) lo = v;
      if (v > h) h = v;
    }
    g->lo[a] = lo;
    hi[a] = h;
    if (fabs(lo) > g->scale) g->scale = fabs(lo);
    if (fabs(h) > g->scale) g->scale = fabs(h);
  }
  if (!(cell > 0.0)) cell = 1.0;
  for (;;) {
    double total = 1.0;
    for (int a = 0; a < 3; ++a) {
      double n = a < g->dim ? floor((hi[a] - g->lo[a]) / cell) + 1.0 : 1.0;
      g->n[a] = (int64_t)n;
      total *= n;
    }
    if (total <= (double)(1 << 26)) break;
    cell *= 1.5;
  }
  g->cell = cell;
  const size_t cells = (size_t)(g->n[0] * g->n[1] * g->n[2]);
  g->start = (uint32_t*)calloc(cells + 1, sizeof(uint32_t));
  g->pts = (uint32_t*)malloc(sizeof(uint32_t) * (s->ns ? s->ns : 1));
  uint32_t* which = (uint32_t*)malloc(sizeof(uint32_t) * (s->ns ? s->ns : 1));
  if (!g->start || !g->pts || !which) { free(which); grid_free(g); return NULL; }
  for (size_t i = 0; i < s->ns; ++i) {
    int64_t c0 = grid_axis(g, 0, s->sx[i]), c1 = grid_axis(g, 1, s->sy[i]);
    int64_t c2 = g->dim == 3 ? grid_axis(g, 2, s->sz ? s->sz[i] : 0.0) : 0;
    which[i] = (uint32_t)((c2 * g->n[1] + c1) * g->n[0] + c0);
    g->start[which[i] + 1]++;
  }
  for (size_t c = 0; c < cells; ++c) g->start[c + 1] += g->start[c];
  uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * (cells ? cells : 1));
  if (!fill) { free(which); grid_free(g); return NULL; }
  memcpy(fill, g->start, sizeof(uint32_t) * cells);
  for (size_t i = 0; i < s->ns; ++i) g->pts[fill[which[i]]++] = (uint32_t)i;
  free(fill);
  free(which);
  return g;
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
  const Grid* grid;    /* NULL: every search point is a candidate */
} Work;

static int grow(Cand** scratch, size_t* cap, size_t need) {
  if (need <= *cap) return 0;
  size_t c = *cap;
  while (c < need) c *= 2;
  Cand* grown = (Cand*)realloc(*scratch, sizeof(Cand) * c);
  if (!grown) return 1;
  *scratch = grown;
  *cap = c;
  return 0;
}

/* Keeps the k best candidates by the full key in scratch[0..*n) (sorted). */
static inline void knn_insert(Cand* scratch, uint32_t* n, uint32_t k, const Cand* c) {
  if (*n == k && !cand_less(c, &scratch[*n - 1])) return;
  uint32_t pos = (*n < k) ? (*n)++ : k - 1;
  while (pos > 0 && cand_less(c, &scratch[pos - 1])) {
    scratch[pos] = scratch[pos - 1];
    --pos;
  }
  scratch[pos] = *c;
}

/* Fixed radius over the grid: cells covering [q - r, q + r] plus one cell. */
static int grid_frn(const Work* w, size_t qi, Cand** scratch, size_t* cap, uint32_t* n_out) {
  const Grid* g = w->grid;
  const Sets* s = w->sets;
  const double r = sqrt(w->radius_sq);
  int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int a = 0; a < g->dim; ++a) {
    double q = axis_value(s, a, qi, 1);
    lo[a] = grid_axis(g, a, q - r) - 1;
    hi[a] = grid_axis(g, a, q + r) + 1;
    if (lo[a] < 0) lo[a] = 0;
    if (hi[a] > g->n[a] - 1) hi[a] = g->n[a] - 1;
  }
  uint32_t n = 0;
  for (int64_t c2 = lo[2]; c2 <= hi[2]; ++c2)
    for (int64_t c1 = lo[1]; c1 <= hi[1]; ++c1) {
      const int64_t row = (c2 * g->n[1] + c1) * g->n[0];
      for (uint32_t j = g->start[row + lo[0]]; j < g->start[row + hi[0] + 1]; ++j) {
        const uint32_t si = g->pts[j];
        double d2 = dist_sq(s, qi, si);
        if (d2 > w->radius_sq) continue;
        if (grow(scratch, cap, (size_t)n + 1)) return 1;
        (*scratch)[n].dist = sqrt(d2);
        (*scratch)[n].id = s->sid[si];
        (*scratch)[n].index = si;
        ++n;
      }
    }
  *n_out = n;
  return 0;
}

/* k nearest over the grid: rings of cells around the query's cell, until the
 * k-th kept distance is clearly below the distance to any unscanned cell. */
static void grid_knn(const Work* w, size_t qi, Cand* scratch, uint32_t* n_out) {
  const Grid* g = w->grid;
  const Sets* s = w->sets;
  const uint32_t k = w->k < s->ns ? w->k : (uint32_t)s->ns;
  int64_t qc[3] = {0, 0, 0};
  double q[3] = {0, 0, 0};
  for (int a = 0; a < g->dim; ++a) {
    q[a] = axis_value(s, a, qi, 1);
    qc[a] = grid_axis(g, a, q[a]);
  }
  int64_t most = 0;
  for (int a = 0; a < g->dim; ++a) {
    int64_t m = qc[a] > g->n[a] - 1 - qc[a] ? qc[a] : g->n[a] - 1 - qc[a];
    if (m > most) most = m;
  }
  uint32_t n = 0;
  for (int64_t ring = 0; ring <= most; ++ring) {
    int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int a = 0; a < g->dim; ++a) {
      lo[a] = qc[a] - ring;
      hi[a] = qc[a] + ring;
    }
    for (int64_t c2 = lo[2]; c2 <= hi[2]; ++c2) {
      if (c2 < 0 || c2 >= g->n[2]) continue;
      for (int64_t c1 = lo[1]; c1 <= hi[1]; ++c1) {
        if (c1 < 0 || c1 >= g->n[1]) continue;
        const int on_shell_12 = (g->dim == 3 && (c2 == lo[2] || c2 == hi[2])) || c1 == lo[1] || c1 == hi[1];
        for (int64_t c0 = lo[0]; c0 <= hi[0]; ++c0) {
          if (c0 < 0 || c0 >= g->n[0]) continue;
          if (!on_shell_12 && c0 != lo[0] && c0 != hi[0]) continue;  /* inner cells were scanned before */
          const int64_t cell = (c2 * g->n[1] + c1) * g->n[0] + c0;
          for (uint32_t j = g->start[cell]; j < g->start[cell + 1]; ++j) {
            const uint32_t si = g->pts[j];
            Cand c;
            c.dist = sqrt(dist_sq(s, qi, si));
            c.id = s->sid[si];
            c.index = si;
            knn_insert(scratch, &n, k, &c);
          }
        }
      }
    }
    if (n == k) {
      /* distance from q to the outside of the scanned block of cells */
      double gap = INFINITY;
      for (int a = 0; a < g->dim; ++a) {
        double below = q[a] - (g->lo[a] + (double)lo[a] * g->cell);
        double above = (g->lo[a] + (double)(hi[a] + 1) * g->cell) - q[a];
        if (lo[a] > 0 && below < gap) gap = below;
        if (hi[a] < g->n[a] - 1 && above < gap) gap = above;
      }
      /* a point's cell can be off by one rounding of its coordinate: keep an
       * absolute margin too, so no unscanned point can tie or beat the k-th */
      if (scratch[n - 1].dist < gap * (1.0 - 1e-9) - 1e-12 * g->scale) break;
    }
  }
  *n_out = n;
}

static void* worker(void* arg) {
  Work* w = (Work*)arg;
  const Sets* s = w->sets;
  size_t cap = 64;
  Cand* scratch = (Cand*)malloc(sizeof(Cand) * cap);
  if (!scratch) { w->failed = 1; return NULL; }
  if (w->mode == 1 && grow(&scratch, &cap, (size_t)w->k + 1)) { w->failed = 1; free(scratch); return NULL; }
  for (size_t qi = w->q_begin; qi < w->q_end; ++qi) {
    uint32_t n = 0, total = 0;
    if (w->grid && w->mode == 0) {
      if (grid_frn(w, qi, &scratch, &cap, &n)) { w->failed = 1; free(scratch); return NULL; }
      total = n;
      qsort(scratch, n, sizeof(Cand), cand_cmp);
      if (n > w->k) n = w->k;
    } else if (w->grid) {
      grid_knn(w, qi, scratch, &n);
      total = (uint32_t)s->ns;
    } else if (w->mode == 0) {
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
static int run_blocks(const Sets* s, int mode, double radius, uint32_t k, int threads, const Grid* grid,
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
    works[t].grid = grid;
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
/* Cell size of the grid candidate generator: the radius for fixed-radius
 * calls (widened to about two points per cell of the search set's box when
 * the radius is tiny), about two points per cell for nearest searches. */
static double grid_cell(const Sets* s, int mode, double radius) {
  const int dim = (s->sz || s->qz) ? 3 : 2;
  double vol = 1.0;
  for (int a = 0; a < dim; ++a) {
    double lo = INFINITY, hi = -INFINITY;
    for (size_t i = 0; i < s->ns; ++i) {
      double v = axis_value(s, a, i, 0);
      if (v < lo) lo = v;
      if (v > hi) hi = v;
    }
    vol *= (hi > lo ? hi - lo : 1e-300);
  }
  double per_point = pow(vol * 2.0 / (double)(s->ns ? s->ns : 1), 1.0 / dim);
  if (mode == 0) return radius > per_point ? radius : per_point;
  return per_point;
}

static int rows_impl(const Sets* s, int mode, double radius, uint32_t k, int ranked, int threads, int use_grid,
                     void** rows_out, size_t* row_count_out, uint32_t* counts_out);

int nn_oracle_rows(const uint32_t* qid, const double* qx, const double* qy, const double* qz, size_t nq,
                   const uint32_t* sid, const double* sx, const double* sy, const double* sz, size_t ns,
                   int mode, double radius, uint32_t k, int ranked, int threads,
                   void** rows_out, size_t* row_count_out, uint32_t* counts_out) {
  Sets s = {qid, qx, qy, qz, sid, sx, sy, sz, nq, ns};
  return rows_impl(&s, mode, radius, k, ranked, threads, 0, rows_out, row_count_out, counts_out);
}

/* The same rows with the uniform-grid candidate generator. */
int nn_oracle_rows_grid(const uint32_t* qid, const double* qx, const double* qy, const double* qz, size_t nq,
                        const uint32_t* sid, const double* sx, const double* sy, const double* sz, size_t ns,
                        int mode, double radius, uint32_t k, int ranked, int threads,
                        void** rows_out, size_t* row_count_out, uint32_t* counts_out) {
  Sets s = {qid, qx, qy, qz, sid, sx, sy, sz, nq, ns};
  return rows_impl(&s, mode, radius, k, ranked, threads, 1, rows_out, row_count_out, counts_out);
}

static int rows_impl(const Sets* sp, int mode, double radius, uint32_t k, int ranked, int threads, int use_grid,
                     void** rows_out, size_t* row_count_out, uint32_t* counts_out) {
  *rows_out = NULL;
  *row_count_out = 0;
  const Sets s = *sp;
  const size_t nq = s.nq;
  QBlock* blocks = NULL;
  QOrder* order = NULL;
  if (nq == 0) return 0;
  Grid* grid = NULL;
  if (use_grid && s.ns > 0) {
    grid = grid_build(&s, grid_cell(&s, mode, radius));
    if (!grid) return 1;
  }
  const int failed = run_blocks(&s, mode, radius, k, threads, grid, &blocks, &order);
  grid_free(grid);
  if (failed) {
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
static int nearest_impl(const Sets* s, int threads, int use_grid, double* dist_out, uint32_t* nid_out) {
  QBlock* blocks = NULL;
  QOrder* order = NULL;
  const size_t nq = s->nq;
  if (nq == 0) return 0;
  if (s->ns == 0) return 1;
  Grid* grid = NULL;
  if (use_grid) {
    grid = grid_build(s, grid_cell(s, 1, 0.0));
    if (!grid) return 1;
  }
  const int failed = run_blocks(s, 1, 0.0, 1, threads, grid, &blocks, &order);
  grid_free(grid);
  if (failed) {
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

int nn_oracle_nearest(const uint32_t* qid, const double* qx, const double* qy, const double* qz, size_t nq,
                      const uint32_t* sid, const double* sx, const double* sy, const double* sz, size_t ns,
                      int threads, double* dist_out, uint32_t* nid_out) {
  Sets s = {qid, qx, qy, qz, sid, sx, sy, sz, nq, ns};
  return nearest_impl(&s, threads, 0, dist_out, nid_out);
}

/* The same with the uniform-grid candidate generator. */
int nn_oracle_nearest_grid(const uint32_t* qid, const double* qx, const double* qy, const double* qz, size_t nq,
                           const uint32_t* sid, const double* sx, const double* sy, const double* sz, size_t ns,
                           int threads, double* dist_out, uint32_t* nid_out) {
  Sets s = {qid, qx, qy, qz, sid, sx, sy, sz, nq, ns};
  return nearest_impl(&s, threads, 1, dist_out, nid_out);
}

void nn_oracle_free(void* p) { free(p); }
