/*
 * pf_oracle.c -- CPU FP64 oracle (TEST INFRASTRUCTURE ONLY, see pf_oracle.h).
 *
 * Restates the reference's CPU FP64 Newton-Raphson pipeline:
 *   Jacobian analysis   cuPF/cpp/src/newton_solver/ops/jacobian/jacobian_analysis.cpp:257-445
 *   CSC storage         cuPF/cpp/src/newton_solver/storage/cpu/cpu_fp64_storage.cpp:219-392
 *   Ibus (CSC SAXPY)    cuPF/cpp/src/newton_solver/ops/ibus/compute_ibus.cpp:12-36
 *   mismatch + norm     cuPF/cpp/src/newton_solver/ops/mismatch/cpu_mismatch.cpp:17-64
 *   Jacobian fill       cuPF/cpp/src/newton_solver/ops/jacobian/fill_jacobian.cpp:28-94
 *   voltage update      cuPF/cpp/src/newton_solver/ops/voltage_update/cpu_voltage_update.cpp:12-43
 *   NR loop             cuPF/cpp/src/newton_solver/core/newton_solver.cpp:497-558
 *   adjoint             cuPF/cpp/src/newton_solver/core/newton_solver_adjoint.cpp:33-153,
 *                       cuPF/cpp/src/newton_solver/core/adjoint_math.cpp:62-154
 * with this file's own sparse LU in place of KLU.
 *
 * Complex products are written out as (ac - bd, ad + bc) in the same
 * association order the reference's std::complex<double> expressions use, and
 * the file is compiled without floating-point contraction, so the Jacobian and
 * mismatch values match the reference bit for bit.
 */
#include "pf_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ======================================================================== */
/* Jacobian analysis                                                         */
/* ======================================================================== */

typedef struct {
  int n_bus, n_pvpq, n_pq, dim;
  int32_t *row_pvpq, *row_pq; /* bus -> J row/col index, -1 = absent */
} jindex;

static int make_index(int n_bus, const int32_t* pv, int n_pv, const int32_t* pq, int n_pq, jindex* ix) {
  if (n_bus <= 0 || n_pv < 0 || n_pq < 0 || n_pv + n_pq <= 0) return -1;
  ix->n_bus = n_bus;
  ix->n_pvpq = n_pv + n_pq;
  ix->n_pq = n_pq;
  ix->dim = ix->n_pvpq + n_pq;
  ix->row_pvpq = (int32_t*)malloc(sizeof(int32_t) * n_bus);
  ix->row_pq = (int32_t*)malloc(sizeof(int32_t) * n_bus);
  for (int i = 0; i < n_bus; ++i) ix->row_pvpq[i] = ix->row_pq[i] = -1;
  for (int i = 0; i < n_pv; ++i) {
    if (pv[i] < 0 || pv[i] >= n_bus) return -1;
    ix->row_pvpq[pv[i]] = i;
  }
  for (int i = 0; i < n_pq; ++i) {
    if (pq[i] < 0 || pq[i] >= n_bus) return -1;
    ix->row_pvpq[pq[i]] = n_pv + i;
    ix->row_pq[pq[i]] = ix->n_pvpq + i;
  }
  return 0;
}

static void free_index(jindex* ix) {
  free(ix->row_pvpq);
  free(ix->row_pq);
}

typedef struct {
  int32_t* v;
  int n, cap;
} ivec;

static void ivec_push(ivec* a, int32_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 8;
    a->v = (int32_t*)realloc(a->v, sizeof(int32_t) * a->cap);
  }
  a->v[a->n++] = x;
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* Emit the (row, col) entries bus pair (rb, cb) contributes to, in the
 * reference's order (J11, J21, J12, J22; jacobian_analysis.cpp:198-221). */
static void append_cols(ivec* rows, const jindex* ix, int rb, int cb) {
  int ri = ix->row_pvpq[rb], rq = ix->row_pq[rb];
  int ci = ix->row_pvpq[cb], cq = ix->row_pq[cb];
  if (ri >= 0 && ci >= 0) ivec_push(&rows[ri], ci);
  if (rq >= 0 && ci >= 0) ivec_push(&rows[rq], ci);
  if (ri >= 0 && cq >= 0) ivec_push(&rows[ri], cq);
  if (rq >= 0 && cq >= 0) ivec_push(&rows[rq], cq);
}

static ivec* build_rows(int n_bus, const int32_t* indptr, const int32_t* indices, const jindex* ix) {
  ivec* rows = (ivec*)calloc(ix->dim, sizeof(ivec));
  /* strict upper triangle of Ybus, both directions, then the diagonal
   * (jacobian_analysis.cpp:342-359) */
  for (int r = 0; r < n_bus; ++r) {
    for (int k = indptr[r]; k < indptr[r + 1]; ++k) {
      int c = indices[k];
      if (c <= r) continue;
      append_cols(rows, ix, r, c);
      append_cols(rows, ix, c, r);
    }
  }
  for (int b = 0; b < n_bus; ++b) append_cols(rows, ix, b, b);
  for (int r = 0; r < ix->dim; ++r) {
    ivec* a = &rows[r];
    if (a->n > 1) qsort(a->v, a->n, sizeof(int32_t), cmp_i32);
    int w = 0;
    for (int i = 0; i < a->n; ++i)
      if (w == 0 || a->v[i] != a->v[w - 1]) a->v[w++] = a->v[i];
    a->n = w;
  }
  return rows;
}

static void free_rows(ivec* rows, int dim) {
  for (int i = 0; i < dim; ++i) free(rows[i].v);
  free(rows);
}

int orc_jacobian_nnz(int n_bus, const int32_t* indptr, const int32_t* indices,
                     const int32_t* pv, int n_pv, const int32_t* pq, int n_pq, int* nnz_j) {
  jindex ix;
  if (make_index(n_bus, pv, n_pv, pq, n_pq, &ix)) return -1;
  ivec* rows = build_rows(n_bus, indptr, indices, &ix);
  long nnz = 0;
  for (int r = 0; r < ix.dim; ++r) nnz += rows[r].n;
  *nnz_j = (int)nnz;
  int dim = ix.dim;
  free_rows(rows, dim);
  free_index(&ix);
  return dim;
}

static int find_slot(const int32_t* row_ptr, const int32_t* col_idx, int dim, int r, int c) {
  if (r < 0 || c < 0 || r >= dim || c >= dim) return -1;
  int lo = row_ptr[r], hi = row_ptr[r + 1];
  while (lo < hi) {
    int mid = lo + (hi - lo) / 2;
    if (col_idx[mid] < c) lo = mid + 1; else hi = mid;
  }
  return (lo < row_ptr[r + 1] && col_idx[lo] == c) ? lo : -1;
}

int orc_jacobian_analysis(int n_bus, const int32_t* indptr, const int32_t* indices,
                          const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                          int32_t* row_ptr, int32_t* col_idx,
                          int32_t* map11, int32_t* map21, int32_t* map12, int32_t* map22,
                          int32_t* diag11, int32_t* diag21, int32_t* diag12, int32_t* diag22) {
  jindex ix;
  if (make_index(n_bus, pv, n_pv, pq, n_pq, &ix)) return -1;
  ivec* rows = build_rows(n_bus, indptr, indices, &ix);
  row_ptr[0] = 0;
  for (int r = 0; r < ix.dim; ++r) {
    memcpy(col_idx + row_ptr[r], rows[r].v, sizeof(int32_t) * rows[r].n);
    row_ptr[r + 1] = row_ptr[r] + rows[r].n;
  }
  for (int b = 0; b < n_bus; ++b) diag11[b] = diag21[b] = diag12[b] = diag22[b] = -1;
  /* scatter maps per Ybus entry (jacobian_analysis.cpp:389-445) */
  for (int r = 0; r < n_bus; ++r) {
    for (int k = indptr[r]; k < indptr[r + 1]; ++k) {
      int c = indices[k];
      int ri = ix.row_pvpq[r], rq = ix.row_pq[r];
      int ci = ix.row_pvpq[c], cq = ix.row_pq[c];
      map11[k] = (ri >= 0 && ci >= 0) ? find_slot(row_ptr, col_idx, ix.dim, ri, ci) : -1;
      map21[k] = (rq >= 0 && ci >= 0) ? find_slot(row_ptr, col_idx, ix.dim, rq, ci) : -1;
      map12[k] = (ri >= 0 && cq >= 0) ? find_slot(row_ptr, col_idx, ix.dim, ri, cq) : -1;
      map22[k] = (rq >= 0 && cq >= 0) ? find_slot(row_ptr, col_idx, ix.dim, rq, cq) : -1;
      if (r == c) {
        diag11[r] = map11[k];
        diag21[r] = map21[k];
        diag12[r] = map12[k];
        diag22[r] = map22[k];
      }
    }
  }
  free_rows(rows, ix.dim);
  free_index(&ix);
  return 0;
}

/* ======================================================================== */
/* Sparse LU: left-looking Gilbert-Peierls with threshold partial pivoting   */
/* ======================================================================== */

struct orc_lu {
  int n;
  int32_t *Lp, *Li; double* Lx; int lcap;  /* unit lower, rows in pivot order */
  int32_t *Up, *Ui; double* Ux; int ucap;  /* upper, diagonal last in each column */
  int32_t* pinv;   /* row -> pivot position */
  int32_t* q;      /* column order new -> old */
  double tol;
  /* workspace */
  double* x;
  int32_t *xi, *stack, *mark, *pstack;
};

static void grow_l(orc_lu* f, int need) {
  if (need <= f->lcap) return;
  while (f->lcap < need) f->lcap *= 2;
  f->Li = (int32_t*)realloc(f->Li, sizeof(int32_t) * f->lcap);
  f->Lx = (double*)realloc(f->Lx, sizeof(double) * f->lcap);
}

static void grow_u(orc_lu* f, int need) {
  if (need <= f->ucap) return;
  while (f->ucap < need) f->ucap *= 2;
  f->Ui = (int32_t*)realloc(f->Ui, sizeof(int32_t) * f->ucap);
  f->Ux = (double*)realloc(f->Ux, sizeof(double) * f->ucap);
}

/* Depth-first reach of the rows of column `col` of A through the graph of the
 * partial L (edges j -> rows of L(:, pinv[j])).  Writes the topologically
 * ordered reach into xi[top..n-1] and returns top. */
static int reach(orc_lu* f, const int32_t* Ap, const int32_t* Ai, int col, int stamp) {
  int n = f->n, top = n;
  for (int p = Ap[col]; p < Ap[col + 1]; ++p) {
    int start = Ai[p];
    if (f->mark[start] == stamp) continue;
    /* iterative DFS */
    int head = 0;
    f->stack[0] = start;
    while (head >= 0) {
      int j = f->stack[head];
      int jpiv = f->pinv[j];
      if (f->mark[j] != stamp) {
        f->mark[j] = stamp;
        f->pstack[head] = (jpiv < 0) ? 0 : f->Lp[jpiv];
      }
      int done = 1;
      int pend = (jpiv < 0) ? 0 : f->Lp[jpiv + 1];
      for (int pp = f->pstack[head]; pp < pend; ++pp) {
        int i = f->Li[pp];
        if (f->mark[i] == stamp) continue;
        f->pstack[head] = pp + 1;
        f->stack[++head] = i;
        done = 0;
        break;
      }
      if (done) {
        --head;
        f->xi[--top] = j;
      }
    }
  }
  return top;
}

static int factor_numeric(orc_lu* f, const int32_t* Ap, const int32_t* Ai, const double* Ax) {
  int n = f->n, lnz = 0, unz = 0;
  for (int i = 0; i < n; ++i) {
    f->pinv[i] = -1;
    f->x[i] = 0.0;
    f->mark[i] = -1;
  }
  for (int k = 0; k < n; ++k) {
    int col = f->q ? f->q[k] : k;
    f->Lp[k] = lnz;
    f->Up[k] = unz;
    grow_l(f, lnz + n);
    grow_u(f, unz + n);
    int top = reach(f, Ap, Ai, col, k);
    for (int p = top; p < n; ++p) f->x[f->xi[p]] = 0.0;
    for (int p = Ap[col]; p < Ap[col + 1]; ++p) f->x[Ai[p]] = Ax[p];
    /* sparse triangular solve x = L \ x over the reach, in topological order */
    for (int p = top; p < n; ++p) {
      int j = f->xi[p];
      int jpiv = f->pinv[j];
      if (jpiv < 0) continue;
      double xj = f->x[j];
      for (int pp = f->Lp[jpiv] + 1; pp < f->Lp[jpiv + 1]; ++pp) f->x[f->Li[pp]] -= f->Lx[pp] * xj;
    }
    /* pivot: largest |x_i| among non-pivotal rows, prefer the diagonal */
    int ipiv = -1;
    double amax = -1.0;
    for (int p = top; p < n; ++p) {
      int i = f->xi[p];
      if (f->pinv[i] < 0) {
        double a = fabs(f->x[i]);
        if (a > amax) { amax = a; ipiv = i; }
      } else {
        f->Ui[unz] = f->pinv[i];
        f->Ux[unz++] = f->x[i];
      }
    }
    if (ipiv < 0 || amax <= 0.0) return -1;
    if (f->pinv[col] < 0 && fabs(f->x[col]) >= f->tol * amax) ipiv = col;
    double piv = f->x[ipiv];
    f->Ui[unz] = k;
    f->Ux[unz++] = piv;
    f->pinv[ipiv] = k;
    f->Li[lnz] = ipiv;
    f->Lx[lnz++] = 1.0;
    for (int p = top; p < n; ++p) {
      int i = f->xi[p];
      if (f->pinv[i] < 0) {
        f->Li[lnz] = i;
        f->Lx[lnz++] = f->x[i] / piv;
      }
      f->x[i] = 0.0;
    }
  }
  f->Lp[n] = lnz;
  f->Up[n] = unz;
  /* relabel L rows into pivot order */
  for (int p = 0; p < lnz; ++p) f->Li[p] = f->pinv[f->Li[p]];
  return 0;
}

orc_lu* orc_lu_factor(int n, const int32_t* Ap, const int32_t* Ai, const double* Ax,
                      const int32_t* col_order, double tol) {
  orc_lu* f = (orc_lu*)calloc(1, sizeof(orc_lu));
  f->n = n;
  f->tol = tol;
  f->lcap = f->ucap = 4 * (Ap[n] + n) + 16;
  f->Lp = (int32_t*)malloc(sizeof(int32_t) * (n + 1));
  f->Up = (int32_t*)malloc(sizeof(int32_t) * (n + 1));
  f->Li = (int32_t*)malloc(sizeof(int32_t) * f->lcap);
  f->Lx = (double*)malloc(sizeof(double) * f->lcap);
  f->Ui = (int32_t*)malloc(sizeof(int32_t) * f->ucap);
  f->Ux = (double*)malloc(sizeof(double) * f->ucap);
  f->pinv = (int32_t*)malloc(sizeof(int32_t) * n);
  f->x = (double*)malloc(sizeof(double) * n);
  f->xi = (int32_t*)malloc(sizeof(int32_t) * n);
  f->stack = (int32_t*)malloc(sizeof(int32_t) * n);
  f->pstack = (int32_t*)malloc(sizeof(int32_t) * n);
  f->mark = (int32_t*)malloc(sizeof(int32_t) * n);
  if (col_order) {
    f->q = (int32_t*)malloc(sizeof(int32_t) * n);
    memcpy(f->q, col_order, sizeof(int32_t) * n);
  }
  if (factor_numeric(f, Ap, Ai, Ax)) {
    orc_lu_free(f);
    return NULL;
  }
  return f;
}

int orc_lu_refactor(orc_lu* f, const int32_t* Ap, const int32_t* Ai, const double* Ax) {
  return factor_numeric(f, Ap, Ai, Ax);
}

int orc_lu_nnz(const orc_lu* f) { return f->Lp[f->n] + f->Up[f->n]; }
int orc_lu_dim(const orc_lu* f) { return f->n; }

void orc_lu_solve(const orc_lu* f, double* b) {
  int n = f->n;
  double* y = (double*)malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) y[f->pinv[i]] = b[i];
  for (int k = 0; k < n; ++k) {           /* L y = P b (unit lower) */
    double yk = y[k];
    for (int p = f->Lp[k] + 1; p < f->Lp[k + 1]; ++p) y[f->Li[p]] -= f->Lx[p] * yk;
  }
  for (int k = n - 1; k >= 0; --k) {      /* U z = y */
    int pd = f->Up[k + 1] - 1;
    y[k] /= f->Ux[pd];
    double yk = y[k];
    for (int p = f->Up[k]; p < pd; ++p) y[f->Ui[p]] -= f->Ux[p] * yk;
  }
  for (int k = 0; k < n; ++k) b[f->q ? f->q[k] : k] = y[k];
  free(y);
}

void orc_lu_tsolve(const orc_lu* f, double* b) {
  int n = f->n;
  double* y = (double*)malloc(sizeof(double) * n);
  for (int k = 0; k < n; ++k) y[k] = b[f->q ? f->q[k] : k];
  for (int k = 0; k < n; ++k) {           /* U^T w = Q^T b */
    int pd = f->Up[k + 1] - 1;
    double s = y[k];
    for (int p = f->Up[k]; p < pd; ++p) s -= f->Ux[p] * y[f->Ui[p]];
    y[k] = s / f->Ux[pd];
  }
  for (int k = n - 1; k >= 0; --k) {      /* L^T v = w */
    double s = y[k];
    for (int p = f->Lp[k] + 1; p < f->Lp[k + 1]; ++p) s -= f->Lx[p] * y[f->Li[p]];
    y[k] = s;
  }
  for (int i = 0; i < n; ++i) b[i] = y[f->pinv[i]];
  free(y);
}

void orc_lu_free(orc_lu* f) {
  if (!f) return;
  free(f->Lp); free(f->Li); free(f->Lx);
  free(f->Up); free(f->Ui); free(f->Ux);
  free(f->pinv); free(f->q); free(f->x);
  free(f->xi); free(f->stack); free(f->pstack); free(f->mark);
  free(f);
}

/* METIS 5.1 C API (64-bit idx_t build shipped with the CUDA toolkit). */
typedef int64_t orc_idx_t;
int METIS_SetDefaultOptions(orc_idx_t* options);
int METIS_NodeND(orc_idx_t* nvtxs, orc_idx_t* xadj, orc_idx_t* adjncy, orc_idx_t* vwgt,
                 orc_idx_t* options, orc_idx_t* perm, orc_idx_t* iperm);

/* METIS keeps its random-number state in globals, so concurrent calls from
 * several threads race and can return different orderings: serialize them. */
static pthread_mutex_t g_metis_lock = PTHREAD_MUTEX_INITIALIZER;

int orc_nd_order(int n, const int32_t* Ap, const int32_t* Ai, int32_t* perm) {
  /* symmetric adjacency without the diagonal, sorted + deduplicated */
  int32_t* deg = (int32_t*)calloc(n + 1, sizeof(int32_t));
  for (int c = 0; c < n; ++c)
    for (int p = Ap[c]; p < Ap[c + 1]; ++p) {
      int r = Ai[p];
      if (r == c) continue;
      deg[r + 1]++;
      deg[c + 1]++;
    }
  for (int i = 0; i < n; ++i) deg[i + 1] += deg[i];
  int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (deg[n] + 1));
  int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (n + 1));
  memcpy(cur, deg, sizeof(int32_t) * (n + 1));
  for (int c = 0; c < n; ++c)
    for (int p = Ap[c]; p < Ap[c + 1]; ++p) {
      int r = Ai[p];
      if (r == c) continue;
      adj[cur[r]++] = c;
      adj[cur[c]++] = r;
    }
  orc_idx_t* xadj = (orc_idx_t*)malloc(sizeof(orc_idx_t) * (n + 1));
  orc_idx_t* adjncy = (orc_idx_t*)malloc(sizeof(orc_idx_t) * (deg[n] + 1));
  long m = 0;
  xadj[0] = 0;
  for (int v = 0; v < n; ++v) {
    int b = deg[v], e = deg[v + 1];
    qsort(adj + b, e - b, sizeof(int32_t), cmp_i32);
    for (int p = b; p < e; ++p)
      if (p == b || adj[p] != adj[p - 1]) adjncy[m++] = adj[p];
    xadj[v + 1] = m;
  }
  int rc = 0;
  if (m == 0) {
    for (int i = 0; i < n; ++i) perm[i] = i;
  } else {
    orc_idx_t opt[40];
    METIS_SetDefaultOptions(opt);
    opt[17] = 0;   /* METIS_OPTION_NUMBERING */
    opt[8] = 42;   /* METIS_OPTION_SEED */
    orc_idx_t nv = n;
    orc_idx_t* p = (orc_idx_t*)malloc(sizeof(orc_idx_t) * n);
    orc_idx_t* ip = (orc_idx_t*)malloc(sizeof(orc_idx_t) * n);
    pthread_mutex_lock(&g_metis_lock);
    const int st = METIS_NodeND(&nv, xadj, adjncy, NULL, opt, p, ip);
    pthread_mutex_unlock(&g_metis_lock);
    if (st != 1) {
      for (int i = 0; i < n; ++i) perm[i] = i;
      rc = 1;
    } else {
      for (int i = 0; i < n; ++i) perm[i] = (int32_t)p[i];
    }
    free(p);
    free(ip);
  }
  free(deg); free(adj); free(cur); free(xadj); free(adjncy);
  return rc;
}

/* ======================================================================== */
/* NR storage and stages                                                     */
/* ======================================================================== */

typedef struct {
  int n_bus, dim, n_pv, n_pq, n_pvpq;
  const int32_t *pv, *pq;
  /* Ybus in CSR (for the Jacobian fill) and CSC (for Ibus) */
  const int32_t *yp, *yi;
  const double* yx;               /* interleaved complex, CSR order */
  int32_t *cp, *ci; double* cx;   /* CSC, rows sorted per column */
  /* Jacobian */
  int32_t *jrow, *jcol;           /* CSR pattern */
  int32_t *jcp, *jci;             /* CSC pattern */
  int32_t* csr_to_csc;
  int32_t *m11, *m21, *m12, *m22, *d11, *d21, *d12, *d22;  /* CSC positions */
  double* jx;                     /* CSC values */
  int nnz_j;
  /* state */
  double *V, *Va, *Vm, *I, *S, *F, *dx;
  orc_lu* lu;
  int32_t* order;
} nrbuf;

static void nrbuf_free(nrbuf* b) {
  free(b->cp); free(b->ci); free(b->cx);
  free(b->jrow); free(b->jcol); free(b->jcp); free(b->jci); free(b->csr_to_csc);
  free(b->m11); free(b->m21); free(b->m12); free(b->m22);
  free(b->d11); free(b->d21); free(b->d12); free(b->d22);
  free(b->jx); free(b->V); free(b->Va); free(b->Vm); free(b->I); free(b->S);
  free(b->F); free(b->dx); free(b->order);
  orc_lu_free(b->lu);
}

static int nrbuf_init(nrbuf* b, int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                      const int32_t* pv, int n_pv, const int32_t* pq, int n_pq) {
  memset(b, 0, sizeof(*b));
  b->n_bus = n_bus; b->n_pv = n_pv; b->n_pq = n_pq; b->n_pvpq = n_pv + n_pq;
  b->pv = pv; b->pq = pq;
  b->yp = indptr; b->yi = indices; b->yx = ydata;
  int nnz_j = 0;
  int dim = orc_jacobian_nnz(n_bus, indptr, indices, pv, n_pv, pq, n_pq, &nnz_j);
  if (dim <= 0) return -1;
  b->dim = dim; b->nnz_j = nnz_j;
  int nnz_y = indptr[n_bus];
  b->jrow = (int32_t*)malloc(sizeof(int32_t) * (dim + 1));
  b->jcol = (int32_t*)malloc(sizeof(int32_t) * nnz_j);
  b->m11 = (int32_t*)malloc(sizeof(int32_t) * nnz_y); b->m21 = (int32_t*)malloc(sizeof(int32_t) * nnz_y);
  b->m12 = (int32_t*)malloc(sizeof(int32_t) * nnz_y); b->m22 = (int32_t*)malloc(sizeof(int32_t) * nnz_y);
  b->d11 = (int32_t*)malloc(sizeof(int32_t) * n_bus); b->d21 = (int32_t*)malloc(sizeof(int32_t) * n_bus);
  b->d12 = (int32_t*)malloc(sizeof(int32_t) * n_bus); b->d22 = (int32_t*)malloc(sizeof(int32_t) * n_bus);
  orc_jacobian_analysis(n_bus, indptr, indices, pv, n_pv, pq, n_pq, b->jrow, b->jcol,
                        b->m11, b->m21, b->m12, b->m22, b->d11, b->d21, b->d12, b->d22);
  /* CSR pattern -> CSC pattern and the csr->csc remap of every map
   * (cpu_fp64_storage.cpp:263-322) */
  b->jcp = (int32_t*)calloc(dim + 1, sizeof(int32_t));
  b->jci = (int32_t*)malloc(sizeof(int32_t) * nnz_j);
  b->csr_to_csc = (int32_t*)malloc(sizeof(int32_t) * nnz_j);
  for (int k = 0; k < nnz_j; ++k) b->jcp[b->jcol[k] + 1]++;
  for (int c = 0; c < dim; ++c) b->jcp[c + 1] += b->jcp[c];
  {
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (dim + 1));
    memcpy(cur, b->jcp, sizeof(int32_t) * (dim + 1));
    for (int r = 0; r < dim; ++r)
      for (int k = b->jrow[r]; k < b->jrow[r + 1]; ++k) {
        int pos = cur[b->jcol[k]]++;
        b->jci[pos] = r;
        b->csr_to_csc[k] = pos;
      }
    free(cur);
  }
  int32_t* maps[4] = {b->m11, b->m21, b->m12, b->m22};
  for (int m = 0; m < 4; ++m)
    for (int k = 0; k < nnz_y; ++k) maps[m][k] = maps[m][k] >= 0 ? b->csr_to_csc[maps[m][k]] : -1;
  int32_t* dmaps[4] = {b->d11, b->d21, b->d12, b->d22};
  for (int m = 0; m < 4; ++m)
    for (int k = 0; k < n_bus; ++k) dmaps[m][k] = dmaps[m][k] >= 0 ? b->csr_to_csc[dmaps[m][k]] : -1;
  b->jx = (double*)calloc(nnz_j, sizeof(double));
  /* Ybus CSC (rows ascending inside each column) */
  b->cp = (int32_t*)calloc(n_bus + 1, sizeof(int32_t));
  b->ci = (int32_t*)malloc(sizeof(int32_t) * nnz_y);
  b->cx = (double*)malloc(sizeof(double) * 2 * nnz_y);
  for (int k = 0; k < nnz_y; ++k) b->cp[indices[k] + 1]++;
  for (int c = 0; c < n_bus; ++c) b->cp[c + 1] += b->cp[c];
  {
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (n_bus + 1));
    memcpy(cur, b->cp, sizeof(int32_t) * (n_bus + 1));
    for (int r = 0; r < n_bus; ++r)
      for (int k = indptr[r]; k < indptr[r + 1]; ++k) {
        int pos = cur[indices[k]]++;
        b->ci[pos] = r;
        b->cx[2 * pos] = ydata[2 * k];
        b->cx[2 * pos + 1] = ydata[2 * k + 1];
      }
    free(cur);
  }
  b->V = (double*)malloc(sizeof(double) * 2 * n_bus);
  b->I = (double*)malloc(sizeof(double) * 2 * n_bus);
  b->S = (double*)malloc(sizeof(double) * 2 * n_bus);
  b->Va = (double*)malloc(sizeof(double) * n_bus);
  b->Vm = (double*)malloc(sizeof(double) * n_bus);
  b->F = (double*)malloc(sizeof(double) * dim);
  b->dx = (double*)malloc(sizeof(double) * dim);
  return 0;
}

/* Ibus = Ybus V by CSC column SAXPY (compute_ibus.cpp:18-34). */
static void stage_ibus(nrbuf* b) {
  int n = b->n_bus;
  for (int i = 0; i < 2 * n; ++i) b->I[i] = 0.0;
  for (int c = 0; c < n; ++c) {
    double vr = b->V[2 * c], vi = b->V[2 * c + 1];
    for (int k = b->cp[c]; k < b->cp[c + 1]; ++k) {
      int r = b->ci[k];
      double yr = b->cx[2 * k], yi = b->cx[2 * k + 1];
      b->I[2 * r] += yr * vr - yi * vi;
      b->I[2 * r + 1] += yr * vi + yi * vr;
    }
  }
}

/* F = [Re mis@pv, Re mis@pq, Im mis@pq], mis = V conj(I) - S
 * (cpu_mismatch.cpp:60-82); returns max |F| (cpu_mismatch.cpp:86-107). */
static double stage_mismatch(nrbuf* b) {
  int k = 0;
  double norm = 0.0;
#define MIS_RE(i) ((b->V[2 * (i)] * b->I[2 * (i)] - b->V[2 * (i) + 1] * (-b->I[2 * (i) + 1])) - b->S[2 * (i)])
#define MIS_IM(i) ((b->V[2 * (i)] * (-b->I[2 * (i) + 1]) + b->V[2 * (i) + 1] * b->I[2 * (i)]) - b->S[2 * (i) + 1])
  for (int i = 0; i < b->n_pv; ++i) b->F[k++] = MIS_RE(b->pv[i]);
  for (int i = 0; i < b->n_pq; ++i) b->F[k++] = MIS_RE(b->pq[i]);
  for (int i = 0; i < b->n_pq; ++i) b->F[k++] = MIS_IM(b->pq[i]);
#undef MIS_RE
#undef MIS_IM
  for (int i = 0; i < b->dim; ++i) {
    double a = fabs(b->F[i]);
    norm = a > norm ? a : norm;
  }
  return norm;
}

/* Jacobian values into the CSC storage (fill_jacobian.cpp:178-244). */
static void stage_jacobian(nrbuf* b) {
  int n = b->n_bus;
  for (int k = 0; k < b->nnz_j; ++k) b->jx[k] = 0.0;
  double* vn = (double*)malloc(sizeof(double) * 2 * n);
  for (int i = 0; i < n; ++i) {
    double vr = b->V[2 * i], vi = b->V[2 * i + 1];
    double vm = hypot(vr, vi);
    if (vm < 1e-8) vm = 1e-8;
    vn[2 * i] = vr / vm;
    vn[2 * i + 1] = vi / vm;
  }
  for (int r = 0; r < n; ++r) {
    double vir = b->V[2 * r], vii = b->V[2 * r + 1];
    /* (-j) * V_i */
    double ar = vii, ai = -vir;
    for (int k = b->yp[r]; k < b->yp[r + 1]; ++k) {
      int c = b->yi[k];
      double yr = b->yx[2 * k], yi = b->yx[2 * k + 1];
      /* conj(y * V_j) */
      double vjr = b->V[2 * c], vji = b->V[2 * c + 1];
      double cr = yr * vjr - yi * vji, ci = -(yr * vji + yi * vjr);
      double va_re = ar * cr - ai * ci, va_im = ar * ci + ai * cr;
      /* V_i * conj(y * Vnorm_j) */
      double nr_ = vn[2 * c], ni = vn[2 * c + 1];
      double dr = yr * nr_ - yi * ni, di = -(yr * ni + yi * nr_);
      double vm_re = vir * dr - vii * di, vm_im = vir * di + vii * dr;
      if (b->m11[k] >= 0) b->jx[b->m11[k]] = va_re;
      if (b->m21[k] >= 0) b->jx[b->m21[k]] = va_im;
      if (b->m12[k] >= 0) b->jx[b->m12[k]] = vm_re;
      if (b->m22[k] >= 0) b->jx[b->m22[k]] = vm_im;
    }
  }
  for (int i = 0; i < n; ++i) {
    double vr = b->V[2 * i], vi = b->V[2 * i + 1];
    double ir = b->I[2 * i], ii = -b->I[2 * i + 1];   /* conj(I) */
    /* j * (V * conj(I)) */
    double pr = vr * ir - vi * ii, pi = vr * ii + vi * ir;
    double va_re = 0.0 * pr - 1.0 * pi, va_im = 0.0 * pi + 1.0 * pr;
    /* conj(I) * Vnorm */
    double nr_ = vn[2 * i], ni = vn[2 * i + 1];
    double vm_re = ir * nr_ - ii * ni, vm_im = ir * ni + ii * nr_;
    if (b->d11[i] >= 0) b->jx[b->d11[i]] += va_re;
    if (b->d21[i] >= 0) b->jx[b->d21[i]] += va_im;
    if (b->d12[i] >= 0) b->jx[b->d12[i]] += vm_re;
    if (b->d22[i] >= 0) b->jx[b->d22[i]] += vm_im;
  }
  free(vn);
}

static int stage_factor_solve(nrbuf* b) {
  if (!b->order) {
    b->order = (int32_t*)malloc(sizeof(int32_t) * b->dim);
    orc_nd_order(b->dim, b->jcp, b->jci, b->order);
  }
  if (!b->lu) {
    b->lu = orc_lu_factor(b->dim, b->jcp, b->jci, b->jx, b->order, 0.001);
    if (!b->lu) return -1;
  } else if (orc_lu_refactor(b->lu, b->jcp, b->jci, b->jx)) {
    return -1;
  }
  memcpy(b->dx, b->F, sizeof(double) * b->dim);
  orc_lu_solve(b->lu, b->dx);
  return 0;
}

/* Va/Vm -= dx, V = Vm (cos Va + j sin Va) (cpu_voltage_update.cpp:19-43). */
static void stage_update(nrbuf* b) {
  for (int i = 0; i < b->n_pv; ++i) b->Va[b->pv[i]] -= b->dx[i];
  for (int i = 0; i < b->n_pq; ++i) b->Va[b->pq[i]] -= b->dx[b->n_pv + i];
  for (int i = 0; i < b->n_pq; ++i) b->Vm[b->pq[i]] -= b->dx[b->n_pvpq + i];
  for (int i = 0; i < b->n_bus; ++i) {
    b->V[2 * i] = b->Vm[i] * cos(b->Va[i]);
    b->V[2 * i + 1] = b->Vm[i] * sin(b->Va[i]);
  }
}

static void set_state(nrbuf* b, const double* sbus, const double* v0) {
  for (int i = 0; i < b->n_bus; ++i) {
    b->V[2 * i] = v0[2 * i];
    b->V[2 * i + 1] = v0[2 * i + 1];
    b->Va[i] = atan2(v0[2 * i + 1], v0[2 * i]);
    b->Vm[i] = hypot(v0[2 * i], v0[2 * i + 1]);
    if (sbus) {
      b->S[2 * i] = sbus[2 * i];
      b->S[2 * i + 1] = sbus[2 * i + 1];
    } else {
      b->S[2 * i] = b->S[2 * i + 1] = 0.0;
    }
  }
}

static int nr_run(nrbuf* b, const double* sbus, const double* v0, orc_nr_config cfg,
                  double* v_out, orc_nr_result* res) {
  set_state(b, sbus, v0);
  int completed = 0;
  double norm = 0.0;
  int status = 0;
  for (int it = 0; it < cfg.max_iter; ++it) {
    completed = it + 1;
    stage_ibus(b);
    norm = stage_mismatch(b);
    if (!isfinite(norm)) { status = 1; break; }
    if (norm <= cfg.tolerance) break;
    stage_jacobian(b);
    if (stage_factor_solve(b)) { status = 2; break; }
    stage_update(b);
  }
  /* final mismatch = the last evaluated norm; when the loop runs out it was
   * taken before the last update, exactly as the reference reports it
   * (newton_solver.cpp:324-341 reads ctx.normF) */
  if (v_out) memcpy(v_out, b->V, sizeof(double) * 2 * b->n_bus);
  if (res) {
    res->iterations = completed;
    res->final_mismatch = norm;
    res->converged = (status == 0 && norm <= cfg.tolerance) ? 1 : 0;
    res->status = status;
  }
  return status;
}

int orc_nr_solve(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                 const double* sbus, const double* v0,
                 const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                 orc_nr_config cfg, double* v_out, orc_nr_result* res) {
  nrbuf b;
  if (nrbuf_init(&b, n_bus, indptr, indices, ydata, pv, n_pv, pq, n_pq)) {
    if (res) res->status = 3;
    return 3;
  }
  int st = nr_run(&b, sbus, v0, cfg, v_out, res);
  nrbuf_free(&b);
  return st;
}

double orc_mismatch(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                    const double* sbus, const double* v,
                    const int32_t* pv, int n_pv, const int32_t* pq, int n_pq, double* F) {
  nrbuf b;
  if (nrbuf_init(&b, n_bus, indptr, indices, ydata, pv, n_pv, pq, n_pq)) return -1.0;
  set_state(&b, sbus, v);
  stage_ibus(&b);
  double norm = stage_mismatch(&b);
  memcpy(F, b.F, sizeof(double) * b.dim);
  nrbuf_free(&b);
  return norm;
}

int orc_jacobian_values(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                        const double* v, const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                        double* jvals_csr) {
  nrbuf b;
  if (nrbuf_init(&b, n_bus, indptr, indices, ydata, pv, n_pv, pq, n_pq)) return -1;
  set_state(&b, NULL, v);
  stage_ibus(&b);
  stage_jacobian(&b);
  for (int k = 0; k < b.nnz_j; ++k) jvals_csr[k] = b.jx[b.csr_to_csc[k]];
  nrbuf_free(&b);
  return 0;
}

double orc_adjoint(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                   const double* v, const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                   const double* grad_va, const double* grad_vm,
                   double* lambda, double* grad_p, double* grad_q) {
  nrbuf b;
  if (nrbuf_init(&b, n_bus, indptr, indices, ydata, pv, n_pv, pq, n_pq)) return -1.0;
  set_state(&b, NULL, v);
  stage_ibus(&b);
  stage_jacobian(&b);
  b.order = (int32_t*)malloc(sizeof(int32_t) * b.dim);
  orc_nd_order(b.dim, b.jcp, b.jci, b.order);
  b.lu = orc_lu_factor(b.dim, b.jcp, b.jci, b.jx, b.order, 0.001);
  if (!b.lu) { nrbuf_free(&b); return -1.0; }
  int dim = b.dim, npvpq = b.n_pvpq;
  double* rhs = (double*)malloc(sizeof(double) * dim);
  /* build_grad_state (adjoint_math.cpp:156-184) */
  for (int i = 0; i < n_pv; ++i) rhs[i] = grad_va[pv[i]];
  for (int i = 0; i < n_pq; ++i) {
    rhs[n_pv + i] = grad_va[pq[i]];
    rhs[npvpq + i] = grad_vm[pq[i]];
  }
  memcpy(lambda, rhs, sizeof(double) * dim);
  orc_lu_tsolve(b.lu, lambda);
  /* relative residual (adjoint_math.cpp:222-248), long double accumulation */
  long double rsq = 0.0L, bsq = 0.0L;
  for (int c = 0; c < dim; ++c) {
    long double acc = 0.0L;
    for (int p = b.jcp[c]; p < b.jcp[c + 1]; ++p) acc += (long double)b.jx[p] * (long double)lambda[b.jci[p]];
    long double d = acc - (long double)rhs[c];
    rsq += d * d;
    bsq += (long double)rhs[c] * (long double)rhs[c];
  }
  long double den = sqrtl(bsq > 1e-60L ? bsq : 1e-60L);
  if (den < 1e-30L) den = 1e-30L;
  double rel = (double)(sqrtl(rsq) / den);
  /* project_load_gradients (adjoint_math.cpp:189-216): grad = -lambda */
  for (int i = 0; i < n_bus; ++i) grad_p[i] = grad_q[i] = 0.0;
  for (int i = 0; i < n_pv; ++i) grad_p[pv[i]] = -lambda[i];
  for (int i = 0; i < n_pq; ++i) {
    grad_p[pq[i]] = -lambda[n_pv + i];
    grad_q[pq[i]] = -lambda[npvpq + i];
  }
  free(rhs);
  nrbuf_free(&b);
  return rel;
}

/* ---- many independent cases over host threads (CPU baseline) ---- */

typedef struct {
  int n_bus;
  const int32_t *indptr, *indices;
  const double* ydata;
  const double *sbus, *v0;
  const int32_t *pv, *pq;
  int n_pv, n_pq, count, threads, tid;
  orc_nr_config cfg;
  double* v_out;
  int32_t* iterations;
  double* final_mismatch;
  int failed;
} many_job;

static void* many_worker(void* arg) {
  many_job* j = (many_job*)arg;
  nrbuf b;
  if (nrbuf_init(&b, j->n_bus, j->indptr, j->indices, j->ydata, j->pv, j->n_pv, j->pq, j->n_pq)) {
    j->failed = 1;
    return NULL;
  }
  size_t stride = 2 * (size_t)j->n_bus;
  for (int c = j->tid; c < j->count; c += j->threads) {
    orc_nr_result r;
    nr_run(&b, j->sbus + c * stride, j->v0 + c * stride, j->cfg,
           j->v_out ? j->v_out + c * stride : NULL, &r);
    if (j->iterations) j->iterations[c] = r.iterations;
    if (j->final_mismatch) j->final_mismatch[c] = r.final_mismatch;
  }
  nrbuf_free(&b);
  return NULL;
}

int orc_nr_solve_many(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                      const double* sbus, const double* v0, int count,
                      const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                      orc_nr_config cfg, int threads, double* v_out,
                      int32_t* iterations, double* final_mismatch) {
  if (threads < 1) threads = 1;
  if (threads > count) threads = count > 0 ? count : 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
  many_job* jobs = (many_job*)malloc(sizeof(many_job) * threads);
  for (int t = 0; t < threads; ++t) {
    many_job j = {n_bus, indptr, indices, ydata, sbus, v0, pv, pq, n_pv, n_pq, count, threads, t,
                  cfg, v_out, iterations, final_mismatch, 0};
    jobs[t] = j;
    pthread_create(&th[t], NULL, many_worker, &jobs[t]);
  }
  int failed = 0;
  for (int t = 0; t < threads; ++t) {
    pthread_join(th[t], NULL);
    failed |= jobs[t].failed;
  }
  free(th);
  free(jobs);
  return failed;
}
