/* Test infrastructure only (checker, never shipped): CPU restatement of the exafmm-dev
 * Laplace FMM hot path.  Each function cites the reference file:line it restates.  Built
 * with -ffp-contract=off so every float operation is a plain IEEE operation, like the
 * reference parity build in oracle/Makefile.
 *
 * Parity pins (tests/test_oracle_vs_reference.py): bounds, adaptive tree cells, body order
 * and interaction lists bit-exact against the reference harness; expansions and potentials
 * within rounding; the examples/kernel.cxx translation chain errors per P. */
#define _DEFAULT_SOURCE
#include "fmm_oracle.h"
#include <tgmath.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
typedef ORACLE_REAL real;

/* deepest level the adaptive builder splits to; a node there keeps all its bodies.
 * (The reference has no cap and recurses forever on > ncrit coincident bodies.) */
#define ORACLE_MAX_LEVEL 21

typedef struct { real re, im; } cplx;
static inline cplx cx(real re, real im) { cplx c = {re, im}; return c; }
static inline cplx cadd(cplx a, cplx b) { return cx(a.re + b.re, a.im + b.im); }
static inline cplx cmul(cplx a, cplx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cplx cscale(cplx a, real s) { return cx(a.re * s, a.im * s); }
static inline cplx cconj(cplx a) { return cx(a.re, -a.im); }
/* a / b as libgcc's complex division evaluates it when b has a zero imaginary part
 * (the case for every monopole M[0], which P2M and M2M leave real) */
static inline cplx cdivm(cplx a, cplx b) {
  if (b.im == 0) return cx(a.re / b.re, a.im / b.re);
  real den = b.re * b.re + b.im * b.im;
  return cx((a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den);
}
#define ODDEVEN(n) ((((n) & 1) == 1) ? -1 : 1)
#define IPOW2N(n) ((n >= 0) ? 1 : ODDEVEN(n))

/* compensated accumulator: include/kahan.h (gpu/kahan.h:35-41); value is s + c there */
typedef struct { real s, c; } kreal;
static inline void kadd(kreal* k, real v) {
  real y = v - k->c;
  real t = k->s + y;
  k->c = (t - k->s) - y;
  k->s = t;
}

typedef struct {
  int begin, count, level;
  real X[3];
  int child[8];
  int nnode;
} Node;

typedef struct {
  int n;
  oracle_params p;
  int nterm, ncoef; /* ncoef: reals per expansion (2*nterm spherical, nterm Cartesian) */
  real eps2;
  /* bodies, permuted into tree order by oracle_build_tree */
  real *x, *q;     /* x: 3 per body */
  int* ibody;
  real* trg;       /* 4 per body */
  kreal* ktrg;     /* 4 per body when kahan */
  /* tree */
  real X0[3], R0;
  Node* nodes;
  int nnodes, capnodes, root;
  int nc, maxlevel;
  int *iparent, *ichild, *nchild, *cibody, *cnbody, *clevel;
  unsigned long long* icell;
  real *cX, *R, *Rbuilt;
  real *M, *L;
  /* lists (target << 32 | source | image << 27) in visiting order */
  long long *m2l, *p2p;
  /* periodic shift of the source tree in the traversal under way, and its image code */
  real xp[3];
  int img;
  int box_fixed; /* the box was set from the bounds of two body sets (oracle_solve_ij) */
  long long nm2l, np2p, capm2l, capp2p;
  /* cartesian index helpers */
  int* cidx;   /* [nx][ny][nz] -> term, size P^3 */
  int* cmi;    /* term -> nx,ny,nz (3 per term) */
} Oracle;

/* ------------------------------------------------------------------ Cartesian indices */
/* Index<nx,ny,nz>::I (kernels/LaplaceCartesianCPU.cxx:3-25): terms ordered by total order,
 * then nx descending, then ny descending. */
static void cart_tables(Oracle* o) {
  int P = o->p.P;
  o->cidx = (int*)malloc(sizeof(int) * P * P * P);
  o->cmi = (int*)malloc(sizeof(int) * 3 * o->nterm);
  for (int i = 0; i < P * P * P; i++) o->cidx[i] = -1;
  int t = 0;
  for (int n = 0; n < P; n++)
    for (int nx = n; nx >= 0; nx--)
      for (int ny = n - nx; ny >= 0; ny--) {
        int nz = n - nx - ny;
        o->cidx[(nx * P + ny) * P + nz] = t;
        o->cmi[3 * t] = nx;
        o->cmi[3 * t + 1] = ny;
        o->cmi[3 * t + 2] = nz;
        t++;
      }
}
static inline int CI(const Oracle* o, int nx, int ny, int nz) {
  int P = o->p.P;
  return o->cidx[(nx * P + ny) * P + nz];
}

/* ------------------------------------------------------------------ handle */
void* oracle_new(int n, const double* x, const double* q, const oracle_params* prm) {
  Oracle* o = (Oracle*)calloc(1, sizeof(Oracle));
  o->n = n;
  o->p = *prm;
  int P = prm->P;
  o->nterm = prm->basis == ORACLE_SPHERICAL ? P * (P + 1) / 2 : P * (P + 1) * (P + 2) / 6;
  o->ncoef = prm->basis == ORACLE_SPHERICAL ? 2 * o->nterm : o->nterm;
  /* Traversal::eps2 is `const int` (include/traversal.h:17) */
  o->eps2 = (real)(int)prm->eps2;
  o->x = (real*)malloc(sizeof(real) * 3 * (n > 0 ? n : 1));
  o->q = (real*)malloc(sizeof(real) * (n > 0 ? n : 1));
  o->ibody = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
  o->trg = (real*)calloc(4 * (n > 0 ? n : 1), sizeof(real));
  o->ktrg = (kreal*)calloc(4 * (n > 0 ? n : 1), sizeof(kreal));
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) o->x[3 * i + d] = (real)x[3 * i + d];
    o->q[i] = (real)q[i];
    o->ibody[i] = i;
  }
  if (prm->basis == ORACLE_CARTESIAN) cart_tables(o);
  o->root = -1;
  return o;
}

static void free_cells(Oracle* o) {
  free(o->iparent); free(o->ichild); free(o->nchild); free(o->cibody); free(o->cnbody);
  free(o->clevel); free(o->icell); free(o->cX); free(o->R); free(o->Rbuilt); free(o->M);
  free(o->L);
}

void oracle_free(void* h) {
  Oracle* o = (Oracle*)h;
  if (!o) return;
  free(o->x); free(o->q); free(o->ibody); free(o->trg); free(o->ktrg); free(o->nodes);
  free_cells(o);
  free(o->m2l); free(o->p2p); free(o->cidx); free(o->cmi);
  free(o);
}

int oracle_real_bytes(void) { return (int)sizeof(real); }

/* ------------------------------------------------------------------ bounds and box */
/* BoundBox::getBounds (include/bound_box.h:76-88, BodiesRecursion :20-39) and
 * BuildTree::bounds2box (include/build_tree_tbb.h:298-310). */
static void update_bounds(const Oracle* o, real* Xmin, real* Xmax) {
  for (int i = 0; i < o->n; i++)
    for (int d = 0; d < 3; d++) {
      real v = o->x[3 * i + d];
      Xmin[d] = v < Xmin[d] ? v : Xmin[d];
      Xmax[d] = v > Xmax[d] ? v : Xmax[d];
    }
}
static void bounds2box(Oracle* o, const real* Xmin, const real* Xmax);
static void make_box(Oracle* o) {
  real Xmin[3], Xmax[3];
  if (o->n == 0) {
    for (int d = 0; d < 3; d++) Xmin[d] = Xmax[d] = 0;
  } else {
    for (int d = 0; d < 3; d++) Xmin[d] = Xmax[d] = o->x[d];
    update_bounds(o, Xmin, Xmax);
  }
  bounds2box(o, Xmin, Xmax);
}
static void bounds2box(Oracle* o, const real* Xmin, const real* Xmax) {
  real R = 0;
  for (int d = 0; d < 3; d++) o->X0[d] = (Xmax[d] + Xmin[d]) / 2;
  for (int d = 0; d < 3; d++) {
    real a = o->X0[d] - Xmin[d];
    R = a > R ? a : R;
    real b = Xmax[d] - o->X0[d];
    R = b > R ? b : R;
  }
  o->R0 = (real)((double)R * 1.00001);
}

/* ------------------------------------------------------------------ adaptive tree */
static int new_node(Oracle* o) {
  if (o->nnodes == o->capnodes) {
    o->capnodes = o->capnodes ? 2 * o->capnodes : 1024;
    o->nodes = (Node*)realloc(o->nodes, sizeof(Node) * o->capnodes);
  }
  return o->nnodes++;
}

/* BuildNodes (include/build_tree_tbb.h:165-218): leaf when NBODY <= ncrit (:172); else
 * stable scatter by octant (x > X) + 2 (y > Y) + 4 (z > Z) (CountBodies :52-81, MoveBodies
 * :97-115), child centre X +- R0 / 2^(level+1) (:199-203), empty octants dropped (:168). */
static int build_nodes(Oracle* o, int begin, int end, const real X[3], int level, real* xb,
                       real* qb, int* ib) {
  if (begin == end) return -1;
  int v = new_node(o);
  Node* nd = &o->nodes[v];
  nd->begin = begin;
  nd->count = end - begin;
  nd->level = level;
  for (int d = 0; d < 3; d++) nd->X[d] = X[d];
  for (int i = 0; i < 8; i++) nd->child[i] = -1;
  nd->nnode = 1;
  if (end - begin <= o->p.ncrit || level >= ORACLE_MAX_LEVEL) return v;
  int cnt[8] = {0}, off[8];
  for (int i = begin; i < end; i++) {
    const real* x = &o->x[3 * i];
    int oct = (x[0] > X[0]) + ((x[1] > X[1]) << 1) + ((x[2] > X[2]) << 2);
    cnt[oct]++;
  }
  int s = begin;
  for (int i = 0; i < 8; i++) { off[i] = s; s += cnt[i]; }
  int pos[8];
  memcpy(pos, off, sizeof(pos));
  for (int i = begin; i < end; i++) {
    const real* x = &o->x[3 * i];
    int oct = (x[0] > X[0]) + ((x[1] > X[1]) << 1) + ((x[2] > X[2]) << 2);
    int p = pos[oct]++;
    for (int d = 0; d < 3; d++) xb[3 * p + d] = x[d];
    qb[p] = o->q[i];
    ib[p] = o->ibody[i];
  }
  memcpy(&o->x[3 * begin], &xb[3 * begin], sizeof(real) * 3 * (end - begin));
  memcpy(&o->q[begin], &qb[begin], sizeof(real) * (end - begin));
  memcpy(&o->ibody[begin], &ib[begin], sizeof(int) * (end - begin));
  int nnode = 1;
  for (int i = 0; i < 8; i++) {
    real Xc[3];
    real r = o->R0 / (1 << (level + 1));
    for (int d = 0; d < 3; d++) Xc[d] = X[d] + r * (((i & 1 << d) >> d) * 2 - 1);
    int c = build_nodes(o, off[i], off[i] + cnt[i], Xc, level + 1, xb, qb, ib);
    o->nodes[v].child[i] = c;
    if (c >= 0) nnode += o->nodes[c].nnode;
  }
  o->nodes[v].nnode = nnode;
  return v;
}

/* Nodes2cells::getKey (include/build_tree_tbb.h:240-249), with 64-bit shifts throughout
 * (the reference's 32-bit `1 << 3*level` and `<< (3*l+d)` overflow above level 10). */
static unsigned long long cell_key(const real X[3], const real Xmin[3], real diameter, int level) {
  int iX[3];
  for (int d = 0; d < 3; d++) iX[d] = (int)((X[d] - Xmin[d]) / diameter);
  unsigned long long index = ((1ULL << (3 * level)) - 1) / 7;
  for (int l = 0; l < level; l++) {
    for (int d = 0; d < 3; d++) index += (unsigned long long)(iX[d] & 1) << (3 * l + d);
    for (int d = 0; d < 3; d++) iX[d] >>= 1;
  }
  return index;
}

/* Nodes2cells::operator() (include/build_tree_tbb.h:250-294): children contiguous at CN,
 * each child's subtree placed after the previous child's (:272-286). */
static void nodes2cells(Oracle* o, int v, int c, int CN, int level, int iparent) {
  Node* nd = &o->nodes[v];
  o->iparent[c] = iparent;
  o->R[c] = o->R0 / (1 << level);
  for (int d = 0; d < 3; d++) o->cX[3 * c + d] = nd->X[d];
  o->cnbody[c] = nd->count;
  o->cibody[c] = nd->begin;
  o->clevel[c] = level;
  real Xmin[3];
  for (int d = 0; d < 3; d++) Xmin[d] = o->X0[d] - o->R0;
  o->icell[c] = cell_key(nd->X, Xmin, 2 * o->R[c], level);
  if (level > o->maxlevel) o->maxlevel = level;
  if (nd->nnode == 1) {
    o->ichild[c] = 0;
    o->nchild[c] = 0;
    return;
  }
  int nch = 0;
  for (int i = 0; i < 8; i++) nch += nd->child[i] >= 0;
  int ci = CN;
  o->ichild[c] = ci;
  o->nchild[c] = nch;
  CN += nch;
  for (int i = 0; i < 8; i++) {
    int ch = nd->child[i];
    if (ch < 0) continue;
    nodes2cells(o, ch, ci, CN, level + 1, c);
    ci++;
    CN += o->nodes[ch].nnode - 1;
  }
}

static int build_uniform(Oracle* o);

/* BuildTree::buildTree (include/build_tree_tbb.h:365-374) = growTree (:313) + linkTree (:347);
 * with tree = ORACLE_TREE_UNIFORM, BuildTree::buildTree of include/build_tree_omp.h:216-262 */
int oracle_build_tree(void* h) {
  Oracle* o = (Oracle*)h;
  if (!o->box_fixed) make_box(o);
  o->nnodes = 0;
  o->maxlevel = 0;
  free_cells(o);
  o->iparent = o->ichild = o->nchild = o->cibody = o->cnbody = o->clevel = NULL;
  o->icell = NULL;
  o->cX = o->R = o->Rbuilt = o->M = o->L = NULL;
  o->nc = 0;
  if (o->n == 0) return 0;
  if (o->p.tree == ORACLE_TREE_UNIFORM) return build_uniform(o);
  real* xb = (real*)malloc(sizeof(real) * 3 * o->n);
  real* qb = (real*)malloc(sizeof(real) * o->n);
  int* ib = (int*)malloc(sizeof(int) * o->n);
  o->root = build_nodes(o, 0, o->n, o->X0, 0, xb, qb, ib);
  free(xb); free(qb); free(ib);
  int nc = o->nodes[o->root].nnode;
  o->nc = nc;
  /* cell arrays hold 27 more cells past the tree: the periodic cells of traversePeriodic */
  int na = nc + 27;
  o->iparent = (int*)calloc(na, sizeof(int));
  o->ichild = (int*)calloc(na, sizeof(int));
  o->nchild = (int*)calloc(na, sizeof(int));
  o->cibody = (int*)calloc(na, sizeof(int));
  o->cnbody = (int*)calloc(na, sizeof(int));
  o->clevel = (int*)calloc(na, sizeof(int));
  o->icell = (unsigned long long*)calloc(na, sizeof(unsigned long long));
  o->cX = (real*)calloc(3 * na, sizeof(real));
  o->R = (real*)calloc(na, sizeof(real));
  o->Rbuilt = (real*)calloc(na, sizeof(real));
  o->M = (real*)calloc((size_t)na * o->ncoef, sizeof(real));
  o->L = (real*)calloc((size_t)na * o->ncoef, sizeof(real));
  nodes2cells(o, o->root, 0, 1, 0, 0);
  memcpy(o->Rbuilt, o->R, sizeof(real) * nc);
  return 0;
}

/* ------------------------------------------------------------------ uniform Morton tree */
/* BuildTree of include/build_tree_omp.h:214-262, the builder an OpenMP build without TBB
 * uses (include/build_tree.h:12-13): every leaf at depth
 * level = 1 + int(log(N / ncrit) / ln 2 / 3) (integer N / ncrit, :218), or 0 for N < ncrit. */
int oracle_uniform_level(int n, int ncrit) {
  return n >= ncrit ? 1 + (int)(log((double)(n / ncrit)) / M_LN2 / 3) : 0;
}

/* the cell size of a level, as getKey / bodies2leafs declare it: `float d`, computed as
 * 2 R / 2^level in real_t (:38, :135) */
static float uniform_d(const Oracle* o, int level) { return (float)(2 * o->R0 / (1 << level)); }

/* grid index of a position along one axis: (X - Xmin) / d truncated to int, with d a float
 * promoted to real_t (:42-44) */
static int uniform_ix(real x, real xmin, float d) { return (int)((x - xmin) / d); }

typedef struct { unsigned long long key; int idx; } KeyIdx;
static int cmp_keyidx(const void* a, const void* b) {
  const KeyIdx *u = (const KeyIdx*)a, *v = (const KeyIdx*)b;
  if (u->key != v->key) return u->key < v->key ? -1 : 1;
  return u->idx < v->idx ? -1 : (u->idx > v->idx);
}

static int build_uniform(Oracle* o) {
  const int n = o->n, level = oracle_uniform_level(n, o->p.ncrit);
  /* the reference's `int id` holds bits up to 3 level - 1; above level 10 its shifts leave
   * the int (:47-49), which neither this restatement nor the device reproduces */
  if (level > 10) return 1;
  real Xmin[3], Xmax[3];
  for (int d = 0; d < 3; d++) Xmin[d] = Xmax[d] = o->x[d];
  update_bounds(o, Xmin, Xmax);
  /* getKey (:36-57) */
  const float d = uniform_d(o, level);
  KeyIdx* ki = (KeyIdx*)malloc(sizeof(KeyIdx) * n);
  for (int b = 0; b < n; b++) {
    int ix = uniform_ix(o->x[3 * b], Xmin[0], d), iy = uniform_ix(o->x[3 * b + 1], Xmin[1], d),
        iz = uniform_ix(o->x[3 * b + 2], Xmin[2], d);
    int id = 0;
    for (int l = 0; l != level; ++l) {
      id += (ix & 1) << (3 * l);
      id += (iy & 1) << (3 * l + 1);
      id += (iz & 1) << (3 * l + 2);
      ix >>= 1;
      iy >>= 1;
      iz >>= 1;
    }
    ki[b].key = (unsigned long long)id;
    ki[b].idx = b;
  }
  /* radixSort (:59-121) is an LSD sort, stable in the input order; permute (:123-128) */
  qsort(ki, n, sizeof(KeyIdx), cmp_keyidx);
  real* xb = (real*)malloc(sizeof(real) * 3 * n);
  real* qb = (real*)malloc(sizeof(real) * n);
  int* ib = (int*)malloc(sizeof(int) * n);
  unsigned long long* key = (unsigned long long*)malloc(sizeof(unsigned long long) * n);
  for (int b = 0; b < n; b++) {
    const int s = ki[b].idx;
    for (int k = 0; k < 3; k++) xb[3 * b + k] = o->x[3 * s + k];
    qb[b] = o->q[s];
    ib[b] = o->ibody[s];
    key[b] = ki[b].key;
  }
  memcpy(o->x, xb, sizeof(real) * 3 * n);
  memcpy(o->q, qb, sizeof(real) * n);
  memcpy(o->ibody, ib, sizeof(int) * n);
  free(xb); free(qb); free(ib); free(ki);
  /* cells in construction order: bodies2leafs (:130-158) then leafs2cells (:160-198) */
  int cap = n + 16, nc = 0;
  int *fb = (int*)malloc(sizeof(int) * cap), *nb = (int*)malloc(sizeof(int) * cap);
  int *ch0 = (int*)malloc(sizeof(int) * cap), *nch = (int*)malloc(sizeof(int) * cap);
  int *par = (int*)malloc(sizeof(int) * cap), *lev = (int*)malloc(sizeof(int) * cap);
  unsigned long long* ic = (unsigned long long*)malloc(sizeof(unsigned long long) * cap);
  real* X = (real*)malloc(sizeof(real) * 3 * cap);
  real* R = (real*)malloc(sizeof(real) * cap);
  /* cell centre and radius at cell size dl from the cell's first body (:148-151, :182-185):
   * d (ix + .5) + Xmin evaluated in double, stored in real_t */
#define UNIFORM_CELL(c, b, dl)                                                         \
  do {                                                                                 \
    for (int k = 0; k < 3; k++) {                                                      \
      int ik = uniform_ix(o->x[3 * (b) + k], Xmin[k], dl);                             \
      X[3 * (c) + k] = (real)((double)(dl) * (ik + .5) + (double)Xmin[k]);             \
    }                                                                                  \
    R[c] = (real)((double)(dl) * .5);                                                  \
  } while (0)
  {
    long long prev = -1;
    for (int b = 0; b < n; b++) {
      const int IC = (int)key[b];
      if (IC != prev) {
        fb[nc] = b; nb[nc] = 0; ch0[nc] = 0; nch[nc] = 0; lev[nc] = level; ic[nc] = IC;
        UNIFORM_CELL(nc, b, d);
        nc++;
        prev = IC;
      }
      nb[nc - 1]++;
    }
  }
  int begin = 0, end = nc;
  float dl = d;
  for (int l = 1; l <= level; l++) {
    const int div = 1 << (3 * l);
    dl *= 2;
    long long prev = -1;
    int p = end - 1;
    for (int c = begin; c != end; c++) {
      const int b = fb[c];
      const int IC = (int)(key[b] / div);
      if (IC != prev) {
        fb[nc] = b; nb[nc] = 0; ch0[nc] = c; nch[nc] = 0; lev[nc] = level - l; ic[nc] = IC;
        UNIFORM_CELL(nc, b, dl);
        nc++;
        p++;
        prev = IC;
      }
      nch[p]++;
      nb[p] += nb[c];
      par[c] = p;
    }
    begin = end;
    end = nc;
  }
#undef UNIFORM_CELL
  par[nc - 1] = 0;
  /* reverseOrder (:200-211): cell c goes to nc - 1 - c, ICHILD to the lowest index of its
   * (now descending) children, leaves (ICHILD 0) to nc, the root's parent 0 to nc - 1 */
  free_cells(o);
  int na = nc + 27;  /* + the periodic cells of traversePeriodic, as the adaptive build */
  o->iparent = (int*)calloc(na, sizeof(int));
  o->ichild = (int*)calloc(na, sizeof(int));
  o->nchild = (int*)calloc(na, sizeof(int));
  o->cibody = (int*)calloc(na, sizeof(int));
  o->cnbody = (int*)calloc(na, sizeof(int));
  o->clevel = (int*)calloc(na, sizeof(int));
  o->icell = (unsigned long long*)calloc(na, sizeof(unsigned long long));
  o->cX = (real*)calloc(3 * na, sizeof(real));
  o->R = (real*)calloc(na, sizeof(real));
  o->Rbuilt = (real*)calloc(na, sizeof(real));
  o->M = (real*)calloc((size_t)na * o->ncoef, sizeof(real));
  o->L = (real*)calloc((size_t)na * o->ncoef, sizeof(real));
  for (int c = 0; c < nc; c++) {
    const int f = nc - 1 - c;
    o->ichild[f] = (nc - 1 - ch0[c]) - nch[c] + 1;
    o->iparent[f] = nc - 1 - par[c];
    o->nchild[f] = nch[c];
    o->cibody[f] = fb[c];
    o->cnbody[f] = nb[c];
    o->clevel[f] = lev[c];
    o->icell[f] = ic[c];
    for (int k = 0; k < 3; k++) o->cX[3 * f + k] = X[3 * c + k];
    o->R[f] = R[c];
  }
  o->nc = nc;
  o->maxlevel = level;
  memcpy(o->Rbuilt, o->R, sizeof(real) * nc);
  /* the root box the upward pass and the traversal never read; kept for get_box */
  free(fb); free(nb); free(ch0); free(nch); free(par); free(lev); free(ic); free(X); free(R);
  free(key);
  return 0;
}

/* ------------------------------------------------------------------ spherical harmonics */
/* cart2sph (kernels/LaplaceSphericalCPU.cxx:9-13) */
static void cart2sph(real* r, real* theta, real* phi, const real dX[3]) {
  *r = sqrt(dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2]);
  *theta = *r == 0 ? 0 : acos(dX[2] / *r);
  *phi = atan2(dX[1], dX[0]);
}

/* evalMultipole (kernels/LaplaceSphericalCPU.cxx:29-65): r^n Y_n^m / (n+|m|)! style solid
 * harmonics at index n*n+n+m, plus their theta derivatives. */
static void eval_multipole(int P, real rho, real alpha, real beta, cplx* Ynm, cplx* YnmTheta) {
  real x = cos(alpha), y = sin(alpha);
  real fact = 1, pn = 1, rhom = 1;
  cplx ei = cx(cos(beta), sin(beta)), eim = cx(1, 0);
  for (int m = 0; m < P; m++) {
    real p = pn;
    int npn = m * m + 2 * m, nmn = m * m;
    Ynm[npn] = cscale(eim, rhom * p);
    Ynm[nmn] = cconj(Ynm[npn]);
    real p1 = p;
    p = x * (2 * m + 1) * p1;
    if (YnmTheta) YnmTheta[npn] = cscale(eim, rhom * (p - (m + 1) * x * p1) / y);
    rhom *= rho;
    real rhon = rhom;
    for (int n = m + 1; n < P; n++) {
      int npm = n * n + n + m, nmm = n * n + n - m;
      rhon /= -(n + m);
      Ynm[npm] = cscale(eim, rhon * p);
      Ynm[nmm] = cconj(Ynm[npm]);
      real p2 = p1;
      p1 = p;
      p = (x * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      if (YnmTheta) YnmTheta[npm] = cscale(eim, rhon * ((n - m + 1) * p - (n + 1) * x * p1) / y);
      rhon *= rho;
    }
    rhom /= -(2 * m + 2) * (2 * m + 1);
    pn = -pn * fact * y;
    fact += 2;
    eim = cmul(eim, ei);
  }
}

/* evalLocal (kernels/LaplaceSphericalCPU.cxx:68-101): singular harmonics r^(-n-1) Y_n^m */
static void eval_local(int P, real rho, real alpha, real beta, cplx* Ynm) {
  real x = cos(alpha), y = sin(alpha);
  real fact = 1, pn = 1;
  real invR = -1.0 / rho;
  real rhom = -invR;
  cplx ei = cx(cos(beta), sin(beta)), eim = cx(1, 0);
  for (int m = 0; m < P; m++) {
    real p = pn;
    int npn = m * m + 2 * m, nmn = m * m;
    Ynm[npn] = cscale(eim, rhom * p);
    Ynm[nmn] = cconj(Ynm[npn]);
    real p1 = p;
    p = x * (2 * m + 1) * p1;
    rhom *= invR;
    real rhon = rhom;
    for (int n = m + 1; n < P; n++) {
      int npm = n * n + n + m, nmm = n * n + n - m;
      Ynm[npm] = cscale(eim, rhon * p);
      Ynm[nmm] = cconj(Ynm[npm]);
      real p2 = p1;
      p1 = p;
      p = (x * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      rhon *= invR * (n - m + 1);
    }
    pn = -pn * fact * y;
    fact += 2;
    eim = cmul(eim, ei);
  }
}

#define CM(o, c) ((cplx*)&(o)->M[(size_t)(c) * (o)->ncoef])
#define CL(o, c) ((cplx*)&(o)->L[(size_t)(c) * (o)->ncoef])

/* P2M spherical (kernels/LaplaceSphericalCPU.cxx:103-118) */
static void sph_p2m(Oracle* o, int c) {
  int P = o->p.P;
  cplx Ynm[P * P], YnmTheta[P * P];
  cplx* M = CM(o, c);
  for (int b = o->cibody[c]; b < o->cibody[c] + o->cnbody[c]; b++) {
    real dX[3];
    for (int d = 0; d < 3; d++) dX[d] = o->x[3 * b + d] - o->cX[3 * c + d];
    real rho, alpha, beta;
    cart2sph(&rho, &alpha, &beta, dX);
    eval_multipole(P, rho, alpha, beta, Ynm, YnmTheta);
    for (int n = 0; n < P; n++)
      for (int m = 0; m <= n; m++) {
        int nm = n * n + n - m, nms = n * (n + 1) / 2 + m;
        M[nms] = cadd(M[nms], cscale(Ynm[nm], o->q[b]));
      }
  }
}

/* M2M spherical (kernels/LaplaceSphericalCPU.cxx:120-147) */
static void sph_m2m(Oracle* o, int ci) {
  int P = o->p.P;
  cplx Ynm[P * P], YnmTheta[P * P];
  cplx* Mi = CM(o, ci);
  for (int cj = o->ichild[ci]; cj < o->ichild[ci] + o->nchild[ci]; cj++) {
    cplx* Mj = CM(o, cj);
    real dX[3];
    for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - o->cX[3 * cj + d];
    real rho, alpha, beta;
    cart2sph(&rho, &alpha, &beta, dX);
    eval_multipole(P, rho, alpha, beta, Ynm, YnmTheta);
    for (int j = 0; j < P; j++)
      for (int k = 0; k <= j; k++) {
        int jks = j * (j + 1) / 2 + k;
        cplx M = cx(0, 0);
        for (int n = 0; n <= j; n++) {
          int mlo = -n > -j + k + n ? -n : -j + k + n;
          int mhi = k - 1 < n ? k - 1 : n;
          for (int m = mlo; m <= mhi; m++) {
            int jnkms = (j - n) * (j - n + 1) / 2 + k - m;
            int nm = n * n + n - m;
            M = cadd(M, cscale(cmul(Mj[jnkms], Ynm[nm]), (real)(IPOW2N(m) * ODDEVEN(n))));
          }
          int mhi2 = n < j + k - n ? n : j + k - n;
          for (int m = k; m <= mhi2; m++) {
            int jnkms = (j - n) * (j - n + 1) / 2 - k + m;
            int nm = n * n + n - m;
            M = cadd(M, cscale(cmul(cconj(Mj[jnkms]), Ynm[nm]), (real)ODDEVEN(k + n + m)));
          }
        }
        Mi[jks] = cadd(Mi[jks], M);
      }
  }
}

/* M2L spherical, non-mutual (kernels/LaplaceSphericalCPU.cxx:149-191) */
static void sph_m2l2(Oracle* o, int ci, Oracle* oj, int cj) {
  int P = o->p.P;
  cplx Ynmi[P * P];
  cplx *Mi = CM(o, ci), *Mj = CM(oj, cj), *Li = CL(o, ci);
  real dX[3];
  for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - oj->cX[3 * cj + d] - o->xp[d];
  real rho, alpha, beta;
  cart2sph(&rho, &alpha, &beta, dX);
  eval_local(P, rho, alpha, beta, Ynmi);
  for (int j = 0; j < P; j++) {
    real Cnm = o->p.mass ? cmul(Mi[0], Mj[0]).re * ODDEVEN(j) : (real)ODDEVEN(j);
    for (int k = 0; k <= j; k++) {
      int jks = j * (j + 1) / 2 + k;
      cplx L = cx(0, 0);
      int n0 = 0;
      if (o->p.mass) {
        int jk = j * j + j - k;
        L = cadd(L, cscale(Ynmi[jk], Cnm));
        n0 = 1;
      }
      for (int n = n0; n < P - j; n++) {
        for (int m = -n; m < 0; m++) {
          int nms = n * (n + 1) / 2 - m;
          int jnkm = (j + n) * (j + n) + j + n + m - k;
          L = cadd(L, cmul(cscale(cconj(Mj[nms]), Cnm), Ynmi[jnkm]));
        }
        for (int m = 0; m <= n; m++) {
          int nms = n * (n + 1) / 2 + m;
          int jnkm = (j + n) * (j + n) + j + n + m - k;
          real Cnm2 = Cnm * ODDEVEN((k - m) * (k < m) + m);
          L = cadd(L, cmul(cscale(Mj[nms], Cnm2), Ynmi[jnkm]));
        }
      }
      Li[jks] = cadd(Li[jks], L);
    }
  }
}

static void sph_m2l(Oracle* o, int ci, int cj) { sph_m2l2(o, ci, o, cj); }

/* L2L spherical (kernels/LaplaceSphericalCPU.cxx:193-224) */
static void sph_l2l(Oracle* o, int ci) {
  int P = o->p.P;
  cplx Ynm[P * P], YnmTheta[P * P];
  int cj = o->iparent[ci];
  cplx *Lj = CL(o, cj), *Li = CL(o, ci);
  real dX[3];
  for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - o->cX[3 * cj + d];
  real rho, alpha, beta;
  cart2sph(&rho, &alpha, &beta, dX);
  eval_multipole(P, rho, alpha, beta, Ynm, YnmTheta);
  if (o->p.mass) {
    /* Ci->L /= Ci->M[0] with complex division by a real-valued M[0] */
    cplx m0 = CM(o, ci)[0];
    for (int i = 0; i < o->nterm; i++) Li[i] = cdivm(Li[i], m0);
  }
  for (int j = 0; j < P; j++)
    for (int k = 0; k <= j; k++) {
      int jks = j * (j + 1) / 2 + k;
      cplx L = cx(0, 0);
      for (int n = j; n < P; n++) {
        for (int m = j + k - n; m < 0; m++) {
          int jnkm = (n - j) * (n - j) + n - j + m - k;
          int nms = n * (n + 1) / 2 - m;
          L = cadd(L, cscale(cmul(cconj(Lj[nms]), Ynm[jnkm]), (real)ODDEVEN(k)));
        }
        for (int m = 0; m <= n; m++) {
          if (n - j >= abs(m - k)) {
            int jnkm = (n - j) * (n - j) + n - j + m - k;
            int nms = n * (n + 1) / 2 + m;
            L = cadd(L, cscale(cmul(Lj[nms], Ynm[jnkm]), (real)ODDEVEN((m - k) * (m < k))));
          }
        }
      }
      Li[jks] = cadd(Li[jks], L);
    }
}

static inline real trg_get(Oracle* o, int b, int d) {
  return o->p.kahan ? o->ktrg[4 * b + d].s + o->ktrg[4 * b + d].c : o->trg[4 * b + d];
}
static inline void trg_add(Oracle* o, int b, int d, real v) {
  if (o->p.kahan) kadd(&o->ktrg[4 * b + d], v);
  else o->trg[4 * b + d] += v;
}
/* TRG /= SRC (kvec4 /= real: kahan operator/= divides s and c, include/kahan.h:57-61) */
static inline void trg_div(Oracle* o, int b, real s) {
  for (int d = 0; d < 4; d++) {
    if (o->p.kahan) {
      o->ktrg[4 * b + d].c /= s;
      o->ktrg[4 * b + d].s /= s;
    } else {
      o->trg[4 * b + d] /= s;
    }
  }
}

/* L2P spherical (kernels/LaplaceSphericalCPU.cxx:226-256) */
static void sph_l2p(Oracle* o, int ci) {
  int P = o->p.P;
  cplx Ynm[P * P], YnmTheta[P * P];
  cplx* L = CL(o, ci);
  for (int b = o->cibody[ci]; b < o->cibody[ci] + o->cnbody[ci]; b++) {
    real dX[3], sph[3] = {0, 0, 0}, cart[3];
    for (int d = 0; d < 3; d++) dX[d] = o->x[3 * b + d] - o->cX[3 * ci + d];
    real r, theta, phi;
    cart2sph(&r, &theta, &phi, dX);
    eval_multipole(P, r, theta, phi, Ynm, YnmTheta);
    trg_div(o, b, o->q[b]);
    for (int n = 0; n < P; n++) {
      int nm = n * n + n, nms = n * (n + 1) / 2;
      trg_add(o, b, 0, cmul(L[nms], Ynm[nm]).re);
      sph[0] += cmul(L[nms], Ynm[nm]).re / r * n;
      sph[1] += cmul(L[nms], YnmTheta[nm]).re;
      for (int m = 1; m <= n; m++) {
        nm = n * n + n + m;
        nms = n * (n + 1) / 2 + m;
        trg_add(o, b, 0, 2 * cmul(L[nms], Ynm[nm]).re);
        sph[0] += 2 * cmul(L[nms], Ynm[nm]).re / r * n;
        sph[1] += 2 * cmul(L[nms], YnmTheta[nm]).re;
        sph[2] += 2 * cmul(cmul(L[nms], Ynm[nm]), cx(0, 1)).re * m;
      }
    }
    /* sph2cart (kernels/LaplaceSphericalCPU.cxx:17-26) */
    cart[0] = sin(theta) * cos(phi) * sph[0] + cos(theta) * cos(phi) / r * sph[1] -
              sin(phi) / r / sin(theta) * sph[2];
    cart[1] = sin(theta) * sin(phi) * sph[0] + cos(theta) * sin(phi) / r * sph[1] +
              cos(phi) / r / sin(theta) * sph[2];
    cart[2] = cos(theta) * sph[0] - sin(theta) / r * sph[1];
    for (int d = 0; d < 3; d++) trg_add(o, b, d + 1, cart[d]);
  }
}

/* ------------------------------------------------------------------ Cartesian Taylor */
/* Kernels::power (kernels/LaplaceCartesianCPU.cxx:171-174,204-207,237-240):
 * C[k] = C[k - e_d] * dX[d] / k_d with d the last nonzero component of k. */
static void cart_power(const Oracle* o, real* C, const real dX[3]) {
  for (int t = 1; t < o->nterm; t++) {
    int nx = o->cmi[3 * t], ny = o->cmi[3 * t + 1], nz = o->cmi[3 * t + 2];
    if (nz > 0) C[t] = C[CI(o, nx, ny, nz - 1)] * dX[2] / nz;
    else if (ny > 0) C[t] = C[CI(o, nx, ny - 1, 0)] * dX[1] / ny;
    else C[t] = C[CI(o, nx - 1, 0, 0)] * dX[0] / nx;
  }
}

/* getCoef (kernels/LaplaceCartesianCPU.cxx:280-285) with Kernels::derivative (:175-179)
 * and DerivativeSum/DerivativeTerm (:28-106): the Taylor coefficients of 1/r by the
 * recurrence n r^2 a_k = (1-2n) sum_d x_d a_{k-e_d} + (1-n) sum_d a_{k-2e_d}, then
 * Kernels::scale (:180-183) multiplies by nx! ny! nz!. */
static void cart_coef(const Oracle* o, real* C, const real dX[3], real invR2, real invR) {
  C[0] = invR;
  for (int t = 1; t < o->nterm; t++) {
    int k[3] = {o->cmi[3 * t], o->cmi[3 * t + 1], o->cmi[3 * t + 2]};
    int n = k[0] + k[1] + k[2];
    real s = 0;
    for (int d = 2; d >= 0; d--) {
      if (k[d] >= 1) {
        int km[3] = {k[0], k[1], k[2]};
        km[d] -= 1;
        s += (1 - 2 * n) * dX[d] * C[CI(o, km[0], km[1], km[2])];
      }
      if (k[d] >= 2) {
        int km[3] = {k[0], k[1], k[2]};
        km[d] -= 2;
        s += (1 - n) * C[CI(o, km[0], km[1], km[2])];
      }
    }
    C[t] = s / n * invR2;
  }
  for (int t = 1; t < o->nterm; t++) {
    unsigned long long F = 1;
    for (int d = 0; d < 3; d++)
      for (int i = 2; i <= o->cmi[3 * t + d]; i++) F *= i;
    C[t] *= (real)F;
  }
}

/* P2M Cartesian (kernels/LaplaceCartesianCPU.cxx:635-643) */
static void cart_p2m(Oracle* o, int c) {
  real C[o->nterm];
  real* M = &o->M[(size_t)c * o->ncoef];
  for (int b = o->cibody[c]; b < o->cibody[c] + o->cnbody[c]; b++) {
    real dX[3];
    for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * c + d] - o->x[3 * b + d];
    C[0] = o->q[b];
    cart_power(o, C, dX);
    for (int i = 0; i < o->nterm; i++) M[i] += C[i];
  }
}

/* M2M Cartesian (kernels/LaplaceCartesianCPU.cxx:645-656, MultipoleSum :109-136) */
static void cart_m2m(Oracle* o, int ci) {
  real C[o->nterm];
  real* Mi = &o->M[(size_t)ci * o->ncoef];
  for (int cj = o->ichild[ci]; cj < o->ichild[ci] + o->nchild[ci]; cj++) {
    real* Mj = &o->M[(size_t)cj * o->ncoef];
    real dX[3];
    for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - o->cX[3 * cj + d];
    C[0] = 1;
    cart_power(o, C, dX);
    for (int i = 0; i < o->nterm; i++) Mi[i] += C[i] * Mj[0];
    for (int t = 1; t < o->nterm; t++) {
      int n[3] = {o->cmi[3 * t], o->cmi[3 * t + 1], o->cmi[3 * t + 2]};
      real s = 0;
      for (int kx = 0; kx <= n[0]; kx++)
        for (int ky = 0; ky <= n[1]; ky++)
          for (int kz = 0; kz <= n[2]; kz++) {
            if (kx + ky + kz == 0) continue;
            s += C[CI(o, n[0] - kx, n[1] - ky, n[2] - kz)] * Mj[CI(o, kx, ky, kz)];
          }
      Mi[t] += s;
    }
  }
}

/* M2L Cartesian, non-mutual (kernels/LaplaceCartesianCPU.cxx:658-673; sumM2L :442-451,
 * LocalSum :139-166): L_n += sum_{|n|+|k|<=P-1} M_k C_{n+k}. */
static void cart_m2l2(Oracle* o, int ci, Oracle* oj, int cj) {
  int P = o->p.P;
  real C[o->nterm];
  real *Mi = &o->M[(size_t)ci * o->ncoef], *Mj = &oj->M[(size_t)cj * o->ncoef];
  real* Li = &o->L[(size_t)ci * o->ncoef];
  real dX[3];
  for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - oj->cX[3 * cj + d] - o->xp[d];
  real invR2 = 1 / (dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2]);
  real invR = o->p.mass ? Mi[0] * Mj[0] * sqrt(invR2) : sqrt(invR2);
  cart_coef(o, C, dX, invR2, invR);
  for (int i = 0; i < o->nterm; i++) Li[i] += o->p.mass ? C[i] : Mj[0] * C[i];
  /* The unrolled sumM2L<1..6> (:453-610), used whenever P <= 7, add to L[0] only the
   * multipole terms of order <= P-2; the generic sumM2L (:442-451) adds them all. */
  int l0max = P <= 7 ? P - 2 : P - 1;
  for (int i = 1; i < o->nterm; i++) {
    int ok = o->cmi[3 * i] + o->cmi[3 * i + 1] + o->cmi[3 * i + 2];
    if (ok <= l0max) Li[0] += Mj[i] * C[i];
  }
  for (int t = 1; t < o->nterm; t++) {
    int n[3] = {o->cmi[3 * t], o->cmi[3 * t + 1], o->cmi[3 * t + 2]};
    int on = n[0] + n[1] + n[2];
    if (on > P - 2) continue;
    real s = 0;
    for (int u = 1; u < o->nterm; u++) {
      int k[3] = {o->cmi[3 * u], o->cmi[3 * u + 1], o->cmi[3 * u + 2]};
      if (on + k[0] + k[1] + k[2] > P - 1) continue;
      s += Mj[u] * C[CI(o, n[0] + k[0], n[1] + k[1], n[2] + k[2])];
    }
    Li[t] += s;
  }
}

static void cart_m2l(Oracle* o, int ci, int cj) { cart_m2l2(o, ci, o, cj); }

/* L2L Cartesian (kernels/LaplaceCartesianCPU.cxx:675-687) */
static void cart_l2l(Oracle* o, int ci) {
  int P = o->p.P;
  real C[o->nterm];
  int cj = o->iparent[ci];
  real *Lj = &o->L[(size_t)cj * o->ncoef], *Li = &o->L[(size_t)ci * o->ncoef];
  real dX[3];
  for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - o->cX[3 * cj + d];
  C[0] = 1;
  cart_power(o, C, dX);
  if (o->p.mass) {
    real m0 = o->M[(size_t)ci * o->ncoef];
    for (int i = 0; i < o->nterm; i++) Li[i] /= m0;
  }
  for (int i = 0; i < o->nterm; i++) Li[i] += Lj[i];
  for (int i = 1; i < o->nterm; i++) Li[0] += C[i] * Lj[i];
  for (int t = 1; t < o->nterm; t++) {
    int n[3] = {o->cmi[3 * t], o->cmi[3 * t + 1], o->cmi[3 * t + 2]};
    int on = n[0] + n[1] + n[2];
    real s = 0;
    for (int u = 1; u < o->nterm; u++) {
      int k[3] = {o->cmi[3 * u], o->cmi[3 * u + 1], o->cmi[3 * u + 2]};
      if (on + k[0] + k[1] + k[2] > P - 1) continue;
      s += C[u] * Lj[CI(o, n[0] + k[0], n[1] + k[1], n[2] + k[2])];
    }
    Li[t] += s;
  }
}

/* L2P Cartesian (kernels/LaplaceCartesianCPU.cxx:689-704) */
static void cart_l2p(Oracle* o, int ci) {
  int P = o->p.P;
  real C[o->nterm];
  real* L = &o->L[(size_t)ci * o->ncoef];
  for (int b = o->cibody[ci]; b < o->cibody[ci] + o->cnbody[ci]; b++) {
    real dX[3];
    for (int d = 0; d < 3; d++) dX[d] = o->x[3 * b + d] - o->cX[3 * ci + d];
    C[0] = 1;
    cart_power(o, C, dX);
    trg_div(o, b, o->q[b]);
    for (int d = 0; d < 4; d++) trg_add(o, b, d, L[d]);
    real s0 = 0;
    for (int i = 1; i < o->nterm; i++) s0 += C[i] * L[i];
    trg_add(o, b, 0, s0);
    for (int d = 0; d < 3; d++) {
      int e[3] = {0, 0, 0};
      e[d] = 1;
      real s = 0;
      for (int u = 1; u < o->nterm; u++) {
        int k[3] = {o->cmi[3 * u], o->cmi[3 * u + 1], o->cmi[3 * u + 2]};
        if (k[0] + k[1] + k[2] > P - 2) continue;
        s += C[u] * L[CI(o, e[0] + k[0], e[1] + k[1], e[2] + k[2])];
      }
      trg_add(o, b, d + 1, s);
    }
  }
}

/* ------------------------------------------------------------------ P2P */
/* P2P between cells, non-mutual (kernels/LaplaceP2PCPU.cxx:141-169, the scalar form of the
 * SIMD loop :10-139): TRG_i += q_i q_j / r, grad -= q_i q_j (x_i - x_j) / r^3. */
static void p2p_pair2(Oracle* o, int ci, Oracle* oj, int cj) {
  for (int i = o->cibody[ci]; i < o->cibody[ci] + o->cnbody[ci]; i++) {
    kreal pot = {0, 0}, ax = {0, 0}, ay = {0, 0}, az = {0, 0};
    real ppot = 0, pax = 0, pay = 0, paz = 0;
    for (int j = oj->cibody[cj]; j < oj->cibody[cj] + oj->cnbody[cj]; j++) {
      real dX[3];
      for (int d = 0; d < 3; d++) dX[d] = o->x[3 * i + d] - oj->x[3 * j + d] - o->xp[d];
      real R2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2] + o->eps2;
      if (R2 != 0) {
        real invR2 = 1.0 / R2;
        real invR = o->q[i] * oj->q[j] * sqrt(invR2);
        for (int d = 0; d < 3; d++) dX[d] *= invR2 * invR;
        if (o->p.kahan) {
          kadd(&pot, invR); kadd(&ax, dX[0]); kadd(&ay, dX[1]); kadd(&az, dX[2]);
        } else {
          ppot += invR; pax += dX[0]; pay += dX[1]; paz += dX[2];
        }
      }
    }
    if (o->p.kahan) {
      ppot = pot.s + pot.c; pax = ax.s + ax.c; pay = ay.s + ay.c; paz = az.s + az.c;
    }
    trg_add(o, i, 0, ppot);
    trg_add(o, i, 1, -pax);
    trg_add(o, i, 2, -pay);
    trg_add(o, i, 3, -paz);
  }
}

static void p2p_pair(Oracle* o, int ci, int cj) { p2p_pair2(o, ci, o, cj); }

/* P2P within one cell (kernels/LaplaceP2PCPU.cxx:304-330): each unordered pair once,
 * updating both bodies. */
static void p2p_self(Oracle* o, int c) {
  int b0 = o->cibody[c], n = o->cnbody[c];
  for (int i = b0; i < b0 + n; i++) {
    real pot = 0, ax = 0, ay = 0, az = 0;
    for (int j = i + 1; j < b0 + n; j++) {
      real dX[3];
      for (int d = 0; d < 3; d++) dX[d] = o->x[3 * i + d] - o->x[3 * j + d];
      real R2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2] + o->eps2;
      if (R2 != 0) {
        real invR2 = 1.0 / R2;
        real invR = o->q[i] * o->q[j] * sqrt(invR2);
        for (int d = 0; d < 3; d++) dX[d] *= invR2 * invR;
        pot += invR; ax += dX[0]; ay += dX[1]; az += dX[2];
        trg_add(o, j, 0, invR);
        trg_add(o, j, 1, dX[0]);
        trg_add(o, j, 2, dX[1]);
        trg_add(o, j, 3, dX[2]);
      }
    }
    trg_add(o, i, 0, pot);
    trg_add(o, i, 1, -ax);
    trg_add(o, i, 2, -ay);
    trg_add(o, i, 3, -az);
  }
}

/* ------------------------------------------------------------------ upward pass */
/* PostOrderTraversal (include/up_down_pass.h:45-84) with setRmax (:51-67), then the root
 * coefficient and SetRopt (:15-42, :125-129). Children always sit at higher cell indices
 * than their parent, so a reverse sweep is a post-order. */
int oracle_upward(void* h) {
  Oracle* o = (Oracle*)h;
  int P = o->p.P;
  real theta = (real)o->p.theta;
  if (o->nc == 0) return 0;
  memset(o->M, 0, sizeof(real) * (size_t)o->nc * o->ncoef);
  memset(o->L, 0, sizeof(real) * (size_t)o->nc * o->ncoef);
  for (int c = o->nc - 1; c >= 0; c--) {
    if (o->nchild[c] == 0) {
      if (o->p.basis == ORACLE_SPHERICAL) sph_p2m(o, c); else cart_p2m(o, c);
    } else {
      if (o->p.basis == ORACLE_SPHERICAL) sph_m2m(o, c); else cart_m2m(o, c);
    }
    if (o->p.use_rmax) {
      real Rmax = 0;
      if (o->nchild[c] == 0) {
        for (int b = o->cibody[c]; b < o->cibody[c] + o->cnbody[c]; b++) {
          real dX[3];
          for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * c + d] - o->x[3 * b + d];
          real R = sqrt(dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2]);
          if (R > Rmax) Rmax = R;
        }
      } else {
        for (int cc = o->ichild[c]; cc < o->ichild[c] + o->nchild[c]; cc++) {
          real dX[3];
          for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * c + d] - o->cX[3 * cc + d];
          real R = sqrt(dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2]) + o->R[cc];
          if (R > Rmax) Rmax = R;
        }
      }
      o->R[c] = o->R[c] < Rmax ? o->R[c] : Rmax;
    }
    o->R[c] /= theta;
  }
  /* |M[0]| of a real-valued complex monopole (std::abs -> hypot(re, 0)) */
  real m0root = o->M[0] < 0 ? -o->M[0] : o->M[0];
  real cc = (real)((double)((1 - theta) * (1 - theta)) / pow((double)theta, (double)(P + 2)) /
                   (double)powf((float)m0root, (float)(1.0 / 3)));
  if (o->p.use_ropt) {
    for (int c = 0; c < o->nc; c++) {
      real* M = &o->M[(size_t)c * o->ncoef];
      if (o->p.mass) {
        if (o->p.basis == ORACLE_SPHERICAL) {
          cplx* Mc = (cplx*)M;
          for (int i = 1; i < o->nterm; i++) Mc[i] = cdivm(Mc[i], Mc[0]);
        } else {
          for (int i = 1; i < o->nterm; i++) M[i] /= M[0];
        }
      }
      real x = (real)(1.0 / theta);
      real m0 = M[0] < 0 ? -M[0] : M[0];
      real a = cc * (real)powf((float)m0, (float)(1.0 / 3));
      for (int i = 0; i < 5; i++) {
        real f = (real)((double)(x * x - 2 * x + 1) - (double)a * pow((double)x, (double)(-P)));
        real df = (P + 2) * x - 2 * (P + 1) + P / x;
        x -= f / df;
      }
      o->R[c] *= x * theta;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ traversal */
static void push_pair(long long** a, long long* n, long long* cap, int i, int j, int img) {
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 4096;
    *a = (long long*)realloc(*a, sizeof(long long) * *cap);
  }
  (*a)[(*n)++] = ((long long)i << 32) | (long long)j | ((long long)img << 27);
}

/* target tree o, source tree oj (the same tree except for oracle_solve_ij) */
static void traverse(Oracle* o, int ci, Oracle* oj, int cj);

/* the traversal under way is mutual: one tree, open boundary, the mutual flag */
static int is_mutual(const Oracle* o, const Oracle* oj) {
  return o->p.mutual && o == oj && o->p.images == 0;
}

/* TraverseRange::operator() (include/traversal.h:81-123); mutual drops the (latter, former)
 * quarter of a range against itself, so each unordered pair is visited once */
static void traverse_range(Oracle* o, int ib, int ie, Oracle* oj, int jb, int je) {
  if (ie - ib == 1 || je - jb == 1) {
    if (ib == jb && o == oj) {
      traverse(o, ib, oj, jb);
    } else {
      for (int i = ib; i < ie; i++)
        for (int j = jb; j < je; j++) traverse(o, i, oj, j);
    }
  } else {
    int im = ib + (ie - ib) / 2, jm = jb + (je - jb) / 2;
    traverse_range(o, ib, im, oj, jb, jm);
    traverse_range(o, im, ie, oj, jm, je);
    traverse_range(o, ib, im, oj, jm, je);
    if (!is_mutual(o, oj) || ib != jb) traverse_range(o, im, ie, oj, jb, jm);
  }
}

/* splitCell (include/traversal.h:188-212) */
static void split_cell(Oracle* o, int ci, Oracle* oj, int cj) {
  if (oj->nchild[cj] == 0) {
    for (int c = o->ichild[ci]; c < o->ichild[ci] + o->nchild[ci]; c++) traverse(o, c, oj, cj);
  } else if (o->nchild[ci] == 0) {
    for (int c = oj->ichild[cj]; c < oj->ichild[cj] + oj->nchild[cj]; c++) traverse(o, ci, oj, c);
  } else if (o->cnbody[ci] + oj->cnbody[cj] >= o->p.nspawn || (is_mutual(o, oj) && ci == cj)) {
    traverse_range(o, o->ichild[ci], o->ichild[ci] + o->nchild[ci], oj, oj->ichild[cj],
                   oj->ichild[cj] + oj->nchild[cj]);
  } else if (o->R[ci] >= oj->R[cj]) {
    for (int c = o->ichild[ci]; c < o->ichild[ci] + o->nchild[ci]; c++) traverse(o, c, oj, cj);
  } else {
    for (int c = oj->ichild[cj]; c < oj->ichild[cj] + oj->nchild[cj]; c++) traverse(o, ci, oj, c);
  }
}

/* Traversal::traverse (include/traversal.h:37-62), kernels applied as pairs are visited */
static void traverse(Oracle* o, int ci, Oracle* oj, int cj) {
  real dX[3];
  for (int d = 0; d < 3; d++) dX[d] = o->cX[3 * ci + d] - oj->cX[3 * cj + d] - o->xp[d];
  real R2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2];
  real Rs = o->R[ci] + oj->R[cj];
  if (R2 > Rs * Rs) {
    push_pair(&o->m2l, &o->nm2l, &o->capm2l, ci, cj, o->img);
    if (o->p.basis == ORACLE_SPHERICAL) sph_m2l2(o, ci, oj, cj); else cart_m2l2(o, ci, oj, cj);
    if (is_mutual(o, oj)) {  /* kernel::M2L with mutual also updates Cj->L */
      if (o->p.basis == ORACLE_SPHERICAL) sph_m2l2(oj, cj, o, ci); else cart_m2l2(oj, cj, o, ci);
    }
  } else if (o->nchild[ci] == 0 && oj->nchild[cj] == 0) {
    push_pair(&o->p2p, &o->np2p, &o->capp2p, ci, cj, o->img);
    if (R2 == 0 && ci == cj && o == oj) {
      p2p_self(o, ci);
    } else {
      p2p_pair2(o, ci, oj, cj);
      if (is_mutual(o, oj)) p2p_pair2(oj, cj, o, ci);  /* kernel::P2P mutual: Cj's bodies */
    }
  } else {
    split_cell(o, ci, oj, cj);
  }
}

static int img_digit(int i) { return i < 0 ? 2 : i; }

/* Traversal::traversePeriodic (include/traversal.h:127-185) for a non-MASS build: the
 * periodic parent cell (scratch cell nc + 26, the source root's copy with the 26 scratch
 * cells nc .. nc + 25 as children) sends M2L to the target root from the 26 x 27 images
 * around the 3 x 3 x 3 block of each sub-level, then becomes the M2M of its 26 shifted
 * copies (the centre copy is not among the children, as in the reference), and the
 * period grows three times. */
static void traverse_periodic(Oracle* o) {
  const int base = o->nc, pc = o->nc + 26;
  const int nco = o->ncoef;
  for (int d = 0; d < 3; d++) o->cX[3 * pc + d] = o->cX[d];
  o->R[pc] = o->R[0];
  memcpy(&o->M[(size_t)pc * nco], &o->M[0], sizeof(real) * nco);
  o->ichild[pc] = base;
  o->nchild[pc] = 26;
  real cycle = (real)o->p.cycle;
  for (int level = 0; level < o->p.images - 1; level++) {
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++)
        for (int iz = -1; iz <= 1; iz++) {
          if (ix == 0 && iy == 0 && iz == 0) continue;
          for (int cx = -1; cx <= 1; cx++)
            for (int cy = -1; cy <= 1; cy++)
              for (int cz = -1; cz <= 1; cz++) {
                o->xp[0] = (real)(ix * 3 + cx) * cycle;
                o->xp[1] = (real)(iy * 3 + cy) * cycle;
                o->xp[2] = (real)(iz * 3 + cz) * cycle;
                if (o->p.basis == ORACLE_SPHERICAL) sph_m2l(o, 0, pc); else cart_m2l(o, 0, pc);
              }
        }
    int k = base;
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++)
        for (int iz = -1; iz <= 1; iz++) {
          if (ix == 0 && iy == 0 && iz == 0) continue;
          o->cX[3 * k] = o->cX[3 * pc] + (real)ix * cycle;
          o->cX[3 * k + 1] = o->cX[3 * pc + 1] + (real)iy * cycle;
          o->cX[3 * k + 2] = o->cX[3 * pc + 2] + (real)iz * cycle;
          memcpy(&o->M[(size_t)k * nco], &o->M[(size_t)pc * nco], sizeof(real) * nco);
          k++;
        }
    memset(&o->M[(size_t)pc * nco], 0, sizeof(real) * nco);
    if (o->p.basis == ORACLE_SPHERICAL) sph_m2m(o, pc); else cart_m2m(o, pc);
    cycle *= 3;
  }
  o->xp[0] = o->xp[1] = o->xp[2] = 0;
}

/* Traversal::dualTreeTraversal (include/traversal.h:240-264), mutual = false: from
 * (root, root) once, or for images > 0 once per shift of the source tree by
 * (ix, iy, iz) cycle, |i| <= 1, then traversePeriodic. */
int oracle_traverse(void* h) {
  Oracle* o = (Oracle*)h;
  o->nm2l = o->np2p = 0;
  o->xp[0] = o->xp[1] = o->xp[2] = 0;
  o->img = 0;
  if (o->nc == 0) return 0;
  if (o->p.images == 0) {
    traverse(o, 0, o, 0);
    return 0;
  }
  if (o->p.mass) return -1; /* the MASS normalisations of traversePeriodic are not restated */
  const real cycle = (real)o->p.cycle;
  for (int ix = -1; ix <= 1; ix++)
    for (int iy = -1; iy <= 1; iy++)
      for (int iz = -1; iz <= 1; iz++) {
        o->xp[0] = (real)ix * cycle;
        o->xp[1] = (real)iy * cycle;
        o->xp[2] = (real)iz * cycle;
        o->img = 9 * img_digit(ix) + 3 * img_digit(iy) + img_digit(iz);
        traverse(o, 0, o, 0);
      }
  o->xp[0] = o->xp[1] = o->xp[2] = 0;
  o->img = 0;
  traverse_periodic(o);
  return 0;
}

/* UpDownPass::downwardPass (include/up_down_pass.h:135-148, PreOrderTraversal :87-111):
 * parents precede children in cell order, so a forward sweep is a pre-order. */
int oracle_downward(void* h) {
  Oracle* o = (Oracle*)h;
  if (o->nc == 0) return 0;
  if (o->nchild[0] == 0) {
    if (o->p.basis == ORACLE_SPHERICAL) sph_l2p(o, 0); else cart_l2p(o, 0);
  }
  for (int c = 1; c < o->nc; c++) {
    if (o->p.basis == ORACLE_SPHERICAL) sph_l2l(o, c); else cart_l2l(o, c);
    if (o->nchild[c] == 0) {
      if (o->p.basis == ORACLE_SPHERICAL) sph_l2p(o, c); else cart_l2p(o, c);
    }
  }
  return 0;
}

/* examples/serial.cxx with IneJ (:30-55): targets hi and sources hj in two trees, on the box
 * of their common bounds (common_box; BoundBox::getBounds(jbodies, bounds),
 * include/bound_box.h:91-97) or each on its own bodies' box (wrappers/petiga.cxx:134-139),
 * both upward passes, dualTreeTraversal(cells, jcells) with mutual = false and no periodic
 * images, and the targets' downward pass.  Returns 0 on success. */
int oracle_solve_ij(void* hi, void* hj, int common_box) {
  Oracle *o = (Oracle*)hi, *oj = (Oracle*)hj;
  if (o->p.images != 0) return -1;
  if (common_box) {
    real Xmin[3], Xmax[3];
    if (o->n == 0) {
      for (int d = 0; d < 3; d++) Xmin[d] = Xmax[d] = 0;
    } else {
      for (int d = 0; d < 3; d++) Xmin[d] = Xmax[d] = o->x[d];
      update_bounds(o, Xmin, Xmax);
    }
    update_bounds(oj, Xmin, Xmax);
    bounds2box(o, Xmin, Xmax);
    bounds2box(oj, Xmin, Xmax);
  }
  o->box_fixed = oj->box_fixed = common_box != 0;
  int r = oracle_build_tree(o);
  if (!r) r = oracle_upward(o);
  if (!r) r = oracle_build_tree(oj);
  if (!r) r = oracle_upward(oj);
  if (r) return r;
  o->nm2l = o->np2p = 0;
  o->xp[0] = o->xp[1] = o->xp[2] = 0;
  o->img = 0;
  if (o->nc > 0 && oj->nc > 0) traverse(o, 0, oj, 0);
  return oracle_downward(o);
}

int oracle_solve(void* h) {
  int r = oracle_build_tree(h);
  if (!r) r = oracle_upward(h);
  if (!r) r = oracle_traverse(h);
  if (!r) r = oracle_downward(h);
  return r;
}

/* ------------------------------------------------------------------ getters */
int oracle_num_cells(void* h) { return ((Oracle*)h)->nc; }
int oracle_maxlevel(void* h) { return ((Oracle*)h)->maxlevel; }
void oracle_get_box(void* h, double* X0R0) {
  Oracle* o = (Oracle*)h;
  for (int d = 0; d < 3; d++) X0R0[d] = o->X0[d];
  X0R0[3] = o->R0;
}
void oracle_get_cells(void* h, int* iparent, int* ichild, int* nchild, int* ibody, int* nbody,
                      unsigned long long* icell, int* level, double* X, double* R_built,
                      double* R) {
  Oracle* o = (Oracle*)h;
  for (int c = 0; c < o->nc; c++) {
    iparent[c] = o->iparent[c];
    ichild[c] = o->ichild[c];
    nchild[c] = o->nchild[c];
    ibody[c] = o->cibody[c];
    nbody[c] = o->cnbody[c];
    icell[c] = o->icell[c];
    level[c] = o->clevel[c];
    for (int d = 0; d < 3; d++) X[3 * c + d] = o->cX[3 * c + d];
    R_built[c] = o->Rbuilt[c];
    R[c] = o->R[c];
  }
}
void oracle_get_order(void* h, int* ibody) {
  Oracle* o = (Oracle*)h;
  memcpy(ibody, o->ibody, sizeof(int) * o->n);
}
void oracle_get_expansion(void* h, int which, double* out) {
  Oracle* o = (Oracle*)h;
  real* src = which == 0 ? o->M : o->L;
  for (size_t i = 0; i < (size_t)o->nc * o->ncoef; i++) out[i] = src[i];
}
void oracle_get_trg(void* h, double* trg) {
  Oracle* o = (Oracle*)h;
  for (int b = 0; b < o->n; b++)
    for (int d = 0; d < 4; d++) trg[4 * o->ibody[b] + d] = trg_get(o, b, d);
}
long long oracle_num_m2l(void* h) { return ((Oracle*)h)->nm2l; }
long long oracle_num_p2p(void* h) { return ((Oracle*)h)->np2p; }
void oracle_get_m2l(void* h, long long* out) {
  Oracle* o = (Oracle*)h;
  memcpy(out, o->m2l, sizeof(long long) * o->nm2l);
}
void oracle_get_p2p(void* h, long long* out) {
  Oracle* o = (Oracle*)h;
  memcpy(out, o->p2p, sizeof(long long) * o->np2p);
}

/* ------------------------------------------------------------------ direct + verify */
void oracle_direct(int nt, const double* xt, int ns, const double* xs, const double* qs,
                   double eps2, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double pot = 0, ax = 0, ay = 0, az = 0;
    for (int j = 0; j < ns; j++) {
      double dx = xt[3 * i] - xs[3 * j], dy = xt[3 * i + 1] - xs[3 * j + 1],
             dz = xt[3 * i + 2] - xs[3 * j + 2];
      double R2 = dx * dx + dy * dy + dz * dz + eps2;
      if (R2 != 0) {
        double invR = 1.0 / sqrt(R2);
        double invR3 = qs[j] * invR * invR * invR;
        pot += qs[j] * invR;
        ax -= dx * invR3;
        ay -= dy * invR3;
        az -= dz * invR3;
      }
    }
    out[4 * i] = pot;
    out[4 * i + 1] = ax;
    out[4 * i + 2] = ay;
    out[4 * i + 3] = az;
  }
}

void oracle_direct_periodic(int nt, const double* xt, int ns, const double* xs,
                            const double* qs, double eps2, int images, double cycle,
                            double* out) {
  int prange = 0;
  for (int i = 0, p3 = 1; i < images; i++, p3 *= 3) prange += p3;
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nt; i++) {
    double pot = 0, ax = 0, ay = 0, az = 0;
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++)
        for (int iz = -prange; iz <= prange; iz++)
          for (int j = 0; j < ns; j++) {
            double dx = xt[3 * i] - xs[3 * j] - ix * cycle;
            double dy = xt[3 * i + 1] - xs[3 * j + 1] - iy * cycle;
            double dz = xt[3 * i + 2] - xs[3 * j + 2] - iz * cycle;
            double R2 = dx * dx + dy * dy + dz * dz + eps2;
            if (R2 != 0) {
              double invR = 1.0 / sqrt(R2);
              double invR3 = qs[j] * invR * invR * invR;
              pot += qs[j] * invR;
              ax -= dx * invR3;
              ay -= dy * invR3;
              az -= dz * invR3;
            }
          }
    out[4 * i] = pot;
    out[4 * i + 1] = ax;
    out[4 * i + 2] = ay;
    out[4 * i + 3] = az;
  }
}

void oracle_rel_l2(int n, const double* trg, const double* ref, double* pot_acc) {
  double pd = 0, pn = 0, ad = 0, an = 0;
  for (int i = 0; i < n; i++) {
    double e = trg[4 * i] - ref[4 * i];
    pd += e * e;
    pn += ref[4 * i] * ref[4 * i];
    for (int d = 1; d < 4; d++) {
      double f = trg[4 * i + d] - ref[4 * i + d];
      ad += f * f;
      an += ref[4 * i + d] * ref[4 * i + d];
    }
  }
  pot_acc[0] = sqrt(pd / pn);
  pot_acc[1] = sqrt(ad / an);
}

/* ------------------------------------------------------------------ kernel chain KAT */
/* examples/kernel.cxx:5-93: P2M -> M2M -> M2L -> L2L -> L2P against P2P on a fixed
 * geometry (theta = 0.5, unit boxes), 16 sources and 16 targets from drand48. */
double oracle_kernel_chain(int basis, int P, int mass, long seed) {
  if (seed >= 0) {
    srand48(seed);
  } else {
    unsigned short x0[3] = {0, 0, 0};
    seed48(x0);
  }
  const real theta = 0.5;
  const real R = 2 / theta;
  double xs[48], qs[16], xt[48], qt[16];
  for (int b = 0; b < 16; b++) {
    xs[3 * b] = (real)(2 * drand48());
    xs[3 * b + 1] = (real)(2 * drand48());
    xs[3 * b + 2] = (real)(2 * drand48());
    qs[b] = (real)drand48();
  }
  for (int b = 0; b < 16; b++) {
    xt[3 * b] = (real)(R + 2 + 2 * drand48());
    xt[3 * b + 1] = (real)(R + 2 + 2 * drand48());
    xt[3 * b + 2] = (real)(R + 2 + 2 * drand48());
    qt[b] = (real)drand48();
  }
  /* cells: 0 = Cj (sources, centre 1), 1 = CJ (parent, centre 0), 2 = CI (centre R+4),
   * 3 = Ci (child of CI, centre R+3); bodies 0..15 sources, 16..31 targets */
  double xall[96], qall[32];
  memcpy(xall, xs, sizeof(xs));
  memcpy(xall + 48, xt, sizeof(xt));
  memcpy(qall, qs, sizeof(qs));
  memcpy(qall + 16, qt, sizeof(qt));
  oracle_params prm = {basis, P, 0.5, 16, 1000, 0, 0, mass, 0, 0.0};
  Oracle* o = (Oracle*)oracle_new(32, xall, qall, &prm);
  o->nc = 4;
  o->iparent = (int*)calloc(4, sizeof(int));
  o->ichild = (int*)calloc(4, sizeof(int));
  o->nchild = (int*)calloc(4, sizeof(int));
  o->cibody = (int*)calloc(4, sizeof(int));
  o->cnbody = (int*)calloc(4, sizeof(int));
  o->cX = (real*)calloc(12, sizeof(real));
  o->M = (real*)calloc(4 * o->ncoef, sizeof(real));
  o->L = (real*)calloc(4 * o->ncoef, sizeof(real));
  real cen[4] = {1, 0, R + 4, R + 3};
  for (int c = 0; c < 4; c++)
    for (int d = 0; d < 3; d++) o->cX[3 * c + d] = cen[c];
  o->cibody[0] = 0; o->cnbody[0] = 16;
  o->cibody[3] = 16; o->cnbody[3] = 16;
  o->ichild[1] = 0; o->nchild[1] = 1;
  o->iparent[3] = 2;
  if (basis == ORACLE_SPHERICAL) sph_p2m(o, 0); else cart_p2m(o, 0);
  if (basis == ORACLE_SPHERICAL) sph_m2m(o, 1); else cart_m2m(o, 1);
  /* CI->M = 1, Ci->M = 1 (every coefficient; a complex 1 for the spherical basis) */
  for (int c = 2; c < 4; c++)
    for (int i = 0; i < o->nterm; i++) {
      if (basis == ORACLE_SPHERICAL) {
        CM(o, c)[i] = cx(1, 0);
      } else {
        o->M[(size_t)c * o->ncoef + i] = 1;
      }
    }
  if (mass) {
    if (basis == ORACLE_SPHERICAL) {
      cplx* Mc = CM(o, 1);
      for (int i = 1; i < o->nterm; i++) Mc[i] = cdivm(Mc[i], Mc[0]);
    } else {
      real* M1 = &o->M[o->ncoef];
      for (int i = 1; i < o->nterm; i++) M1[i] /= M1[0];
    }
  }
  if (basis == ORACLE_SPHERICAL) sph_m2l(o, 2, 1); else cart_m2l(o, 2, 1);
  if (basis == ORACLE_SPHERICAL) sph_l2l(o, 3); else cart_l2l(o, 3);
  if (basis == ORACLE_SPHERICAL) sph_l2p(o, 3); else cart_l2p(o, 3);
  double fmm[16];
  for (int b = 0; b < 16; b++) fmm[b] = trg_get(o, 16 + b, 0);
  /* direct: P2P(Ci, Cj) then TRG /= SRC (kernel.cxx:74-80) */
  for (int b = 0; b < 16; b++)
    for (int d = 0; d < 4; d++) o->trg[4 * (16 + b) + d] = 0;
  p2p_pair(o, 3, 0);
  double diff = 0, norm = 0;
  for (int b = 0; b < 16; b++) {
    double dir = trg_get(o, 16 + b, 0) / o->q[16 + b];
    diff += (fmm[b] - dir) * (fmm[b] - dir);
    norm += dir * dir;
  }
  oracle_free(o);
  return sqrt(diff / norm);
}

/* ------------------------------------------------------------------ single operators */
/* One kernel::P2M / M2M / M2L / L2L / L2P application (include/kernel.h:6-14) on cells set
 * up by hand, as examples/kernel.cxx does; expansions as ncoef doubles, accumulating into
 * the output.  Unnormalised (non-MASS) multipoles. */
static Oracle* op_setup(int basis, int P, int nb, const double* xq) {
  double zx[3] = {0, 0, 0}, zq[1] = {1};
  double* x = nb ? (double*)malloc(sizeof(double) * 3 * nb) : zx;
  double* q = nb ? (double*)malloc(sizeof(double) * nb) : zq;
  for (int b = 0; b < nb; b++) {
    for (int d = 0; d < 3; d++) x[3 * b + d] = xq[4 * b + d];
    q[b] = xq[4 * b + 3];
  }
  oracle_params prm = {.basis = basis, .P = P, .theta = 0.5, .ncrit = 16, .nspawn = 1000};
  Oracle* o = (Oracle*)oracle_new(nb, x, q, &prm);
  if (nb) { free(x); free(q); }
  o->nc = 2;
  o->iparent = (int*)calloc(2, sizeof(int));
  o->ichild = (int*)calloc(2, sizeof(int));
  o->nchild = (int*)calloc(2, sizeof(int));
  o->cibody = (int*)calloc(2, sizeof(int));
  o->cnbody = (int*)calloc(2, sizeof(int));
  o->cX = (real*)calloc(6, sizeof(real));
  o->M = (real*)calloc(2 * o->ncoef, sizeof(real));
  o->L = (real*)calloc(2 * o->ncoef, sizeof(real));
  o->cnbody[0] = nb;
  return o;
}
static void op_set(Oracle* o, int c, const double* X, const double* M, const double* L) {
  for (int d = 0; d < 3; d++) o->cX[3 * c + d] = (real)X[d];
  for (int i = 0; i < o->ncoef; i++) {
    if (M) o->M[(size_t)c * o->ncoef + i] = (real)M[i];
    if (L) o->L[(size_t)c * o->ncoef + i] = (real)L[i];
  }
}
static void op_get(Oracle* o, const real* src, double* out) {
  for (int i = 0; i < o->ncoef; i++) out[i] += src[i];
}

void oracle_op_m2l(int basis, int P, const double* Xi, const double* Xj, const double* Mj,
                   double* Li) {
  Oracle* o = op_setup(basis, P, 0, NULL);
  op_set(o, 0, Xi, NULL, NULL);
  op_set(o, 1, Xj, Mj, NULL);
  if (basis == ORACLE_SPHERICAL) sph_m2l(o, 0, 1); else cart_m2l(o, 0, 1);
  op_get(o, o->L, Li);
  oracle_free(o);
}

void oracle_op_m2m(int basis, int P, const double* Xp, const double* Xc, const double* Mc,
                   double* Mp) {
  Oracle* o = op_setup(basis, P, 0, NULL);
  op_set(o, 0, Xp, NULL, NULL);
  op_set(o, 1, Xc, Mc, NULL);
  o->ichild[0] = 1;
  o->nchild[0] = 1;
  if (basis == ORACLE_SPHERICAL) sph_m2m(o, 0); else cart_m2m(o, 0);
  op_get(o, o->M, Mp);
  oracle_free(o);
}

void oracle_op_l2l(int basis, int P, const double* Xc, const double* Xp, const double* Lp,
                   double* Lc) {
  Oracle* o = op_setup(basis, P, 0, NULL);
  op_set(o, 0, Xc, NULL, NULL);
  op_set(o, 1, Xp, NULL, Lp);
  o->iparent[0] = 1;
  if (basis == ORACLE_SPHERICAL) sph_l2l(o, 0); else cart_l2l(o, 0);
  op_get(o, o->L, Lc);
  oracle_free(o);
}

void oracle_op_p2m(int basis, int P, const double* Xc, int nb, const double* xq, double* M) {
  Oracle* o = op_setup(basis, P, nb, xq);
  op_set(o, 0, Xc, NULL, NULL);
  if (basis == ORACLE_SPHERICAL) sph_p2m(o, 0); else cart_p2m(o, 0);
  op_get(o, o->M, M);
  oracle_free(o);
}

/* potential and gradient of the local expansion L at the bodies (unit charges) */
void oracle_op_l2p(int basis, int P, const double* Xc, const double* L, int nb,
                   const double* x, double* trg) {
  double* xq = (double*)malloc(sizeof(double) * 4 * (nb ? nb : 1));
  for (int b = 0; b < nb; b++) {
    for (int d = 0; d < 3; d++) xq[4 * b + d] = x[3 * b + d];
    xq[4 * b + 3] = 1;
  }
  Oracle* o = op_setup(basis, P, nb, xq);
  free(xq);
  op_set(o, 0, Xc, NULL, L);
  if (basis == ORACLE_SPHERICAL) sph_l2p(o, 0); else cart_l2p(o, 0);
  for (int b = 0; b < nb; b++)
    for (int d = 0; d < 4; d++) trg[4 * b + d] = o->trg[4 * b + d];
  oracle_free(o);
}
