/* Test infrastructure only: CPU restatement of the exafmm-dev Laplace FMM hot path, used
 * as the checker for the CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it; the product never does.
 *
 * Built twice (oracle/Makefile): liboracle_f32.so (ORACLE_REAL=float) and
 * liboracle_f64.so (ORACLE_REAL=double), matching the reference's real_t
 * (include/types.h:12-18).  All geometry, expansions and accumulators use that type, as
 * the reference does, so trees and interaction lists come out bit-exact against the
 * reference compiled with the same real_t (pinned in tests/test_oracle_vs_reference.py).
 *
 * Handle-based API, all plain C types (ctypes-callable). */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_SPHERICAL = 0, ORACLE_CARTESIAN = 1 };

typedef struct oracle_params {
  int basis;      /* ORACLE_SPHERICAL / ORACLE_CARTESIAN */
  int P;          /* expansion order (include/types.h:38) */
  double theta;   /* multipole acceptance (include/up_down_pass.h:9) */
  int ncrit;      /* max bodies per leaf (include/build_tree_tbb.h:172) */
  int nspawn;     /* 2x2 split threshold (include/traversal.h:199) */
  int use_rmax;   /* include/up_down_pass.h:81 */
  int use_ropt;   /* include/up_down_pass.h:126 */
  int mass;       /* MASS semantics: normalised multipoles (up_down_pass.h:29-31) */
  int kahan;      /* compensated TRG accumulation (include/types.h:27-35) */
  double eps2;    /* softening; the reference truncates it to int (traversal.h:17) */
  int images;     /* periodic image levels (include/traversal.h:21; 0 = open boundary) */
  double cycle;   /* period of the box (Traversal::dualTreeTraversal's cycle) */
  int mutual;     /* dualTreeTraversal's mutual flag (open boundary, one tree): each
                   * unordered cell pair visited once and applied both ways */
  int tree;       /* ORACLE_TREE_ADAPTIVE: BuildTree of include/build_tree_tbb.h;
                   * ORACLE_TREE_UNIFORM: BuildTree of include/build_tree_omp.h */
} oracle_params;

enum { ORACLE_TREE_ADAPTIVE = 0, ORACLE_TREE_UNIFORM = 1 };

/* Pairs in the lists are packed (target << 32) | source | image << 27, image 0 for the
 * unshifted source and, for periodic runs, the shift (ix, iy, iz) in {-1, 0, 1}^3 coded
 * as 9 d(ix) + 3 d(iy) + d(iz) with d(0) = 0, d(1) = 1, d(-1) = 2. */

void* oracle_new(int n, const double* x, const double* q, const oracle_params* prm);
void oracle_free(void* h);
/* Stages as in examples/serial.cxx:46-60. Return 0 on success. */
int oracle_build_tree(void* h);
/* depth of the uniform tree for n bodies (include/build_tree_omp.h:218) */
int oracle_uniform_level(int n, int ncrit);
int oracle_upward(void* h);
int oracle_traverse(void* h); /* also applies M2L/P2P as the traversal visits pairs */
int oracle_downward(void* h);
int oracle_solve(void* h);    /* all of the above */
/* targets (hi) and sources (hj) in two trees (examples/serial.cxx IneJ with common_box = 1;
 * the petiga wrapper's trees on their own boxes with 0): both upward passes,
 * dualTreeTraversal(cells, jcells), the targets' downward pass */
int oracle_solve_ij(void* hi, void* hj, int common_box);

int oracle_num_cells(void* h);
int oracle_maxlevel(void* h);
void oracle_get_cells(void* h, int* iparent, int* ichild, int* nchild, int* ibody, int* nbody,
                      unsigned long long* icell, int* level, double* X, double* R_built,
                      double* R);
void oracle_get_order(void* h, int* ibody);
void oracle_get_box(void* h, double* X0R0);
void oracle_get_expansion(void* h, int which, double* out);
void oracle_get_trg(void* h, double* trg);
long long oracle_num_m2l(void* h);
long long oracle_num_p2p(void* h);
void oracle_get_m2l(void* h, long long* out);
void oracle_get_p2p(void* h, long long* out);

/* FP64 direct sum (include/traversal.h:304-337 with double accumulation): targets t (3*nt),
 * sources (3*ns positions, ns charges); out 4*nt = (phi, dphi/dx, dphi/dy, dphi/dz). */
void oracle_direct(int nt, const double* xt, int ns, const double* xs, const double* qs,
                   double eps2, double* out);
/* the same over the periodic images Traversal::direct sums (include/traversal.h:304-320):
 * shifts (ix, iy, iz) cycle with |i| <= prange = sum_{l < images} 3^l */
void oracle_direct_periodic(int nt, const double* xt, int ns, const double* xs,
                            const double* qs, double eps2, int images, double cycle,
                            double* out);
/* rel-L2 (include/verify.h:18-83): returns sqrt(sum dif^2 / sum ref^2) for pot and grad */
void oracle_rel_l2(int n, const double* trg, const double* ref, double* pot_acc);
/* examples/kernel.cxx:5-93 chain in this precision; seed < 0 = glibc unseeded drand48 */
double oracle_kernel_chain(int basis, int P, int mass, long seed);
int oracle_real_bytes(void);

/* single operators (include/kernel.h:6-14) on hand-made cells, accumulating outputs;
 * expansions as ncoef doubles (2 NTERM spherical, NTERM Cartesian), unnormalised */
void oracle_op_m2l(int basis, int P, const double* Xi, const double* Xj, const double* Mj,
                   double* Li);
void oracle_op_m2m(int basis, int P, const double* Xp, const double* Xc, const double* Mc,
                   double* Mp);
void oracle_op_l2l(int basis, int P, const double* Xc, const double* Xp, const double* Lp,
                   double* Lc);
void oracle_op_p2m(int basis, int P, const double* Xc, int nb, const double* xq, double* M);
void oracle_op_l2p(int basis, int P, const double* Xc, const double* L, int nb,
                   const double* x, double* trg);

#ifdef __cplusplus
}
#endif
#endif
