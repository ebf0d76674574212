/* exafmm_b200_petiga.h -- the PetIGA wrapper ABI of exafmm-dev (wrappers/petiga.cxx:45-316)
 * on one GPU, single rank: libexafmm_b200_petiga.so, a library of its own because its
 * FMM_Init / FMM_Partition / FMM_Finalize share their names with the gromacs wrapper's.
 *
 * Two body sets, b and v, with positions as separate x, y, z arrays and one value (charge)
 * per body.  Each interaction call sets the charges it is given and ADDS the potential per
 * unit target charge to its output:
 *   FMM_B2B(vi, vb): b on b, charges vb, into vi      (wrappers/petiga.cxx:141-170)
 *   FMM_V2B(vb, vv): v on b, charges vv, into vb      (:172-204; two trees, own boxes)
 *   FMM_B2V(vv, vb): b on v, charges vb, into vv      (:206-238; two trees, own boxes)
 *   FMM_V2V(vi, vv): v on v, charges vv, into vi      (:240-269)
 *   Direct(...):     direct sum of j on i (charges vj), into vi (:271-298; FP64 on the GPU)
 * FMM_Partition leaves the bodies where they are (one rank); FMM_BuildTree does nothing
 * (every interaction call builds its trees from the same positions).  Parameters as the
 * reference's FMM_Init (:45-92): nspawn 1000, theta 0.4, use_rmax and use_ropt on,
 * images 0, eps2 truncated to an integer, the given ncrit; spherical basis at
 * EXAFMM_B200_P (default 10) in FP32; `threads` and `verbose` are ignored. */
#ifndef EXAFMM_B200_PETIGA_H
#define EXAFMM_B200_PETIGA_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

void FMM_Init(double eps2, int ncrit, int threads, int nb, double* xb, double* yb, double* zb,
              double* vb, int nv, double* xv, double* yv, double* zv, double* vv);
void FMM_Finalize(void);
#ifdef __cplusplus
void FMM_Partition(int& nb, double* xb, double* yb, double* zb, double* vb, int& nv, double* xv,
                   double* yv, double* zv, double* vv);
#else
void FMM_Partition(int* nb, double* xb, double* yb, double* zb, double* vb, int* nv, double* xv,
                   double* yv, double* zv, double* vv);
#endif
void FMM_BuildTree(void);
void FMM_B2B(double* vi, double* vb, bool verbose);
void FMM_V2B(double* vb, double* vv, bool verbose);
void FMM_B2V(double* vv, double* vb, bool verbose);
void FMM_V2V(double* vi, double* vv, bool verbose);
void Direct(int ni, double* xi, double* yi, double* zi, double* vi, int nj, double* xj,
            double* yj, double* zj, double* vj);

#ifdef __cplusplus
}
#endif
#endif
