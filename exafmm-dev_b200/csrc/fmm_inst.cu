// One expansion-kernel instantiation: basis FMM_INST_BASIS (0 spherical, 1 Cartesian),
// precision FMM_INST_REAL, order FMM_INST_P.  The Makefile compiles this file once per
// entry of its order lists so the unrolled kernels build in parallel.
#if FMM_INST_BASIS == 0
#include "fmm_spherical.cuh"
#define FMM_INST_FILL sph_fill
#else
#include "fmm_cartesian.cuh"
#define FMM_INST_FILL cart_fill
#endif
#define FMM_CAT2(a, b, c, d) a##b##c##d
#define FMM_CAT(a, b, c, d) FMM_CAT2(a, b, c, d)

namespace fmmb200 {
void FMM_CAT(fmm_ops_, FMM_INST_BASIS, FMM_INST_TAG, FMM_INST_P)(ExpansionOps<FMM_INST_REAL>* ops) {
  FMM_INST_FILL<FMM_INST_REAL, FMM_INST_P>(ops);
}
}  // namespace fmmb200
