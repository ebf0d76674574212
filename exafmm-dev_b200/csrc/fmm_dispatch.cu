// Order dispatch of the expansion kernels.  FMM_SPH_ORDERS / FMM_CART_ORDERS (X-macro
// lists of the compiled orders) come from the Makefile, which builds one fmm_inst.cu object
// per entry.
#include "fmm_solver.cuh"

namespace fmmb200 {

#define FMM_DECL(b, p)                                  \
  void fmm_ops_##b##f##p(ExpansionOps<float>* ops);   \
  void fmm_ops_##b##d##p(ExpansionOps<double>* ops);
#define FMM_DECL_S(p) FMM_DECL(0, p)
#define FMM_DECL_C(p) FMM_DECL(1, p)
FMM_SPH_ORDERS(FMM_DECL_S)
FMM_CART_ORDERS(FMM_DECL_C)

template <> bool spherical_ops<float>(int P, ExpansionOps<float>* ops) {
  switch (P) {
#define FMM_CASE(p) case p: fmm_ops_0f##p(ops); return true;
    FMM_SPH_ORDERS(FMM_CASE)
#undef FMM_CASE
    default: return false;
  }
}
template <> bool spherical_ops<double>(int P, ExpansionOps<double>* ops) {
  switch (P) {
#define FMM_CASE(p) case p: fmm_ops_0d##p(ops); return true;
    FMM_SPH_ORDERS(FMM_CASE)
#undef FMM_CASE
    default: return false;
  }
}
template <> bool cartesian_ops<float>(int P, ExpansionOps<float>* ops) {
  switch (P) {
#define FMM_CASE(p) case p: fmm_ops_1f##p(ops); return true;
    FMM_CART_ORDERS(FMM_CASE)
#undef FMM_CASE
    default: return false;
  }
}
template <> bool cartesian_ops<double>(int P, ExpansionOps<double>* ops) {
  switch (P) {
#define FMM_CASE(p) case p: fmm_ops_1d##p(ops); return true;
    FMM_CART_ORDERS(FMM_CASE)
#undef FMM_CASE
    default: return false;
  }
}

std::vector<int> spherical_orders() {
  std::vector<int> v;
#define FMM_PUSH(p) v.push_back(p);
  FMM_SPH_ORDERS(FMM_PUSH)
  return v;
}
std::vector<int> cartesian_orders() {
  std::vector<int> v;
  FMM_CART_ORDERS(FMM_PUSH)
#undef FMM_PUSH
  return v;
}

}  // namespace fmmb200
