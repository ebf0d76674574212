// The solver handle behind the C ABI and the helpers every entry point uses to reach it:
// a handle owns one Solver<float> or Solver<double>; guarded() runs a call on the handle's
// device and turns exceptions into status codes (the message stays readable through
// fmm_b200_last_error); FMM_DISPATCH runs a body with `s` bound to the typed solver.
#pragma once
#include <cuda_runtime.h>

#include <exception>

#include "fmm_solver.cuh"

struct fmm_b200_solver {
  int precision = FMM_FP32;
  fmmb200::SolverBase* base = nullptr;
};

namespace fmmb200 {

template <typename T> Solver<T>& S(fmm_b200_solver* h) { return *static_cast<Solver<T>*>(h->base); }

template <typename F> inline int guarded(fmm_b200_solver* h, F&& f) {
  if (!h || !h->base) return FMM_ERR_INVALID;
  try {
    FMM_CUDA(cudaSetDevice(h->base->cfg.device));
    f();
    h->base->err.clear();
    return FMM_OK;
  } catch (const FmmError& e) {
    h->base->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->base->err = e.what();
    return FMM_ERR_INVALID;
  }
}

}  // namespace fmmb200

#define FMM_DISPATCH(h, ...)                                   \
  guarded(h, [&] {                                             \
    if (h->precision == FMM_FP64) {                            \
      using T = double;                                        \
      Solver<T>& s = S<T>(h);                                  \
      __VA_ARGS__;                                             \
    } else {                                                   \
      using T = float;                                         \
      Solver<T>& s = S<T>(h);                                  \
      __VA_ARGS__;                                             \
    }                                                          \
  })

