// Shared device/host definitions for the B200 Laplace FMM.
//
// Working precision T is float (FP32 expansions, compensated potential/gradient sums) or
// double (the plain FP64 path).  Bodies travel as 4-vectors (x, y, z, q); cells as
// 4-vectors (x, y, z, R); expansions as T arrays of ncoef values per cell (2 * NTERM for the
// spherical basis: (re, im) pairs; NTERM for the Cartesian basis).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/exafmm_b200.h"

namespace fmmb200 {

// Deepest level the adaptive builder splits to (3 key bits per level in a 63-bit key).
constexpr int kMaxLevel = 21;

template <typename T> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };
template <typename T> using vec4 = typename V4<T>::type;
template <typename T> struct V2;
template <> struct V2<float> { using type = float2; };
template <> struct V2<double> { using type = double2; };
template <typename T> using vec2 = typename V2<T>::type;

template <typename T> __host__ __device__ __forceinline__ vec4<T> make_v4(T a, T b, T c, T d) {
  vec4<T> v;
  v.x = a; v.y = b; v.z = c; v.w = d;
  return v;
}

// ------------------------------------------------------------------ IEEE helpers
// Geometry that decides tree structure and interaction lists is evaluated with explicitly
// rounded operations so that it matches the reference's un-fused arithmetic bit for bit.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float rsqrt_(float a) { return rsqrtf(a); }
__device__ __forceinline__ double rsqrt_(double a) { return rsqrt(a); }

// Source field of a packed list pair (target << 32 | source): the source cell in bits 0-26
// and the periodic image of the source tree in bits 27-31, coded 9 d(ix) + 3 d(iy) + d(iz)
// for a shift of (ix, iy, iz) periods with d(0) = 0, d(1) = 1, d(-1) = 2 (0: no shift).
constexpr int kImgShift = 27;
constexpr unsigned kCellMask = (1u << kImgShift) - 1;
__host__ __device__ __forceinline__ int pair_cell(unsigned src) { return (int)(src & kCellMask); }
__host__ __device__ __forceinline__ int pair_img(unsigned src) { return (int)(src >> kImgShift); }
__host__ __device__ __forceinline__ int img_code(int ix, int iy, int iz) {
  return 9 * (ix < 0 ? 2 : ix) + 3 * (iy < 0 ? 2 : iy) + (iz < 0 ? 2 : iz);
}
// shift of image code c: (ix, iy, iz) times the period (exact: |i| <= 1)
template <typename T>
__host__ __device__ __forceinline__ void img_shift(int c, T cycle, T& sx, T& sy, T& sz) {
  const int dx = c / 9, dy = (c / 3) % 3, dz = c % 3;
  sx = (T)(dx == 2 ? -1 : dx) * cycle;
  sy = (T)(dy == 2 ? -1 : dy) * cycle;
  sz = (T)(dz == 2 ? -1 : dz) * cycle;
}

// |d|^2 as ((dx*dx + dy*dy) + dz*dz) with every step rounded (vec.h norm, no fusion)
template <typename T> __device__ __forceinline__ T norm_rn(T dx, T dy, T dz) {
  return add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
}

// ------------------------------------------------------------------ compensated sums
// Two-term sum (Knuth TwoSum): value = s + e, exact representation of the running sum's
// rounding error, used to fold per-tile plain sums into the potential and gradient.
template <typename T> struct Comp {
  T s, e;
};
template <typename T> __device__ __forceinline__ void comp_add(Comp<T>& a, T v) {
  T t = add_rn(a.s, v);
  T bp = sub_rn(t, a.s);
  T err = add_rn(sub_rn(a.s, sub_rn(t, bp)), sub_rn(v, bp));
  a.s = t;
  a.e = add_rn(a.e, err);
}
template <typename T> __device__ __forceinline__ void comp_merge(Comp<T>& a, const Comp<T>& b) {
  comp_add(a, b.s);
  a.e = add_rn(a.e, b.e);
}

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// a partitioned solve (fmm_b200_set_partition): does the cell whose (NCHILD, ICHILD, NBODY,
// IBODY) record is f hold a body of the part's range [range[0], range[1])?
__device__ __forceinline__ bool part_holds(int4 f, const int* __restrict__ range) {
  return f.w < range[1] && f.w + f.z > range[0];
}

// ------------------------------------------------------------------ host error plumbing
struct FmmError : std::runtime_error {
  int code;
  FmmError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define FMM_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::fmmb200::FmmError(FMM_ERR_CUDA, std::string(#call) + ": " +             \
                                                  cudaGetErrorString(e_));            \
  } while (0)

// every kernel launch of this library is followed by FMM_LAUNCH_CHECK(): it counts the
// launch (fmm_b200_kernel_launches) and surfaces launch errors
extern std::atomic<long long> g_launches;
extern std::atomic<long long> g_device_allocs;  // cudaMalloc calls of the solvers' arrays
#define FMM_LAUNCH_CHECK()                                          \
  do {                                                              \
    ::fmmb200::g_launches.fetch_add(1, std::memory_order_relaxed);  \
    FMM_CUDA(cudaGetLastError());                                   \
  } while (0)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Spherical / Cartesian term counts (include/types.h:38-45)
__host__ __device__ constexpr int nterm_sph(int P) { return P * (P + 1) / 2; }
__host__ __device__ constexpr int nterm_cart(int P) { return P * (P + 1) * (P + 2) / 6; }

// Position of the Cartesian multi-index (nx, ny, nz) in the reference's term order
// (Index<nx,ny,nz>::I, kernels/LaplaceCartesianCPU.cxx:3-25): by total order o, then nx
// descending, then ny descending.
__host__ __device__ constexpr int cidx(int nx, int ny, int nz) {
  return (nx + ny + nz) * (nx + ny + nz + 1) * (nx + ny + nz + 2) / 6 +
         (ny + nz) * (ny + nz + 1) / 2 + nz;
}

}  // namespace fmmb200
