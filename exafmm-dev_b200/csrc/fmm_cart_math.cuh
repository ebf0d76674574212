// Cartesian Taylor-basis translation operators of the Laplace FMM, P known at compile time.
//
// Restates kernels/LaplaceCartesianCPU.cxx: terms are multi-indices k = (kx, ky, kz) of
// total order < P in the order of Index<> (:3-25); multipoles M_k = sum q (Xc - x)^k / k!
// (P2M :635-643, Kernels::power :171-174), locals L_n = sum_k M_k d^(n+k)(1/r) (M2L
// :658-673 with getCoef :280-439 and sumM2L :442-610), shifted by exact Taylor shifts
// (M2M :645-656, L2L :675-687) and evaluated with their first derivatives (L2P :689-704).
// The derivative tensor d^k(1/r) comes from the three-term recurrence
//   |k| r^2 a_k = (1 - 2|k|) sum_d x_d a_{k - e_d} + (1 - |k|) sum_d a_{k - 2 e_d},
//   d^k(1/r) = k! a_k,
// which the reference's DerivativeSum (:28-106) and its unrolled getCoef<1..6> implement.
// As in the reference's unrolled sumM2L<1..6> (used for P <= 7), the potential coefficient
// L_0 omits multipole terms of the highest order P-1 (the generic sumM2L keeps them).
#pragma once
#include <cmath>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace fmmb200 {
namespace cart {

__host__ __device__ constexpr int NT(int P) { return P * (P + 1) * (P + 2) / 6; }
__host__ __device__ constexpr int idx(int nx, int ny, int nz) {
  return (nx + ny + nz) * (nx + ny + nz + 1) * (nx + ny + nz + 2) / 6 +
         (ny + nz) * (ny + nz + 1) / 2 + nz;
}
__host__ __device__ constexpr double fact(int n) {
  double r = 1;
  for (int i = 2; i <= n; i++) r *= i;
  return r;
}

// C[k] = C[k - e_d] * dX[d] / k_d (Kernels::power), C[0] set by the caller
template <typename T, int P>
__host__ __device__ __forceinline__ void power(T* C, T dx, T dy, T dz) {
#pragma unroll
  for (int n = 1; n < P; n++)
#pragma unroll
    for (int nx = n; nx >= 0; nx--)
#pragma unroll
      for (int ny = n - nx; ny >= 0; ny--) {
        const int nz = n - nx - ny;
        if (nz > 0) C[idx(nx, ny, nz)] = C[idx(nx, ny, nz - 1)] * dz / T(nz);
        else if (ny > 0) C[idx(nx, ny, 0)] = C[idx(nx, ny - 1, 0)] * dy / T(ny);
        else C[idx(nx, 0, 0)] = C[idx(nx - 1, 0, 0)] * dx / T(nx);
      }
}

// C[k] = d^k (1/r) at dX (getCoef), C[0] = invR
template <typename T, int P>
__host__ __device__ __forceinline__ void derivs(T* C, T dx, T dy, T dz, T invR2, T invR) {
  C[0] = invR;
#pragma unroll
  for (int n = 1; n < P; n++)
#pragma unroll
    for (int nx = n; nx >= 0; nx--)
#pragma unroll
      for (int ny = n - nx; ny >= 0; ny--) {
        const int nz = n - nx - ny;
        T s = 0;
        if (nz >= 1) s += T(1 - 2 * n) * dz * C[idx(nx, ny, nz - 1)];
        if (nz >= 2) s += T(1 - n) * C[idx(nx, ny, nz - 2)];
        if (ny >= 1) s += T(1 - 2 * n) * dy * C[idx(nx, ny - 1, nz)];
        if (ny >= 2) s += T(1 - n) * C[idx(nx, ny - 2, nz)];
        if (nx >= 1) s += T(1 - 2 * n) * dx * C[idx(nx - 1, ny, nz)];
        if (nx >= 2) s += T(1 - n) * C[idx(nx - 2, ny, nz)];
        C[idx(nx, ny, nz)] = s * (T(1) / T(n)) * invR2;
      }
#pragma unroll
  for (int n = 2; n < P; n++)
#pragma unroll
    for (int nx = n; nx >= 0; nx--)
#pragma unroll
      for (int ny = n - nx; ny >= 0; ny--) {
        const int nz = n - nx - ny;
        C[idx(nx, ny, nz)] *= T(fact(nx) * fact(ny) * fact(nz));
      }
}

// L += M2L(M) for one source (sumM2L), C from derivs()
template <typename T, int P>
__host__ __device__ __forceinline__ void m2l_pair(const T* C, const T* M, T* L) {
  constexpr int l0max = P <= 7 ? P - 2 : P - 1;
#pragma unroll
  for (int n = 0; n < P; n++)
#pragma unroll
    for (int nx = n; nx >= 0; nx--)
#pragma unroll
      for (int ny = n - nx; ny >= 0; ny--) {
        const int nz = n - nx - ny;
        T s = 0;
#pragma unroll
        for (int o = 0; o + n < P; o++) {
          if (n == 0 && o > l0max) continue;
#pragma unroll
          for (int kx = o; kx >= 0; kx--)
#pragma unroll
            for (int ky = o - kx; ky >= 0; ky--) {
              const int kz = o - kx - ky;
              s += M[idx(kx, ky, kz)] * C[idx(nx + kx, ny + ky, nz + kz)];
            }
        }
        L[idx(nx, ny, nz)] += s;
      }
}

// M2M of one child into the parent's expansion: every output n of m2m_term below, the same
// terms in the same order, with compile-time indices
template <typename T, int P>
__host__ __device__ __forceinline__ void m2m_child(const T* C, const T* Mc, T* acc) {
#pragma unroll
  for (int n = 0; n < P; n++)
#pragma unroll
    for (int nx = n; nx >= 0; nx--)
#pragma unroll
      for (int ny = n - nx; ny >= 0; ny--) {
        const int nz = n - nx - ny;
        T s = 0;
#pragma unroll
        for (int kx = 0; kx <= nx; kx++)
#pragma unroll
          for (int ky = 0; ky <= ny; ky++)
#pragma unroll
            for (int kz = 0; kz <= nz; kz++)
              s += C[idx(nx - kx, ny - ky, nz - kz)] * Mc[idx(kx, ky, kz)];
        acc[idx(nx, ny, nz)] += s;
      }
}

// L2L from the parent into one child: every output n of l2l_term below, the same terms in
// the same order, with compile-time indices
template <typename T, int P>
__host__ __device__ __forceinline__ void l2l_child(const T* C, const T* Lp, T* Lc) {
#pragma unroll
  for (int n = 0; n < P; n++)
#pragma unroll
    for (int nx = n; nx >= 0; nx--)
#pragma unroll
      for (int ny = n - nx; ny >= 0; ny--) {
        const int nz = n - nx - ny;
        T s = 0;
#pragma unroll
        for (int o = 0; o + n < P; o++)
#pragma unroll
          for (int kx = o; kx >= 0; kx--)
#pragma unroll
            for (int ky = o - kx; ky >= 0; ky--) {
              const int kz = o - kx - ky;
              s += C[idx(kx, ky, kz)] * Lp[idx(nx + kx, ny + ky, nz + kz)];
            }
        Lc[idx(nx, ny, nz)] += s;
      }
}

// one M2M output term n from one child (Kernels::M2M, MultipoleSum), runtime indices
template <typename T>
__host__ __device__ __forceinline__ T m2m_term(int nx, int ny, int nz, const T* C, const T* Mc) {
  T s = 0;
  for (int kx = 0; kx <= nx; kx++)
    for (int ky = 0; ky <= ny; ky++)
      for (int kz = 0; kz <= nz; kz++) s += C[idx(nx - kx, ny - ky, nz - kz)] * Mc[idx(kx, ky, kz)];
  return s;
}

// one L2L output term n from the parent (Kernels::L2L, LocalSum), runtime indices
template <typename T>
__host__ __device__ __forceinline__ T l2l_term(int P, int nx, int ny, int nz, const T* C,
                                               const T* Lp) {
  T s = 0;
  const int n = nx + ny + nz;
  for (int o = 0; o + n < P; o++)
    for (int kx = o; kx >= 0; kx--)
      for (int ky = o - kx; ky >= 0; ky--) {
        const int kz = o - kx - ky;
        s += C[idx(kx, ky, kz)] * Lp[idx(nx + kx, ny + ky, nz + kz)];
      }
  return s;
}

// L2P of one body: potential and gradient of L at offset dX from the cell centre
template <typename T, int P>
__host__ __device__ __forceinline__ void l2p_body(T dx, T dy, T dz, const T* L, T& pot, T& gx,
                                                  T& gy, T& gz) {
  T C[NT(P)];
  C[0] = 1;
  power<T, P>(C, dx, dy, dz);
  T p = 0, x = 0, y = 0, z = 0;
#pragma unroll
  for (int o = 0; o < P; o++)
#pragma unroll
    for (int kx = o; kx >= 0; kx--)
#pragma unroll
      for (int ky = o - kx; ky >= 0; ky--) {
        const int kz = o - kx - ky;
        const T c = C[idx(kx, ky, kz)];
        p += c * L[idx(kx, ky, kz)];
        if (o + 1 < P) {
          x += c * L[idx(kx + 1, ky, kz)];
          y += c * L[idx(kx, ky + 1, kz)];
          z += c * L[idx(kx, ky, kz + 1)];
        }
      }
  pot = p;
  gx = x;
  gy = y;
  gz = z;
}

// multi-index of term t (runtime)
__host__ __device__ __forceinline__ void mi_of(int t, int& nx, int& ny, int& nz) {
  int n = 0;
  while ((n + 1) * (n + 2) * (n + 3) / 6 <= t) n++;
  int r = t - n * (n + 1) * (n + 2) / 6;  // position within order n
  int s = 0;                               // s = ny + nz
  while ((s + 1) * (s + 2) / 2 <= r) s++;
  nz = r - s * (s + 1) / 2;
  ny = s - nz;
  nx = n - s;
}

}  // namespace cart
}  // namespace fmmb200
