// Spherical-harmonic translation operators of the Laplace FMM, P known at compile time.
//
// Restates kernels/LaplaceSphericalCPU.cxx (evalMultipole :29-65, evalLocal :68-101,
// P2M :103-118, M2M :120-147, M2L :149-191, L2L :193-224, L2P :226-256) for the device:
//   * angles come straight from the Cartesian offset: cos(alpha) = dz / r,
//     sin(alpha) = |(dx, dy)| / r, e^(i beta) = (dx + i dy) / |(dx, dy)|, in place of the
//     reference's acos / atan2 / cos / sin round trip (same values up to rounding);
//   * harmonics are stored for m >= 0 only, Y[n, -m] = conj(Y[n, m]) (the reference keeps
//     both halves, :41-42), at index n (n + 1) / 2 + m, the layout of the expansions;
//   * the M2L sum over m < 0 and m >= 0 is folded into per-(n, |m|) terms with the signs
//     of :158-185 resolved at compile time.
// Every function is __host__ __device__ so the CPU tests run the exact device arithmetic.
#pragma once
#include <cmath>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace fmmb200 {
namespace sph {

__host__ __device__ constexpr int NT(int P) { return P * (P + 1) / 2; }
__host__ __device__ constexpr int sidx(int n, int m) { return n * (n + 1) / 2 + m; }

template <typename T> struct Angles {
  T r, x, y, cb, sb;  // |dX|, cos(alpha), sin(alpha), cos(beta), sin(beta)
};

template <typename T> __host__ __device__ __forceinline__ T hsqrt(T v) { return std::sqrt(v); }

// cart2sph (:9-13): alpha = acos(dz / r) (0 when r = 0), beta = atan2(dy, dx)
template <typename T> __host__ __device__ __forceinline__ Angles<T> angles(T dx, T dy, T dz) {
  Angles<T> a;
  T rxy2 = dx * dx + dy * dy;
  a.r = hsqrt(rxy2 + dz * dz);
  T rxy = hsqrt(rxy2);
  if (a.r > T(0)) {
    T inv = T(1) / a.r;
    a.x = dz * inv;
    a.y = rxy * inv;
  } else {
    a.x = T(1);
    a.y = T(0);
  }
  if (rxy > T(0)) {
    T inv = T(1) / rxy;
    a.cb = dx * inv;
    a.sb = dy * inv;
  } else {
    a.cb = dx < T(0) ? T(-1) : T(1);  // atan2(+-0, x) = 0 or pi
    a.sb = T(0);
  }
  return a;
}

// 1 / sqrt(v): the device's reciprocal square root (rsqrtf, rsqrt), the quotient on the host
template <typename T> __host__ __device__ __forceinline__ T hrsqrt(T v) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == 4) return rsqrtf(v);
  else return rsqrt(v);
#else
  return T(1) / std::sqrt(v);
#endif
}

// angles() for an offset of nonzero length with reciprocal square roots instead of two
// square roots and two divisions (r = r^2 / sqrt(r^2)); invr = 1 / r.  For the M2L pairs,
// whose cells are well separated.
template <typename T>
__host__ __device__ __forceinline__ Angles<T> angles_rs(T dx, T dy, T dz, T& invr) {
  Angles<T> a;
  const T rxy2 = dx * dx + dy * dy, r2 = rxy2 + dz * dz;
  invr = hrsqrt(r2);
  a.r = r2 * invr;
  a.x = dz * invr;
  if (rxy2 > T(0)) {
    const T ixy = hrsqrt(rxy2);
    a.y = rxy2 * ixy * invr;
    a.cb = dx * ixy;
    a.sb = dy * ixy;
  } else {
    a.y = T(0);
    a.cb = dx < T(0) ? T(-1) : T(1);
    a.sb = T(0);
  }
  return a;
}

// evalMultipole (:29-65) without the theta derivative: Y[n, m] = rho^n P_n^m e^(i m beta)
// / (-1)^n (n + m)!-style normalisation of the reference; its divisions by -(n + m) and
// (2m + 2)(2m + 1) are multiplications by the reciprocals here.
template <typename T, int P>
__host__ __device__ __forceinline__ void multipole(const Angles<T>& a, T rho, T* yr, T* yi) {
  T fact = 1, pn = 1, rhom = 1;
  T er = 1, ei = 0;
#pragma unroll
  for (int m = 0; m < P; m++) {
    T p = pn;
    yr[sidx(m, m)] = rhom * p * er;
    yi[sidx(m, m)] = rhom * p * ei;
    T p1 = p;
    p = a.x * (2 * m + 1) * p1;
    rhom *= rho;
    T rhon = rhom;
#pragma unroll
    for (int n = m + 1; n < P; n++) {
      rhon *= T(-1) / T(n + m);
      yr[sidx(n, m)] = rhon * p * er;
      yi[sidx(n, m)] = rhon * p * ei;
      T p2 = p1;
      p1 = p;
      p = (a.x * (2 * n + 1) * p1 - (n + m) * p2) * (T(1) / T(n - m + 1));
      rhon *= rho;
    }
    rhom *= T(-1) / T((2 * m + 2) * (2 * m + 1));
    pn = -pn * fact * a.y;
    fact += 2;
    T t = er * a.cb - ei * a.sb;
    ei = er * a.sb + ei * a.cb;
    er = t;
  }
}

// evalLocal (:68-101): singular harmonics y[n, m] = (-1)^n r^-(n+1) (n - m)! P_n^m e^(i m beta)
// with the reference's P_n^m.  Q[n] = (n - m)! P_n^m follows
//   Q[m] = P_m^m,   Q[n + 1] = (2n + 1) x Q[n] - (n + m)(n - m) Q[n - 1]
// (the reference's recurrence times (n + 1 - m)!), so each term costs one multiply and one
// fused multiply-add, and the radial factor is a table of P powers of -1/r.
template <typename T, int P>
__host__ __device__ __forceinline__ void local(const Angles<T>& a, T* yr, T* yi) {
  const T ninvr = -T(1) / a.r;
  T fact = 1, pn = 1;
  T rpm = -ninvr;  // (-1)^m / r^(m+1)
  T er = 1, ei = 0;
#pragma unroll
  for (int m = 0; m < P; m++) {
    T q = pn, qm1 = 0;  // Q[m] = P_m^m
    {
      const T t = q * rpm;
      yr[sidx(m, m)] = t * er;
      yi[sidx(m, m)] = t * ei;
    }
    T rpn = rpm;
#pragma unroll
    for (int n = m + 1; n < P; n++) {
      // Q[n] = (2n - 1) x Q[n-1] - (n - 1 + m)(n - 1 - m) Q[n-2]
      const T qn = fma(T(2 * n - 1) * a.x, q, T(-(n - 1 + m) * (n - 1 - m)) * qm1);
      qm1 = q;
      q = qn;
      rpn *= ninvr;
      const T t = q * rpn;
      yr[sidx(n, m)] = t * er;
      yi[sidx(n, m)] = t * ei;
    }
    rpm *= ninvr;
    pn = -pn * fact * a.y;
    fact += 2;
    const T tt = er * a.cb - ei * a.sb;
    ei = er * a.sb + ei * a.cb;
    er = tt;
  }
}

// M2L of one source multipole into a register local expansion (:149-191, mutual = false,
// unnormalised multipoles), for the output degrees j in [J0, J1) only (the FP32 kernel
// splits the outputs into passes).  Mj holds NT (re, im) pairs.  The loop bounds are
// compile-time after unrolling, so the whole contraction resolves to register operands.
// (re, im) of one coefficient; on the device one 8-byte (float) or 16-byte (double) load,
// for a row that starts on a multiple of 2 reals (every expansion row does: its length is
// even)
__host__ __device__ __forceinline__ void load_pair(const float* p, float& a, float& b) {
#ifdef __CUDA_ARCH__
  const float2 v = *reinterpret_cast<const float2*>(p);
  a = v.x;
  b = v.y;
#else
  a = p[0];
  b = p[1];
#endif
}
__host__ __device__ __forceinline__ void load_pair(const double* p, double& a, double& b) {
#ifdef __CUDA_ARCH__
  const double2 v = *reinterpret_cast<const double2*>(p);
  a = v.x;
  b = v.y;
#else
  a = p[0];
  b = p[1];
#endif
}

template <typename T, int P, int J0 = 0, int J1 = P>
__host__ __device__ __forceinline__ void m2l_pair(const T* yr, const T* yi, const T* Mj, T* Lr,
                                                  T* Li) {
  // Every product goes straight into its accumulator as one fused multiply-add; the signs
  // ((-1)^j of :189, (-1)^min(k, mu) of the m > 0 half, the conjugations) are compile-time
  // after unrolling and become operand negations.
#pragma unroll
  for (int n = 0; n < P - J0; n++) {
#pragma unroll
    for (int mu = 0; mu <= n; mu++) {
      T mr, mi;
      load_pair(Mj + 2 * sidx(n, mu), mr, mi);
#pragma unroll
      for (int j = J0; j < J1; j++) {
        if (j + n >= P) break;
        const int a = j + n;
        const T sr = (j & 1) ? -mr : mr, si = (j & 1) ? -mi : mi;  // (-1)^j M[n, mu]
#pragma unroll
        for (int k = 0; k <= j; k++) {
          const int t = sidx(j, k);
          if (mu == 0) {
            // M[n,0] conj(Y[a,k])
            const T ur = yr[sidx(a, k)], ui = yi[sidx(a, k)];
            Lr[t] = fma(sr, ur, Lr[t]);
            Lr[t] = fma(si, ui, Lr[t]);
            Li[t] = fma(si, ur, Li[t]);
            Li[t] = fma(-sr, ui, Li[t]);
          } else {
            // m = -mu: conj(M[n,mu] Y[a, k+mu])
            const T ur = yr[sidx(a, k + mu)], ui = yi[sidx(a, k + mu)];
            Lr[t] = fma(sr, ur, Lr[t]);
            Lr[t] = fma(-si, ui, Lr[t]);
            Li[t] = fma(-sr, ui, Li[t]);
            Li[t] = fma(-si, ur, Li[t]);
            // m = +mu: (-1)^(k < mu ? k : mu) M[n,mu] Y[a, mu-k] (conj Y[a, k-mu] if k > mu)
            const bool neg = ((k < mu ? k : mu) & 1) != 0;
            const T br = neg ? -sr : sr, bi = neg ? -si : si;
            if (mu >= k) {
              const T wr = yr[sidx(a, mu - k)], wi = yi[sidx(a, mu - k)];
              Lr[t] = fma(br, wr, Lr[t]);
              Lr[t] = fma(-bi, wi, Lr[t]);
              Li[t] = fma(br, wi, Li[t]);
              Li[t] = fma(bi, wr, Li[t]);
            } else {
              const T wr = yr[sidx(a, k - mu)], wi = yi[sidx(a, k - mu)];
              Lr[t] = fma(br, wr, Lr[t]);
              Lr[t] = fma(bi, wi, Lr[t]);
              Li[t] = fma(bi, wr, Li[t]);
              Li[t] = fma(-br, wi, Li[t]);
            }
          }
        }
      }
    }
  }
}

// The local harmonics split into a real factor and an azimuthal phase: Y[n, m] =
// rho[n, m] e^(i m beta) for m >= 0 (rho = the t of local(), the same arithmetic given
// invr = 1 / r).  rho is stored for the degrees n >= A0 only, at sidx(n, m) - sidx(A0, 0);
// (cr[m], ci[m]) = e^(i m beta) for m < P.
template <typename T, int P, int A0>
__host__ __device__ __forceinline__ void local_rho(const Angles<T>& a, T invr, T* rho, T* cr,
                                                   T* ci) {
  const T ninvr = -invr;
  T fact = 1, pn = 1;
  T rpm = -ninvr;  // (-1)^m / r^(m+1)
  T er = 1, ei = 0;
#pragma unroll
  for (int m = 0; m < P; m++) {
    cr[m] = er;
    ci[m] = ei;
    T q = pn, qm1 = 0;  // Q[m] = P_m^m
    if (m >= A0) rho[sidx(m, m) - sidx(A0, 0)] = q * rpm;
    T rpn = rpm;
#pragma unroll
    for (int n = m + 1; n < P; n++) {
      const T qn = fma(T(2 * n - 1) * a.x, q, T(-(n - 1 + m) * (n - 1 - m)) * qm1);
      qm1 = q;
      q = qn;
      rpn *= ninvr;
      if (n >= A0) rho[sidx(n, m) - sidx(A0, 0)] = q * rpn;
    }
    rpm *= ninvr;
    pn = -pn * fact * a.y;
    fact += 2;
    const T tt = er * a.cb - ei * a.sb;
    ei = er * a.sb + ei * a.cb;
    er = tt;
  }
}

// The M2L of m2l_pair in the source's azimuthal frame.  Every term of output (j, k) carries
// the phase e^(i (m - k) beta) of its harmonic, so with M'[n, mu] = M[n, mu] e^(i mu beta)
//   L[j, k] += e^(-i k beta) A[j, k],   A[j, k] = sum over (n, mu) of real rho times M' or
//   conj(M'),
// and each term of A is two real multiply-adds instead of a complex one (four): the
// source is rotated once on entry (one complex product per mu > 0 coefficient) and each
// output once on exit.  Terms and signs as m2l_pair: mu = 0: (-1)^j rho[a, k] M';
// m = -mu: (-1)^j rho[a, k + mu] conj(M'); m = +mu: (-1)^(j + min(k, mu)) rho[a, |mu - k|] M'.
template <typename T, int P, int J0, int J1>
__host__ __device__ __forceinline__ void m2l_pair_rot(const T* rho, const T* cr, const T* ci,
                                                      const T* Mj, T* Lr, T* Li) {
  constexpr int O0 = sidx(J0, 0), NO = sidx(J1, 0) - sidx(J0, 0);
  T Ar[NO], Ai[NO];
#pragma unroll
  for (int t = 0; t < NO; t++) Ar[t] = Ai[t] = T(0);
#pragma unroll
  for (int n = 0; n < P - J0; n++) {
#pragma unroll
    for (int mu = 0; mu <= n; mu++) {
      T mr, mi;
      load_pair(Mj + 2 * sidx(n, mu), mr, mi);
      if (mu > 0) {
        const T r = mr * cr[mu] - mi * ci[mu];
        mi = mr * ci[mu] + mi * cr[mu];
        mr = r;
      }
#pragma unroll
      for (int j = J0; j < J1; j++) {
        if (j + n >= P) break;
        const int a = j + n;
        const bool oj = (j & 1) != 0;
#pragma unroll
        for (int k = 0; k <= j; k++) {
          const int t = sidx(j, k) - O0;
          if (mu == 0) {
            const T p = rho[sidx(a, k) - O0];
            const T ps = oj ? -p : p;
            Ar[t] = fma(ps, mr, Ar[t]);
            Ai[t] = fma(ps, mi, Ai[t]);
          } else {
            const T p1 = rho[sidx(a, k + mu) - O0];
            const T s1 = oj ? -p1 : p1;
            Ar[t] = fma(s1, mr, Ar[t]);
            Ai[t] = fma(-s1, mi, Ai[t]);
            const T p2 = rho[sidx(a, mu >= k ? mu - k : k - mu) - O0];
            const bool o2 = oj != (((k < mu ? k : mu) & 1) != 0);
            const T s2 = o2 ? -p2 : p2;
            Ar[t] = fma(s2, mr, Ar[t]);
            Ai[t] = fma(s2, mi, Ai[t]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = J0; j < J1; j++)
#pragma unroll
    for (int k = 0; k <= j; k++) {
      const int t = sidx(j, k) - O0, g = sidx(j, k);
      if (k == 0) {
        Lr[g] += Ar[t];
        Li[g] += Ai[t];
      } else {
        Lr[g] = fma(cr[k], Ar[t], fma(ci[k], Ai[t], Lr[g]));
        Li[g] = fma(cr[k], Ai[t], fma(-ci[k], Ar[t], Li[g]));
      }
    }
}

// m2l_pair_rot with the loops the other way round: the rotated source coefficients of the
// degrees n < P - J0 held in registers and each output's sum A[j, k] finished and rotated
// before the next (the same terms in the same order, so the same results); for the
// passes of high output degree, which take few source coefficients and many outputs.
template <typename T, int P, int J0, int J1>
__host__ __device__ __forceinline__ void m2l_pair_rot_out(const T* rho, const T* cr,
                                                          const T* ci, const T* Mj, T* Lr,
                                                          T* Li) {
  constexpr int O0 = sidx(J0, 0), NIN = sidx(P - J0, 0);
  T Mr[NIN], Mi[NIN];
#pragma unroll
  for (int n = 0; n < P - J0; n++)
#pragma unroll
    for (int mu = 0; mu <= n; mu++) {
      T mr, mi;
      load_pair(Mj + 2 * sidx(n, mu), mr, mi);
      if (mu > 0) {
        const T r = mr * cr[mu] - mi * ci[mu];
        mi = mr * ci[mu] + mi * cr[mu];
        mr = r;
      }
      Mr[sidx(n, mu)] = mr;
      Mi[sidx(n, mu)] = mi;
    }
  // outputs by order k, then degree: e^(i k beta) advances by one rotation per k, so the
  // phases need not stay live in registers
  T er = T(1), ei = T(0);
#pragma unroll
  for (int k = 0; k < J1; k++) {
#pragma unroll
    for (int j = (k > J0 ? k : J0); j < J1; j++) {
      const bool oj = (j & 1) != 0;
      T ar = T(0), ai = T(0);
#pragma unroll
      for (int n = 0; n < P - j; n++) {
        const int a = j + n;
#pragma unroll
        for (int mu = 0; mu <= n; mu++) {
          const T mr = Mr[sidx(n, mu)], mi = Mi[sidx(n, mu)];
          if (mu == 0) {
            const T p = rho[sidx(a, k) - O0];
            const T ps = oj ? -p : p;
            ar = fma(ps, mr, ar);
            ai = fma(ps, mi, ai);
          } else {
            const T p1 = rho[sidx(a, k + mu) - O0];
            const T s1 = oj ? -p1 : p1;
            ar = fma(s1, mr, ar);
            ai = fma(-s1, mi, ai);
            const T p2 = rho[sidx(a, mu >= k ? mu - k : k - mu) - O0];
            const bool o2 = oj != (((k < mu ? k : mu) & 1) != 0);
            const T s2 = o2 ? -p2 : p2;
            ar = fma(s2, mr, ar);
            ai = fma(s2, mi, ai);
          }
        }
      }
      const int g = sidx(j, k);
      if (k == 0) {
        Lr[g] += ar;
        Li[g] += ai;
      } else {
        Lr[g] = fma(er, ar, fma(ei, ai, Lr[g]));
        Li[g] = fma(er, ai, fma(-ei, ar, Li[g]));
      }
    }
    const T tt = er * cr[1] - ei * ci[1];
    ei = er * ci[1] + ei * cr[1];
    er = tt;
  }
}

// Y[a, b] for any sign of b from the m >= 0 store (real parts yr, imaginary parts yi)
template <typename T>
__host__ __device__ __forceinline__ void yget(const T* yr, const T* yi, int a, int b, T& r,
                                              T& i) {
  if (b >= 0) {
    r = yr[sidx(a, b)];
    i = yi[sidx(a, b)];
  } else {
    r = yr[sidx(a, -b)];
    i = -yi[sidx(a, -b)];
  }
}

// M2M output coefficient (j, k) from one child (:127-144); Y (yr, yi) from multipole() at
// Xparent - Xchild, Mc the child's NT (re, im) pairs.  Runtime indices when (j, k) are
// runtime values, register operands when they are unrolled constants.
template <typename T>
__host__ __device__ __forceinline__ void m2m_term(int j, int k, const T* yr, const T* yi,
                                                  const T* Mc, T& outr, T& outi) {
  T sr = 0, si = 0;
#pragma unroll
  for (int n = 0; n <= j; n++) {
    // m in [max(-n, -j+k+n), min(k-1, n)]
#pragma unroll
    for (int m = -n; m <= n; m++) {
      if (m < -j + k + n) continue;
      if (m > k - 1) break;
      // Cj->M[(j-n)(j-n+1)/2 + k - m] * Ynm[n*n+n-m] * IPOW2N(m) * ODDEVEN(n)
      const int q = (j - n) * (j - n + 1) / 2 + k - m;
      const T Mr = Mc[2 * q], Mi = Mc[2 * q + 1];
      T ur, ui;
      yget(yr, yi, n, -m, ur, ui);
      const T pr = Mr * ur - Mi * ui, pi = Mr * ui + Mi * ur;
      const int sgn = ((m < 0 && (m & 1)) ? -1 : 1) * ((n & 1) ? -1 : 1);
      sr += sgn * pr;
      si += sgn * pi;
    }
    // m in [k, min(n, j+k-n)]
#pragma unroll
    for (int m = k; m <= n; m++) {
      if (m > j + k - n) break;
      // conj(Cj->M[(j-n)(j-n+1)/2 - k + m]) * Ynm[n*n+n-m] * ODDEVEN(k+n+m)
      const int q = (j - n) * (j - n + 1) / 2 - k + m;
      const T Mr = Mc[2 * q], Mi = -Mc[2 * q + 1];
      T ur, ui;
      yget(yr, yi, n, -m, ur, ui);
      const T pr = Mr * ur - Mi * ui, pi = Mr * ui + Mi * ur;
      const int sgn = ((k + n + m) & 1) ? -1 : 1;
      sr += sgn * pr;
      si += sgn * pi;
    }
  }
  outr = sr;
  outi = si;
}

// L2L output coefficient (j, k) from the parent (:203-222); Y (yr, yi) from multipole() at
// Xchild - Xparent, Lp the parent's NT (re, im) pairs.
template <typename T>
__host__ __device__ __forceinline__ void l2l_term(int P, int j, int k, const T* yr,
                                                  const T* yi, const T* Lp, T& outr, T& outi) {
  T sr = 0, si = 0;
#pragma unroll
  for (int n = j; n < P; n++) {
    // m in [j+k-n, -1]
#pragma unroll
    for (int m = -n; m < 0; m++) {
      if (m < j + k - n) continue;
      // conj(Cj->L[n(n+1)/2 - m]) * Ynm[(n-j)^2 + n-j + m-k] * ODDEVEN(k)
      const int q = n * (n + 1) / 2 - m;
      const T Lr = Lp[2 * q], Li = -Lp[2 * q + 1];
      T ur, ui;
      yget(yr, yi, n - j, m - k, ur, ui);
      const T pr = Lr * ur - Li * ui, pi = Lr * ui + Li * ur;
      const int sgn = (k & 1) ? -1 : 1;
      sr += sgn * pr;
      si += sgn * pi;
    }
#pragma unroll
    for (int m = 0; m <= n; m++) {
      const int d = m - k;
      if (n - j < (d < 0 ? -d : d)) continue;
      // Cj->L[n(n+1)/2 + m] * Ynm[(n-j)^2 + n-j + m-k] * ODDEVEN((m-k)(m<k))
      const int q = n * (n + 1) / 2 + m;
      const T Lr = Lp[2 * q], Li = Lp[2 * q + 1];
      T ur, ui;
      yget(yr, yi, n - j, d, ur, ui);
      const T pr = Lr * ur - Li * ui, pi = Lr * ui + Li * ur;
      const int sgn = (d < 0 && (d & 1)) ? -1 : 1;
      sr += sgn * pr;
      si += sgn * pi;
    }
  }
  outr = sr;
  outi = si;
}

// Whole M2M / L2L translations for the output degrees j in [J0, J1) with compile-time
// indices (register operands); out[t - sidx(J0, 0)] holds output t as (re, im).
template <typename T, int P, int J0 = 0, int J1 = P>
__host__ __device__ __forceinline__ void m2m_range(const T* yr, const T* yi, const T* Mc,
                                                   T* out) {
#pragma unroll
  for (int j = J0; j < J1; j++)
#pragma unroll
    for (int k = 0; k <= j; k++) {
      T r, i;
      m2m_term<T>(j, k, yr, yi, Mc, r, i);
      out[2 * (sidx(j, k) - sidx(J0, 0))] += r;
      out[2 * (sidx(j, k) - sidx(J0, 0)) + 1] += i;
    }
}
template <typename T, int P, int J0 = 0, int J1 = P>
__host__ __device__ __forceinline__ void l2l_range(const T* yr, const T* yi, const T* Lp,
                                                   T* out) {
#pragma unroll
  for (int j = J0; j < J1; j++)
#pragma unroll
    for (int k = 0; k <= j; k++) {
      T r, i;
      l2l_term<T>(P, j, k, yr, yi, Lp, r, i);
      out[2 * (sidx(j, k) - sidx(J0, 0))] += r;
      out[2 * (sidx(j, k) - sidx(J0, 0)) + 1] += i;
    }
}

// L2P of one body (:226-256): potential and gradient of the local expansion L (NT (re, im)
// pairs) at offset dX from the cell centre.  Harmonics and their theta derivatives are
// generated column by column and consumed on the fly.
template <typename T, int P>
__host__ __device__ __forceinline__ void l2p_body(T dx, T dy, T dz, const T* L, T& pot, T& gx,
                                                  T& gy, T& gz) {
  // the divisions of the reference (by rho per term, by -(n+m) and (2m+2)(2m+1) per
  // step) are multiplications by reciprocals here: one division per body
  Angles<T> a = angles(dx, dy, dz);
  const T rho = a.r, invrho = T(1) / rho;
  T s0 = 0, s1 = 0, s2 = 0, ph = 0;
  T fact = 1, pn = 1, rhom = 1;
  T er = 1, ei = 0;
  const T invy = T(1) / a.y;
#pragma unroll
  for (int m = 0; m < P; m++) {
    const T w = m == 0 ? T(1) : T(2);
    T p = pn;
    T p1 = p;
    p = a.x * (2 * m + 1) * p1;
    {
      // Y[m,m] and its theta derivative
      const T yv = rhom * p1;
      const T tv = rhom * (p - (m + 1) * a.x * p1) * invy;
      const T Lr = L[2 * sidx(m, m)], Li = L[2 * sidx(m, m) + 1];
      const T re = Lr * er - Li * ei, im = Lr * ei + Li * er;  // L * e^(i m beta)
      ph += w * yv * re;
      s0 += w * yv * re * invrho * m;
      s1 += w * tv * re;
      s2 -= w * yv * im * m;
    }
    rhom *= rho;
    T rhon = rhom;
#pragma unroll
    for (int n = m + 1; n < P; n++) {
      rhon *= T(-1) / T(n + m);
      const T yv = rhon * p;
      T p2 = p1;
      p1 = p;
      p = (a.x * (2 * n + 1) * p1 - (n + m) * p2) * (T(1) / T(n - m + 1));
      const T tv = rhon * ((n - m + 1) * p - (n + 1) * a.x * p1) * invy;
      const T Lr = L[2 * sidx(n, m)], Li = L[2 * sidx(n, m) + 1];
      const T re = Lr * er - Li * ei, im = Lr * ei + Li * er;
      ph += w * yv * re;
      s0 += w * yv * re * invrho * n;
      s1 += w * tv * re;
      s2 -= w * yv * im * m;
      rhon *= rho;
    }
    rhom *= T(-1) / T((2 * m + 2) * (2 * m + 1));
    pn = -pn * fact * a.y;
    fact += 2;
    T t = er * a.cb - ei * a.sb;
    ei = er * a.sb + ei * a.cb;
    er = t;
  }
  // sph2cart (:17-26)
  pot = ph;
  gx = a.y * a.cb * s0 + a.x * a.cb * invrho * s1 - a.sb * invrho * invy * s2;
  gy = a.y * a.sb * s0 + a.x * a.sb * invrho * s1 + a.cb * invrho * invy * s2;
  gz = a.x * s0 - a.y * invrho * s1;
}

}  // namespace sph
}  // namespace fmmb200
