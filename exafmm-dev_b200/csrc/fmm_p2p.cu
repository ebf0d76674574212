// Near-field P2P over the per-target-leaf source lists (kernel::P2P,
// kernels/LaplaceP2PCPU.cxx:4-170 and the self form :172-331).
//
// One warp owns one target leaf.  Its lanes split into groups of G (1, 2 or 4) so that a
// small leaf still keeps the warp busy: each group holds one target body and its G lanes
// take every G-th source; a leaf of 33..64 bodies gives each lane two targets that share
// every staged source.  Source leaves stream through shared memory 32 bodies at a time
// (one coalesced 16-byte load per lane); in FP32 the staged sources are taken two at a time
// with the packed two-wide instructions of sm_100 (half the issue slots of the scalar pair
// arithmetic).  The inner loop is FMA + one rsqrt per pair (no r^2 == 0 test outside the
// target leaf itself), and each source leaf's plain partial sum is folded into a
// compensated (TwoSum) accumulator, so the accumulation error does not grow with the number
// of source leaves.  Pairs with r^2 == 0 are skipped, as the reference does (:149); the
// result is per unit target charge (the reference multiplies by q_i in P2P and divides
// again in L2P / normalize).
#include <algorithm>

#include "fmm_solver.cuh"

namespace fmmb200 {

constexpr int kP2PWarps = 4;

// 1/sqrt with subnormal inputs flushed to zero (PTX rsqrt.approx.ftz.f32): no handling of
// subnormal inputs and no r^2 == 0 test, for the source leaves where neither can occur
__device__ __forceinline__ float rsqrt_ftz(float a) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ double rsqrt_ftz(double a) { return rsqrt(a); }

// one pair; EXACT: skip r^2 == 0 and take subnormal r^2 as it is (the reference's
// arithmetic); otherwise an r^2 of zero or below the normal range makes `pot` non-finite
// SHIFT: the source is a periodic image shifted by (px, py, pz); the offset is formed as
// (xj - xi) + p, the negation of the reference's (xi - xj) - Xperiodic
template <typename T, bool EXACT = true, bool SHIFT = false>
__device__ __forceinline__ void p2p_accum(const vec4<T>& sj, const vec4<T>& xi, T eps2, T& pot,
                                          T& ax, T& ay, T& az, T px = 0, T py = 0, T pz = 0) {
  T dx = sj.x - xi.x, dy = sj.y - xi.y, dz = sj.z - xi.z;
  if (SHIFT) {
    dx += px;
    dy += py;
    dz += pz;
  }
  const T r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
  const T inv = EXACT ? (r2 > T(0) ? rsqrt_(r2) : T(0)) : rsqrt_ftz(r2);
  const T qinv = sj.w * inv;
  const T inv3 = qinv * inv * inv;
  pot += qinv;
  ax = fma(dx, inv3, ax);
  ay = fma(dy, inv3, ay);
  az = fma(dz, inv3, az);
}

// FP32 source leaf: the staged sources are taken two at a time with the packed two-wide
// instructions of sm_100 (add.f32x2, mul.f32x2, fma.f32x2: one instruction for both, each
// component rounded as the scalar operation, so each pair's terms are those of p2p_accum);
// a target's two partial sums are added at the end of the leaf.  The warp's row holds
// A[i] = (x, x', y, y') and B[i] = (z, z', q, q') for the sources 2i and 2i + 1; a missing
// partner is a far-away zero charge, which adds exactly zero.
template <int TPL, bool EXACT, bool SHIFT>
__device__ __forceinline__ void source_leaf_pairs(int lane, float4* row, int sub, int G, int j0,
                                                  int nj, const vec4<float>* __restrict__ bodies,
                                                  float eps2, const vec4<float>* xi, float* pot,
                                                  float* ax, float* ay, float* az, float px,
                                                  float py, float pz) {
  float4* A = row;
  float4* B = row + 16;
  float2 nx[TPL], ny[TPL], nz[TPL], sp[TPL], sx[TPL], sy[TPL], sz[TPL];
#pragma unroll
  for (int u = 0; u < TPL; u++) {
    nx[u] = make_float2(-xi[u].x, -xi[u].x);
    ny[u] = make_float2(-xi[u].y, -xi[u].y);
    nz[u] = make_float2(-xi[u].z, -xi[u].z);
    sp[u] = sx[u] = sy[u] = sz[u] = make_float2(0.f, 0.f);
  }
  const float2 e2 = make_float2(eps2, eps2);
  const float2 p2x = make_float2(px, px), p2y = make_float2(py, py), p2z = make_float2(pz, pz);
  for (int jb = 0; jb < nj; jb += 32) {
    const int cnt = min(32, nj - jb);
    __syncwarp();
    {
      const vec4<float> b =
          lane < cnt ? bodies[j0 + jb + lane] : make_v4<float>(1e30f, 1e30f, 1e30f, 0.f);
      float* a = reinterpret_cast<float*>(&A[lane >> 1]);
      float* c = reinterpret_cast<float*>(&B[lane >> 1]);
      const int h = lane & 1;
      a[h] = b.x;
      a[2 + h] = b.y;
      c[h] = b.z;
      c[2 + h] = b.w;
    }
    __syncwarp();
    const int np = (cnt + 1) >> 1;
#pragma unroll 2
    for (int i = sub; i < np; i += G) {
      const float4 a = A[i], c = B[i];
      const float2 x2 = make_float2(a.x, a.y), y2 = make_float2(a.z, a.w);
      const float2 z2 = make_float2(c.x, c.y), q2 = make_float2(c.z, c.w);
#pragma unroll
      for (int u = 0; u < TPL; u++) {
        float2 dx = __fadd2_rn(x2, nx[u]), dy = __fadd2_rn(y2, ny[u]), dz = __fadd2_rn(z2, nz[u]);
        if (SHIFT) {
          dx = __fadd2_rn(dx, p2x);
          dy = __fadd2_rn(dy, p2y);
          dz = __fadd2_rn(dz, p2z);
        }
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
        float2 inv;
        inv.x = EXACT ? (r2.x > 0.f ? rsqrt_(r2.x) : 0.f) : rsqrt_ftz(r2.x);
        inv.y = EXACT ? (r2.y > 0.f ? rsqrt_(r2.y) : 0.f) : rsqrt_ftz(r2.y);
        const float2 qinv = __fmul2_rn(q2, inv);
        const float2 inv3 = __fmul2_rn(__fmul2_rn(qinv, inv), inv);
        sp[u] = __fadd2_rn(sp[u], qinv);
        sx[u] = __ffma2_rn(dx, inv3, sx[u]);
        sy[u] = __ffma2_rn(dy, inv3, sy[u]);
        sz[u] = __ffma2_rn(dz, inv3, sz[u]);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < TPL; u++) {
    pot[u] = sp[u].x + sp[u].y;
    ax[u] = sx[u].x + sx[u].y;
    ay[u] = sy[u].x + sy[u].y;
    az[u] = sz[u].x + sz[u].y;
  }
}

// all bodies of one source leaf (first body j0, nj bodies) on the lane's TPL targets, its
// sums started from zero; sources are staged through the warp's shared row 32 at a time
template <typename T, int TPL, bool EXACT, bool SHIFT = false>
__device__ __forceinline__ void source_leaf(int lane, int wl, vec4<T> (*sh)[32], int sub, int G,
                                            int j0, int nj, const vec4<T>* __restrict__ bodies,
                                            T eps2, const vec4<T>* xi, T* pot, T* ax, T* ay,
                                            T* az, T px = 0, T py = 0, T pz = 0) {
  if constexpr (sizeof(T) == 4) {
    source_leaf_pairs<TPL, EXACT, SHIFT>(lane, reinterpret_cast<float4*>(sh[wl]), sub, G, j0,
                                         nj, bodies, eps2, xi, pot, ax, ay, az, px, py, pz);
  } else {
#pragma unroll
  for (int u = 0; u < TPL; u++) pot[u] = ax[u] = ay[u] = az[u] = 0;
  for (int jb = 0; jb < nj; jb += 32) {
    const int cnt = min(32, nj - jb);
    __syncwarp();
    if (lane < cnt) sh[wl][lane] = bodies[j0 + jb + lane];
    __syncwarp();
#pragma unroll 4
    for (int k = sub; k < cnt; k += G) {
      const vec4<T> sj = sh[wl][k];
#pragma unroll
      for (int u = 0; u < TPL; u++)
        p2p_accum<T, EXACT, SHIFT>(sj, xi[u], eps2, pot[u], ax[u], ay[u], az[u], px, py, pz);
    }
  }
  }
}

// TPL targets per lane (1 or 2): a lane holds targets ti and ti + 32 / G and reuses every
// staged source for both.
template <typename T, bool COMP, int TPL>
__device__ __forceinline__ void p2p_leaf(int lane, int wl, vec4<T> (*sh)[32], int b0, int nb,
                                         int base, int G, int s0, int s1,
                                         const unsigned long long* __restrict__ pairs,
                                         const int* __restrict__ ibody,
                                         const int* __restrict__ nbody,
                                         const vec4<T>* __restrict__ bodies, T eps2, T cycle,
                                         vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e) {
  const int tpp = 32 / G;
  const int sub = lane % G;
  int ti[TPL];
  bool act[TPL];
  vec4<T> xi[TPL];
  Comp<T> acc[TPL][4];
#pragma unroll
  for (int u = 0; u < TPL; u++) {
    ti[u] = base + u * tpp + lane / G;
    act[u] = ti[u] < nb;
    xi[u] = act[u] ? bodies[b0 + ti[u]] : make_v4<T>(0, 0, 0, 0);
#pragma unroll
    for (int d = 0; d < 4; d++) acc[u][d] = Comp<T>{0, 0};
  }
  // source leaf s: (first body, count, periodic image), the next one prefetched
  const unsigned src0 = s0 < s1 ? (unsigned)pairs[s0] : 0u;
  int j0 = s0 < s1 ? ibody[pair_cell(src0)] : 0, nj = s0 < s1 ? nbody[pair_cell(src0)] : 0;
  int img = pair_img(src0);
  for (int s = s0; s < s1; s++) {
    int j0n = 0, njn = 0, imgn = 0;
    if (s + 1 < s1) {
      const unsigned srcn = (unsigned)pairs[s + 1];
      j0n = ibody[pair_cell(srcn)];
      njn = nbody[pair_cell(srcn)];
      imgn = pair_img(srcn);
    }
    T pot[TPL], ax[TPL], ay[TPL], az[TPL];
    // Bodies at one position share every octant and so one leaf: only the target leaf
    // itself can hold a pair at r^2 == 0.  Other source leaves take the fast pair form;
    // if a pair underflowed to r^2 == 0 or below the normal range there, its sum is not
    // finite and the leaf is summed again in the exact form, so results are always those
    // of the exact form.
    if (img != 0) {
      // a periodic image of a source leaf (r^2 == 0 would take bodies exactly one period
      // apart): fast form, exact re-sum if not finite
      T px, py, pz;
      img_shift<T>(img, cycle, px, py, pz);
      source_leaf<T, TPL, false, true>(lane, wl, sh, sub, G, j0, nj, bodies, eps2, xi, pot, ax,
                                       ay, az, px, py, pz);
      bool bad = false;
#pragma unroll
      for (int u = 0; u < TPL; u++) bad |= act[u] && !isfinite(pot[u]);
      if (__any_sync(0xffffffffu, bad))
        source_leaf<T, TPL, true, true>(lane, wl, sh, sub, G, j0, nj, bodies, eps2, xi, pot, ax,
                                        ay, az, px, py, pz);
    } else if (j0 != b0) {
      source_leaf<T, TPL, false>(lane, wl, sh, sub, G, j0, nj, bodies, eps2, xi, pot, ax, ay, az);
      bool bad = false;
#pragma unroll
      for (int u = 0; u < TPL; u++) bad |= act[u] && !isfinite(pot[u]);
      if (__any_sync(0xffffffffu, bad))
        source_leaf<T, TPL, true>(lane, wl, sh, sub, G, j0, nj, bodies, eps2, xi, pot, ax, ay, az);
    } else {
      source_leaf<T, TPL, true>(lane, wl, sh, sub, G, j0, nj, bodies, eps2, xi, pot, ax, ay, az);
    }
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      if (COMP) {
        comp_add(acc[u][0], pot[u]);
        comp_add(acc[u][1], ax[u]);
        comp_add(acc[u][2], ay[u]);
        comp_add(acc[u][3], az[u]);
      } else {
        acc[u][0].s += pot[u];
        acc[u][1].s += ax[u];
        acc[u][2].s += ay[u];
        acc[u][3].s += az[u];
      }
    }
    j0 = j0n;
    nj = njn;
    img = imgn;
  }
  for (int o = 1; o < G; o <<= 1) {
#pragma unroll
    for (int u = 0; u < TPL; u++)
#pragma unroll
      for (int d = 0; d < 4; d++) {
        Comp<T> r;
        r.s = __shfl_xor_sync(0xffffffffu, acc[u][d].s, o);
        r.e = __shfl_xor_sync(0xffffffffu, acc[u][d].e, o);
        if (COMP) comp_merge(acc[u][d], r);
        else acc[u][d].s += r.s;
      }
  }
  if (sub == 0) {
#pragma unroll
    for (int u = 0; u < TPL; u++)
      if (act[u]) {
        trg_s[b0 + ti[u]] = make_v4<T>(acc[u][0].s, acc[u][1].s, acc[u][2].s, acc[u][3].s);
        trg_e[b0 + ti[u]] = make_v4<T>(acc[u][0].e, acc[u][1].e, acc[u][2].e, acc[u][3].e);
      }
  }
}

template <typename T, bool COMP>
__global__ void __launch_bounds__(32 * kP2PWarps)
    k_p2p(const int* __restrict__ leaves, int nleaves, const int* __restrict__ off,
          const unsigned long long* __restrict__ pairs, const int* __restrict__ ibody,
          const int* __restrict__ nbody, const vec4<T>* __restrict__ bodies, T eps2, T cycle,
          vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e) {
  __shared__ vec4<T> sh[kP2PWarps][32];
  const int wl = threadIdx.x >> 5;
  const int w = blockIdx.x * kP2PWarps + wl;
  if (w >= nleaves) return;
  const int lane = lane_id();
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const int G = nb <= 8 ? 4 : (nb <= 16 ? 2 : 1);
  const int s0 = off[c], s1 = off[c + 1];
  if (nb <= 32) {
    p2p_leaf<T, COMP, 1>(lane, wl, sh, b0, nb, 0, G, s0, s1, pairs, ibody, nbody, bodies, eps2,
                         cycle, trg_s, trg_e);
  } else {
    for (int base = 0; base < nb; base += 64)
      p2p_leaf<T, COMP, 2>(lane, wl, sh, b0, nb, base, 1, s0, s1, pairs, ibody, nbody, bodies,
                           eps2, cycle, trg_s, trg_e);
  }
}

template <typename T> void run_p2p(Solver<T>& s) {
  if (s.nleaves == 0) return;
  constexpr bool comp = sizeof(T) == 4;
  k_p2p<T, comp><<<ceil_div(s.nleaves, kP2PWarps), 32 * kP2PWarps, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.p2p_off.p, s.p2p.p, s.c_ibody.p, s.c_nbody.p, s.bodies.p,
      (T)s.cfg.eps2, (T)s.cfg.cycle, s.trg_s.p, s.trg_e.p);
  FMM_LAUNCH_CHECK();
}

template void run_p2p<float>(Solver<float>&);
template void run_p2p<double>(Solver<double>&);

}  // namespace fmmb200
