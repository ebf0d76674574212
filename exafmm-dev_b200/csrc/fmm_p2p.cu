// Near-field P2P over the per-target-leaf source lists (kernel::P2P,
// kernels/LaplaceP2PCPU.cxx:4-170 and the self form :172-331).
//
// One warp owns one target leaf.  Its lanes split into groups of G (1, 2 or 4) so that a
// small leaf still keeps the warp busy: each group holds one target body and its G lanes
// take every G-th source; a leaf of 33..64 bodies gives each lane two targets that share
// every staged source.  Sources stream through shared memory 32 bodies at a time (one
// coalesced load per lane), a chunk of 32 running on across source leaves; in FP32 the
// staged sources are taken two at a time with the packed two-wide instructions of sm_100
// (half the issue slots of the scalar pair arithmetic).  The inner loop is FMA + one rsqrt
// per pair (no r^2 == 0 test away from the target leaf itself).  FP32 folds each chunk's
// plain partial sum into a compensated (TwoSum) accumulator, so the accumulation error does
// not grow with the length of the list; FP64 sums plainly.  Pairs with r^2 == 0 are
// skipped, as the reference does (:149); the result is per unit target charge (the
// reference multiplies by q_i in P2P and divides again in L2P / normalize).
#include <algorithm>
#include <type_traits>

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

// FP32 rows: the staged sources are taken two at a time with the packed two-wide
// instructions of sm_100 (add.f32x2, mul.f32x2, fma.f32x2: one instruction for both, each
// component rounded as the scalar operation, so each pair's terms are those of p2p_accum).
// A warp's row holds A[i] = (x, x', y, y') and B[i] = (z, z', q, q') for the sources 2i and
// 2i + 1 (A in float4 0..15, B in 16..31); a missing partner is a far-away zero charge,
// which adds exactly zero.

// the pairs of one staged row (np source pairs) on the lane's TPL targets, added to the
// two-wide sums; nx, ny, nz are the negated target coordinates in both halves
template <int TPL, bool EXACT, bool SHIFT>
__device__ __forceinline__ void row_pairs(const float4* row, int sub, int G, int np,
                                          const float2* nx, const float2* ny, const float2* nz,
                                          float2 e2, float2 p2x, float2 p2y, float2 p2z,
                                          float2* sp, float2* sx, float2* sy, float2* sz) {
  const float4* A = row;
  const float4* B = row + 16;
#pragma unroll (4 / TPL)
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

// FP64 rows: one source per entry (x, y, z, q); the pairs of a staged row (cnt sources) on
// the lane's TPL targets, added to the plain sums
template <int TPL, bool EXACT, bool SHIFT>
__device__ __forceinline__ void row_pairs(const vec4<double>* row, int sub, int G, int cnt,
                                          const vec4<double>* xi, double eps2, double px,
                                          double py, double pz, double* sp, double* sx,
                                          double* sy, double* sz) {
#pragma unroll (4 / TPL)
  for (int k = sub; k < cnt; k += G) {
    const vec4<double> sj = row[k];
#pragma unroll
    for (int u = 0; u < TPL; u++)
      p2p_accum<double, EXACT, SHIFT>(sj, xi[u], eps2, sp[u], sx[u], sy[u], sz[u], px, py, pz);
  }
}

// Target leaf, either precision: the bodies of its source leaves, taken in list order, are
// staged 32 at a time whatever the leaves' sizes (a chunk runs on into the next source leaf,
// and ends early only where the periodic image changes or after 32 source leaves), so that
// the rows are full and the per-chunk work (staging, the finite test, the compensated fold)
// is shared by all of its source leaves.  The source leaves' descriptors (first body,
// count, image) are read 32 at a time, one per lane; a lane finds the leaf of its chunk
// position by a scan of the counts and a binary search over the lanes.  A chunk that holds
// bodies of the target leaf itself is summed in the exact form; any other chunk in the fast
// form, and again in the exact form (from the same row) if a sum is not finite, so the
// results are those of the exact form throughout.  FP32 takes the staged sources two at a
// time with the packed f32x2 instructions; FP64 one at a time.
template <typename T, bool COMP, int TPL>
__device__ __forceinline__ void p2p_leaf_chunked(int lane, void* rowmem, int b0, int nb,
                                                 int base, int G, int s0, int s1,
                                                 const unsigned long long* __restrict__ pairs,
                                                 const int* __restrict__ ibody,
                                                 const int* __restrict__ nbody,
                                                 const vec4<T>* __restrict__ bodies, T eps2,
                                                 T cycle, vec4<T>* __restrict__ trg_s,
                                                 vec4<T>* __restrict__ trg_e) {
  constexpr bool F32 = sizeof(T) == 4;
  // per-lane pair sums: float2 (two halves of the packed form) or T
  using Acc = typename std::conditional<F32, float2, T>::type;
  const unsigned full = 0xffffffffu;
  const int tpp = 32 / G;
  const int sub = lane % G;
  int ti[TPL];
  bool act[TPL];
  vec4<T> xi[TPL];
  float2 nx[TPL], ny[TPL], nz[TPL];  // FP32: negated target coordinates in both halves
  Comp<T> acc[TPL][4];
#pragma unroll
  for (int u = 0; u < TPL; u++) {
    ti[u] = base + u * tpp + lane / G;
    act[u] = ti[u] < nb;
    xi[u] = act[u] ? bodies[b0 + ti[u]] : make_v4<T>(0, 0, 0, 0);
    if constexpr (F32) {
      nx[u] = make_float2(-xi[u].x, -xi[u].x);
      ny[u] = make_float2(-xi[u].y, -xi[u].y);
      nz[u] = make_float2(-xi[u].z, -xi[u].z);
    }
#pragma unroll
    for (int d = 0; d < 4; d++) acc[u][d] = Comp<T>{0, 0};
  }
  const float2 e2 = make_float2((float)eps2, (float)eps2);
  for (int sb = s0; sb < s1; sb += 32) {
    // lane k: source leaf sb + k (image -1 past the end of the list)
    int dj0 = 0, dnj = 0, dimg = -1;
    if (sb + lane < s1) {
      const unsigned src = (unsigned)pairs[sb + lane];
      dj0 = ibody[pair_cell(src)];
      dnj = nbody[pair_cell(src)];
      dimg = pair_img(src);
    }
    int k = 0, o = 0;  // the chunk starts at body o of leaf k
    while (k < 32) {
      const int img = __shfl_sync(full, dimg, k);
      if (img < 0) break;
      const unsigned other = ~__ballot_sync(full, dimg == img) & (full << k);
      const int cut = other ? __ffs(other) - 1 : 32;  // leaves k .. cut - 1 share the image
      const int avail = lane >= k && lane < cut ? dnj - (lane == k ? o : 0) : 0;
      int incl = avail;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(full, incl, d);
        if (lane >= d) incl += v;
      }
      const int total = __shfl_sync(full, incl, 31);
      const int cnt = min(32, total);
      // f: the leaf of chunk position `lane`.  Each leaf of the chunk sets the bit of its
      // first position; f is k plus the number of bits at or below `lane`, less one (with
      // an empty leaf in the range, whose start would coincide with the next one's: the
      // number of leaves whose counts end at or before `lane`, by binary search)
      int f;
      if (!__any_sync(full, lane >= k && lane < cut && avail == 0)) {
        const unsigned starts =
            __reduce_or_sync(full, avail > 0 && incl - avail < 32 ? 1u << (incl - avail) : 0u);
        f = k + __popc(starts & (full >> (31 - lane))) - 1;
      } else {
        f = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1)
          if (__shfl_sync(full, incl, f + step - 1) <= lane) f += step;
      }
      const int ex = __shfl_sync(full, incl - avail, f);
      const int jf = __shfl_sync(full, dj0 + (lane == k ? o : 0), f);
      const int bj = jf + lane - ex;
      const vec4<T> b = lane < cnt ? bodies[bj] : make_v4<T>(T(1e30), T(1e30), T(1e30), T(0));
      const bool self = __any_sync(full, lane < cnt && img == 0 && bj >= b0 && bj < b0 + nb);
      T px = 0, py = 0, pz = 0;
      if (img != 0) img_shift<T>(img, cycle, px, py, pz);
      Acc sp[TPL], sx[TPL], sy[TPL], sz[TPL];
      auto zero = [&]() {
#pragma unroll
        for (int u = 0; u < TPL; u++) {
          if constexpr (F32) sp[u] = sx[u] = sy[u] = sz[u] = make_float2(0.f, 0.f);
          else sp[u] = sx[u] = sy[u] = sz[u] = T(0);
        }
      };
      auto finite = [&]() {
        bool bad = false;
#pragma unroll
        for (int u = 0; u < TPL; u++) {
          if constexpr (F32) bad |= act[u] && !isfinite(sp[u].x + sp[u].y);
          else bad |= act[u] && !isfinite(sp[u]);
        }
        return !__any_sync(full, bad);
      };
      __syncwarp();
      if constexpr (F32) {
        // A[i] = (x, x', y, y'), B[i] = (z, z', q, q') for the sources 2i and 2i + 1
        float4* A = static_cast<float4*>(rowmem);
        float4* B = A + 16;
        float* a = reinterpret_cast<float*>(&A[lane >> 1]);
        float* c = reinterpret_cast<float*>(&B[lane >> 1]);
        const int h = lane & 1;
        a[h] = b.x;
        a[2 + h] = b.y;
        c[h] = b.z;
        c[2 + h] = b.w;
      } else {
        static_cast<vec4<T>*>(rowmem)[lane] = b;
      }
      __syncwarp();
      // evaluate the row in the fast or the exact pair form (with or without the shift)
      auto pairs_of = [&](auto exact, auto shift) {
        constexpr bool EX = decltype(exact)::value, SH = decltype(shift)::value;
        if constexpr (F32) {
          const float2 p2x = make_float2(px, px), p2y = make_float2(py, py),
                       p2z = make_float2(pz, pz);
          row_pairs<TPL, EX, SH>(static_cast<const float4*>(rowmem), sub, G, (cnt + 1) >> 1,
                                 nx, ny, nz, e2, p2x, p2y, p2z, sp, sx, sy, sz);
        } else {
          row_pairs<TPL, EX, SH>(static_cast<const vec4<T>*>(rowmem), sub, G, cnt, xi, eps2,
                                 px, py, pz, sp, sx, sy, sz);
        }
      };
      using TT = std::true_type;
      using FF = std::false_type;
      zero();
      if (img != 0) {
        pairs_of(FF(), TT());
        if (!finite()) {
          zero();
          pairs_of(TT(), TT());
        }
      } else if (self) {
        pairs_of(TT(), FF());
      } else {
        pairs_of(FF(), FF());
        if (!finite()) {
          zero();
          pairs_of(TT(), FF());
        }
      }
#pragma unroll
      for (int u = 0; u < TPL; u++) {
        T pot, ax, ay, az;
        if constexpr (F32) {
          pot = sp[u].x + sp[u].y;
          ax = sx[u].x + sx[u].y;
          ay = sy[u].x + sy[u].y;
          az = sz[u].x + sz[u].y;
        } else {
          pot = sp[u];
          ax = sx[u];
          ay = sy[u];
          az = sz[u];
        }
        if (COMP) {
          comp_add(acc[u][0], pot);
          comp_add(acc[u][1], ax);
          comp_add(acc[u][2], ay);
          comp_add(acc[u][3], az);
        } else {
          acc[u][0].s += pot;
          acc[u][1].s += ax;
          acc[u][2].s += ay;
          acc[u][3].s += az;
        }
      }
      // the next chunk: past leaves k .. cut - 1, or inside the leaf holding position 32
      if (total <= 32) {
        k = cut;
        o = 0;
      } else {
        const int kn = __popc(__ballot_sync(full, lane < cut && incl <= 32));
        const int exn = __shfl_sync(full, incl - avail, kn);
        o = (kn == k ? o : 0) + 32 - exn;
        k = kn;
      }
    }
  }
  for (int o = 1; o < G; o <<= 1) {
#pragma unroll
    for (int u = 0; u < TPL; u++)
#pragma unroll
      for (int d = 0; d < 4; d++) {
        Comp<T> r;
        r.s = __shfl_xor_sync(full, acc[u][d].s, o);
        r.e = __shfl_xor_sync(full, acc[u][d].e, o);
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
          vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e, int g4, int g2) {
  // one row of 32 sources per warp
  __shared__ __align__(16) unsigned char smem[kP2PWarps][32 * sizeof(vec4<T>)];
  const int wl = threadIdx.x >> 5;
  const int w = blockIdx.x * kP2PWarps + wl;
  if (w >= nleaves) return;
  const int lane = lane_id();
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const int G = nb <= g4 ? 4 : (nb <= g2 ? 2 : 1);
  const int s0 = off[c], s1 = off[c + 1];
  void* row = smem[wl];
  if (nb <= 32) {
    p2p_leaf_chunked<T, COMP, 1>(lane, row, b0, nb, 0, G, s0, s1, pairs, ibody, nbody, bodies,
                                 eps2, cycle, trg_s, trg_e);
  } else {
    for (int base = 0; base < nb; base += 64)
      p2p_leaf_chunked<T, COMP, 2>(lane, row, b0, nb, base, 1, s0, s1, pairs, ibody, nbody,
                                   bodies, eps2, cycle, trg_s, trg_e);
  }
}

template <typename T> void run_p2p(Solver<T>& s) {
  if (s.nleaves == 0) return;
  constexpr bool comp = sizeof(T) == 4;
  k_p2p<T, comp><<<ceil_div(s.nleaves, kP2PWarps), 32 * kP2PWarps, 0, s.stream>>>(
      s.p2p_ordered ? s.p2p_order.p : s.leaves.p, s.nleaves, s.p2p_off.p, s.p2p.p, s.c_ibody.p, s.c_nbody.p, s.bodies.p,
      (T)s.cfg.eps2, (T)s.cfg.cycle, s.trg_s.p, s.trg_e.p, std::min(s.p2p_g4, 8),
      std::min(s.p2p_g2, 16));
  FMM_LAUNCH_CHECK();
}

template void run_p2p<float>(Solver<float>&);
template void run_p2p<double>(Solver<double>&);

}  // namespace fmmb200
