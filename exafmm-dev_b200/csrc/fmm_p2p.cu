// Near-field P2P over the per-target-leaf source lists (kernel::P2P,
// kernels/LaplaceP2PCPU.cxx:4-170 and the self form :172-331).
//
// One warp owns one target leaf.  Its lanes split into groups of G (1, 2 or 4) so that a
// small leaf still keeps the warp busy: each group holds one target body and its G lanes
// take every G-th source.  Source leaves stream through shared memory 32 bodies at a time
// (one coalesced 16-byte load per lane, read back as a broadcast), the inner loop is
// FP32 FMA + one rsqrt per pair, and each source leaf's plain FP32 partial sum is folded
// into a compensated (TwoSum) accumulator, so the accumulation error does not grow with
// the number of source leaves.  Pairs with r^2 == 0 are skipped, as the reference does
// (:149); the result is per unit target charge (the reference multiplies by q_i in P2P
// and divides again in L2P / normalize).
#include <algorithm>

#include "fmm_solver.cuh"

namespace fmmb200 {

constexpr int kP2PWarps = 4;

template <typename T, bool COMP>
__global__ void __launch_bounds__(32 * kP2PWarps)
    k_p2p(const int* __restrict__ leaves, int nleaves, const int* __restrict__ off,
          const unsigned long long* __restrict__ pairs, const int* __restrict__ ibody,
          const int* __restrict__ nbody, const vec4<T>* __restrict__ bodies, T eps2,
          vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e) {
  __shared__ vec4<T> sh[kP2PWarps][32];
  const int wl = threadIdx.x >> 5;
  const int w = blockIdx.x * kP2PWarps + wl;
  if (w >= nleaves) return;
  const int lane = lane_id();
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const int G = nb <= 8 ? 4 : (nb <= 16 ? 2 : 1);
  const int tpp = 32 / G;
  const int s0 = off[c], s1 = off[c + 1];
  for (int base = 0; base < nb; base += tpp) {
    const int ti = base + lane / G;
    const int sub = lane % G;
    const bool active = ti < nb;
    vec4<T> xi = active ? bodies[b0 + ti] : make_v4<T>(0, 0, 0, 0);
    Comp<T> acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int s = s0; s < s1; s++) {
      const int cj = (int)(pairs[s] & 0xffffffffULL);
      const int j0 = ibody[cj], nj = nbody[cj];
      T pot = 0, ax = 0, ay = 0, az = 0;
      for (int jb = 0; jb < nj; jb += 32) {
        const int cnt = min(32, nj - jb);
        __syncwarp();
        if (lane < cnt) sh[wl][lane] = bodies[j0 + jb + lane];
        __syncwarp();
#pragma unroll 4
        for (int k = sub; k < cnt; k += G) {
          const vec4<T> sj = sh[wl][k];
          const T dx = sj.x - xi.x, dy = sj.y - xi.y, dz = sj.z - xi.z;
          const T r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
          const T inv = r2 > T(0) ? rsqrt_(r2) : T(0);
          const T qinv = sj.w * inv;
          const T inv3 = qinv * inv * inv;
          pot += qinv;
          ax = fma(dx, inv3, ax);
          ay = fma(dy, inv3, ay);
          az = fma(dz, inv3, az);
        }
      }
      if (COMP) {
        comp_add(acc[0], pot);
        comp_add(acc[1], ax);
        comp_add(acc[2], ay);
        comp_add(acc[3], az);
      } else {
        acc[0].s += pot;
        acc[1].s += ax;
        acc[2].s += ay;
        acc[3].s += az;
      }
    }
    for (int o = 1; o < G; o <<= 1) {
#pragma unroll
      for (int d = 0; d < 4; d++) {
        Comp<T> r;
        r.s = __shfl_xor_sync(0xffffffffu, acc[d].s, o);
        r.e = __shfl_xor_sync(0xffffffffu, acc[d].e, o);
        if (COMP) comp_merge(acc[d], r);
        else acc[d].s += r.s;
      }
    }
    if (active && sub == 0) {
      trg_s[b0 + ti] = make_v4<T>(acc[0].s, acc[1].s, acc[2].s, acc[3].s);
      trg_e[b0 + ti] = make_v4<T>(acc[0].e, acc[1].e, acc[2].e, acc[3].e);
    }
  }
}

template <typename T> void run_p2p(Solver<T>& s) {
  if (s.nleaves == 0) return;
  constexpr bool comp = sizeof(T) == 4;
  k_p2p<T, comp><<<ceil_div(s.nleaves, kP2PWarps), 32 * kP2PWarps, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.p2p_off.p, s.p2p.p, s.c_ibody.p, s.c_nbody.p, s.bodies.p,
      (T)s.cfg.eps2, s.trg_s.p, s.trg_e.p);
  FMM_LAUNCH_CHECK();
}

template void run_p2p<float>(Solver<float>&);
template void run_p2p<double>(Solver<double>&);

}  // namespace fmmb200
