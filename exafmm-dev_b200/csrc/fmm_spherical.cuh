// Spherical-basis expansion kernels (P2M, M2M, M2L, L2L, L2P) for compile-time P.
//
// Mappings (the same kernels in FP32 and FP64; register and thread budgets per precision):
//   P2M  warp per leaf, lane per body; each lane's q conj(Y) row goes to shared memory and
//        the warp sums columns in body order, so M[0] is the reference's sequential sum.
//   M2M  8 lanes per parent, one child each, compile-time indices; children summed in a
//        fixed order and the monopole in the reference's child order
//        (include/up_down_pass.h:79-80 / LaplaceSphericalCPU.cxx:143).
//   M2L  warp per target cell, lane per source cell, each pair contracted in the source's
//        azimuthal frame with the harmonics and the local expansion held in registers,
//        passes over the output degrees, one warp reduction per target.
//   L2L  thread per cell, the parent's local staged in the thread's row of shared memory.
//   L2P  thread per body, harmonics generated and consumed on the fly.
// setRmax / R /= theta (include/up_down_pass.h:51-67, :81-82) are fused into P2M and M2M.
#pragma once
#include <algorithm>

#include "fmm_solver.cuh"
#include "fmm_sph_math.cuh"

namespace fmmb200 {

// P2M keeps one row of 2 NT (+1 pad) values per lane in shared memory: as many warps per
// block as fit in 40 KB of static shared memory.
template <typename T, int P> struct P2MCfg {
  static constexpr int RS = (2 * sph::NT(P)) | 1;
  static constexpr int BYTES = 32 * RS * (int)sizeof(T);
  static constexpr int W = 40960 / BYTES >= 4 ? 4 : (40960 / BYTES >= 2 ? 2 : 1);
};

// ---------------------------------------------------------------- P2M (+ setRmax)
template <typename T, int P>
__global__ void __launch_bounds__(32 * P2MCfg<T, P>::W)
    k_p2m(const int* __restrict__ leaves, int nleaves, const int* __restrict__ ibody,
          const int* __restrict__ nbody, vec4<T>* __restrict__ cX,
          const vec4<T>* __restrict__ bodies, T* __restrict__ M, int ncoef, int use_rmax,
          T theta, int write_r, int* __restrict__ body_leaf) {
  constexpr int NT = sph::NT(P), NC = 2 * NT, RS = NC | 1, KA = (NC + 31) / 32;
  constexpr int W = P2MCfg<T, P>::W;
  __shared__ T rows[W][32 * RS];
  const int wl = threadIdx.x >> 5, lane = lane_id();
  const int w = blockIdx.x * W + wl;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const vec4<T> C = cX[c];
  T acc[KA];
#pragma unroll
  for (int i = 0; i < KA; i++) acc[i] = 0;
  T rmax = 0;
  for (int base = 0; base < nb; base += 32) {
    const int cnt = min(32, nb - base);
    __syncwarp();
    if (lane < cnt) {
      body_leaf[b0 + base + lane] = c;
      const vec4<T> b = bodies[b0 + base + lane];
      const T dx = b.x - C.x, dy = b.y - C.y, dz = b.z - C.z;
      T yr[NT], yi[NT];
      sph::Angles<T> a = sph::angles(dx, dy, dz);
      sph::multipole<T, P>(a, a.r, yr, yi);
      T* row = &rows[wl][lane * RS];
#pragma unroll
      for (int t = 0; t < NT; t++) {
        row[2 * t] = b.w * yr[t];
        row[2 * t + 1] = -(b.w * yi[t]);
      }
      const T r = sqrt_rn(norm_rn(sub_rn(C.x, b.x), sub_rn(C.y, b.y), sub_rn(C.z, b.z)));
      rmax = r > rmax ? r : rmax;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KA; i++) {
      const int t = lane + 32 * i;
      if (t < NC)
        for (int r = 0; r < cnt; r++) acc[i] += rows[wl][r * RS + t];
    }
  }
#pragma unroll
  for (int i = 0; i < KA; i++) {
    const int t = lane + 32 * i;
    if (t < NC) M[(size_t)c * ncoef + t] = acc[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T v = __shfl_xor_sync(0xffffffffu, rmax, o);
    rmax = v > rmax ? v : rmax;
  }
  if (lane == 0 && write_r) {
    T R = C.w;
    if (use_rmax) R = rmax < R ? rmax : R;
    cX[c].w = div_rn(R, theta);
  }
}

// write the register harmonics of one lane's pair into shared memory, entry t by lane t%32
template <typename T, int NT>
__device__ __forceinline__ void spread_y(const T* yr, const T* yi, T* sy, int lane) {
#pragma unroll
  for (int t = 0; t < NT; t++)
    if ((t & 31) == lane) {
      sy[t] = yr[t];
      sy[NT + t] = yi[t];
    }
}

__device__ __forceinline__ void jk_of(int t, int& j, int& k) {
  j = 0;
  while ((j + 1) * (j + 2) / 2 <= t) j++;
  k = t - j * (j + 1) / 2;
}

// ---------------------------------------------------------------- M2M (+ setRmax)
// output degrees per M2M / L2L pass: at most 24 complex outputs per pass in FP32, 12 in
// FP64 (the same registers)
template <typename T> __host__ __device__ constexpr int tr_pass_outs() {
  return sizeof(T) == 4 ? 24 : 12;
}
template <typename T>
__host__ __device__ constexpr int tr_pass_end(int P, int J0) {
  int j = J0 + 1;
  while (j < P && sph::NT(j + 1) - sph::NT(J0) <= tr_pass_outs<T>()) j++;
  return j;
}

// M2M passes for one child lane; outputs summed over the 8-lane group and written.
template <typename T, int P, int J0>
__device__ __forceinline__ void m2m_passes(const T* yr, const T* yi, const T* Mc, bool has,
                                           int slot, T* Mp, T m0) {
  if constexpr (J0 < P) {
    constexpr int J1 = tr_pass_end<T>(P, J0);
    constexpr int NO = 2 * (sph::sidx(J1, 0) - sph::sidx(J0, 0));
    T acc[NO];
#pragma unroll
    for (int t = 0; t < NO; t++) acc[t] = 0;
    if (has) sph::m2m_range<T, P, J0, J1>(yr, yi, Mc, acc);
#pragma unroll
    for (int o = 1; o < 8; o <<= 1)
#pragma unroll
      for (int t = 0; t < NO; t++) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], o);
    if (J0 == 0) acc[0] = m0;
    if (Mp) {
#pragma unroll
      for (int t = 0; t < NO; t++)
        if ((t & 7) == slot) Mp[2 * sph::sidx(J0, 0) + t] = acc[t];
    }
    m2m_passes<T, P, J1>(yr, yi, Mc, has, slot, Mp, m0);
  }
}

// M2M (either precision): 8 lanes per parent (one per child slot), 4 parents per warp;
// each lane translates its child with compile-time indices, the group sums in a fixed
// order, and the monopole is re-summed in child order (the reference's sequence) so that
// the radii of the error-optimised MAC see the same M[0] bits.
// Threads per block of the M2M / L2L kernels (64 in FP32, 32 in FP64: the same shared
// memory); each thread stages the expansion it translates (its child's multipole, its
// parent's local) in its own row of shared memory first, with all the loads issued at once:
// read term by term from global memory, their latencies added up along the translation's
// dependent chain (~40 us per level).
template <typename T> constexpr int tr_threads() { return sizeof(T) == 4 ? 64 : 32; }

template <typename T, int P>
__global__ void __launch_bounds__(tr_threads<T>())
    k_m2m_reg(int lo, int hi, const int* __restrict__ npos, const int* __restrict__ ichild,
              const int* __restrict__ nchild, vec4<T>* __restrict__ cX, T* __restrict__ M,
              int ncoef, int use_rmax, T theta, int write_r) {
  constexpr int NT = sph::NT(P), STR = (2 * NT) | 1;  // odd row stride: no bank conflicts
  __shared__ T rows[tr_threads<T>() * STR];
  T* row = rows + threadIdx.x * STR;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = lo + (gt >> 3);
  const int slot = gt & 7;
  int c = 0, nch = 0, c0 = 0;
  if (v < hi) {
    c = npos[v];
    nch = nchild[c];
    c0 = ichild[c];
  }
  const bool has = slot < nch;
  T rr = 0;
  vec4<T> Xp = make_v4<T>(0, 0, 0, 0);
  if (v < hi) Xp = cX[c];
  T yr[NT], yi[NT];
  const T* Mc = M;
  if (has) {
    const int cc = c0 + slot;
    const T* src = M + (size_t)cc * ncoef;
#pragma unroll
    for (int t = 0; t < NT; t++) sph::load_pair(src + 2 * t, row[2 * t], row[2 * t + 1]);
    const vec4<T> Xc = cX[cc];
    sph::Angles<T> a = sph::angles(Xp.x - Xc.x, Xp.y - Xc.y, Xp.z - Xc.z);
    sph::multipole<T, P>(a, a.r, yr, yi);
    Mc = row;
    rr = add_rn(sqrt_rn(norm_rn(sub_rn(Xp.x, Xc.x), sub_rn(Xp.y, Xc.y), sub_rn(Xp.z, Xc.z))), Xc.w);
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    const T x = __shfl_xor_sync(0xffffffffu, rr, o);
    rr = x > rr ? x : rr;
  }
  T m0 = 0;
  if (slot == 0)
    for (int k = 0; k < nch; k++) m0 = add_rn(m0, M[(size_t)(c0 + k) * ncoef]);
  const bool write = v < hi && nch > 0;
  m2m_passes<T, P, 0>(yr, yi, Mc, has, slot, write ? M + (size_t)c * ncoef : nullptr, m0);
  if (write && slot == 0 && write_r) {
    T R = Xp.w;
    if (use_rmax) R = rr < R ? rr : R;
    cX[c].w = div_rn(R, theta);
  }
}

template <typename T, int P, int J0>
__device__ __forceinline__ void l2l_passes(const T* yr, const T* yi, const T* Lp, T* Lc) {
  if constexpr (J0 < P) {
    constexpr int J1 = tr_pass_end<T>(P, J0);
    constexpr int NO = 2 * (sph::sidx(J1, 0) - sph::sidx(J0, 0));
    T acc[NO];
#pragma unroll
    for (int t = 0; t < NO; t++) acc[t] = Lc[2 * sph::sidx(J0, 0) + t];
    sph::l2l_range<T, P, J0, J1>(yr, yi, Lp, acc);
#pragma unroll
    for (int t = 0; t < NO; t++) Lc[2 * sph::sidx(J0, 0) + t] = acc[t];
    l2l_passes<T, P, J1>(yr, yi, Lp, Lc);
  }
}

// L2L (either precision): thread per cell, compile-time indices, the parent's local staged
// in the thread's shared row.
template <typename T, int P>
__global__ void __launch_bounds__(tr_threads<T>())
    k_l2l_reg(int lo, int hi, const int* __restrict__ npos, const int* __restrict__ iparent,
              const vec4<T>* __restrict__ cX, T* __restrict__ L, int ncoef,
              const int4* __restrict__ info, const int* __restrict__ range) {
  constexpr int NT = sph::NT(P), STR = (2 * NT) | 1;
  __shared__ T rows[tr_threads<T>() * STR];
  T* row = rows + threadIdx.x * STR;
  const int v = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= hi) return;
  const int c = npos[v];
  if (range && !part_holds(info[c], range)) return;  // no body of this part below the cell
  const int p = iparent[c];
  const T* src = L + (size_t)p * ncoef;
#pragma unroll
  for (int t = 0; t < NT; t++) sph::load_pair(src + 2 * t, row[2 * t], row[2 * t + 1]);
  const vec4<T> Xc = cX[c], Xp = cX[p];
  T yr[NT], yi[NT];
  sph::Angles<T> a = sph::angles(Xc.x - Xp.x, Xc.y - Xp.y, Xc.z - Xp.z);
  sph::multipole<T, P>(a, a.r, yr, yi);
  l2l_passes<T, P, 0>(yr, yi, row, L + (size_t)c * ncoef);
}

// ---------------------------------------------------------------- M2L
// Warp per target, lane per source cell, harmonics and local expansion in registers, one
// warp reduction per target cell at the end (either precision).  Each pair is contracted in
// the source's azimuthal frame (m2l_pair_rot: real harmonic factors, half the multiply-adds
// of the complex form).  The outputs are split into passes over their degree (separate
// launches) so that each pass's registers stay within its block's share.
// Passes over the output degrees.  Registers of a pass [J0, J1) (besides the phases
// e^(i m beta)): the real harmonic factors of degrees >= J0, the accumulators (two per
// output), and either the pair's rotated sums A (two per output: source coefficients
// streamed, m2l_pair_rot) or the rotated source coefficients of degrees < P - J0 (two per
// coefficient: outputs streamed, m2l_pair_rot_out).  The last pass streams its outputs once
// the remaining degrees fit OUT values; the passes before it stream the source and add
// degrees while they fit IN values.
//   FP32: 12 warps per block (3 per SM sub-partition, whose 16 K registers then allow 168
//         per thread); P = 10 takes the passes [0, 5) and [5, 10), at 168 registers each,
//         the second with a small spill.
//   FP64: 8 warps per block (255 registers per thread), the budgets in values about half
//         of FP32's in registers; P = 10 takes four passes, none spilling.
template <typename T> struct M2LBudget {
  static constexpr int W = sizeof(T) == 4 ? 12 : 8;
  static constexpr int IN = sizeof(T) == 4 ? 139 : 100;
  static constexpr int OUT = sizeof(T) == 4 ? 149 : 105;
};
__host__ __device__ constexpr int m2l_regs_out(int P, int J0) {
  return sph::NT(P) - sph::sidx(J0, 0) + 2 * (sph::NT(P) - sph::sidx(J0, 0)) +
         2 * sph::NT(P - J0);
}
template <typename T> __host__ __device__ constexpr bool m2l_pass_out(int P, int J0) {
  return m2l_regs_out(P, J0) <= M2LBudget<T>::OUT;
}
// A source-streaming pass takes every degree its registers hold: it runs faster per term
// than the output-streaming pass that finishes the remaining degrees.
template <typename T> __host__ __device__ constexpr int m2l_pass_end(int P, int J0) {
  if (m2l_pass_out<T>(P, J0)) return P;
  const int rho = sph::NT(P) - sph::sidx(J0, 0);
  int j = J0, outs = 0;
  while (j < P) {
    const int o = outs + j + 1;
    if (j > J0 && rho + 4 * o > M2LBudget<T>::IN)
      break;
    outs = o;
    j++;
  }
  return j;
}

// Each warp runs its target's batches of 32 sources on its own; targets arrive ordered by
// their number of batches, so the warps of a block have about the same amount of work and
// the block's registers free up together.  (Holding a block's warps in lockstep with a
// barrier per batch, so that they share fetched instruction lines, measured 3 % slower at
// P = 10: the warps waited at the barriers.)
template <typename T, int P, int J0, int J1, int W>
__global__ void __launch_bounds__(32 * W)
    k_m2l_reg(int ntgt, const int* __restrict__ tgt, const int* __restrict__ off,
              const unsigned long long* __restrict__ pairs, const vec4<T>* __restrict__ cX,
              const T* __restrict__ M, T* __restrict__ L, int ncoef, T cycle) {
  constexpr int NT = sph::NT(P);
  const int lane = lane_id();
  const int w = blockIdx.x * W + (threadIdx.x >> 5);
  if (w >= ntgt) return;
  const int c = tgt[w];
  const int s0 = off[c], s1 = off[c + 1];
  if (s1 == s0) return;
  const vec4<T> Xi = cX[c];
  T Lr[NT], Li[NT];
#pragma unroll
  for (int t = 0; t < NT; t++) Lr[t] = Li[t] = 0;
  for (int sb = s0; sb < s1; sb += 32) {
    const int s = sb + lane;
    if (s < s1) {
      const unsigned src = (unsigned)pairs[s];
      const int j = pair_cell(src);
      T px, py, pz;  // periodic shift of the source (0 without images)
      img_shift<T>(pair_img(src), cycle, px, py, pz);
      const vec4<T> Xj = cX[j];
      T rho[NT - sph::sidx(J0, 0)], cr[P], ci[P];
      T invr;
      sph::Angles<T> a =
          sph::angles_rs(Xi.x - Xj.x - px, Xi.y - Xj.y - py, Xi.z - Xj.z - pz, invr);
      sph::local_rho<T, P, J0>(a, invr, rho, cr, ci);
      if constexpr (m2l_pass_out<T>(P, J0))
        sph::m2l_pair_rot_out<T, P, J0, J1>(rho, cr, ci, M + (size_t)j * ncoef, Lr, Li);
      else
        sph::m2l_pair_rot<T, P, J0, J1>(rho, cr, ci, M + (size_t)j * ncoef, Lr, Li);
    }
  }
#pragma unroll
  for (int t = sph::sidx(J0, 0); t < sph::sidx(J1, 0); t++) {
    const T r = warp_sum(Lr[t]);
    const T i = warp_sum(Li[t]);
    if (lane == (t & 31)) {
      L[(size_t)c * ncoef + 2 * t] += r;
      L[(size_t)c * ncoef + 2 * t + 1] += i;
    }
  }
}

template <typename T, int P, int J0>
static void launch_m2l_passes(Solver<T>& s) {
  if constexpr (J0 < P) {
    constexpr int J1 = m2l_pass_end<T>(P, J0);
    constexpr int W = M2LBudget<T>::W;
    k_m2l_reg<T, P, J0, J1, W><<<ceil_div(s.m2l_ntgt, W), 32 * W, 0, s.stream>>>(
        s.m2l_ntgt, s.m2l_tgt.p, s.m2l_off.p, s.m2l.p, s.cX.p, s.M.p, s.L.p, s.ncoef,
        (T)s.cfg.cycle);
    FMM_LAUNCH_CHECK();
    launch_m2l_passes<T, P, J1>(s);
  }
}

// M2L output coefficient (j, k) from one source (:156-189), runtime indices
template <typename T>
__device__ __forceinline__ void m2l_term(int P, int j, int k, const T* y, const T* Mj, T& outr,
                                         T& outi) {
  const int NTy = P * (P + 1) / 2;  // y holds NT real parts, then NT imaginary parts
  T sr = 0, si = 0;
  for (int n = 0; n < P - j; n++) {
    const int a = j + n;
    for (int mu = 1; mu <= n; mu++) {
      const T mr = Mj[2 * sph::sidx(n, mu)], mi = Mj[2 * sph::sidx(n, mu) + 1];
      const T ur = y[sph::sidx(a, k + mu)], ui = y[NTy + sph::sidx(a, k + mu)];
      sr += mr * ur - mi * ui;
      si -= mr * ui + mi * ur;
    }
    for (int m = 0; m <= n; m++) {
      const T mr = Mj[2 * sph::sidx(n, m)], mi = Mj[2 * sph::sidx(n, m) + 1];
      T vr, vi;
      if (m >= k) {
        const T wr = y[sph::sidx(a, m - k)], wi = y[NTy + sph::sidx(a, m - k)];
        vr = mr * wr - mi * wi;
        vi = mr * wi + mi * wr;
      } else {
        const T wr = y[sph::sidx(a, k - m)], wi = y[NTy + sph::sidx(a, k - m)];
        vr = mr * wr + mi * wi;
        vi = mi * wr - mr * wi;
      }
      if ((k < m ? k : m) & 1) {
        sr -= vr;
        si -= vi;
      } else {
        sr += vr;
        si += vi;
      }
    }
  }
  if (j & 1) {
    sr = -sr;
    si = -si;
  }
  outr = sr;
  outi = si;
}

// L2P with one thread per body (tree order), its leaf from the map P2M wrote, the leaf's
// local expansion read through L1 (the bodies of a warp share one to three leaves): every
// lane busy whatever the leaf sizes; the arithmetic per body is that of k_l2p
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_l2p_bodies(int n, const int* __restrict__ body_leaf, const vec4<T>* __restrict__ cX,
                 const vec4<T>* __restrict__ bodies, const T* __restrict__ L, int ncoef,
                 vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e,
                 const int* __restrict__ range) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (range && (i < range[0] || i >= range[1])) return;  // another part's body
  const int c = body_leaf[i];
  if (c < 0) return;  // a body outside the cells of a single-operator call
  const vec4<T> C = cX[c];
  const vec4<T> b = bodies[i];
  T pot, gx, gy, gz;
  sph::l2p_body<T, P>(b.x - C.x, b.y - C.y, b.z - C.z, L + (size_t)c * ncoef, pot, gx, gy, gz);
  vec4<T> s = trg_s[i], e = trg_e[i];
  Comp<T> a0 = {s.x, e.x}, a1 = {s.y, e.y}, a2 = {s.z, e.z}, a3 = {s.w, e.w};
  comp_add(a0, pot);
  comp_add(a1, gx);
  comp_add(a2, gy);
  comp_add(a3, gz);
  trg_s[i] = make_v4<T>(a0.s, a1.s, a2.s, a3.s);
  trg_e[i] = make_v4<T>(a0.e, a1.e, a2.e, a3.e);
}

// ---------------------------------------------------------------- dispatch
template <typename T, int P> static void p2m_(Solver<T>& s) {
  constexpr int W = P2MCfg<T, P>::W;
  if (!s.nleaves) return;
  s.body_leaf.ensure(std::max(s.n, 1));
  k_p2m<T, P><<<ceil_div(s.nleaves, W), 32 * W, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.c_ibody.p, s.c_nbody.p, s.cX.p, s.bodies.p, s.M.p, s.ncoef,
      s.cfg.use_rmax, (T)s.cfg.theta, s.write_r, s.body_leaf.p);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void m2m_(Solver<T>& s, int lo, int hi) {
  constexpr int NTH = tr_threads<T>();
  k_m2m_reg<T, P><<<ceil_div(8LL * (hi - lo), NTH), NTH, 0, s.stream>>>(
      lo, hi, s.npos.p, s.c_ichild.p, s.c_nchild.p, s.cX.p, s.M.p, s.ncoef, s.cfg.use_rmax,
      (T)s.cfg.theta, s.write_r);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void m2l_(Solver<T>& s) { launch_m2l_passes<T, P, 0>(s); }
template <typename T, int P> static void l2l_(Solver<T>& s, int lo, int hi) {
  constexpr int NTH = tr_threads<T>();
  k_l2l_reg<T, P><<<ceil_div(hi - lo, NTH), NTH, 0, s.stream>>>(lo, hi, s.npos.p, s.c_iparent.p,
                                                                s.cX.p, s.L.p, s.ncoef,
                                                                s.c_info.p, s.part_ptr());
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void l2p_(Solver<T>& s) {
  if (!s.nleaves) return;
  k_l2p_bodies<T, P><<<ceil_div(s.n, 128), 128, 0, s.stream>>>(
      s.n, s.body_leaf.p, s.cX.p, s.bodies.p, s.L.p, s.ncoef, s.trg_s.p, s.trg_e.p,
      s.part_ptr());
  FMM_LAUNCH_CHECK();
}


// fill the dispatch table for one (precision, order); one object file per instantiation
// ---------------------------------------------------------------- periodic far field
// Traversal::traversePeriodic (include/traversal.h:127-185), one root per solve of the
// batch.  Per sub-level of images: the periodic cell (the root's multipole, at the root's
// centre) sends M2L into the root from the 26 x 27 shifts (3 ix + cx, ...) cycle, |i|,
// |c| <= 1, (ix, iy, iz) != 0 (k_per_m2l: one warp per shift, lanes over outputs; then
// k_per_reduce adds the 702 terms to the root's local expansion in the reference's loop
// order); then the periodic cell becomes the M2M of its 26 copies shifted by
// (ix, iy, iz) cycle, (ix, iy, iz) != 0 (k_per_m2m; as in the reference, the unshifted copy
// is not among them), and the period grows three times.
constexpr int kPerShifts = 26 * 27;

__device__ __forceinline__ void per_outer(int o, int& ix, int& iy, int& iz) {
  const int q = o < 13 ? o : o + 1;  // the 26 of {-1,0,1}^3 other than (0,0,0), loop order
  ix = q / 9 - 1;
  iy = (q / 3) % 3 - 1;
  iz = q % 3 - 1;
}

template <typename T, int P>
__global__ void __launch_bounds__(32)
    k_per_m2l(const T* __restrict__ Mp, T cycle, int ncoef, T* __restrict__ contrib) {
  constexpr int NT = sph::NT(P), NC = 2 * NT, KO = (NT + 31) / 32;
  __shared__ T sy[NC], sm[NC];
  const int lane = lane_id();
  const int sidx = blockIdx.x, r = blockIdx.y;
  int ix, iy, iz;
  per_outer(sidx / 27, ix, iy, iz);
  const int c = sidx % 27, cx = c / 9 - 1, cy = (c / 3) % 3 - 1, cz = c % 3 - 1;
  // dX = Ci0->X - Ci->X - Xperiodic with Ci at the root's own centre: -Xperiodic
  const T px = (T)(ix * 3 + cx) * cycle, py = (T)(iy * 3 + cy) * cycle,
          pz = (T)(iz * 3 + cz) * cycle;
  {
    T yr[NT], yi[NT];
    sph::Angles<T> a = sph::angles(T(0) - px, T(0) - py, T(0) - pz);
    sph::local<T, P>(a, yr, yi);
    spread_y<T, NT>(yr, yi, sy, lane);
    for (int t = lane; t < NC; t += 32) sm[t] = Mp[(size_t)r * ncoef + t];
  }
  __syncwarp();
  T* out = contrib + ((size_t)r * kPerShifts + sidx) * NC;
#pragma unroll
  for (int i = 0; i < KO; i++) {
    const int t = lane + 32 * i;
    if (t < NT) {
      int j, kk;
      jk_of(t, j, kk);
      T re, im;
      m2l_term<T>(P, j, kk, sy, sm, re, im);
      out[2 * t] = re;
      out[2 * t + 1] = im;
    }
  }
}

template <typename T>
__global__ void k_per_reduce(int nroots, int nc, const int* __restrict__ root_cell,
                             const T* __restrict__ contrib, T* __restrict__ L, int ncoef) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nroots * nc) return;
  const int r = t / nc, e = t % nc;
  T acc = L[(size_t)root_cell[r] * ncoef + e];
  for (int q = 0; q < kPerShifts; q++) acc += contrib[((size_t)r * kPerShifts + q) * nc + e];
  L[(size_t)root_cell[r] * ncoef + e] = acc;
}

template <typename T, int P>
__global__ void __launch_bounds__(32)
    k_per_m2m(const T* __restrict__ Mp, const int* __restrict__ root_cell,
              const vec4<T>* __restrict__ cX, T cycle, int ncoef, T* __restrict__ Mout) {
  constexpr int NT = sph::NT(P), NC = 2 * NT, KO = (NT + 31) / 32;
  __shared__ T sy[NC], sm[NC];
  const int lane = lane_id(), r = blockIdx.x;
  const vec4<T> X = cX[root_cell[r]];
  for (int t = lane; t < NC; t += 32) sm[t] = Mp[(size_t)r * ncoef + t];
  T ar[KO], ai[KO];
#pragma unroll
  for (int i = 0; i < KO; i++) ar[i] = ai[i] = 0;
  for (int o = 0; o < 26; o++) {
    int ix, iy, iz;
    per_outer(o, ix, iy, iz);
    // child centre X + (ix, iy, iz) cycle, then dX = Xparent - Xchild as the reference rounds
    const T xc = X.x + (T)ix * cycle, yc = X.y + (T)iy * cycle, zc = X.z + (T)iz * cycle;
    __syncwarp();
    {
      T yr[NT], yi[NT];
      sph::Angles<T> a = sph::angles(X.x - xc, X.y - yc, X.z - zc);
      sph::multipole<T, P>(a, a.r, yr, yi);
      spread_y<T, NT>(yr, yi, sy, lane);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KO; i++) {
      const int t = lane + 32 * i;
      if (t < NT) {
        int j, kk;
        jk_of(t, j, kk);
        T re, im;
        sph::m2m_term<T>(j, kk, sy, sy + NT, sm, re, im);
        ar[i] += re;
        ai[i] += im;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < KO; i++) {
    const int t = lane + 32 * i;
    if (t < NT) {
      Mout[(size_t)r * ncoef + 2 * t] = ar[i];
      Mout[(size_t)r * ncoef + 2 * t + 1] = ai[i];
    }
  }
}

template <typename T>
__global__ void k_per_init(int nroots, const int* __restrict__ root_cell, const T* __restrict__ M,
                           int ncoef, T* __restrict__ Mp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nroots * ncoef) return;
  const int r = t / ncoef, e = t % ncoef;
  Mp[t] = M[(size_t)root_cell[r] * ncoef + e];
}

template <typename T, int P> static void periodic_(Solver<T>& s) {
  const int R = s.nroots, nc = 2 * sph::NT(P);
  if (s.cfg.images < 2 || R == 0) return;
  s.pM.ensure((size_t)R * s.ncoef);
  s.pM2.ensure((size_t)R * s.ncoef);
  s.pC.ensure((size_t)R * kPerShifts * nc);
  s.c_root_cells.ensure(R);
  FMM_CUDA(cudaMemcpyAsync(s.c_root_cells.p, s.root_cell.data(), sizeof(int) * R,
                           cudaMemcpyHostToDevice, s.stream));
  k_per_init<T><<<ceil_div((long long)R * s.ncoef, 256), 256, 0, s.stream>>>(
      R, s.c_root_cells.p, s.M.p, s.ncoef, s.pM.p);
  FMM_LAUNCH_CHECK();
  T cycle = (T)s.cfg.cycle;
  for (int level = 0; level < s.cfg.images - 1; level++) {
    k_per_m2l<T, P><<<dim3(kPerShifts, R), 32, 0, s.stream>>>(s.pM.p, cycle, s.ncoef, s.pC.p);
    FMM_LAUNCH_CHECK();
    k_per_reduce<T><<<ceil_div((long long)R * nc, 128), 128, 0, s.stream>>>(
        R, nc, s.c_root_cells.p, s.pC.p, s.L.p, s.ncoef);
    FMM_LAUNCH_CHECK();
    k_per_m2m<T, P><<<R, 32, 0, s.stream>>>(s.pM.p, s.c_root_cells.p, s.cX.p, cycle, s.ncoef,
                                            s.pM2.p);
    FMM_LAUNCH_CHECK();
    std::swap(s.pM, s.pM2);
    cycle = cycle * (T)3;
  }
}

template <typename T, int P> void sph_fill(ExpansionOps<T>* ops) {
  ops->periodic = &periodic_<T, P>;
  ops->p2m = &p2m_<T, P>;
  ops->m2m_level = &m2m_<T, P>;
  ops->m2l = &m2l_<T, P>;
  ops->l2l_level = &l2l_<T, P>;
  ops->l2p = &l2p_<T, P>;
}

}  // namespace fmmb200
