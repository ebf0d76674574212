// Cartesian-basis expansion kernels (P2M, M2M, M2L, L2L, L2P) for compile-time P.
// Same warp mappings as the spherical kernels; M2L is lane per source cell in both
// precisions (NTERM = 35 at P = 5 keeps the derivative tensor and the local expansion in
// registers).
#pragma once
#include <algorithm>

#include "fmm_cart_math.cuh"
#include "fmm_solver.cuh"

namespace fmmb200 {

template <typename T, int P> struct CartCfg {
  static constexpr int RS = cart::NT(P) | 1;
  static constexpr int BYTES = 32 * RS * (int)sizeof(T);
  static constexpr int W = 40960 / BYTES >= 4 ? 4 : (40960 / BYTES >= 2 ? 2 : 1);
};

template <typename T, int P>
__global__ void __launch_bounds__(32 * CartCfg<T, P>::W)
    k_cp2m(const int* __restrict__ leaves, int nleaves, const int* __restrict__ ibody,
           const int* __restrict__ nbody, vec4<T>* __restrict__ cX,
           const vec4<T>* __restrict__ bodies, T* __restrict__ M, int ncoef, int use_rmax,
           T theta, int write_r, int* __restrict__ body_leaf) {
  constexpr int NT = cart::NT(P), RS = CartCfg<T, P>::RS, KA = (NT + 31) / 32;
  constexpr int W = CartCfg<T, P>::W;
  __shared__ T rows[W][32 * RS];
  const int wl = threadIdx.x >> 5, lane = lane_id();
  const int w = blockIdx.x * W + wl;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const vec4<T> X = cX[c];
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
      T C[NT];
      C[0] = b.w;
      cart::power<T, P>(C, X.x - b.x, X.y - b.y, X.z - b.z);
      T* row = &rows[wl][lane * RS];
#pragma unroll
      for (int t = 0; t < NT; t++) row[t] = C[t];
      const T r = sqrt_rn(norm_rn(sub_rn(X.x, b.x), sub_rn(X.y, b.y), sub_rn(X.z, b.z)));
      rmax = r > rmax ? r : rmax;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KA; i++) {
      const int t = lane + 32 * i;
      if (t < NT)
        for (int r = 0; r < cnt; r++) acc[i] += rows[wl][r * RS + t];
    }
  }
#pragma unroll
  for (int i = 0; i < KA; i++) {
    const int t = lane + 32 * i;
    if (t < NT) M[(size_t)c * ncoef + t] = acc[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T v = __shfl_xor_sync(0xffffffffu, rmax, o);
    rmax = v > rmax ? v : rmax;
  }
  if (lane == 0 && write_r) {
    T R = X.w;
    if (use_rmax) R = rmax < R ? rmax : R;
    cX[c].w = div_rn(R, theta);
  }
}

template <typename T, int NT>
__device__ __forceinline__ void spread_c(const T* C, T* sc, int lane) {
#pragma unroll
  for (int t = 0; t < NT; t++)
    if ((t & 31) == lane) sc[t] = C[t];
}

// M2M, thread per parent cell of the level: the children's multipoles shifted one after
// the other (cart::m2m_child, unrolled) into the parent's expansion held in registers
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cm2m(int lo, int hi, const int* __restrict__ npos, const int* __restrict__ ichild,
           const int* __restrict__ nchild, vec4<T>* __restrict__ cX, T* __restrict__ M,
           int ncoef, int use_rmax, T theta, int write_r) {
  constexpr int NT = cart::NT(P);
  const int v = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= hi) return;
  const int c = npos[v];
  const int nch = nchild[c];
  if (nch == 0) return;
  const int c0 = ichild[c];
  const vec4<T> Xp = cX[c];
  T acc[NT];
#pragma unroll
  for (int t = 0; t < NT; t++) acc[t] = 0;
  T rmax = 0;
  for (int ch = 0; ch < nch; ch++) {
    const int cc = c0 + ch;
    const vec4<T> Xc = cX[cc];
    T C[NT];
    C[0] = 1;
    cart::power<T, P>(C, Xp.x - Xc.x, Xp.y - Xc.y, Xp.z - Xc.z);
    if constexpr (3 * NT * sizeof(T) <= 1024) {  // the child's expansion in registers too
      T Mc[NT];
#pragma unroll
      for (int t = 0; t < NT; t++) Mc[t] = M[(size_t)cc * ncoef + t];
      cart::m2m_child<T, P>(C, Mc, acc);
    } else {  // FP64 at P >= 6: read through L1 where used
      cart::m2m_child<T, P>(C, M + (size_t)cc * ncoef, acc);
    }
    const T d = sqrt_rn(norm_rn(sub_rn(Xp.x, Xc.x), sub_rn(Xp.y, Xc.y), sub_rn(Xp.z, Xc.z)));
    const T r = add_rn(d, Xc.w);
    rmax = r > rmax ? r : rmax;
  }
#pragma unroll
  for (int t = 0; t < NT; t++) M[(size_t)c * ncoef + t] = acc[t];
  if (write_r) {
    T R = Xp.w;
    if (use_rmax) R = rmax < R ? rmax : R;
    cX[c].w = div_rn(R, theta);
  }
}

// M2L, thread per target: the targets with pairs in order of descending pair count (so
// the threads of a warp run about the same number of pairs), each contracting its sources
// one after the other into the whole local expansion held in registers; no reduction.
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cm2l(int ntgt, const int* __restrict__ tgt, const int* __restrict__ off,
           const unsigned long long* __restrict__ pairs, const vec4<T>* __restrict__ cX,
           const T* __restrict__ M, T* __restrict__ L, int ncoef, T cycle) {
  constexpr int NT = cart::NT(P);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntgt) return;
  const int c = tgt[t];
  const int s0 = off[c], s1 = off[c + 1];
  const vec4<T> Xi = cX[c];
  T acc[NT];
#pragma unroll
  for (int k = 0; k < NT; k++) acc[k] = 0;
  for (int s = s0; s < s1; s++) {
    const unsigned src = (unsigned)pairs[s];
    const int j = pair_cell(src);
    T px, py, pz;  // periodic shift of the source (0 without images)
    img_shift<T>(pair_img(src), cycle, px, py, pz);
    const vec4<T> Xj = cX[j];
    // dX = Xi - Xj - Xperiodic (kernels/LaplaceCartesianCPU.cxx:658-673)
    const T dx = Xi.x - Xj.x - px, dy = Xi.y - Xj.y - py, dz = Xi.z - Xj.z - pz;
    const T invR2 = T(1) / (dx * dx + dy * dy + dz * dz);
    T C[NT];
    cart::derivs<T, P>(C, dx, dy, dz, invR2, sqrt(invR2));
    cart::m2l_pair<T, P>(C, M + (size_t)j * ncoef, acc);
  }
  T* Lc = L + (size_t)c * ncoef;
#pragma unroll
  for (int k = 0; k < NT; k++) Lc[k] += acc[k];
}

// L2L, thread per cell of the level: the parent's local expansion shifted to the cell
// (cart::l2l_child, unrolled) and added to the cell's
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cl2l(int lo, int hi, const int* __restrict__ npos, const int* __restrict__ iparent,
           const vec4<T>* __restrict__ cX, T* __restrict__ L, int ncoef,
           const int4* __restrict__ info, const int* __restrict__ range) {
  constexpr int NT = cart::NT(P);
  const int v = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= hi) return;
  const int c = npos[v];
  if (range && !part_holds(info[c], range)) return;  // no body of this part below the cell
  const int p = iparent[c];
  const vec4<T> Xc = cX[c], Xp = cX[p];
  T C[NT], Lp[NT];
  C[0] = 1;
  cart::power<T, P>(C, Xc.x - Xp.x, Xc.y - Xp.y, Xc.z - Xp.z);
#pragma unroll
  for (int t = 0; t < NT; t++) Lp[t] = L[(size_t)p * ncoef + t];
  cart::l2l_child<T, P>(C, Lp, L + (size_t)c * ncoef);
}

// L2P with one thread per body (tree order), its leaf from the map P2M wrote, the leaf's
// local expansion read through L1 (the bodies of a warp share one to three leaves)
template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cl2p_bodies(int n, const int* __restrict__ body_leaf, const vec4<T>* __restrict__ cX,
                  const vec4<T>* __restrict__ bodies, const T* __restrict__ L, int ncoef,
                  vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e,
                  const int* __restrict__ range) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (range && (i < range[0] || i >= range[1])) return;  // another part's body
  const int c = body_leaf[i];
  if (c < 0) return;  // a body outside the cells of a single-operator call
  const vec4<T> X = cX[c];
  const vec4<T> b = bodies[i];
  T pot, gx, gy, gz;
  cart::l2p_body<T, P>(b.x - X.x, b.y - X.y, b.z - X.z, L + (size_t)c * ncoef, pot, gx, gy, gz);
  vec4<T> s = trg_s[i], e = trg_e[i];
  Comp<T> a0 = {s.x, e.x}, a1 = {s.y, e.y}, a2 = {s.z, e.z}, a3 = {s.w, e.w};
  comp_add(a0, pot);
  comp_add(a1, gx);
  comp_add(a2, gy);
  comp_add(a3, gz);
  trg_s[i] = make_v4<T>(a0.s, a1.s, a2.s, a3.s);
  trg_e[i] = make_v4<T>(a0.e, a1.e, a2.e, a3.e);
}

template <typename T, int P> static void p2m_(Solver<T>& s) {
  constexpr int W = CartCfg<T, P>::W;
  if (!s.nleaves) return;
  s.body_leaf.ensure(std::max(s.n, 1));
  k_cp2m<T, P><<<ceil_div(s.nleaves, W), 32 * W, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.c_ibody.p, s.c_nbody.p, s.cX.p, s.bodies.p, s.M.p, s.ncoef,
      s.cfg.use_rmax, (T)s.cfg.theta, s.write_r, s.body_leaf.p);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void m2m_(Solver<T>& s, int lo, int hi) {
  k_cm2m<T, P><<<ceil_div(hi - lo, 128), 128, 0, s.stream>>>(lo, hi, s.npos.p, s.c_ichild.p,
                                                             s.c_nchild.p, s.cX.p, s.M.p,
                                                             s.ncoef, s.cfg.use_rmax,
                                                             (T)s.cfg.theta, s.write_r);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void m2l_(Solver<T>& s) {
  if (!s.m2l_ntgt) return;
  k_cm2l<T, P><<<ceil_div(s.m2l_ntgt, 128), 128, 0, s.stream>>>(
      s.m2l_ntgt, s.m2l_tgt.p, s.m2l_off.p, s.m2l.p, s.cX.p, s.M.p, s.L.p, s.ncoef,
      (T)s.cfg.cycle);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void l2l_(Solver<T>& s, int lo, int hi) {
  k_cl2l<T, P><<<ceil_div(hi - lo, 128), 128, 0, s.stream>>>(lo, hi, s.npos.p, s.c_iparent.p,
                                                             s.cX.p, s.L.p, s.ncoef,
                                                             s.c_info.p, s.part_ptr());
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void l2p_(Solver<T>& s) {
  if (!s.nleaves) return;
  k_cl2p_bodies<T, P><<<ceil_div(s.n, 128), 128, 0, s.stream>>>(
      s.n, s.body_leaf.p, s.cX.p, s.bodies.p, s.L.p, s.ncoef, s.trg_s.p, s.trg_e.p,
      s.part_ptr());
  FMM_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- periodic far field
// Traversal::traversePeriodic (include/traversal.h:127-185) on this basis, one root per
// solve of the batch.  Per sub-level of images: the periodic cell (the root's multipole, at
// the root's centre) sends M2L into the root from the 26 x 27 shifts (3 ix + cx, ...) cycle,
// |i|, |c| <= 1, (ix, iy, iz) != 0 (k_cper_m2l: one thread per shift, the whole local
// expansion in registers as in k_cm2l; k_cper_reduce adds the 702 terms to the root's local
// expansion in the reference's loop order); then the periodic cell becomes the M2M of its
// 26 copies shifted by (ix, iy, iz) cycle, (ix, iy, iz) != 0 (k_cper_m2m; the unshifted copy
// is not among them, as in the reference), and the period grows three times.
constexpr int kCPerShifts = 26 * 27;

__device__ __forceinline__ void cper_outer(int o, int& ix, int& iy, int& iz) {
  const int q = o < 13 ? o : o + 1;  // the 26 of {-1,0,1}^3 other than (0,0,0), loop order
  ix = q / 9 - 1;
  iy = (q / 3) % 3 - 1;
  iz = q % 3 - 1;
}

template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cper_m2l(int nroots, const T* __restrict__ Mp, T cycle, int ncoef, T* __restrict__ contrib) {
  constexpr int NT = cart::NT(P);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nroots * kCPerShifts) return;
  const int r = t / kCPerShifts, sidx = t % kCPerShifts;
  int ix, iy, iz;
  cper_outer(sidx / 27, ix, iy, iz);
  const int c = sidx % 27, cx = c / 9 - 1, cy = (c / 3) % 3 - 1, cz = c % 3 - 1;
  // dX = Ci0->X - Ci->X - Xperiodic with Ci at the root's own centre: -Xperiodic
  const T dx = T(0) - (T)(ix * 3 + cx) * cycle, dy = T(0) - (T)(iy * 3 + cy) * cycle,
          dz = T(0) - (T)(iz * 3 + cz) * cycle;
  const T invR2 = T(1) / (dx * dx + dy * dy + dz * dz);
  T C[NT], acc[NT];
  cart::derivs<T, P>(C, dx, dy, dz, invR2, sqrt(invR2));
#pragma unroll
  for (int u = 0; u < NT; u++) acc[u] = 0;
  cart::m2l_pair<T, P>(C, Mp + (size_t)r * ncoef, acc);
  T* out = contrib + (size_t)t * NT;
#pragma unroll
  for (int u = 0; u < NT; u++) out[u] = acc[u];
}

template <typename T>
__global__ void k_cper_reduce(int nroots, int nt, const int* __restrict__ root_cell,
                              const T* __restrict__ contrib, T* __restrict__ L, int ncoef) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nroots * nt) return;
  const int r = t / nt, e = t % nt;
  T acc = L[(size_t)root_cell[r] * ncoef + e];
  for (int q = 0; q < kCPerShifts; q++) acc += contrib[((size_t)r * kCPerShifts + q) * nt + e];
  L[(size_t)root_cell[r] * ncoef + e] = acc;
}

template <typename T, int P>
__global__ void __launch_bounds__(32)
    k_cper_m2m(const T* __restrict__ Mp, const int* __restrict__ root_cell,
               const vec4<T>* __restrict__ cX, T cycle, int ncoef, T* __restrict__ Mout) {
  constexpr int NT = cart::NT(P), KO = (NT + 31) / 32;
  __shared__ T sc[NT], sm[NT];
  const int lane = lane_id(), r = blockIdx.x;
  const vec4<T> X = cX[root_cell[r]];
  for (int t = lane; t < NT; t += 32) sm[t] = Mp[(size_t)r * ncoef + t];
  T acc[KO];
  int ox[KO], oy[KO], oz[KO];
#pragma unroll
  for (int i = 0; i < KO; i++) {
    acc[i] = 0;
    cart::mi_of(lane + 32 * i, ox[i], oy[i], oz[i]);
  }
  for (int o = 0; o < 26; o++) {
    int ix, iy, iz;
    cper_outer(o, ix, iy, iz);
    // child centre X + (ix, iy, iz) cycle, then dX = Xparent - Xchild as the reference rounds
    const T xc = X.x + (T)ix * cycle, yc = X.y + (T)iy * cycle, zc = X.z + (T)iz * cycle;
    {
      T C[NT];
      C[0] = 1;
      cart::power<T, P>(C, X.x - xc, X.y - yc, X.z - zc);
      __syncwarp();
      spread_c<T, NT>(C, sc, lane);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KO; i++)
      if (lane + 32 * i < NT) acc[i] += cart::m2m_term<T>(ox[i], oy[i], oz[i], sc, sm);
  }
#pragma unroll
  for (int i = 0; i < KO; i++)
    if (lane + 32 * i < NT) Mout[(size_t)r * ncoef + lane + 32 * i] = acc[i];
}

template <typename T>
__global__ void k_cper_init(int nroots, const int* __restrict__ root_cell,
                            const T* __restrict__ M, int ncoef, T* __restrict__ Mp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nroots * ncoef) return;
  const int r = t / ncoef, e = t % ncoef;
  Mp[t] = M[(size_t)root_cell[r] * ncoef + e];
}

template <typename T, int P> static void cperiodic_(Solver<T>& s) {
  constexpr int NT = cart::NT(P);
  const int R = s.nroots;
  if (s.cfg.images < 2 || R == 0) return;
  s.pM.ensure((size_t)R * s.ncoef);
  s.pM2.ensure((size_t)R * s.ncoef);
  s.pC.ensure((size_t)R * kCPerShifts * NT);
  s.c_root_cells.ensure(R);
  FMM_CUDA(cudaMemcpyAsync(s.c_root_cells.p, s.root_cell.data(), sizeof(int) * R,
                           cudaMemcpyHostToDevice, s.stream));
  k_cper_init<T><<<ceil_div((long long)R * s.ncoef, 256), 256, 0, s.stream>>>(
      R, s.c_root_cells.p, s.M.p, s.ncoef, s.pM.p);
  FMM_LAUNCH_CHECK();
  T cycle = (T)s.cfg.cycle;
  for (int level = 0; level < s.cfg.images - 1; level++) {
    k_cper_m2l<T, P><<<ceil_div(R * kCPerShifts, 128), 128, 0, s.stream>>>(R, s.pM.p, cycle,
                                                                            s.ncoef, s.pC.p);
    FMM_LAUNCH_CHECK();
    k_cper_reduce<T><<<ceil_div((long long)R * NT, 128), 128, 0, s.stream>>>(
        R, NT, s.c_root_cells.p, s.pC.p, s.L.p, s.ncoef);
    FMM_LAUNCH_CHECK();
    k_cper_m2m<T, P><<<R, 32, 0, s.stream>>>(s.pM.p, s.c_root_cells.p, s.cX.p, cycle, s.ncoef,
                                             s.pM2.p);
    FMM_LAUNCH_CHECK();
    std::swap(s.pM, s.pM2);
    cycle = cycle * (T)3;
  }
}

// fill the dispatch table for one (precision, order); one object file per instantiation
template <typename T, int P> void cart_fill(ExpansionOps<T>* ops) {
  ops->periodic = &cperiodic_<T, P>;
  ops->p2m = &p2m_<T, P>;
  ops->m2m_level = &m2m_<T, P>;
  ops->m2l = &m2l_<T, P>;
  ops->l2l_level = &l2l_<T, P>;
  ops->l2p = &l2p_<T, P>;
}

}  // namespace fmmb200
