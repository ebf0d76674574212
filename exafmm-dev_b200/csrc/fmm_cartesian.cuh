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
           T theta) {
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
  if (lane == 0) {
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

template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cm2m(int lo, int hi, const int* __restrict__ npos, const int* __restrict__ ichild,
           const int* __restrict__ nchild, vec4<T>* __restrict__ cX, T* __restrict__ M,
           int ncoef, int use_rmax, T theta) {
  constexpr int NT = cart::NT(P), KO = (NT + 31) / 32, W = 4;
  __shared__ T sc[W][NT], sm[W][NT];
  const int wl = threadIdx.x >> 5, lane = lane_id();
  const int v = lo + blockIdx.x * W + wl;
  if (v >= hi) return;
  const int c = npos[v];
  const int nch = nchild[c];
  if (nch == 0) return;
  const int c0 = ichild[c];
  const vec4<T> Xp = cX[c];
  T acc[KO];
  int ox[KO], oy[KO], oz[KO];
#pragma unroll
  for (int i = 0; i < KO; i++) {
    acc[i] = 0;
    cart::mi_of(lane + 32 * i, ox[i], oy[i], oz[i]);
  }
  T rmax = 0;
  for (int ch = 0; ch < nch; ch++) {
    const int cc = c0 + ch;
    const vec4<T> Xc = cX[cc];
    {
      T C[NT];
      C[0] = 1;
      cart::power<T, P>(C, Xp.x - Xc.x, Xp.y - Xc.y, Xp.z - Xc.z);
      __syncwarp();
      spread_c<T, NT>(C, sc[wl], lane);
      for (int t = lane; t < NT; t += 32) sm[wl][t] = M[(size_t)cc * ncoef + t];
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KO; i++)
      if (lane + 32 * i < NT) acc[i] += cart::m2m_term<T>(ox[i], oy[i], oz[i], sc[wl], sm[wl]);
    if (lane == ch) {
      const T d = sqrt_rn(norm_rn(sub_rn(Xp.x, Xc.x), sub_rn(Xp.y, Xc.y), sub_rn(Xp.z, Xc.z)));
      rmax = add_rn(d, Xc.w);
    }
  }
#pragma unroll
  for (int i = 0; i < KO; i++)
    if (lane + 32 * i < NT) M[(size_t)c * ncoef + lane + 32 * i] = acc[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T x = __shfl_xor_sync(0xffffffffu, rmax, o);
    rmax = x > rmax ? x : rmax;
  }
  if (lane == 0) {
    T R = Xp.w;
    if (use_rmax) R = rmax < R ? rmax : R;
    cX[c].w = div_rn(R, theta);
  }
}

template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cm2l(int ncells, const int* __restrict__ off, const unsigned long long* __restrict__ pairs,
           const vec4<T>* __restrict__ cX, const T* __restrict__ M, T* __restrict__ L, int ncoef) {
  constexpr int NT = cart::NT(P);
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = lane_id();
  if (c >= ncells) return;
  const int s0 = off[c], s1 = off[c + 1];
  if (s0 == s1) return;
  const vec4<T> Xi = cX[c];
  T acc[NT];
#pragma unroll
  for (int t = 0; t < NT; t++) acc[t] = 0;
  for (int s = s0 + lane; s < s1; s += 32) {
    const int j = pair_cell((unsigned)pairs[s]);  // no periodic images on this basis
    const vec4<T> Xj = cX[j];
    const T dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
    const T invR2 = T(1) / (dx * dx + dy * dy + dz * dz);
    T C[NT];
    cart::derivs<T, P>(C, dx, dy, dz, invR2, sqrt(invR2));
    cart::m2l_pair<T, P>(C, M + (size_t)j * ncoef, acc);
  }
#pragma unroll
  for (int t = 0; t < NT; t++) {
    const T r = warp_sum(acc[t]);
    if (lane == (t & 31)) L[(size_t)c * ncoef + t] += r;
  }
}

template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cl2l(int lo, int hi, const int* __restrict__ npos, const int* __restrict__ iparent,
           const vec4<T>* __restrict__ cX, T* __restrict__ L, int ncoef) {
  constexpr int NT = cart::NT(P), KO = (NT + 31) / 32, W = 4;
  __shared__ T sc[W][NT], sl[W][NT];
  const int wl = threadIdx.x >> 5, lane = lane_id();
  const int v = lo + blockIdx.x * W + wl;
  if (v >= hi) return;
  const int c = npos[v];
  const int p = iparent[c];
  const vec4<T> Xc = cX[c], Xp = cX[p];
  {
    T C[NT];
    C[0] = 1;
    cart::power<T, P>(C, Xc.x - Xp.x, Xc.y - Xp.y, Xc.z - Xp.z);
    spread_c<T, NT>(C, sc[wl], lane);
    for (int t = lane; t < NT; t += 32) sl[wl][t] = L[(size_t)p * ncoef + t];
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < KO; i++) {
    const int t = lane + 32 * i;
    if (t < NT) {
      int nx, ny, nz;
      cart::mi_of(t, nx, ny, nz);
      L[(size_t)c * ncoef + t] += cart::l2l_term<T>(P, nx, ny, nz, sc[wl], sl[wl]);
    }
  }
}

template <typename T, int P>
__global__ void __launch_bounds__(128)
    k_cl2p(const int* __restrict__ leaves, int nleaves, const int* __restrict__ ibody,
           const int* __restrict__ nbody, const vec4<T>* __restrict__ cX,
           const vec4<T>* __restrict__ bodies, const T* __restrict__ L, int ncoef,
           vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e) {
  constexpr int NT = cart::NT(P), W = 4;
  __shared__ T sl[W][NT];
  const int wl = threadIdx.x >> 5, lane = lane_id();
  const int w = blockIdx.x * W + wl;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const vec4<T> X = cX[c];
  for (int t = lane; t < NT; t += 32) sl[wl][t] = L[(size_t)c * ncoef + t];
  __syncwarp();
  for (int i = lane; i < nb; i += 32) {
    const vec4<T> b = bodies[b0 + i];
    T pot, gx, gy, gz;
    cart::l2p_body<T, P>(b.x - X.x, b.y - X.y, b.z - X.z, sl[wl], pot, gx, gy, gz);
    vec4<T> s = trg_s[b0 + i], e = trg_e[b0 + i];
    Comp<T> a0 = {s.x, e.x}, a1 = {s.y, e.y}, a2 = {s.z, e.z}, a3 = {s.w, e.w};
    comp_add(a0, pot);
    comp_add(a1, gx);
    comp_add(a2, gy);
    comp_add(a3, gz);
    trg_s[b0 + i] = make_v4<T>(a0.s, a1.s, a2.s, a3.s);
    trg_e[b0 + i] = make_v4<T>(a0.e, a1.e, a2.e, a3.e);
  }
}

template <typename T, int P> static void p2m_(Solver<T>& s) {
  constexpr int W = CartCfg<T, P>::W;
  if (!s.nleaves) return;
  k_cp2m<T, P><<<ceil_div(s.nleaves, W), 32 * W, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.c_ibody.p, s.c_nbody.p, s.cX.p, s.bodies.p, s.M.p, s.ncoef,
      s.cfg.use_rmax, (T)s.cfg.theta);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void m2m_(Solver<T>& s, int lo, int hi) {
  k_cm2m<T, P><<<ceil_div(hi - lo, 4), 128, 0, s.stream>>>(lo, hi, s.npos.p, s.c_ichild.p,
                                                             s.c_nchild.p, s.cX.p, s.M.p,
                                                             s.ncoef, s.cfg.use_rmax,
                                                             (T)s.cfg.theta);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void m2l_(Solver<T>& s) {
  k_cm2l<T, P><<<ceil_div(s.ncells, 4), 128, 0, s.stream>>>(s.ncells, s.m2l_off.p, s.m2l.p,
                                                              s.cX.p, s.M.p, s.L.p, s.ncoef);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void l2l_(Solver<T>& s, int lo, int hi) {
  k_cl2l<T, P><<<ceil_div(hi - lo, 4), 128, 0, s.stream>>>(lo, hi, s.npos.p, s.c_iparent.p,
                                                             s.cX.p, s.L.p, s.ncoef);
  FMM_LAUNCH_CHECK();
}
template <typename T, int P> static void l2p_(Solver<T>& s) {
  if (!s.nleaves) return;
  k_cl2p<T, P><<<ceil_div(s.nleaves, 4), 128, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.c_ibody.p, s.c_nbody.p, s.cX.p, s.bodies.p, s.L.p, s.ncoef,
      s.trg_s.p, s.trg_e.p);
  FMM_LAUNCH_CHECK();
}


// fill the dispatch table for one (precision, order); one object file per instantiation
template <typename T, int P> void cart_fill(ExpansionOps<T>* ops) {
  ops->periodic = nullptr;  // periodic images are spherical-basis only
  ops->p2m = &p2m_<T, P>;
  ops->m2m_level = &m2m_<T, P>;
  ops->m2l = &m2l_<T, P>;
  ops->l2l_level = &l2l_<T, P>;
  ops->l2p = &l2p_<T, P>;
}

}  // namespace fmmb200
