// Level-synchronous upward and downward passes (UpDownPass, include/up_down_pass.h).
//
// The reference walks the tree recursively: post-order P2M / M2M with setRmax and
// R /= theta (:45-84), then SetRopt over every cell (:15-42), and pre-order L2L / L2P
// (:87-111).  Here each tree level is one launch: P2M over all leaves, M2M from the
// deepest parent level up to the root, one launch of the error-optimised radius over all
// cells; after the traversal, L2L from level 1 down and L2P over all leaves.
#include <algorithm>

#include "fmm_solver.cuh"

namespace fmmb200 {

// SetRopt (include/up_down_pass.h:22-41) with the root coefficient of :125, evaluated in
// the reference's mix of real_t and double arithmetic.  Multipoles stay unnormalised
// here (the reference's MASS normalisation M[i] /= M[0] is a change of scale that the
// M2L / L2L of the MASS build undo again), so only |M[0]| enters.
// The monopole of each cell is read at M[c * stride] (the multipoles, stride ncoef, or the
// monopoles of the structure pass, stride 1).
template <typename T>
__global__ void k_ropt(int ncells, vec4<T>* __restrict__ cX, const T* __restrict__ M,
                       const int* __restrict__ croot, int ncoef, int P, T theta) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const T m0root = fabs(M[(size_t)croot[c] * ncoef]);  // the monopole of this cell's root
  const T omt = sub_rn((T)1, theta);
  const T cc = (T)__ddiv_rn(__ddiv_rn((double)mul_rn(omt, omt), pow((double)theta, (double)(P + 2))),
                           (double)powf((float)m0root, (float)(1.0 / 3)));
  T x = (T)__ddiv_rn(1.0, (double)theta);
  const T m0 = fabs(M[(size_t)c * ncoef]);
  const T a = mul_rn(cc, (T)powf((float)m0, (float)(1.0 / 3)));
  for (int i = 0; i < 5; i++) {
    const T q = add_rn(sub_rn(mul_rn(x, x), mul_rn((T)2, x)), (T)1);
    const T f = (T)__dsub_rn((double)q, __dmul_rn((double)a, pow((double)x, (double)(-P))));
    const T df = add_rn(sub_rn(mul_rn((T)(P + 2), x), (T)(2 * (P + 1))), div_rn((T)P, x));
    x = sub_rn(x, div_rn(f, df));
  }
  cX[c].w = mul_rn(cX[c].w, mul_rn(x, theta));
}

// The cell radii of the upward pass and the monopoles, without the expansions (the
// structure pass): setRmax and R /= theta (include/up_down_pass.h:45-84) with the same
// rounded arithmetic as the P2M / M2M kernels, and each monopole as the sum the P2M / M2M
// kernels form for M[0] (a leaf's charges in body order, then its children's monopoles in
// child order), so that radii, monopoles and the error-optimised radii match those of the
// expansion passes bit for bit.  It lets the traversal start while the expansions are
// still being formed.
// a warp per leaf: the bodies' distances to the centre 32 at a time (their maximum by
// shuffles: max is exact), the charges added in body order by lane 0 from shuffles
template <typename T>
__global__ void k_struct_leaves(const int* __restrict__ leaves, int nleaves,
                                const int* __restrict__ ibody, const int* __restrict__ nbody,
                                vec4<T>* __restrict__ cX, const vec4<T>* __restrict__ bodies,
                                T* __restrict__ m0, int use_rmax, T theta) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = lane_id();
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = ibody[c], nb = nbody[c];
  const vec4<T> C = cX[c];
  T rmax = 0, q = 0;
  for (int base = 0; base < nb; base += 32) {
    const int cnt = min(32, nb - base);
    vec4<T> b = make_v4<T>(C.x, C.y, C.z, 0);
    if (lane < cnt) b = bodies[b0 + base + lane];
    const T r = sqrt_rn(norm_rn(sub_rn(C.x, b.x), sub_rn(C.y, b.y), sub_rn(C.z, b.z)));
    rmax = r > rmax ? r : rmax;
    for (int i = 0; i < cnt; i++) {
      const T qi = __shfl_sync(0xffffffffu, b.w, i);
      q = add_rn(q, qi);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T v = __shfl_xor_sync(0xffffffffu, rmax, o);
    rmax = v > rmax ? v : rmax;
  }
  if (lane == 0) {
    T R = C.w;
    if (use_rmax) R = rmax < R ? rmax : R;
    cX[c].w = div_rn(R, theta);
    m0[c] = q;
  }
}

template <typename T>
__global__ void k_struct_level(int lo, int hi, const int* __restrict__ npos,
                               const int* __restrict__ ichild, const int* __restrict__ nchild,
                               vec4<T>* __restrict__ cX, T* __restrict__ m0, int use_rmax,
                               T theta) {
  const int v = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= hi) return;
  const int c = npos[v], nch = nchild[c];
  if (nch == 0) return;
  const int c0 = ichild[c];
  const vec4<T> Xp = cX[c];
  T rr = 0, q = 0;
  for (int k = 0; k < nch; k++) {
    const vec4<T> Xc = cX[c0 + k];
    const T d = add_rn(sqrt_rn(norm_rn(sub_rn(Xp.x, Xc.x), sub_rn(Xp.y, Xc.y), sub_rn(Xp.z, Xc.z))),
                       Xc.w);
    rr = d > rr ? d : rr;
    q = add_rn(q, m0[c0 + k]);
  }
  T R = Xp.w;
  if (use_rmax) R = rr < R ? rr : R;
  cX[c].w = div_rn(R, theta);
  m0[c] = q;
}

template <typename T>
__global__ void k_output(int n, const int* __restrict__ order, const vec4<T>* __restrict__ s,
                         const vec4<T>* __restrict__ e, vec4<T>* __restrict__ out) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  vec4<T> a = s[b], c = e[b];
  out[order[b]] = make_v4<T>(a.x + c.x, a.y + c.y, a.z + c.z, a.w + c.w);
}

template <typename T> static ExpansionOps<T> ops_of(const Solver<T>& s) {
  ExpansionOps<T> ops;
  bool ok = s.cfg.basis == FMM_SPHERICAL ? spherical_ops<T>(s.cfg.P, &ops)
                                         : cartesian_ops<T>(s.cfg.P, &ops);
  if (!ok) throw FmmError(FMM_ERR_INVALID, "expansion order not compiled");
  return ops;
}

// the expansions of the upward pass (P2M, M2M); with s.write_r the kernels also set the
// cell radii (setRmax, R /= theta), else the structure pass has set them
template <typename T> void upward_expansions(Solver<T>& s) {
  if (s.ncells == 0) return;
  ExpansionOps<T> ops = ops_of(s);
  const size_t ne = (size_t)s.ncells * s.ncoef;
  s.M.ensure(ne);
  s.L.ensure(ne);
  FMM_CUDA(cudaMemsetAsync(s.M.p, 0, ne * sizeof(T), s.stream));
  FMM_CUDA(cudaMemsetAsync(s.L.p, 0, ne * sizeof(T), s.stream));
  ops.p2m(s);
  for (int l = s.maxlevel - 1; l >= 0; l--) ops.m2m_level(s, s.level_lo[l], s.level_lo[l + 1]);
}

template <typename T> void upward_pass(Solver<T>& s) {
  if (s.ncells == 0) return;
  s.write_r = 1;
  upward_expansions(s);
  if (s.cfg.use_ropt) {
    k_ropt<T><<<ceil_div(s.ncells, 256), 256, 0, s.stream>>>(s.ncells, s.cX.p, s.M.p, s.c_root.p,
                                                            s.ncoef, s.cfg.P, (T)s.cfg.theta);
    FMM_LAUNCH_CHECK();
  }
}

// the final cell radii (radii, then the error-optimised radii) without the expansions
template <typename T> void structure_pass(Solver<T>& s) {
  if (s.ncells == 0) return;
  const int TB = 128;
  s.m0.ensure(s.ncells);
  k_struct_leaves<T><<<ceil_div(32LL * s.nleaves, TB), TB, 0, s.stream>>>(
      s.leaves.p, s.nleaves, s.c_ibody.p, s.c_nbody.p, s.cX.p, s.bodies.p, s.m0.p,
      s.cfg.use_rmax, (T)s.cfg.theta);
  FMM_LAUNCH_CHECK();
  for (int l = s.maxlevel - 1; l >= 0; l--) {
    const int lo = s.level_lo[l], hi = s.level_lo[l + 1];
    k_struct_level<T><<<ceil_div(hi - lo, TB), TB, 0, s.stream>>>(
        lo, hi, s.npos.p, s.c_ichild.p, s.c_nchild.p, s.cX.p, s.m0.p, s.cfg.use_rmax,
        (T)s.cfg.theta);
    FMM_LAUNCH_CHECK();
  }
  if (s.cfg.use_ropt) {
    k_ropt<T><<<ceil_div(s.ncells, 256), 256, 0, s.stream>>>(s.ncells, s.cX.p, s.m0.p, s.c_root.p,
                                                            1, s.cfg.P, (T)s.cfg.theta);
    FMM_LAUNCH_CHECK();
  }
}

template <typename T> void run_m2l(Solver<T>& s) {
  if (s.ncells == 0) return;
  ExpansionOps<T> ops = ops_of(s);
  if (s.nm2l > 0) ops.m2l(s);
  if (s.cfg.images > 1) {
    if (!ops.periodic) throw FmmError(FMM_ERR_NOT_SUPPORTED, "periodic images on this basis");
    ops.periodic(s);
  }
}

template <typename T> void downward_l2l(Solver<T>& s) {
  if (s.ncells == 0) return;
  ExpansionOps<T> ops = ops_of(s);
  for (int l = 1; l <= s.maxlevel; l++) ops.l2l_level(s, s.level_lo[l], s.level_lo[l + 1]);
}

template <typename T> void downward_l2p(Solver<T>& s) {
  if (s.ncells == 0) return;
  ExpansionOps<T> ops = ops_of(s);
  ops.l2p(s);
  s.trg_out.ensure(s.n);
  k_output<T><<<ceil_div(s.n, 256), 256, 0, s.stream>>>(s.n, s.order.p, s.trg_s.p, s.trg_e.p,
                                                        s.trg_out.p);
  FMM_LAUNCH_CHECK();
}

template <typename T> void downward_pass(Solver<T>& s) {
  downward_l2l(s);
  downward_l2p(s);
}

template void upward_pass<float>(Solver<float>&);
template void upward_pass<double>(Solver<double>&);
template void upward_expansions<float>(Solver<float>&);
template void upward_expansions<double>(Solver<double>&);
template void structure_pass<float>(Solver<float>&);
template void structure_pass<double>(Solver<double>&);
template void run_m2l<float>(Solver<float>&);
template void run_m2l<double>(Solver<double>&);
template void downward_pass<float>(Solver<float>&);
template void downward_pass<double>(Solver<double>&);
template void downward_l2l<float>(Solver<float>&);
template void downward_l2l<double>(Solver<double>&);
template void downward_l2p<float>(Solver<float>&);
template void downward_l2p<double>(Solver<double>&);

}  // namespace fmmb200
