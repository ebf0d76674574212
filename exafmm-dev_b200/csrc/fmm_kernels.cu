// Single translation operators on caller-chosen cells: the kernel plugin interface of the
// reference (namespace kernel, include/kernel.h:6-14: P2P pair and self, P2M, M2M, M2L,
// L2L, L2P; driven one cell at a time by examples/kernel.cxx:23-92 and by the traversal and
// the up/down passes) as C-ABI calls over lists of cells of a solver handle.
//
// The cells are those of the handle's last tree build, or cells the caller sets up by hand
// (fmm_b200_kernel_set_cells, over the bodies of fmm_b200_set_bodies_* in their given
// order).  Each call runs the solver's own kernels (the P2M / M2M / M2L / L2L / L2P of the
// handle's basis, order and precision, and the P2P) over the listed cells, with the
// reference's accumulate semantics: M, L and the targets receive += (the solver's P2M, M2M
// and P2P kernels write their results, so the rows they write are saved first and added
// back).  All host arguments are checked before any device work, so an out-of-range index
// is an FMM_ERR_INVALID, never a device access.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "fmm_handle.cuh"

using namespace fmmb200;

namespace fmmb200 {

template <typename T>
__global__ void k_kcells(int nc, const double* __restrict__ X, const double* __restrict__ R,
                         vec4<T>* __restrict__ cX) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc) cX[c] = make_v4<T>((T)X[3 * c], (T)X[3 * c + 1], (T)X[3 * c + 2], (T)R[c]);
}

template <typename T>
__global__ void k_kconvert(size_t n, const double* __restrict__ in, T* __restrict__ out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (T)in[i];
}

// expansion rows of the listed cells: save (dst = src, src = 0) or add back (dst += src)
template <typename T>
__global__ void k_krows(int n, const int* __restrict__ list, int ncoef, T* __restrict__ src,
                        T* __restrict__ dst, bool add) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * ncoef) return;
  const size_t e = (size_t)list[t / ncoef] * ncoef + t % ncoef;
  if (add) {
    dst[e] += src[e];
  } else {
    dst[e] = src[e];
    src[e] = 0;
  }
}

// the bodies of the listed cells, warp per cell: mark them with their cell (L2P), or add the
// targets saved before a P2P back to its sums (compensated merge)
__global__ void k_kmark(int n, const int* __restrict__ list, const int* __restrict__ ibody,
                        const int* __restrict__ nbody, int* __restrict__ body_leaf) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;
  const int c = list[w];
  for (int b = ibody[c] + lane_id(); b < ibody[c] + nbody[c]; b += 32) body_leaf[b] = c;
}
template <typename T>
__global__ void k_kmerge(int n, const int* __restrict__ list, const int* __restrict__ ibody,
                         const int* __restrict__ nbody, const vec4<T>* __restrict__ saved,
                         int nb, vec4<T>* __restrict__ trg_s, vec4<T>* __restrict__ trg_e) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;
  const int c = list[w];
  for (int b = ibody[c] + lane_id(); b < ibody[c] + nbody[c]; b += 32) {
    const vec4<T> s = trg_s[b], e = trg_e[b], os = saved[b], oe = saved[nb + b];
    Comp<T> a[4] = {{s.x, e.x}, {s.y, e.y}, {s.z, e.z}, {s.w, e.w}};
    const Comp<T> o[4] = {{os.x, oe.x}, {os.y, oe.y}, {os.z, oe.z}, {os.w, oe.w}};
    for (int d = 0; d < 4; d++) comp_merge(a[d], o[d]);
    trg_s[b] = make_v4<T>(a[0].s, a[1].s, a[2].s, a[3].s);
    trg_e[b] = make_v4<T>(a[0].e, a[1].e, a[2].e, a[3].e);
  }
}

template <typename T>
__global__ void k_ktrg_in(int n, const double* __restrict__ in, vec4<T>* __restrict__ trg_s,
                          vec4<T>* __restrict__ trg_e) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  trg_s[i] = in ? make_v4<T>((T)in[4 * i], (T)in[4 * i + 1], (T)in[4 * i + 2], (T)in[4 * i + 3])
                : make_v4<T>(0, 0, 0, 0);
  trg_e[i] = make_v4<T>(0, 0, 0, 0);
}
template <typename T>
__global__ void k_ktrg_out(int n, const vec4<T>* __restrict__ trg_s,
                           const vec4<T>* __restrict__ trg_e, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const vec4<T> s = trg_s[i], e = trg_e[i];
  out[4 * i] = (double)s.x + (double)e.x;
  out[4 * i + 1] = (double)s.y + (double)e.y;
  out[4 * i + 2] = (double)s.z + (double)e.z;
  out[4 * i + 3] = (double)s.w + (double)e.w;
}

}  // namespace fmmb200

namespace {

template <typename T> ExpansionOps<T> kops(const Solver<T>& s) {
  ExpansionOps<T> ops;
  const bool ok = s.cfg.basis == FMM_SPHERICAL ? spherical_ops<T>(s.cfg.P, &ops)
                                               : cartesian_ops<T>(s.cfg.P, &ops);
  if (!ok) throw FmmError(FMM_ERR_INVALID, "expansion order not compiled");
  return ops;
}

void bad(const std::string& msg) { throw FmmError(FMM_ERR_INVALID, msg); }

// Cells to operate on: a built tree (or set cells) with host copies of their index fields,
// expansions allocated (zero when the upward pass has not run), targets allocated.
// The operators apply to the listed cells whatever the handle's target partition
// (fmm_b200_set_partition): the partition is set aside for the call.
struct WholeSolve {
  SolverBase& s;
  int nparts;
  explicit WholeSolve(SolverBase& s_) : s(s_), nparts(s_.nparts) { s.nparts = 1; }
  ~WholeSolve() { s.nparts = nparts; }
};

template <typename T> void prepare(Solver<T>& s) {
  if (s.stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "no cells: build a tree or set cells");
  const int nc = s.ncells;
  if (!s.kc_valid) {
    std::vector<int>* h[] = {&s.kc_ibody, &s.kc_nbody, &s.kc_ichild, &s.kc_nchild, &s.kc_iparent};
    const int* d[] = {s.c_ibody.p, s.c_nbody.p, s.c_ichild.p, s.c_nchild.p, s.c_iparent.p};
    for (int k = 0; k < 5; k++) {
      h[k]->resize(nc);
      if (nc)
        FMM_CUDA(cudaMemcpyAsync(h[k]->data(), d[k], sizeof(int) * nc, cudaMemcpyDeviceToHost,
                                 s.stream));
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
    s.kc_valid = true;
  }
  if (s.stage < ST_UP) {
    const size_t ne = std::max<size_t>((size_t)nc * s.ncoef, 1);
    s.M.ensure(ne);
    s.L.ensure(ne);
    FMM_CUDA(cudaMemsetAsync(s.M.p, 0, ne * sizeof(T), s.stream));
    FMM_CUDA(cudaMemsetAsync(s.L.p, 0, ne * sizeof(T), s.stream));
    s.stage = ST_UP;
  }
  s.trg_s.ensure(std::max(s.n, 1));
  s.trg_e.ensure(std::max(s.n, 1));
  s.body_leaf.ensure(std::max(s.n, 1));
}

// an operator call leaves the expansions readable but the handle's interaction lists and
// downward pass stale
void finish(SolverBase& s) {
  if (s.stage > ST_UP) s.stage = ST_UP;
  s.trav_sized = false;
}

void check_list(const SolverBase& s, int n, const int* cells, const char* what) {
  if (n < 0 || (n > 0 && !cells)) bad(std::string(what) + ": invalid list");
  std::vector<char> seen(s.ncells, 0);
  for (int k = 0; k < n; k++) {
    const int c = cells[k];
    if (c < 0 || c >= s.ncells) bad(std::string(what) + ": cell index out of range");
    if (seen[c]) bad(std::string(what) + ": a cell is listed twice");
    seen[c] = 1;
  }
}

// the bodies of the listed cells must not overlap (their targets are written concurrently)
void check_disjoint_bodies(const SolverBase& s, const std::vector<int>& cells, const char* what) {
  std::vector<std::pair<int, int>> r;
  for (int c : cells)
    if (s.kc_nbody[c] > 0) r.push_back({s.kc_ibody[c], s.kc_ibody[c] + s.kc_nbody[c]});
  std::sort(r.begin(), r.end());
  for (size_t k = 1; k < r.size(); k++)
    if (r[k].first < r[k - 1].second)
      bad(std::string(what) + ": the target cells' bodies overlap");
}

void upload_list(SolverBase& s, int n, const int* cells) {
  s.k_list.ensure(std::max(n, 1));
  if (n)
    FMM_CUDA(cudaMemcpyAsync(s.k_list.p, cells, sizeof(int) * n, cudaMemcpyHostToDevice,
                             s.stream));
}

// the reverse image code: the shift (-ix, -iy, -iz) of code 9 d(ix) + 3 d(iy) + d(iz),
// d(0) = 0, d(1) = 1, d(-1) = 2
int neg_image(int code) {
  static const int swap[3] = {0, 2, 1};
  return 9 * swap[code / 9] + 3 * swap[(code / 3) % 3] + swap[code % 3];
}

// Cell pairs grouped by target, in call order within a target (mutual: each pair of two
// different cells also in reverse, with the reverse shift), as the solver's lists: packed
// (target << 32) | image << 27 | source, CSR offsets per cell, the targets in order.
struct PairList {
  std::vector<unsigned long long> pairs;
  std::vector<int> off, targets;
};
PairList pair_list(const SolverBase& s, int n, const int* ci, const int* cj, const int* image,
                   int mutual, const char* what) {
  if (n < 0 || (n > 0 && (!ci || !cj)) || (mutual != 0 && mutual != 1))
    bad(std::string(what) + ": invalid arguments");
  std::vector<std::vector<unsigned>> per(s.ncells);
  for (int k = 0; k < n; k++) {
    const int a = ci[k], b = cj[k], img = image ? image[k] : 0;
    if (a < 0 || a >= s.ncells || b < 0 || b >= s.ncells)
      bad(std::string(what) + ": cell index out of range");
    if (img < 0 || img >= 27) bad(std::string(what) + ": image code out of range");
    if (b >= (1 << kImgShift)) bad(std::string(what) + ": source index above the pair format");
    per[a].push_back((unsigned)b | ((unsigned)img << kImgShift));
    if (mutual && a != b) per[b].push_back((unsigned)a | ((unsigned)neg_image(img) << kImgShift));
  }
  PairList L;
  L.off.assign(s.ncells + 1, 0);
  for (int c = 0; c < s.ncells; c++) {
    L.off[c + 1] = L.off[c] + (int)per[c].size();
    if (!per[c].empty()) L.targets.push_back(c);
    for (unsigned src : per[c]) L.pairs.push_back(((unsigned long long)c << 32) | src);
  }
  return L;
}

void upload_pairs(SolverBase& s, const PairList& L, DevArr<unsigned long long>& pairs,
                  DevArr<int>& off) {
  pairs.ensure(std::max<size_t>(L.pairs.size(), 1));
  off.ensure(s.ncells + 1);
  if (!L.pairs.empty())
    FMM_CUDA(cudaMemcpyAsync(pairs.p, L.pairs.data(), 8 * L.pairs.size(), cudaMemcpyHostToDevice,
                             s.stream));
  FMM_CUDA(cudaMemcpyAsync(off.p, L.off.data(), sizeof(int) * (s.ncells + 1),
                           cudaMemcpyHostToDevice, s.stream));
}

// P2M and M2M write the rows of their cells (and the cell radii): the listed rows are saved
// and zeroed, the operator runs, the saved rows are added back and the radii restored
template <typename T, typename F> void with_saved_rows(Solver<T>& s, int n, F&& op) {
  const size_t ne = (size_t)s.ncells * s.ncoef;
  s.k_rows.ensure(std::max<size_t>(ne, 1));
  s.k_cx.ensure(std::max(s.ncells, 1));
  FMM_CUDA(cudaMemcpyAsync(s.k_cx.p, s.cX.p, sizeof(vec4<T>) * s.ncells, cudaMemcpyDeviceToDevice,
                           s.stream));
  const long long work = (long long)n * s.ncoef;
  k_krows<T><<<ceil_div(work, 256), 256, 0, s.stream>>>(n, s.k_list.p, s.ncoef, s.M.p,
                                                        s.k_rows.p, false);
  FMM_LAUNCH_CHECK();
  op();
  k_krows<T><<<ceil_div(work, 256), 256, 0, s.stream>>>(n, s.k_list.p, s.ncoef, s.k_rows.p,
                                                        s.M.p, true);
  FMM_LAUNCH_CHECK();
  FMM_CUDA(cudaMemcpyAsync(s.cX.p, s.k_cx.p, sizeof(vec4<T>) * s.ncells, cudaMemcpyDeviceToDevice,
                           s.stream));
}

// body_leaf belongs to the solve (P2M writes it for L2P): kept across an operator call
template <typename T, typename F> void with_saved_body_leaf(Solver<T>& s, F&& op) {
  s.k_saved_leaves.ensure(std::max(s.n, 1));
  if (s.n)
    FMM_CUDA(cudaMemcpyAsync(s.k_saved_leaves.p, s.body_leaf.p, sizeof(int) * s.n,
                             cudaMemcpyDeviceToDevice, s.stream));
  op();
  if (s.n)
    FMM_CUDA(cudaMemcpyAsync(s.body_leaf.p, s.k_saved_leaves.p, sizeof(int) * s.n,
                             cudaMemcpyDeviceToDevice, s.stream));
}

template <typename T> void op_p2m(Solver<T>& s, int n, const int* cells) {
  WholeSolve whole(s);
  prepare(s);
  check_list(s, n, cells, "P2M");
  if (!n) return;
  upload_list(s, n, cells);
  ExpansionOps<T> ops = kops(s);
  with_saved_body_leaf(s, [&] {
    with_saved_rows(s, n, [&] {
      std::swap(s.leaves, s.k_list);
      const int nl = s.nleaves, wr = s.write_r;
      s.nleaves = n;
      s.write_r = 0;
      try {
        ops.p2m(s);
      } catch (...) {
        std::swap(s.leaves, s.k_list);
        s.nleaves = nl;
        s.write_r = wr;
        throw;
      }
      std::swap(s.leaves, s.k_list);
      s.nleaves = nl;
      s.write_r = wr;
    });
  });
  finish(s);
}

template <typename T> void op_m2m(Solver<T>& s, int n, const int* cells) {
  WholeSolve whole(s);
  prepare(s);
  check_list(s, n, cells, "M2M");
  std::vector<char> listed(s.ncells, 0);
  for (int k = 0; k < n; k++) listed[cells[k]] = 1;
  for (int k = 0; k < n; k++) {
    const int c = cells[k], c0 = s.kc_ichild[c], nch = s.kc_nchild[c];
    if (nch < 0 || nch > 8 || (nch > 0 && (c0 < 0 || c0 + nch > s.ncells)))
      bad("M2M: children out of range");
    for (int i = 0; i < nch; i++)
      if (listed[c0 + i]) bad("M2M: a cell and its child in one call (translate the child first)");
  }
  if (!n) return;
  upload_list(s, n, cells);
  ExpansionOps<T> ops = kops(s);
  with_saved_rows(s, n, [&] {
    std::swap(s.npos, s.k_list);
    const int wr = s.write_r;
    s.write_r = 0;
    try {
      ops.m2m_level(s, 0, n);
    } catch (...) {
      std::swap(s.npos, s.k_list);
      s.write_r = wr;
      throw;
    }
    std::swap(s.npos, s.k_list);
    s.write_r = wr;
  });
  finish(s);
}

template <typename T> void op_l2l(Solver<T>& s, int n, const int* cells) {
  WholeSolve whole(s);
  prepare(s);
  check_list(s, n, cells, "L2L");
  std::vector<char> listed(s.ncells, 0);
  for (int k = 0; k < n; k++) listed[cells[k]] = 1;
  for (int k = 0; k < n; k++) {
    const int p = s.kc_iparent[cells[k]];
    if (p < 0 || p >= s.ncells || p == cells[k]) bad("L2L: parent out of range");
    if (listed[p]) bad("L2L: a cell and its parent in one call (translate the parent first)");
  }
  if (!n) return;
  upload_list(s, n, cells);
  ExpansionOps<T> ops = kops(s);
  std::swap(s.npos, s.k_list);
  try {
    ops.l2l_level(s, 0, n);
  } catch (...) {
    std::swap(s.npos, s.k_list);
    throw;
  }
  std::swap(s.npos, s.k_list);
  finish(s);
}

template <typename T> void op_l2p(Solver<T>& s, int n, const int* cells) {
  WholeSolve whole(s);
  prepare(s);
  check_list(s, n, cells, "L2P");
  check_disjoint_bodies(s, std::vector<int>(cells, cells + n), "L2P");
  if (!n || !s.n) return;
  upload_list(s, n, cells);
  ExpansionOps<T> ops = kops(s);
  with_saved_body_leaf(s, [&] {
    FMM_CUDA(cudaMemsetAsync(s.body_leaf.p, 0xff, sizeof(int) * s.n, s.stream));
    k_kmark<<<ceil_div(32LL * n, 256), 256, 0, s.stream>>>(n, s.k_list.p, s.c_ibody.p,
                                                           s.c_nbody.p, s.body_leaf.p);
    FMM_LAUNCH_CHECK();
    const int nl = s.nleaves;
    s.nleaves = n;  // any non-zero count: the kernel walks every body and skips unmarked ones
    try {
      ops.l2p(s);
    } catch (...) {
      s.nleaves = nl;
      throw;
    }
    s.nleaves = nl;
  });
  finish(s);
}

template <typename T>
void op_m2l(Solver<T>& s, int n, const int* ci, const int* cj, const int* image, int mutual) {
  prepare(s);
  PairList L = pair_list(s, n, ci, cj, image, mutual, "M2L");
  if (L.pairs.empty()) return;
  ExpansionOps<T> ops = kops(s);
  upload_pairs(s, L, s.m2l, s.m2l_off);
  s.m2l_tgt.ensure(L.targets.size());
  FMM_CUDA(cudaMemcpyAsync(s.m2l_tgt.p, L.targets.data(), sizeof(int) * L.targets.size(),
                           cudaMemcpyHostToDevice, s.stream));
  s.nm2l = (long long)L.pairs.size();
  s.m2l_ntgt = (int)L.targets.size();
  ops.m2l(s);
  s.nm2l = 0;
  finish(s);
}

template <typename T>
void op_p2p(Solver<T>& s, int n, const int* ci, const int* cj, const int* image, int mutual,
            double eps2) {
  prepare(s);
  if (!(eps2 >= 0)) bad("P2P: eps2 must be >= 0");
  PairList L = pair_list(s, n, ci, cj, image, mutual, "P2P");
  if (L.pairs.empty() || !s.n) return;
  check_disjoint_bodies(s, L.targets, "P2P");
  const int nt = (int)L.targets.size();
  upload_pairs(s, L, s.p2p, s.p2p_off);
  s.p2p_ordered = false;  // the solver's P2P lists (and their target order) are replaced
  upload_list(s, nt, L.targets.data());
  // save the targets, let the P2P write its sums, add the saved values back
  s.k_trg.ensure(2 * (size_t)s.n);
  FMM_CUDA(cudaMemcpyAsync(s.k_trg.p, s.trg_s.p, sizeof(vec4<T>) * s.n, cudaMemcpyDeviceToDevice,
                           s.stream));
  FMM_CUDA(cudaMemcpyAsync(s.k_trg.p + s.n, s.trg_e.p, sizeof(vec4<T>) * s.n,
                           cudaMemcpyDeviceToDevice, s.stream));
  std::swap(s.leaves, s.k_list);
  const int nl = s.nleaves;
  const double e2 = s.cfg.eps2;
  s.nleaves = nt;
  s.cfg.eps2 = eps2;
  auto restore = [&] {
    std::swap(s.leaves, s.k_list);
    s.nleaves = nl;
    s.cfg.eps2 = e2;
  };
  try {
    s.np2p = (long long)L.pairs.size();
    run_p2p(s);
  } catch (...) {
    restore();
    throw;
  }
  restore();
  k_kmerge<T><<<ceil_div(32LL * nt, 256), 256, 0, s.stream>>>(
      nt, s.k_list.p, s.c_ibody.p, s.c_nbody.p, s.k_trg.p, s.n, s.trg_s.p, s.trg_e.p);
  FMM_LAUNCH_CHECK();
  s.np2p = 0;
  finish(s);
}

}  // namespace

extern "C" {

int fmm_b200_kernel_set_cells(fmm_b200_solver* h, int nc, const double* X, const double* R,
                              const int* ibody, const int* nbody, const int* ichild,
                              const int* nchild, const int* iparent) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_BODIES) throw FmmError(FMM_ERR_STATE, "bodies not set");
    if (nc < 1 || !X || !R || !ibody || !nbody || !ichild || !nchild || !iparent)
      bad("set_cells: invalid arguments");
    if (nc >= (1 << kImgShift)) bad("set_cells: too many cells");
    for (int c = 0; c < nc; c++) {
      if (ibody[c] < 0 || nbody[c] < 0 || (long long)ibody[c] + nbody[c] > s.n)
        bad("set_cells: body range out of range");
      if (nchild[c] < 0 || nchild[c] > 8 ||
          (nchild[c] > 0 && (ichild[c] < 0 || (long long)ichild[c] + nchild[c] > nc)))
        bad("set_cells: child range out of range");
    }
    const int n = s.n;
    // bodies in the given order (no tree permutation), targets zero
    s.bodies.ensure(std::max(n, 1));
    s.order.ensure(std::max(n, 1));
    if (n) {
      FMM_CUDA(cudaMemcpyAsync(s.bodies.p, s.bodies_in.p, sizeof(vec4<T>) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
      std::vector<int> iota(n);
      std::iota(iota.begin(), iota.end(), 0);
      FMM_CUDA(cudaMemcpyAsync(s.order.p, iota.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                               s.stream));
    }
    DevArr<int>* dst[] = {&s.c_ibody, &s.c_nbody, &s.c_ichild, &s.c_nchild, &s.c_iparent};
    const int* src[] = {ibody, nbody, ichild, nchild, iparent};
    for (int k = 0; k < 5; k++) {
      dst[k]->ensure(nc);
      FMM_CUDA(cudaMemcpyAsync(dst[k]->p, src[k], sizeof(int) * nc, cudaMemcpyHostToDevice,
                               s.stream));
    }
    s.c_level.ensure(nc);
    s.c_icell.ensure(nc);
    s.c_root.ensure(nc);
    FMM_CUDA(cudaMemsetAsync(s.c_level.p, 0, sizeof(int) * nc, s.stream));
    FMM_CUDA(cudaMemsetAsync(s.c_icell.p, 0, 8 * (size_t)nc, s.stream));
    FMM_CUDA(cudaMemsetAsync(s.c_root.p, 0, sizeof(int) * nc, s.stream));
    s.dtmp.ensure(4 * (size_t)nc);
    FMM_CUDA(cudaMemcpyAsync(s.dtmp.p, X, 24 * (size_t)nc, cudaMemcpyHostToDevice, s.stream));
    FMM_CUDA(cudaMemcpyAsync(s.dtmp.p + 3 * (size_t)nc, R, 8 * (size_t)nc,
                             cudaMemcpyHostToDevice, s.stream));
    s.cX.ensure(nc);
    k_kcells<T><<<ceil_div(nc, 256), 256, 0, s.stream>>>(nc, s.dtmp.p, s.dtmp.p + 3 * (size_t)nc,
                                                         s.cX.p);
    FMM_LAUNCH_CHECK();
    s.kc_ibody.assign(ibody, ibody + nc);
    s.kc_nbody.assign(nbody, nbody + nc);
    s.kc_ichild.assign(ichild, ichild + nc);
    s.kc_nchild.assign(nchild, nchild + nc);
    s.kc_iparent.assign(iparent, iparent + nc);
    s.kc_valid = true;
    s.ncells = nc;
    s.maxlevel = 0;
    s.nleaves = 0;
    s.nroots = 0;
    s.root_cell.clear();
    s.level_lo.assign({0, nc});
    s.nm2l = s.np2p = 0;
    s.p2p_ordered = false;
    s.trav_sized = false;
    s.stage = ST_TREE;
    prepare(s);  // expansions and targets zero
    FMM_CUDA(cudaMemsetAsync(s.trg_s.p, 0, sizeof(vec4<T>) * std::max(n, 1), s.stream));
    FMM_CUDA(cudaMemsetAsync(s.trg_e.p, 0, sizeof(vec4<T>) * std::max(n, 1), s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_kernel_set_expansion(fmm_b200_solver* h, int which, const double* in) {
  return FMM_DISPATCH(h, {
    if (which != 0 && which != 1) bad("set_expansion: which must be 0 (M) or 1 (L)");
    prepare(s);
    const size_t ne = (size_t)s.ncells * s.ncoef;
    T* dst = which ? s.L.p : s.M.p;
    if (!in) {
      FMM_CUDA(cudaMemsetAsync(dst, 0, ne * sizeof(T), s.stream));
    } else if (ne) {
      s.dtmp.ensure(ne);
      FMM_CUDA(cudaMemcpyAsync(s.dtmp.p, in, ne * sizeof(double), cudaMemcpyHostToDevice,
                               s.stream));
      k_kconvert<T><<<ceil_div((long long)ne, 256), 256, 0, s.stream>>>(ne, s.dtmp.p, dst);
      FMM_LAUNCH_CHECK();
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_kernel_set_trg(fmm_b200_solver* h, const double* trg) {
  return FMM_DISPATCH(h, {
    prepare(s);
    if (s.n) {
      const double* d = nullptr;
      if (trg) {
        s.dtmp.ensure(4 * (size_t)s.n);
        FMM_CUDA(cudaMemcpyAsync(s.dtmp.p, trg, 32 * (size_t)s.n, cudaMemcpyHostToDevice,
                                 s.stream));
        d = s.dtmp.p;
      }
      k_ktrg_in<T><<<ceil_div(s.n, 256), 256, 0, s.stream>>>(s.n, d, s.trg_s.p, s.trg_e.p);
      FMM_LAUNCH_CHECK();
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_kernel_get_trg(fmm_b200_solver* h, double* trg) {
  return FMM_DISPATCH(h, {
    prepare(s);
    if (s.n) {
      if (!trg) bad("get_trg: null output");
      s.dtmp.ensure(4 * (size_t)s.n);
      k_ktrg_out<T><<<ceil_div(s.n, 256), 256, 0, s.stream>>>(s.n, s.trg_s.p, s.trg_e.p,
                                                              s.dtmp.p);
      FMM_LAUNCH_CHECK();
      FMM_CUDA(cudaMemcpyAsync(trg, s.dtmp.p, 32 * (size_t)s.n, cudaMemcpyDeviceToHost,
                               s.stream));
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_kernel_p2m(fmm_b200_solver* h, int n, const int* cells) {
  return FMM_DISPATCH(h, op_p2m(s, n, cells));
}
int fmm_b200_kernel_m2m(fmm_b200_solver* h, int n, const int* cells) {
  return FMM_DISPATCH(h, op_m2m(s, n, cells));
}
int fmm_b200_kernel_m2l(fmm_b200_solver* h, int n, const int* ci, const int* cj,
                        const int* image, int mutual) {
  return FMM_DISPATCH(h, op_m2l(s, n, ci, cj, image, mutual));
}
int fmm_b200_kernel_l2l(fmm_b200_solver* h, int n, const int* cells) {
  return FMM_DISPATCH(h, op_l2l(s, n, cells));
}
int fmm_b200_kernel_l2p(fmm_b200_solver* h, int n, const int* cells) {
  return FMM_DISPATCH(h, op_l2p(s, n, cells));
}
int fmm_b200_kernel_p2p(fmm_b200_solver* h, int n, const int* ci, const int* cj,
                        const int* image, int mutual, double eps2) {
  return FMM_DISPATCH(h, op_p2p(s, n, ci, cj, image, mutual, eps2));
}

}  // extern "C"
