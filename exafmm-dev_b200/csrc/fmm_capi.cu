// The C ABI (include/exafmm_b200.h): handle lifecycle, stages, whole solves, introspection.
// Every entry point converts exceptions into status codes; a handle's last failure message
// stays readable through fmm_b200_last_error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include <string>

#include "fmm_handle.cuh"

using namespace fmmb200;


static thread_local std::string g_create_error;

namespace fmmb200 {

// message of a failed call that has no solver handle (read through fmm_b200_last_error(NULL))
void set_call_error(const char* msg) { g_create_error = msg; }

void phase_begin(SolverBase& s, int ph) {
  FMM_CUDA(cudaEventRecord(s.ev[2 * ph], s.stream));
}
void phase_end(SolverBase& s, int ph) {
  FMM_CUDA(cudaEventRecord(s.ev[2 * ph + 1], s.stream));
  s.ev_used[ph] = true;
}

// double host-side layout (x[3n], q[n]) -> working-precision 4-vectors
template <typename T>
__global__ void k_pack(int n, const double* __restrict__ x, const double* __restrict__ q,
                       vec4<T>* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_v4<T>((T)x[3 * i], (T)x[3 * i + 1], (T)x[3 * i + 2], (T)q[i]);
}
template <typename T>
__global__ void k_unpack(int n, const vec4<T>* __restrict__ in, double* __restrict__ trg4) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    vec4<T> v = in[i];
    trg4[4 * i] = v.x;
    trg4[4 * i + 1] = v.y;
    trg4[4 * i + 2] = v.z;
    trg4[4 * i + 3] = v.w;
  }
}
template <typename T>
__global__ void k_unpack_pf(int n, const vec4<T>* __restrict__ in, double* __restrict__ p,
                            double* __restrict__ f) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    vec4<T> v = in[i];
    p[i] = v.x;
    f[3 * i] = v.y;
    f[3 * i + 1] = v.z;
    f[3 * i + 2] = v.w;
  }
}
template <typename T>
__global__ void k_cells_out(int nc, const vec4<T>* __restrict__ cX, double* __restrict__ X,
                            double* __restrict__ R) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc) {
    vec4<T> v = cX[c];
    X[3 * c] = v.x;
    X[3 * c + 1] = v.y;
    X[3 * c + 2] = v.z;
    R[c] = v.w;
  }
}
template <typename T>
__global__ void k_to_double(size_t n, const T* __restrict__ in, double* __restrict__ out) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

}  // namespace fmmb200

namespace {

// body ranges of a batch of solves from their counts (host); false on a bad count
bool set_segments(SolverBase& s, int nsolves, const int* counts, int* total) {
  if (nsolves < 1 || !counts) return false;
  s.seg.assign(nsolves + 1, 0);
  long long acc = 0;
  for (int q = 0; q < nsolves; q++) {
    if (counts[q] < 0) return false;
    acc += counts[q];
    if (acc > 0x7fffffffLL) return false;
    s.seg[q + 1] = (int)acc;
  }
  *total = (int)acc;
  return true;
}

template <typename T> void set_bodies_host_t(Solver<T>& s, int n, const double* x, const double* q,
                                             DevArr<double>& tmp) {
  s.n = n;
  s.bodies_in.ensure(std::max(n, 1));
  if (n > 0) {
    tmp.ensure(4 * (size_t)n);
    FMM_CUDA(cudaMemcpyAsync(tmp.p, x, 3 * sizeof(double) * n, cudaMemcpyHostToDevice, s.stream));
    FMM_CUDA(cudaMemcpyAsync(tmp.p + 3 * (size_t)n, q, sizeof(double) * n,
                             cudaMemcpyHostToDevice, s.stream));
    k_pack<T><<<ceil_div(n, 256), 256, 0, s.stream>>>(n, tmp.p, tmp.p + 3 * (size_t)n,
                                                      s.bodies_in.p);
    FMM_LAUNCH_CHECK();
  }
  s.stage = ST_BODIES;
}

template <typename T> void stage_tree(Solver<T>& s) {
  if (s.stage < ST_BODIES) throw FmmError(FMM_ERR_STATE, "bodies not set");
  for (int p = 0; p < FMM_NUM_PHASES; p++) s.ev_used[p] = false;
  phase_begin(s, FMM_PHASE_TOTAL);
  phase_begin(s, FMM_PHASE_BOUNDS);
  build_tree(s);
  partition_range(s);
  if (s.n == 0) phase_end(s, FMM_PHASE_BOUNDS);
  else phase_end(s, FMM_PHASE_TREE);
  s.stage = ST_TREE;
}
template <typename T> void stage_up(Solver<T>& s) {
  if (s.stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "tree not built");
  phase_begin(s, FMM_PHASE_UPWARD);
  upward_pass(s);
  phase_end(s, FMM_PHASE_UPWARD);
  s.stage = ST_UP;
}
template <typename T> void stage_trav(Solver<T>& s) {
  if (s.stage < ST_UP) throw FmmError(FMM_ERR_STATE, "upward pass not done");
  phase_begin(s, FMM_PHASE_TRAVERSE);
  build_lists(s);
  phase_end(s, FMM_PHASE_TRAVERSE);
  phase_begin(s, FMM_PHASE_M2L);
  run_m2l(s);
  phase_end(s, FMM_PHASE_M2L);
  phase_begin(s, FMM_PHASE_P2P);
  s.trg_s.ensure(std::max(s.n, 1));
  s.trg_e.ensure(std::max(s.n, 1));
  if (s.n > 0) {
    FMM_CUDA(cudaMemsetAsync(s.trg_s.p, 0, sizeof(vec4<T>) * s.n, s.stream));
    FMM_CUDA(cudaMemsetAsync(s.trg_e.p, 0, sizeof(vec4<T>) * s.n, s.stream));
  }
  run_p2p(s);
  phase_end(s, FMM_PHASE_P2P);
  s.stage = ST_TRAV;
}
template <typename T> void stage_down(Solver<T>& s) {
  if (s.stage < ST_TRAV) throw FmmError(FMM_ERR_STATE, "traversal not done");
  phase_begin(s, FMM_PHASE_DOWNWARD);
  downward_pass(s);
  if (s.n == 0) s.trg_out.ensure(1);
  phase_end(s, FMM_PHASE_DOWNWARD);
  phase_end(s, FMM_PHASE_TOTAL);
  s.stage = ST_DOWN;
}
// A whole solve: the stages in order, with two overlaps on side streams.  (1) Spherical
// basis: the expansions of the upward pass (P2M, M2M) run on a lowest-priority stream
// while the main stream sets the cell radii in a pass of their own (structure_pass: the
// same radii, monopoles and error-optimised radii as the expansion kernels would set) and
// runs the traversal, which needs the radii but not the expansions; M2L waits for both.
// (2) The L2L levels run on a high-priority stream while P2P runs (from the end of M2L to
// the start of L2P).  The L2L levels have few cells each and long dependent chains per cell, so
// alone they leave most of the GPU idle; with the higher priority their blocks start as
// soon as SMs free up.  The results are the same as stage by stage: P2P writes only the
// bodies' sums, L2L only the local expansions, and L2P runs after both.
template <typename T> void solve_all(Solver<T>& s) {
  stage_tree(s);
  if (!s.side) {
    int lo = 0, hi = 0;
    FMM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    FMM_CUDA(cudaStreamCreateWithPriority(&s.side, cudaStreamNonBlocking, hi));
    FMM_CUDA(cudaStreamCreateWithPriority(&s.side_lo, cudaStreamNonBlocking, lo));
    FMM_CUDA(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming));
    FMM_CUDA(cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming));
  }
  cudaStream_t main = s.stream;
  if (s.ncells > 0) {
    FMM_CUDA(cudaEventRecord(s.fork, s.stream));
    FMM_CUDA(cudaStreamWaitEvent(s.side_lo, s.fork, 0));
    s.stream = s.side_lo;  // below the traversal, which is on the critical path
    s.write_r = 0;
    try {
      phase_begin(s, FMM_PHASE_UPWARD);
      upward_expansions(s);
      phase_end(s, FMM_PHASE_UPWARD);
      FMM_CUDA(cudaEventRecord(s.join, s.stream));
    } catch (...) {
      s.stream = main;
      s.write_r = 1;
      throw;
    }
    s.stream = main;
    s.write_r = 1;
    s.stage = ST_UP;
    phase_begin(s, FMM_PHASE_TRAVERSE);
    structure_pass(s);
    build_lists(s, true);
    phase_end(s, FMM_PHASE_TRAVERSE);
    FMM_CUDA(cudaStreamWaitEvent(s.stream, s.join, 0));  // the multipoles, before M2L
  } else {
    stage_up(s);
    phase_begin(s, FMM_PHASE_TRAVERSE);
    build_lists(s, true);
    phase_end(s, FMM_PHASE_TRAVERSE);
  }
  phase_begin(s, FMM_PHASE_M2L);
  run_m2l(s);
  phase_end(s, FMM_PHASE_M2L);
  // fork: the L2L levels on the side stream
  FMM_CUDA(cudaEventRecord(s.fork, s.stream));
  FMM_CUDA(cudaStreamWaitEvent(s.side, s.fork, 0));
  s.stream = s.side;
  try {
    phase_begin(s, FMM_PHASE_DOWNWARD);
    downward_l2l(s);
    FMM_CUDA(cudaEventRecord(s.join, s.stream));
  } catch (...) {
    s.stream = main;
    throw;
  }
  s.stream = main;
  phase_begin(s, FMM_PHASE_P2P);
  s.trg_s.ensure(std::max(s.n, 1));
  s.trg_e.ensure(std::max(s.n, 1));
  if (s.n > 0) {
    FMM_CUDA(cudaMemsetAsync(s.trg_s.p, 0, sizeof(vec4<T>) * s.n, s.stream));
    FMM_CUDA(cudaMemsetAsync(s.trg_e.p, 0, sizeof(vec4<T>) * s.n, s.stream));
  }
  finish_p2p_list(s);  // grouped on the side stream while M2L ran
  run_p2p(s);
  phase_end(s, FMM_PHASE_P2P);
  s.stage = ST_TRAV;
  FMM_CUDA(cudaStreamWaitEvent(s.stream, s.join, 0));  // join before L2P reads the locals
  downward_l2p(s);
  if (s.n == 0) s.trg_out.ensure(1);
  phase_end(s, FMM_PHASE_DOWNWARD);
  phase_end(s, FMM_PHASE_TOTAL);
  s.stage = ST_DOWN;
}

}  // namespace

// ncrit autotuner: each candidate solves the handle's current bodies `repeats` times after
// one untimed solve (which sizes the buffers); the median device time decides.
template <typename T>
static int autotune_ncrit_t(Solver<T>& s, const int* cand, int ncand, int repeats,
                            int* best, double* times_ms) {
  if (s.stage < ST_BODIES) throw FmmError(FMM_ERR_STATE, "bodies not set");
  const int keep = s.cfg.ncrit;
  cudaEvent_t e0, e1;
  FMM_CUDA(cudaEventCreate(&e0));
  FMM_CUDA(cudaEventCreate(&e1));
  double best_ms = 1e300;
  int best_nc = keep;
  try {
    for (int i = 0; i < ncand; i++) {
      s.cfg.ncrit = cand[i];
      s.trav_sized = false;  // list sizes change with the tree
      solve_all(s);
      std::vector<float> ms;
      for (int r = 0; r < repeats; r++) {
        FMM_CUDA(cudaEventRecord(e0, s.stream));
        solve_all(s);
        FMM_CUDA(cudaEventRecord(e1, s.stream));
        FMM_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        FMM_CUDA(cudaEventElapsedTime(&t, e0, e1));
        ms.push_back(t);
      }
      std::sort(ms.begin(), ms.end());
      const double med = ms[ms.size() / 2];
      if (times_ms) times_ms[i] = med;
      if (med < best_ms) {
        best_ms = med;
        best_nc = cand[i];
      }
    }
  } catch (...) {
    s.cfg.ncrit = keep;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s.cfg.ncrit = best_nc;
  s.trav_sized = false;
  s.stage = ST_BODIES;
  if (best) *best = best_nc;
  return FMM_OK;
}

// P2P lane-group autotuner: on the lists of the handle's last solve, each candidate pair of
// leaf-size thresholds (4 lanes per target up to g4 bodies, 2 up to g2) runs the P2P
// `repeats` times after one untimed run; the median device time decides.
template <typename T>
static int autotune_p2p_t(Solver<T>& s, const int* g4, const int* g2, int ncand, int repeats,
                          int* best, double* times_ms) {
  if (s.stage < ST_DOWN) throw FmmError(FMM_ERR_STATE, "solve first: the P2P lists are tuned on");
  const int k4 = s.p2p_g4, k2 = s.p2p_g2;
  cudaEvent_t e0, e1;
  FMM_CUDA(cudaEventCreate(&e0));
  FMM_CUDA(cudaEventCreate(&e1));
  double best_ms = 1e300;
  int bi = 0;
  try {
    for (int i = 0; i < ncand; i++) {
      s.p2p_g4 = g4[i];
      s.p2p_g2 = g2[i];
      run_p2p(s);
      std::vector<float> ms;
      for (int r = 0; r < repeats; r++) {
        FMM_CUDA(cudaEventRecord(e0, s.stream));
        run_p2p(s);
        FMM_CUDA(cudaEventRecord(e1, s.stream));
        FMM_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        FMM_CUDA(cudaEventElapsedTime(&t, e0, e1));
        ms.push_back(t);
      }
      std::sort(ms.begin(), ms.end());
      const double med = ms[ms.size() / 2];
      if (times_ms) times_ms[i] = med;
      if (med < best_ms) {
        best_ms = med;
        bi = i;
      }
    }
  } catch (...) {
    s.p2p_g4 = k4;
    s.p2p_g2 = k2;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s.p2p_g4 = g4[bi];
  s.p2p_g2 = g2[bi];
  s.stage = ST_BODIES;  // the targets now hold the tuning runs' near field: solve again
  if (best) *best = bi;
  return FMM_OK;
}

// targets (segment 0) and sources (segment 1) as two trees on a common box
template <typename T>
static void solve_ij_t(fmm_b200_solver* h, Solver<T>& s, int nt, int ns, int common_box) {
  if (s.cfg.images != 0)
    throw FmmError(FMM_ERR_NOT_SUPPORTED, "separate target and source sets with periodic images");
  const int counts[2] = {nt, ns};
  int n = 0;
  if (!set_segments(*h->base, 2, counts, &n)) throw FmmError(FMM_ERR_INVALID, "sizes");
  s.ij = true;
  s.ij_common_box = common_box != 0;
  s.trav_sized = false;  // the frontier holds one pair, not one per root
  try {
    solve_all(s);
  } catch (...) {
    s.ij = false;
    throw;
  }
  s.ij = false;
}

extern "C" {

int fmm_b200_default_config(fmm_b200_config* c) {
  if (!c) return FMM_ERR_INVALID;
  c->basis = FMM_SPHERICAL;
  c->P = 10;
  c->theta = 0.4;
  c->ncrit = 64;
  c->nspawn = 1000;
  c->use_rmax = 1;
  c->use_ropt = 1;
  c->precision = FMM_FP32;
  c->eps2 = 0.0;
  c->images = 0;
  c->device = 0;
  c->cycle = 2 * M_PI;
  c->mutual = 0;
  c->tree = FMM_TREE_ADAPTIVE;
  return FMM_OK;
}

int fmm_b200_supported_orders(int basis, int* orders, int cap) {
  std::vector<int> v = basis == FMM_CARTESIAN ? cartesian_orders() : spherical_orders();
  for (int i = 0; i < (int)v.size() && i < cap; i++) orders[i] = v[i];
  return (int)v.size();
}

int fmm_b200_create(const fmm_b200_config* cfg, fmm_b200_solver** out) {
  g_create_error.clear();
  if (!cfg || !out) {
    g_create_error = "null argument";
    return FMM_ERR_INVALID;
  }
  *out = nullptr;
  if (cfg->basis != FMM_SPHERICAL && cfg->basis != FMM_CARTESIAN) {
    g_create_error = "unknown basis";
    return FMM_ERR_INVALID;
  }
  if (cfg->images < 0 || (cfg->images > 0 && !(cfg->cycle > 0.0))) {
    g_create_error = "images must be >= 0 and cycle > 0 when images > 0";
    return FMM_ERR_INVALID;
  }
  if (cfg->mutual != 0 && cfg->mutual != 1) {
    g_create_error = "mutual must be 0 or 1";
    return FMM_ERR_INVALID;
  }
  if (cfg->tree != FMM_TREE_ADAPTIVE && cfg->tree != FMM_TREE_UNIFORM) {
    g_create_error = "tree must be FMM_TREE_ADAPTIVE or FMM_TREE_UNIFORM";
    return FMM_ERR_INVALID;
  }
  std::vector<int> ords = cfg->basis == FMM_CARTESIAN ? cartesian_orders() : spherical_orders();
  if (std::find(ords.begin(), ords.end(), cfg->P) == ords.end()) {
    g_create_error = "expansion order P=" + std::to_string(cfg->P) + " not compiled for this basis";
    return FMM_ERR_INVALID;
  }
  if (!(cfg->theta > 0.0 && cfg->theta < 1.0) || cfg->ncrit < 1 || cfg->nspawn < 1 ||
      (cfg->precision != FMM_FP32 && cfg->precision != FMM_FP64) || !(cfg->eps2 >= 0.0)) {
    g_create_error = "invalid theta / ncrit / nspawn / precision / eps2";
    return FMM_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0) {
    (void)cudaGetLastError();
    g_create_error = "no CUDA device " + std::to_string(cfg->device);
    return FMM_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10) {
    (void)cudaGetLastError();
    g_create_error = "kernels are built for sm_100a (B200); device is sm_" +
                     std::to_string(prop.major) + std::to_string(prop.minor);
    return FMM_ERR_NO_DEVICE;
  }
  fmm_b200_solver* h = new fmm_b200_solver();
  h->precision = cfg->precision;
  if (cfg->precision == FMM_FP64) h->base = new Solver<double>();
  else h->base = new Solver<float>();
  SolverBase& s = *h->base;
  s.cfg = *cfg;
  s.nterm = cfg->basis == FMM_SPHERICAL ? nterm_sph(cfg->P) : nterm_cart(cfg->P);
  s.ncoef = cfg->basis == FMM_SPHERICAL ? 2 * s.nterm : s.nterm;
  try {
    FMM_CUDA(cudaSetDevice(cfg->device));
    s.scal.ensure(512);
    FMM_CUDA(cudaMallocHost((void**)&s.scal_host, 512 * sizeof(int)));
    for (int i = 0; i < 2 * FMM_NUM_PHASES; i++) FMM_CUDA(cudaEventCreate(&s.ev[i]));
  } catch (const FmmError& e) {
    g_create_error = e.what();
    delete h->base;
    delete h;
    return e.code;
  }
  *out = h;
  return FMM_OK;
}

// every device array of a handle (the typed ones through the precision); OP is a member
// function of DevArr (release, free_retired)
#define FMM_FOR_ALL_ARRAYS(h, OP)                                                          \
  do {                                                                                     \
    SolverBase& s_ = *(h)->base;                                                           \
    DevArr<int>* ia[] = {&s_.nbegin,   &s_.ncount,   &s_.nparent,  &s_.nchildn, &s_.nfirst, \
                         &s_.nnode,    &s_.npos,     &s_.ncb,      &s_.nlevel,  &s_.nsplit, \
                         &s_.coff,     &s_.leaves,   &s_.idx,      &s_.idx2,    &s_.scal,   \
                         &s_.c_iparent, &s_.c_ichild, &s_.c_nchild, &s_.c_ibody, &s_.c_nbody, \
                         &s_.c_level,  &s_.order,    &s_.m2l_off,  &s_.p2p_off, &s_.seg_cnt, \
                         &s_.d_lvl,    &s_.seg_cnt2, &s_.body_leaf, &s_.d_seg,  &s_.d_root_first, \
                         &s_.d_root_count, &s_.nsid, &s_.c_root,   &s_.cbase,   &s_.fs_pos, \
                         &s_.fs_pos2,  &s_.fs_idx,   &s_.m2l_tgt,  &s_.k_list,  &s_.k_saved_leaves}; \
    for (auto* a : ia) a->OP();                                                            \
    s_.keys.OP(); s_.keys2.OP(); s_.c_icell.OP(); s_.m2l.OP(); s_.fs_keys.OP();            \
    s_.c_info.OP(); s_.fs_root.OP(); s_.fs_root2.OP();                                     \
    s_.p2p.OP(); s_.list_tmp.OP(); s_.p2p_pairs_count.OP();                                \
    s_.cub_tmp.OP(); s_.front.OP(); s_.front2.OP();                                        \
    s_.seg_keys2.OP(); s_.cub_tmp2.OP(); s_.dtmp.OP();                                     \
    if ((h)->precision == FMM_FP64) {                                                      \
      Solver<double>& d_ = *static_cast<Solver<double>*>((h)->base);                       \
      d_.bodies_in.OP(); d_.bodies.OP(); d_.trg_s.OP(); d_.trg_e.OP(); d_.trg_out.OP();    \
      d_.cX.OP(); d_.box.OP(); d_.M.OP(); d_.L.OP(); d_.nX.OP(); d_.m0.OP();               \
      d_.pM.OP(); d_.pM2.OP(); d_.pC.OP(); d_.c_root_cells.OP(); d_.minmax_part.OP();      \
      d_.k_rows.OP(); d_.k_cx.OP(); d_.k_trg.OP();                                         \
    } else {                                                                               \
      Solver<float>& d_ = *static_cast<Solver<float>*>((h)->base);                         \
      d_.bodies_in.OP(); d_.bodies.OP(); d_.trg_s.OP(); d_.trg_e.OP(); d_.trg_out.OP();    \
      d_.cX.OP(); d_.box.OP(); d_.M.OP(); d_.L.OP(); d_.nX.OP(); d_.m0.OP();               \
      d_.pM.OP(); d_.pM2.OP(); d_.pC.OP(); d_.c_root_cells.OP(); d_.minmax_part.OP();      \
      d_.k_rows.OP(); d_.k_cx.OP(); d_.k_trg.OP();                                         \
    }                                                                                      \
  } while (0)

int fmm_b200_trim(fmm_b200_solver* h) {
  return guarded(h, [&] {
    FMM_CUDA(cudaStreamSynchronize(h->base->stream));
    FMM_FOR_ALL_ARRAYS(h, free_retired);
  });
}

int fmm_b200_destroy(fmm_b200_solver* h) {
  if (!h) return FMM_ERR_INVALID;
  if (h->base) {
    SolverBase& s = *h->base;
    cudaSetDevice(s.cfg.device);
    cudaStreamSynchronize(s.stream);
    FMM_FOR_ALL_ARRAYS(h, release);
    for (int i = 0; i < 2 * FMM_NUM_PHASES; i++)
      if (s.ev[i]) cudaEventDestroy(s.ev[i]);
    if (s.fork) cudaEventDestroy(s.fork);
    if (s.join) cudaEventDestroy(s.join);
    if (s.side) cudaStreamDestroy(s.side);
    if (s.side_lo) cudaStreamDestroy(s.side_lo);
    if (s.p2p_ready) cudaEventDestroy(s.p2p_ready);
    if (s.scal_host) cudaFreeHost(s.scal_host);
    if (s.roots_host) cudaFreeHost(s.roots_host);
    for (int2* q : s.roots_retired) cudaFreeHost(q);
    delete h->base;
  }
  delete h;
  return FMM_OK;
}

int fmm_b200_set_mutual(fmm_b200_solver* h, int mutual) {
  if (!h || !h->base || (mutual != 0 && mutual != 1)) return FMM_ERR_INVALID;
  h->base->cfg.mutual = mutual;
  h->base->trav_sized = false;
  return FMM_OK;
}

int fmm_b200_set_periodic(fmm_b200_solver* h, int images, double cycle) {
  if (!h || !h->base) return FMM_ERR_INVALID;
  if (images < 0 || (images > 0 && !(cycle > 0.0))) return FMM_ERR_INVALID;
  h->base->cfg.images = images;
  h->base->cfg.cycle = cycle;
  return FMM_OK;
}

int fmm_b200_set_partition(fmm_b200_solver* h, int part, int nparts) {
  if (!h || !h->base) return FMM_ERR_INVALID;
  if (nparts < 1 || part < 0 || part >= nparts) {
    h->base->err = "partition: need 0 <= part < nparts";
    return FMM_ERR_INVALID;
  }
  h->base->part = part;
  h->base->nparts = nparts;
  h->base->err.clear();
  return FMM_OK;
}

int fmm_b200_get_partition(fmm_b200_solver* h, int* part, int* nparts, int* body_begin,
                           int* body_end) {
  return guarded(h, [&] {
    fmmb200::SolverBase& s = *h->base;
    if (part) *part = s.part;
    if (nparts) *nparts = s.nparts;
    int r[2] = {0, s.n};
    if (s.nparts > 1 && s.stage >= fmmb200::ST_TREE && s.n > 0 && s.part_range.p) {
      FMM_CUDA(cudaMemcpyAsync(r, s.part_range.p, sizeof(r), cudaMemcpyDeviceToHost, s.stream));
      FMM_CUDA(cudaStreamSynchronize(s.stream));
    }
    if (body_begin) *body_begin = r[0];
    if (body_end) *body_end = r[1];
  });
}

int fmm_b200_set_stream(fmm_b200_solver* h, void* stream) {
  return guarded(h, [&] { h->base->stream = (cudaStream_t)stream; });
}

const char* fmm_b200_last_error(const fmm_b200_solver* h) {
  if (!h || !h->base) return g_create_error.c_str();
  return h->base->err.c_str();
}

int fmm_b200_set_bodies_host(fmm_b200_solver* h, int n, const double* x, const double* q) {
  if (n < 0 || (n > 0 && (!x || !q))) return FMM_ERR_INVALID;
  if (!h || !h->base) return FMM_ERR_INVALID;
  h->base->seg = {0, n};
  return FMM_DISPATCH(h, set_bodies_host_t(s, n, x, q, h->base->dtmp));
}

int fmm_b200_set_bodies_device(fmm_b200_solver* h, int n, const void* d_bodies) {
  if (n < 0 || (n > 0 && !d_bodies)) return FMM_ERR_INVALID;
  if (!h || !h->base) return FMM_ERR_INVALID;
  h->base->seg = {0, n};
  return FMM_DISPATCH(h, {
    s.n = n;
    s.bodies_in.ensure(std::max(n, 1));
    if (n > 0)
      FMM_CUDA(cudaMemcpyAsync(s.bodies_in.p, d_bodies, sizeof(s.bodies_in.p[0]) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
    s.stage = ST_BODIES;
  });
}

int fmm_b200_build_tree(fmm_b200_solver* h) { return FMM_DISPATCH(h, stage_tree(s)); }
int fmm_b200_upward_pass(fmm_b200_solver* h) { return FMM_DISPATCH(h, stage_up(s)); }
int fmm_b200_traverse(fmm_b200_solver* h) { return FMM_DISPATCH(h, stage_trav(s)); }
int fmm_b200_downward_pass(fmm_b200_solver* h) { return FMM_DISPATCH(h, stage_down(s)); }

int fmm_b200_autotune_ncrit(fmm_b200_solver* h, const int* candidates, int ncand, int repeats,
                            int* best_ncrit, double* times_ms) {
  if (!h || !h->base || !candidates || ncand < 1 || repeats < 1) return FMM_ERR_INVALID;
  for (int i = 0; i < ncand; i++)
    if (candidates[i] < 1) return FMM_ERR_INVALID;
  return FMM_DISPATCH(h, autotune_ncrit_t(s, candidates, ncand, repeats, best_ncrit, times_ms));
}

int fmm_b200_autotune_p2p(fmm_b200_solver* h, const int* lanes4_max, const int* lanes2_max,
                          int ncand, int repeats, int* best, double* times_ms) {
  if (!h || !h->base || !lanes4_max || !lanes2_max || ncand < 1 || repeats < 1)
    return FMM_ERR_INVALID;
  for (int i = 0; i < ncand; i++)
    if (lanes4_max[i] < 0 || lanes4_max[i] > 8 || lanes2_max[i] < lanes4_max[i] ||
        lanes2_max[i] > 16)
      return FMM_ERR_INVALID;
  return FMM_DISPATCH(h, autotune_p2p_t(s, lanes4_max, lanes2_max, ncand, repeats, best,
                                        times_ms));
}

int fmm_b200_solve_device(fmm_b200_solver* h, int n, const void* d_bodies, void* d_trg) {
  if (n < 0 || (n > 0 && (!d_bodies || !d_trg))) return FMM_ERR_INVALID;
  if (!h || !h->base) return FMM_ERR_INVALID;
  h->base->seg = {0, n};
  return FMM_DISPATCH(h, {
    s.n = n;
    s.bodies_in.ensure(std::max(n, 1));
    if (n > 0)
      FMM_CUDA(cudaMemcpyAsync(s.bodies_in.p, d_bodies, sizeof(s.bodies_in.p[0]) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
    s.stage = ST_BODIES;
    solve_all(s);
    if (n > 0)
      FMM_CUDA(cudaMemcpyAsync(d_trg, s.trg_out.p, sizeof(s.trg_out.p[0]) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
  });
}

int fmm_b200_solve_host(fmm_b200_solver* h, int n, const double* x, const double* q, double* p,
                        double* f) {
  if (n < 0 || (n > 0 && (!x || !q || !p || !f))) return FMM_ERR_INVALID;
  if (!h || !h->base) return FMM_ERR_INVALID;
  h->base->seg = {0, n};
  return FMM_DISPATCH(h, {
    DevArr<double>& tmp = h->base->dtmp;
    set_bodies_host_t(s, n, x, q, tmp);
    solve_all(s);
    if (n > 0) {
      tmp.ensure(4 * (size_t)n);
      k_unpack_pf<T><<<ceil_div(n, 256), 256, 0, s.stream>>>(n, s.trg_out.p, tmp.p, tmp.p + n);
      FMM_LAUNCH_CHECK();
      FMM_CUDA(cudaMemcpyAsync(p, tmp.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s.stream));
      FMM_CUDA(cudaMemcpyAsync(f, tmp.p + n, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost,
                               s.stream));
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_solve_batch_device(fmm_b200_solver* h, int nsolves, const int* counts,
                                const void* d_bodies, void* d_trg) {
  if (!h || !h->base) return FMM_ERR_INVALID;
  int n = 0;
  if (!set_segments(*h->base, nsolves, counts, &n)) return FMM_ERR_INVALID;
  if (n > 0 && (!d_bodies || !d_trg)) return FMM_ERR_INVALID;
  return FMM_DISPATCH(h, {
    s.n = n;
    s.bodies_in.ensure(std::max(n, 1));
    if (n > 0)
      FMM_CUDA(cudaMemcpyAsync(s.bodies_in.p, d_bodies, sizeof(s.bodies_in.p[0]) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
    s.stage = ST_BODIES;
    solve_all(s);
    if (n > 0)
      FMM_CUDA(cudaMemcpyAsync(d_trg, s.trg_out.p, sizeof(s.trg_out.p[0]) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
  });
}

int fmm_b200_solve_batch_host(fmm_b200_solver* h, int nsolves, const int* counts,
                              const double* x, const double* q, double* p, double* f) {
  if (!h || !h->base) return FMM_ERR_INVALID;
  int n = 0;
  if (!set_segments(*h->base, nsolves, counts, &n)) return FMM_ERR_INVALID;
  if (n > 0 && (!x || !q || !p || !f)) return FMM_ERR_INVALID;
  return FMM_DISPATCH(h, {
    DevArr<double>& tmp = h->base->dtmp;
    std::vector<int> seg = s.seg;
    set_bodies_host_t(s, n, x, q, tmp);
    s.seg = seg;
    solve_all(s);
    if (n > 0) {
      tmp.ensure(4 * (size_t)n);
      k_unpack_pf<T><<<ceil_div(n, 256), 256, 0, s.stream>>>(n, s.trg_out.p, tmp.p, tmp.p + n);
      FMM_LAUNCH_CHECK();
      FMM_CUDA(cudaMemcpyAsync(p, tmp.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s.stream));
      FMM_CUDA(cudaMemcpyAsync(f, tmp.p + n, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost,
                               s.stream));
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_solve_ij_host(fmm_b200_solver* h, int nt, const double* xt, const double* qt,
                           int ns, const double* xs, const double* qs, int common_box, double* p,
                           double* f) {
  if (!h || !h->base || nt < 0 || ns < 0) return FMM_ERR_INVALID;
  if ((nt > 0 && (!xt || !qt || !p || !f)) || (ns > 0 && (!xs || !qs))) return FMM_ERR_INVALID;
  if (nt == 0) return FMM_OK;
  std::vector<double> x(3 * ((size_t)nt + ns)), q((size_t)nt + ns);
  std::memcpy(x.data(), xt, sizeof(double) * 3 * nt);
  std::memcpy(q.data(), qt, sizeof(double) * nt);
  if (ns) {
    std::memcpy(x.data() + 3 * (size_t)nt, xs, sizeof(double) * 3 * ns);
    std::memcpy(q.data() + nt, qs, sizeof(double) * ns);
  }
  return FMM_DISPATCH(h, {
    DevArr<double>& tmp = h->base->dtmp;
    set_bodies_host_t(s, nt + ns, x.data(), q.data(), tmp);
    solve_ij_t(h, s, nt, ns, common_box);
    tmp.ensure(4 * (size_t)nt);
    k_unpack_pf<T><<<ceil_div(nt, 256), 256, 0, s.stream>>>(nt, s.trg_out.p, tmp.p, tmp.p + nt);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaMemcpyAsync(p, tmp.p, sizeof(double) * nt, cudaMemcpyDeviceToHost, s.stream));
    FMM_CUDA(cudaMemcpyAsync(f, tmp.p + nt, 3 * sizeof(double) * nt, cudaMemcpyDeviceToHost,
                             s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_solve_ij_device(fmm_b200_solver* h, int nt, const void* d_targets, int ns,
                             const void* d_sources, int common_box, void* d_trg) {
  if (!h || !h->base || nt < 0 || ns < 0) return FMM_ERR_INVALID;
  if ((nt > 0 && (!d_targets || !d_trg)) || (ns > 0 && !d_sources)) return FMM_ERR_INVALID;
  if (nt == 0) return FMM_OK;
  return FMM_DISPATCH(h, {
    s.n = nt + ns;
    s.bodies_in.ensure(std::max(s.n, 1));
    FMM_CUDA(cudaMemcpyAsync(s.bodies_in.p, d_targets, sizeof(s.bodies_in.p[0]) * nt,
                             cudaMemcpyDeviceToDevice, s.stream));
    if (ns)
      FMM_CUDA(cudaMemcpyAsync(s.bodies_in.p + nt, d_sources, sizeof(s.bodies_in.p[0]) * ns,
                               cudaMemcpyDeviceToDevice, s.stream));
    s.stage = ST_BODIES;
    solve_ij_t(h, s, nt, ns, common_box);
    FMM_CUDA(cudaMemcpyAsync(d_trg, s.trg_out.p, sizeof(s.trg_out.p[0]) * nt,
                             cudaMemcpyDeviceToDevice, s.stream));
  });
}

int fmm_b200_set_bodies_batch_device(fmm_b200_solver* h, int nsolves, const int* counts,
                                     const void* d_bodies) {
  if (!h || !h->base) return FMM_ERR_INVALID;
  int n = 0;
  if (!set_segments(*h->base, nsolves, counts, &n)) return FMM_ERR_INVALID;
  if (n > 0 && !d_bodies) return FMM_ERR_INVALID;
  return FMM_DISPATCH(h, {
    s.n = n;
    s.bodies_in.ensure(std::max(n, 1));
    if (n > 0)
      FMM_CUDA(cudaMemcpyAsync(s.bodies_in.p, d_bodies, sizeof(s.bodies_in.p[0]) * n,
                               cudaMemcpyDeviceToDevice, s.stream));
    s.stage = ST_BODIES;
  });
}

int fmm_b200_get_roots(fmm_b200_solver* h, int* nroots, int* root_cells, int* root_solves) {
  return guarded(h, [&] {
    SolverBase& s = *h->base;
    if (s.stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "tree not built");
    if (nroots) *nroots = s.nroots;
    for (int r = 0; r < s.nroots; r++) {
      if (root_cells) root_cells[r] = s.root_cell[r];
      if (root_solves) root_solves[r] = s.root_solve[r];
    }
  });
}

int fmm_b200_get_trg_host(fmm_b200_solver* h, double* trg) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_DOWN) throw FmmError(FMM_ERR_STATE, "downward pass not done");
    if (s.n > 0) {
      DevArr<double>& tmp = h->base->dtmp;
      tmp.ensure(4 * (size_t)s.n);
      k_unpack<T><<<ceil_div(s.n, 256), 256, 0, s.stream>>>(s.n, s.trg_out.p, tmp.p);
      FMM_LAUNCH_CHECK();
      FMM_CUDA(cudaMemcpyAsync(trg, tmp.p, 4 * sizeof(double) * s.n, cudaMemcpyDeviceToHost,
                               s.stream));
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_get_trg_device(fmm_b200_solver* h, void* d_trg) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_DOWN) throw FmmError(FMM_ERR_STATE, "downward pass not done");
    if (s.n > 0)
      FMM_CUDA(cudaMemcpyAsync(d_trg, s.trg_out.p, sizeof(s.trg_out.p[0]) * s.n,
                               cudaMemcpyDeviceToDevice, s.stream));
  });
}

int fmm_b200_num_cells(fmm_b200_solver* h, int* nc, int* ml) {
  return guarded(h, [&] {
    if (h->base->stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "tree not built");
    if (nc) *nc = h->base->ncells;
    if (ml) *ml = h->base->maxlevel;
  });
}

int fmm_b200_get_cells(fmm_b200_solver* h, int* iparent, int* ichild, int* nchild, int* ibody,
                       int* nbody, unsigned long long* icell, int* level, double* X, double* R) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "tree not built");
    const int nc = s.ncells;
    if (nc == 0) return;
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (dst) FMM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s.stream));
    };
    cp(iparent, s.c_iparent.p, 4 * (size_t)nc);
    cp(ichild, s.c_ichild.p, 4 * (size_t)nc);
    cp(nchild, s.c_nchild.p, 4 * (size_t)nc);
    cp(ibody, s.c_ibody.p, 4 * (size_t)nc);
    cp(nbody, s.c_nbody.p, 4 * (size_t)nc);
    cp(icell, s.c_icell.p, 8 * (size_t)nc);
    cp(level, s.c_level.p, 4 * (size_t)nc);
    if (X || R) {
      DevArr<double>& tmp = h->base->dtmp;
      tmp.ensure(4 * (size_t)nc);
      k_cells_out<T><<<ceil_div(nc, 256), 256, 0, s.stream>>>(nc, s.cX.p, tmp.p, tmp.p + 3 * (size_t)nc);
      FMM_LAUNCH_CHECK();
      cp(X, tmp.p, 24 * (size_t)nc);
      cp(R, tmp.p + 3 * (size_t)nc, 8 * (size_t)nc);
    }
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_get_order(fmm_b200_solver* h, int* ibody) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "tree not built");
    if (s.n > 0)
      FMM_CUDA(cudaMemcpyAsync(ibody, s.order.p, 4 * (size_t)s.n, cudaMemcpyDeviceToHost, s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_get_box(fmm_b200_solver* h, double* x0r0) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_TREE) throw FmmError(FMM_ERR_STATE, "tree not built");
    DevArr<double>& tmp = h->base->dtmp;
    tmp.ensure(4);
    k_to_double<T><<<1, 32, 0, s.stream>>>((size_t)4, s.box.p, tmp.p);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaMemcpyAsync(x0r0, tmp.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_get_expansion(fmm_b200_solver* h, int which, double* out) {
  return FMM_DISPATCH(h, {
    if (s.stage < ST_UP) throw FmmError(FMM_ERR_STATE, "upward pass not done");
    const size_t ne = (size_t)s.ncells * s.ncoef;
    if (ne == 0) return;
    DevArr<double>& tmp = h->base->dtmp;
    tmp.ensure(ne);
    k_to_double<T><<<ceil_div((long long)ne, 256), 256, 0, s.stream>>>(ne, which ? s.L.p : s.M.p, tmp.p);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaMemcpyAsync(out, tmp.p, ne * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_num_lists(fmm_b200_solver* h, long long* nm2l, long long* np2p, long long* bp) {
  return guarded(h, [&] {
    if (h->base->stage < ST_TRAV) throw FmmError(FMM_ERR_STATE, "traversal not done");
    if (nm2l) *nm2l = h->base->nm2l;
    if (np2p) *np2p = h->base->np2p;
    if (bp) {
      if (h->base->p2p_body_pairs < 0) h->base->p2p_body_pairs = count_p2p_body_pairs(*h->base);
      *bp = h->base->p2p_body_pairs;
    }
  });
}

int fmm_b200_get_lists(fmm_b200_solver* h, long long* m2l, long long* p2p) {
  return guarded(h, [&] {
    SolverBase& s = *h->base;
    if (s.stage < ST_TRAV) throw FmmError(FMM_ERR_STATE, "traversal not done");
    if (m2l && s.nm2l)
      FMM_CUDA(cudaMemcpyAsync(m2l, s.m2l.p, 8 * (size_t)s.nm2l, cudaMemcpyDeviceToHost, s.stream));
    if (p2p && s.np2p)
      FMM_CUDA(cudaMemcpyAsync(p2p, s.p2p.p, 8 * (size_t)s.np2p, cudaMemcpyDeviceToHost, s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  });
}

int fmm_b200_get_timings(fmm_b200_solver* h, double* ms) {
  return guarded(h, [&] {
    SolverBase& s = *h->base;
    FMM_CUDA(cudaStreamSynchronize(s.stream));
    for (int p = 0; p < FMM_NUM_PHASES; p++) {
      ms[p] = 0;
      if (!s.ev_used[p]) continue;
      float t = 0;
      FMM_CUDA(cudaEventElapsedTime(&t, s.ev[2 * p], s.ev[2 * p + 1]));
      ms[p] = t;
    }
  });
}

}  // extern "C"
