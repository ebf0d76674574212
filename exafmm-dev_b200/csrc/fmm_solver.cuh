// Per-handle solver state and the stage entry points each translation unit implements.
//
// HBM layout of one solve (T = float or double, N bodies, C cells):
//   bodies_in   vec4<T>[N]   caller order (x, y, z, q)
//   bodies      vec4<T>[N]   tree order (the reference's permuted Bodies)
//   order       int[N]       original index of each tree-order body (Body::IBODY)
//   trg_s/trg_e vec4<T>[N]   potential + gradient, compensated sum and its error term
//   cells       SoA over C:  iparent, ichild, nchild, ibody, nbody, level (int),
//                            icell (u64), X = (x, y, z, R) vec4<T>
//   M, L        T[C * ncoef] expansions, ncoef = 2 * NTERM (spherical) or NTERM
//   m2l, p2p    u64 pairs (target << 32 | source) sorted by target, + CSR offsets[C + 1]
// Tree nodes are built breadth first (level by level) and each node knows its cell slot,
// so level-synchronous passes walk node ranges and write cells in the reference layout.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "fmm_common.cuh"

namespace fmmb200 {

// A grow-only device array owned by one solver: freed with it, moved (never copied).
// Buffers it grows out of are retired, not freed, until the array is released: cudaFree
// synchronises the whole device, which would stall every other stream at each growth (the
// serving loop's other workers among them).  Growth doubles, so the retired buffers add up
// to at most the final size, and a handle that meets ever larger inputs grows a few times.
template <typename U> struct DevArr {
  U* p = nullptr;
  size_t cap = 0;
  std::vector<U*> retired;
  DevArr() = default;
  DevArr(const DevArr&) = delete;
  DevArr& operator=(const DevArr&) = delete;
  DevArr(DevArr&& o) noexcept : p(o.p), cap(o.cap), retired(std::move(o.retired)) {
    o.p = nullptr;
    o.cap = 0;
    o.retired.clear();
  }
  DevArr& operator=(DevArr&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      cap = o.cap;
      retired = std::move(o.retired);
      o.p = nullptr;
      o.cap = 0;
      o.retired.clear();
    }
    return *this;
  }
  ~DevArr() { release(); }
  void ensure(size_t n) {
    if (n <= cap) return;
    if (p) retired.push_back(p);
    p = nullptr;
    cap = 0;
    size_t want = 2 * n + 256;
    g_device_allocs.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaMalloc((void**)&p, want * sizeof(U));
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
      throw FmmError(FMM_ERR_NO_MEMORY, "cudaMalloc of " + std::to_string(want * sizeof(U)) +
                                            " bytes failed: " + cudaGetErrorString(e));
    }
    cap = want;
  }
  void free_retired() {
    for (U* q : retired) cudaFree(q);
    retired.clear();
  }
  void release() {
    if (p) cudaFree(p);
    free_retired();
    p = nullptr;
    cap = 0;
  }
};

// Move a's buffers (its current one and those it retired) into b's retired list, leaving a
// empty, for a grow-and-copy that replaces a with b without freeing during a solve.
template <typename U> void retire_into(DevArr<U>& a, DevArr<U>& b) {
  if (a.p) b.retired.push_back(a.p);
  b.retired.insert(b.retired.end(), a.retired.begin(), a.retired.end());
  a.p = nullptr;
  a.cap = 0;
  a.retired.clear();
}

enum Stage { ST_NONE = 0, ST_BODIES = 1, ST_TREE = 2, ST_UP = 3, ST_TRAV = 4, ST_DOWN = 5 };

struct SolverBase {
  fmm_b200_config cfg;
  cudaStream_t stream = nullptr;
  int n = 0;
  // a batch of independent solves ("forest"): body ranges [seg[s], seg[s+1]) per solve;
  // every non-empty solve gets one root (roots in solve order), cells of a root contiguous
  std::vector<int> seg{0, 0};
  std::vector<int> root_solve;  // solve of each root
  std::vector<int> root_cell;   // first cell of each root (host copy)
  int nroots = 0;
  DevArr<int> d_seg, d_root_first, d_root_count, nsid, c_root, cbase;
  int ncoef = 0, nterm = 0;
  Stage stage = ST_NONE;
  std::string err;
  // tree shape (host copies of the few scalars the level loops need)
  int ncells = 0, maxlevel = 0, nleaves = 0;
  std::vector<int> level_lo;  // node index range of level l: [level_lo[l], level_lo[l+1])
  long long nm2l = 0, np2p = 0, p2p_body_pairs = 0;  // body pairs: -1 until counted
  // node arrays (breadth-first)
  DevArr<int> nbegin, ncount, nparent, nchildn, nfirst, nnode, npos, ncb, nlevel, nsplit;
  DevArr<int> coff;
  DevArr<int> leaves;  // cell index of every leaf
  // sort scratch
  DevArr<unsigned long long> keys, keys2;
  DevArr<int> idx, idx2;
  DevArr<char> cub_tmp;
  DevArr<int> scal;          // small device scalars (counters, flags)
  int* scal_host = nullptr;  // pinned mirror of scal
  // pinned staging of the traversal's first frontier (its copy needs no host wait: every
  // solve reads the traversal's totals back before the next one writes here); buffers it
  // grew out of are kept until the handle is destroyed (cudaFreeHost synchronises)
  int2* roots_host = nullptr;
  size_t roots_cap = 0;
  std::vector<int2*> roots_retired;
  // cells
  DevArr<int> c_iparent, c_ichild, c_nchild, c_ibody, c_nbody, c_level;
  DevArr<int4> c_info;  // per cell (NCHILD, ICHILD, NBODY, IBODY): one load for the traversal
  DevArr<unsigned long long> c_icell;
  DevArr<int> order;
  // interaction lists
  DevArr<unsigned> fs_root, fs_root2;  // forest sort: root of each key-sorted body
  DevArr<int> fs_pos, fs_pos2;
  DevArr<unsigned long long> fs_keys;
  DevArr<int> fs_idx;
  DevArr<int2> front, front2;
  bool trav_sized = false;  // list / frontier buffers sized by a counted traversal
  int trav_steps = 0, trav_maxlevel = 0;  // the last traversal's steps, and its tree depth
  int tree_plan = 0;        // levels of the handle's last tree (0: none; builds level by level)
  int write_r = 1;          // P2M / M2M set the cell radii (else the structure pass did)
  // P2P lanes per target by target leaf size: 4 up to p2p_g4 bodies, 2 up to p2p_g2, else 1
  // (p2p_g4 <= 8 and p2p_g2 <= 16: a warp holds 32 / lanes targets); fmm_b200_autotune_p2p
  int p2p_g4 = 8, p2p_g2 = 16;
  DevArr<int> d_lvl;        // level ends of the planned node build
  // targets and sources in two trees (segments 0 and 1) on a common box, traversed from
  // (target root, source root) only (fmm_b200_solve_ij_*)
  bool ij = false;
  bool ij_common_box = true;  // else each tree on its own bodies' box (the petiga wrapper)
  // target partition of one solve over nparts GPUs (fmm_b200_set_partition): the bodies of
  // part `part` in tree order, [part_range[0], part_range[1]), set on the device after the
  // tree build; the traversal keeps the pairs whose target cell holds some of them, and L2L
  // and L2P run on the cells and bodies of the part only
  int part = 0, nparts = 1;
  DevArr<int> part_range;
  const int* part_ptr() const { return nparts > 1 ? part_range.p : nullptr; }
  int nfront0 = 0;          // pairs of the first traversal step (roots x images)
  DevArr<unsigned long long> m2l, p2p, list_tmp;
  DevArr<int> m2l_off, p2p_off;
  DevArr<int> body_leaf;  // the leaf cell of each body (tree order), written by P2M
  DevArr<int> seg_cnt;  // pairs per target while a list is grouped by target
  // the P2P list's grouping when it runs on the side stream beside M2L (whole solves)
  DevArr<int> seg_cnt2;
  DevArr<unsigned> seg_keys2;
  DevArr<char> cub_tmp2;
  bool p2p_pending = false;
  cudaEvent_t p2p_ready = nullptr;
  DevArr<int> m2l_tgt;  // M2L target cells, by descending number of 32-source batches
  // P2P target leaves by descending body pairs (valid while p2p_ordered: the lists of the
  // last traversal), so that the longest leaves start first and none is left alone at the end
  DevArr<int> p2p_order, p2p_widx;
  DevArr<unsigned> p2p_wkey, p2p_wkey2;
  bool p2p_ordered = false;
  int m2l_ntgt = 0;
  DevArr<unsigned long long> p2p_pairs_count;
  DevArr<double> dtmp;  // host <-> device conversion scratch
  // phase timing
  cudaEvent_t ev[2 * FMM_NUM_PHASES] = {};
  bool ev_used[FMM_NUM_PHASES] = {};
  // whole solves run the latency-bound L2L levels on a high-priority side stream, forked
  // after M2L and joined before L2P, so that they overlap P2P
  cudaStream_t side = nullptr;
  cudaStream_t side_lo = nullptr;  // lowest priority: the upward expansions beside the traversal
  cudaEvent_t fork = nullptr, join = nullptr;
  // single-operator calls (fmm_kernels.cu): host copies of the cells' index fields for
  // argument checks (valid while kc_valid), the operator's cell list, saved values
  bool kc_valid = false;
  std::vector<int> kc_ibody, kc_nbody, kc_ichild, kc_nchild, kc_iparent;
  DevArr<int> k_list, k_saved_leaves;
  virtual ~SolverBase() {}
};

template <typename T> struct Solver : SolverBase {
  DevArr<vec4<T>> bodies_in, bodies, trg_s, trg_e, trg_out, cX;
  DevArr<T> box;  // per root, 16 values: X0[3], R0, Xmin[3], Xmax[3]
  DevArr<T> M, L, nX;
  DevArr<T> m0;  // monopole per cell (structure pass)
  DevArr<T> pM, pM2, pC;  // periodic cell multipoles and per-shift M2L terms
  DevArr<int> c_root_cells;
  DevArr<T> minmax_part;
  DevArr<T> k_rows;             // single-operator calls: saved expansion rows
  DevArr<vec4<T>> k_cx, k_trg;  // saved cell centres / radii, saved targets (sum, error)
};

// ---- stage implementations (one translation unit each) ---------------------------------
template <typename T> void build_tree(Solver<T>& s);          // fmm_tree.cu
void partition_range(SolverBase& s);                         // fmm_tree.cu: part_range
long long count_p2p_body_pairs(SolverBase& s);              // fmm_traverse.cu
template <typename T> void upward_pass(Solver<T>& s);         // fmm_passes.cu
template <typename T> void upward_expansions(Solver<T>& s);   // fmm_passes.cu: P2M, M2M
template <typename T> void structure_pass(Solver<T>& s);      // fmm_passes.cu: radii, ropt
template <typename T> void downward_pass(Solver<T>& s);       // fmm_passes.cu
template <typename T> void downward_l2l(Solver<T>& s);        // fmm_passes.cu: L2L levels
template <typename T> void downward_l2p(Solver<T>& s);        // fmm_passes.cu: L2P + output
template <typename T> void build_lists(Solver<T>& s, bool defer_p2p = false);  // fmm_traverse.cu
void finish_p2p_list(SolverBase& s);  // fmm_traverse.cu: after build_lists(s, true)
template <typename T> void run_m2l(Solver<T>& s);             // fmm_passes.cu
template <typename T> void run_p2p(Solver<T>& s);             // fmm_p2p.cu

// dispatch of the P-templated expansion kernels (fmm_spherical.cu, fmm_cartesian.cu)
template <typename T> struct ExpansionOps {
  // leaves: list of leaf cells; level cells given by node range + npos
  void (*p2m)(Solver<T>& s);
  void (*m2m_level)(Solver<T>& s, int lo, int hi);
  void (*m2l)(Solver<T>& s);
  void (*l2l_level)(Solver<T>& s, int lo, int hi);
  void (*l2p)(Solver<T>& s);
  void (*periodic)(Solver<T>& s);  // far field of the periodic images, or null
};
template <typename T> bool spherical_ops(int P, ExpansionOps<T>* ops);
template <typename T> bool cartesian_ops(int P, ExpansionOps<T>* ops);
std::vector<int> spherical_orders();
std::vector<int> cartesian_orders();

// phase timing helpers (fmm_capi.cu)
void phase_begin(SolverBase& s, int phase);
void phase_end(SolverBase& s, int phase);
// message of a failed call without a solver handle, read by fmm_b200_last_error(NULL)
void set_call_error(const char* msg);

// CUB wrappers compiled once (fmm_sort.cu)
void sort_pairs_u64(SolverBase& s, const unsigned long long* kin, unsigned long long* kout,
                    const int* vin, int* vout, int n, int end_bit,
                    int begin_bit = 0);
void sort_keys_u64(SolverBase& s, const unsigned long long* kin, unsigned long long* kout,
                   int n, int end_bit);
void sort_pairs_u32(SolverBase& s, const unsigned* kin, unsigned* kout, const int* vin,
                    int* vout, int n, int end_bit, DevArr<char>* tmp = nullptr);
// scratch: s.cub_tmp, or tmp for a scan that may run beside other CUB calls of the solver
void exclusive_sum_int(SolverBase& s, const int* in, int* out, int n,
                       DevArr<char>* tmp = nullptr);
void segmented_sort_pairs_u64(SolverBase& s, const unsigned long long* kin,
                              unsigned long long* kout, const int* vin, int* vout, int n,
                              int nseg, const int* begin, const int* end, int end_bit);
void sum_u64(SolverBase& s, const unsigned long long* in, unsigned long long* out, int n);

}  // namespace fmmb200
