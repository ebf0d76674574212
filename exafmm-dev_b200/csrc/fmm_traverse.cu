// Dual-tree traversal on the device (Traversal::dualTreeTraversal, include/traversal.h).
//
// The reference recurses from (root, root) (:248): a pair is far (M2L) when
// |Xi - Xj|^2 > (Ri + Rj)^2 (:40), two leaves interact directly (P2P, :44-58), and
// otherwise splitCell (:188-212) descends into the children of the leaf-less side, of both
// sides when NBODY_i + NBODY_j >= nspawn (TraverseRange :65-124, which for mutual = false
// visits every child pair), or of the larger cell (ties split Ci).  The set of emitted
// pairs depends only on each pair, so here the recursion runs breadth first: every
// iteration classifies a frontier of pairs in parallel (count pass + write pass, exact
// sizes, no overflow) and emits M2L pairs, P2P pairs and the next frontier.  Lists are
// then grouped by target (per-target CSR for the M2L and P2P kernels) and sorted by source
// within each target.
#include <algorithm>
#include <climits>
#include <vector>

#include "fmm_solver.cuh"

namespace fmmb200 {

enum {
  PAIR_DROP = -1,  // a partitioned solve: the target cell holds none of the part's bodies
  PAIR_M2L = 0, PAIR_P2P = 1, PAIR_SPLIT_I = 2, PAIR_SPLIT_J = 3, PAIR_SPLIT_IJ = 4,
  PAIR_SPLIT_SELF = 5  // mutual: a cell against itself, its children pairs (a, b), a <= b
};

// cj: source cell with the periodic image of the source tree in its top bits (pair_cell,
// pair_img); the distance is (Xi - Xj) - Xperiodic as the reference rounds it (:38)
// mutual (dualTreeTraversal's flag, open boundary): each unordered pair is visited once
// (TraverseRange drops the (latter, former) quarter of a range against itself, :108-113),
// a cell against itself always splits both sides (:200), and an M2L or a P2P between two
// different cells is emitted in both directions (the mutual kernels update both cells);
// *nout counts those outputs
// The pair's cell data (centres with radii, and (NCHILD, ICHILD, NBODY, IBODY)) are loaded
// together, so that a pair costs one round trip to memory rather than one per decision.
// A partitioned solve drops the pairs whose target cell holds none of the bodies [b0, b1):
// every pair below them has a target inside that cell, so the pairs kept are exactly the
// whole traversal's pairs of the part's targets (b0 = INT_MIN, b1 = INT_MAX keep all).
template <typename T>
__device__ __forceinline__ int classify_data(int ci, int cjp, const vec4<T>& a, const vec4<T>& b,
                                             const int4& fi, const int4& fj, int nspawn, T cycle,
                                             int mutual, int b0, int b1, int* nout) {
  const int cj = pair_cell((unsigned)cjp);
  T px, py, pz;
  img_shift<T>(pair_img((unsigned)cjp), cycle, px, py, pz);
  if (!(fi.w < b1 && fi.w + fi.z > b0)) {
    *nout = 0;
    return PAIR_DROP;
  }
  T R2 = norm_rn(sub_rn(sub_rn(a.x, b.x), px), sub_rn(sub_rn(a.y, b.y), py),
                 sub_rn(sub_rn(a.z, b.z), pz));
  T Rs = add_rn(a.w, b.w);
  if (R2 > mul_rn(Rs, Rs)) {
    *nout = mutual ? 2 : 1;
    return PAIR_M2L;
  }
  const int ni = fi.x, nj = fj.x;
  if (ni == 0 && nj == 0) {
    *nout = mutual && ci != cj ? 2 : 1;
    return PAIR_P2P;
  }
  if (nj == 0) {
    *nout = ni;
    return PAIR_SPLIT_I;
  }
  if (ni == 0) {
    *nout = nj;
    return PAIR_SPLIT_J;
  }
  if (mutual && ci == cj) {
    *nout = ni * (ni + 1) / 2;
    return PAIR_SPLIT_SELF;
  }
  if (fi.z + fj.z >= nspawn) {
    *nout = ni * nj;
    return PAIR_SPLIT_IJ;
  }
  if (a.w >= b.w) {
    *nout = ni;
    return PAIR_SPLIT_I;
  }
  *nout = nj;
  return PAIR_SPLIT_J;
}
template <typename T>
__device__ __forceinline__ int classify(int ci, int cjp, const vec4<T>* __restrict__ X,
                                        const int4* __restrict__ info, int nspawn, T cycle,
                                        int mutual, int b0, int b1, int* nout) {
  const int cj = pair_cell((unsigned)cjp);
  return classify_data<T>(ci, cjp, X[ci], X[cj], info[ci], info[cj], nspawn, cycle, mutual,
                          b0, b1, nout);
}

// pass 1: per-block totals of (M2L, P2P, children) added to three device counters
// the part's body range [range[0], range[1]) of a partitioned solve, else everything
__device__ __forceinline__ void part_bounds(const int* __restrict__ range, int& b0, int& b1) {
  b0 = INT_MIN;
  b1 = INT_MAX;
  if (range) {
    b0 = range[0];
    b1 = range[1];
  }
}

template <typename T>
__global__ void k_trav_count(const int2* __restrict__ front, int nfront,
                             const vec4<T>* __restrict__ X, const int4* __restrict__ info,
                             int nspawn, T cycle, int mutual, const int* __restrict__ range,
                             unsigned long long* __restrict__ counters) {
  int b0, b1;
  part_bounds(range, b0, b1);
  unsigned long long c[3] = {0, 0, 0};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nfront; t += gridDim.x * blockDim.x) {
    int2 p = front[t];
    int k;
    int ty = classify<T>(p.x, p.y, X, info, nspawn, cycle, mutual, b0, b1, &k);
    c[ty == PAIR_M2L ? 0 : ty == PAIR_P2P ? 1 : 2] += k;
  }
  for (int i = 0; i < 3; i++) {
    unsigned long long v = warp_sum(c[i]);
    if (lane_id() == 0 && v) atomicAdd(&counters[i], v);
  }
}

// pass 2: write.  Output slots come from one atomic per warp and output kind (the lanes'
// offsets from a warp prefix sum); the final lists are sorted afterwards, so their order
// does not depend on scheduling.
__device__ __forceinline__ unsigned long long warp_alloc(unsigned long long* counter,
                                                         unsigned k) {
  const int lane = lane_id();
  unsigned incl = k;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, (unsigned long long)total);
  base = __shfl_sync(0xffffffffu, base, 31);
  return base + (incl - k);
}

template <typename T>
__global__ void k_trav_write(const int2* __restrict__ front, int nfront,
                             const vec4<T>* __restrict__ X, const int4* __restrict__ info,
                             int nspawn, T cycle, int mutual, const int* __restrict__ range,
                             unsigned long long* __restrict__ counters,
                             unsigned long long* __restrict__ m2l,
                             unsigned long long* __restrict__ p2p, int2* __restrict__ next) {
  int b0, b1;
  part_bounds(range, b0, b1);
  const int stride = gridDim.x * blockDim.x;
  // every lane of a warp runs the same number of iterations (warp-uniform trip count)
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int wbase = t0 - lane_id();
  for (int w = wbase; w < nfront; w += stride) {
    const int t = w + lane_id();
    int ty = -1, k = 0;
    int2 p = make_int2(0, 0);
    if (t < nfront) {
      p = front[t];
      ty = classify<T>(p.x, p.y, X, info, nspawn, cycle, mutual, b0, b1, &k);
    }
    const unsigned long long packed = ((unsigned long long)(unsigned)p.x << 32) | (unsigned)p.y;
    // the reverse of a mutual pair (no periodic image with mutual)
    const unsigned long long rev = ((unsigned long long)(unsigned)p.y << 32) | (unsigned)p.x;
    const int cj = pair_cell((unsigned)p.y), img = (int)((unsigned)p.y & ~kCellMask);
    const unsigned long long om = warp_alloc(&counters[0], ty == PAIR_M2L ? (unsigned)k : 0u);
    const unsigned long long op = warp_alloc(&counters[1], ty == PAIR_P2P ? (unsigned)k : 0u);
    const unsigned long long o = warp_alloc(&counters[2], ty >= PAIR_SPLIT_I ? (unsigned)k : 0u);
    if (ty == PAIR_M2L) {
      m2l[om] = packed;
      if (k == 2) m2l[om + 1] = rev;
    } else if (ty == PAIR_P2P) {
      p2p[op] = packed;
      if (k == 2) p2p[op + 1] = rev;
    } else if (ty == PAIR_SPLIT_SELF) {
      const int c0 = info[p.x].y, n = info[p.x].x;
      unsigned long long q = o;
      for (int a = 0; a < n; a++)
        for (int b = a; b < n; b++) next[q++] = make_int2(c0 + a, c0 + b);
    } else if (ty == PAIR_SPLIT_I) {
      int c0 = info[p.x].y;
      for (int i = 0; i < k; i++) next[o + i] = make_int2(c0 + i, p.y);
    } else if (ty == PAIR_SPLIT_J) {
      int c0 = info[cj].y;
      for (int j = 0; j < k; j++) next[o + j] = make_int2(p.x, (c0 + j) | img);
    } else if (ty == PAIR_SPLIT_IJ) {
      int ci0 = info[p.x].y, cj0 = info[cj].y;
      int nj = info[cj].x;
      for (int i = 0; i < k; i++) next[o + i] = make_int2(ci0 + i / nj, (cj0 + i % nj) | img);
    }
  }
}

// One traversal step without a count pass, for a solver whose list and frontier buffers
// were sized by an earlier solve.  The frontier size is read on the device (no host round
// trip per step).  Each lane takes kTravItems consecutive frontier pairs (their loads are
// independent); output slots come from one warp-wide scan of the lanes' packed (M2L, P2P,
// children) counts and three atomics per warp.  Writes beyond a buffer's capacity are
// skipped but every slot below it is written and all are counted, so the host can tell an
// overflow from the final counts and redo the traversal in the counted form.
constexpr int kTravItems = 4;

template <typename T>
__global__ void __launch_bounds__(256)
    k_trav_step(const int2* __restrict__ front, const unsigned long long* __restrict__ nfront_p,
                unsigned long long front_cap, const vec4<T>* __restrict__ X,
                const int4* __restrict__ info, int nspawn, T cycle, int mutual, int ncells,
                const int* __restrict__ range,
                unsigned long long* __restrict__ ctr,  // [0] M2L, [1] P2P, [2] bad index
                unsigned long long* __restrict__ next_count, unsigned long long* __restrict__ m2l,
                unsigned long long m2l_cap, unsigned long long* __restrict__ p2p,
                unsigned long long p2p_cap, int2* __restrict__ next,
                unsigned long long next_cap) {
  const long long nfront = (long long)min(*nfront_p, front_cap);
  int b0, b1;
  part_bounds(range, b0, b1);
  const int lane = lane_id();
  const long long stride = (long long)gridDim.x * blockDim.x * kTravItems;
  const long long wbase =
      ((long long)blockIdx.x * blockDim.x + threadIdx.x - lane) * kTravItems;
  for (long long w = wbase; w < nfront; w += stride) {  // warp-uniform trip count
    const long long t0 = w + (long long)lane * kTravItems;
    int ty[kTravItems], k[kTravItems];
    int2 p[kTravItems];
    unsigned v = 0;  // packed: M2L in bits 0-8, P2P in 9-17, children in 18-31 (warp totals:
                     // <= 256, <= 256, <= 8192)
#pragma unroll
    for (int u = 0; u < kTravItems; u++) {
      ty[u] = -1;
      k[u] = 0;
      p[u] = t0 + u < nfront ? front[t0 + u] : make_int2(0, 0);
    }
    bool okp[kTravItems];
#pragma unroll
    for (int u = 0; u < kTravItems; u++)
      okp[u] = t0 + u < nfront && (unsigned)p[u].x < (unsigned)ncells &&
               (unsigned)pair_cell((unsigned)p[u].y) < (unsigned)ncells &&
               pair_img((unsigned)p[u].y) < 27;
    if constexpr (sizeof(T) == 4) {
      // FP32: all the items' cell data loaded before any is classified, so that the gathers
      // of the four pairs are in flight together (FP64 cells take twice the registers: one
      // pair at a time)
      vec4<T> ca[kTravItems], cb[kTravItems];
      int4 fa[kTravItems], fb[kTravItems];
#pragma unroll
      for (int u = 0; u < kTravItems; u++)
        if (okp[u]) {
          const int cj = pair_cell((unsigned)p[u].y);
          ca[u] = X[p[u].x];
          cb[u] = X[cj];
          fa[u] = info[p[u].x];
          fb[u] = info[cj];
        }
#pragma unroll
      for (int u = 0; u < kTravItems; u++)
        if (okp[u])
          ty[u] = classify_data<T>(p[u].x, p[u].y, ca[u], cb[u], fa[u], fb[u], nspawn, cycle,
                                   mutual, b0, b1, &k[u]);
    } else {
#pragma unroll
      for (int u = 0; u < kTravItems; u++)
        if (okp[u])
          ty[u] = classify<T>(p[u].x, p[u].y, X, info, nspawn, cycle, mutual, b0, b1, &k[u]);
    }
#pragma unroll
    for (int u = 0; u < kTravItems; u++) {
      if (t0 + u < nfront && !okp[u])
        atomicOr(&ctr[2], 1ULL);  // never expected: reported to the host, pair skipped
      v += (ty[u] == PAIR_M2L ? (unsigned)k[u] : 0u) |
           (ty[u] == PAIR_P2P ? (unsigned)k[u] << 9 : 0u) |
           (ty[u] >= PAIR_SPLIT_I ? (unsigned)k[u] << 18 : 0u);
    }
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    const unsigned tot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long bm = 0, bp = 0, bn = 0;
    if (lane == 31) {
      if (tot & 0x1ffu) bm = atomicAdd(&ctr[0], (unsigned long long)(tot & 0x1ffu));
      if ((tot >> 9) & 0x1ffu) bp = atomicAdd(&ctr[1], (unsigned long long)((tot >> 9) & 0x1ffu));
      if (tot >> 18) bn = atomicAdd(next_count, (unsigned long long)(tot >> 18));
    }
    bm = __shfl_sync(0xffffffffu, bm, 31) + ((incl - v) & 0x1ffu);
    bp = __shfl_sync(0xffffffffu, bp, 31) + (((incl - v) >> 9) & 0x1ffu);
    bn = __shfl_sync(0xffffffffu, bn, 31) + ((incl - v) >> 18);
#pragma unroll
    for (int u = 0; u < kTravItems; u++) {
      const unsigned long long packed =
          ((unsigned long long)(unsigned)p[u].x << 32) | (unsigned)p[u].y;
      const unsigned long long rev =
          ((unsigned long long)(unsigned)p[u].y << 32) | (unsigned)p[u].x;
      if (ty[u] == PAIR_M2L) {
        if (bm < m2l_cap) m2l[bm] = packed;
        if (k[u] == 2 && bm + 1 < m2l_cap) m2l[bm + 1] = rev;
        bm += k[u];
      } else if (ty[u] == PAIR_P2P) {
        if (bp < p2p_cap) p2p[bp] = packed;
        if (k[u] == 2 && bp + 1 < p2p_cap) p2p[bp + 1] = rev;
        bp += k[u];
      } else if (ty[u] >= PAIR_SPLIT_I) {
        // every slot below the capacity is written (the next step reads up to it)
        const unsigned long long o = bn;
        const int kw = o >= next_cap ? 0 : (int)min((unsigned long long)k[u], next_cap - o);
        const int cj = pair_cell((unsigned)p[u].y), img = (int)((unsigned)p[u].y & ~kCellMask);
        if (ty[u] == PAIR_SPLIT_SELF) {
          const int c0 = info[p[u].x].y, n = info[p[u].x].x;
          int w = 0;
          for (int a = 0; a < n; a++)
            for (int b = a; b < n; b++, w++)
              if (w < kw) next[o + w] = make_int2(c0 + a, c0 + b);
        } else if (ty[u] == PAIR_SPLIT_I) {
          const int c0 = info[p[u].x].y;
          for (int i = 0; i < kw; i++) next[o + i] = make_int2(c0 + i, p[u].y);
        } else if (ty[u] == PAIR_SPLIT_J) {
          const int c0 = info[cj].y;
          for (int j = 0; j < kw; j++) next[o + j] = make_int2(p[u].x, (c0 + j) | img);
        } else {
          const int ci0 = info[p[u].x].y, cj0 = info[cj].y, nj = info[cj].x;
          for (int i = 0; i < kw; i++)
            next[o + i] = make_int2(ci0 + i / nj, (cj0 + i % nj) | img);
        }
        bn += k[u];
      }
    }
  }
}

// ---------------------------------------------------------------- grouping by target
// A list leaves the traversal in the order its pairs were found (atomic slots).  It is
// grouped by target with a count per target (warp-aggregated atomics), an exclusive scan
// of the counts into the CSR offsets, and a scatter of every pair's source key
// (image << b | cell) into its target's range; each range is then sorted in shared memory
// and written back as (target << 32 | image << 27 | cell).  The result is the order of a
// global sort of the packed pairs (target, then image, then source cell), so it does not
// depend on the order in which the traversal emitted them.
constexpr int kSegWarpCap = 1024;   // keys one warp sorts in its registers
constexpr int kSegBlockCap = 8192;  // keys one block sorts; longer ranges: global sort
constexpr int kSegWarps = 8;
constexpr int kSegBlock = 512;

__global__ void k_seg_count(const unsigned long long* __restrict__ pairs, long long n,
                            int* __restrict__ cnt) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t0 = blockIdx.x * (long long)blockDim.x; t0 < n; t0 += stride) {
    const long long t = t0 + threadIdx.x;
    const unsigned act = __ballot_sync(0xffffffffu, t < n);
    if (t >= n) continue;
    const int tgt = (int)(pairs[t] >> 32);
    const unsigned grp = __match_any_sync(act, tgt);
    if (lane_id() == __ffs(grp) - 1) atomicAdd(&cnt[tgt], __popc(grp));
  }
}

// cnt holds the counts on entry and zeros on exit; each warp's pairs of one target take
// consecutive slots from the top of the target's remaining range
__global__ void k_seg_scatter(const unsigned long long* __restrict__ pairs, long long n,
                              const int* __restrict__ off, int* __restrict__ cnt, int b,
                              unsigned* __restrict__ keys) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int lane = lane_id();
  for (long long t0 = blockIdx.x * (long long)blockDim.x; t0 < n; t0 += stride) {
    const long long t = t0 + threadIdx.x;
    const unsigned act = __ballot_sync(0xffffffffu, t < n);
    if (t >= n) continue;
    const unsigned long long v = pairs[t];
    const int tgt = (int)(v >> 32);
    const unsigned src = (unsigned)v;
    const unsigned grp = __match_any_sync(act, tgt);
    const int leader = __ffs(grp) - 1, k = __popc(grp);
    int top = 0;
    if (lane == leader) top = atomicSub(&cnt[tgt], k);
    top = __shfl_sync(grp, top, leader);
    const int rank = __popc(grp & ((1u << lane) - 1));
    keys[off[tgt] + top - k + rank] = ((unsigned)pair_img(src) << b) | (unsigned)pair_cell(src);
  }
}

__device__ __forceinline__ unsigned long long seg_pair(int c, unsigned key, int b) {
  const unsigned src = ((key >> b) << kImgShift) | (key & ((1u << b) - 1));
  return ((unsigned long long)(unsigned)c << 32) | src;
}

// ascending bitonic sort of a[0, n2), n2 a power of two, by nt threads (tid) that sync
// with __syncthreads (BLOCK) or __syncwarp
template <bool BLOCK>
__device__ __forceinline__ void bitonic_sort(unsigned* a, int n2, int tid, int nt) {
  for (int k = 2; k <= n2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int p = tid; p < (n2 >> 1); p += nt) {
        const int i = ((p & ~(j - 1)) << 1) | (p & (j - 1));  // bit j of i clear
        const int l = i | j;
        const unsigned x = a[i], y = a[l];
        if ((x > y) == ((i & k) == 0)) {
          a[i] = y;
          a[l] = x;
        }
      }
      if (BLOCK) __syncthreads();
      else __syncwarp();
    }
}

// A warp's range of n <= 32 K keys sorted in registers: lane l holds keys l K .. l K + K - 1
// (padded with 0xffffffff), the bitonic network's stages of partner distance j < K run
// within each lane, those with j >= K pair the lanes l and l ^ (j / K) by shuffles; every
// index and, for k < K, every direction is a compile-time constant.
template <int K>
__device__ __forceinline__ void warp_sort_range(const unsigned* __restrict__ keys, int n, int c,
                                                int b, unsigned long long* __restrict__ out) {
  const int lane = lane_id();
  unsigned v[K];
#pragma unroll
  for (int r = 0; r < K; r++) {
    const int e = lane * K + r;
    v[r] = e < n ? keys[e] : 0xffffffffu;
  }
#pragma unroll
  for (int k = 2; k <= 32 * K; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j < K) {
#pragma unroll
        for (int r = 0; r < K; r++) {
          if (r & j) continue;
          const bool up = k < K ? (r & k) == 0 : (lane & (k / K)) == 0;
          const unsigned x = v[r], y = v[r | j];
          const unsigned lo = min(x, y), hi = max(x, y);
          v[r] = up ? lo : hi;
          v[r | j] = up ? hi : lo;
        }
      } else {
        const bool keep_min = ((lane & (j / K)) == 0) == ((lane & (k / K)) == 0);
#pragma unroll
        for (int r = 0; r < K; r++) {
          const unsigned y = __shfl_xor_sync(0xffffffffu, v[r], j / K);
          v[r] = keep_min ? min(v[r], y) : max(v[r], y);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < K; r++) {
    const int e = lane * K + r;
    if (e < n) out[e] = seg_pair(c, v[r], b);
  }
}

// one warp per target with at most kSegWarpCap pairs
__global__ void __launch_bounds__(32 * kSegWarps, 5)
    k_seg_sort_warp(int ncells, const int* __restrict__ off, const unsigned* __restrict__ keys,
                    int b, unsigned long long* __restrict__ out) {
  const int c = blockIdx.x * kSegWarps + (threadIdx.x >> 5);
  if (c >= ncells) return;
  const int s0 = off[c], n = off[c + 1] - s0;
  if (n == 0 || n > kSegWarpCap) return;
  keys += s0;
  out += s0;
  if (n <= 32) warp_sort_range<1>(keys, n, c, b, out);
  else if (n <= 64) warp_sort_range<2>(keys, n, c, b, out);
  else if (n <= 128) warp_sort_range<4>(keys, n, c, b, out);
  else if (n <= 256) warp_sort_range<8>(keys, n, c, b, out);
  else if (n <= 512) warp_sort_range<16>(keys, n, c, b, out);
  else warp_sort_range<32>(keys, n, c, b, out);
}

// the longer ranges, one block at a time; a range above kSegBlockCap is written unsorted and
// flagged for the global sort
__global__ void __launch_bounds__(kSegBlock)
    k_seg_sort_block(int ncells, const int* __restrict__ off, const unsigned* __restrict__ keys,
                     int b, unsigned long long* __restrict__ out, int* __restrict__ overflow) {
  __shared__ unsigned a[kSegBlockCap];
  __shared__ int todo[kSegBlock];
  __shared__ int ntodo;
  for (int base = blockIdx.x * kSegBlock; base < ncells; base += gridDim.x * kSegBlock) {
    if (threadIdx.x == 0) ntodo = 0;
    __syncthreads();
    const int cc = base + threadIdx.x;
    if (cc < ncells && off[cc + 1] - off[cc] > kSegWarpCap) todo[atomicAdd(&ntodo, 1)] = cc;
    __syncthreads();
    const int m = ntodo;
    for (int q = 0; q < m; q++) {
      const int c = todo[q];
      const int s0 = off[c], n = off[c + 1] - s0;
      if (n > kSegBlockCap) {
        for (int i = threadIdx.x; i < n; i += kSegBlock) out[s0 + i] = seg_pair(c, keys[s0 + i], b);
        if (threadIdx.x == 0) atomicExch(overflow, 1);
        continue;
      }
      int n2 = 32;
      while (n2 < n) n2 <<= 1;
      for (int i = threadIdx.x; i < n2; i += kSegBlock) a[i] = i < n ? keys[s0 + i] : 0xffffffffu;
      __syncthreads();
      bitonic_sort<true>(a, n2, threadIdx.x, kSegBlock);
      for (int i = threadIdx.x; i < n; i += kSegBlock) out[s0 + i] = seg_pair(c, a[i], b);
      __syncthreads();
    }
    __syncthreads();
  }
}

// M2L targets (cells with at least one source) keyed by their number of 32-source batches,
// largest first, so that the warps of an M2L block have about the same amount of work
// M2L targets by descending pair count in buckets of 2^shift pairs (targets of one bucket in
// cell order, which keeps neighbouring targets, and so their shared sources, together);
// cells without pairs last.  The spherical kernel takes sources in batches of 32 (shift 5),
// the Cartesian one a thread per target (shift 0: exact counts, even warps).
constexpr int kTgtKeyBits = 20, kTgtKeyMax = (1 << kTgtKeyBits) - 1;
__global__ void k_m2l_targets(int ncells, const int* __restrict__ off, int shift,
                              unsigned long long* __restrict__ key, int* __restrict__ cell,
                              int* __restrict__ count) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int n = off[c + 1] - off[c];
  const int b = (n + (1 << shift) - 1) >> shift;
  key[c] = n ? (unsigned long long)(kTgtKeyMax - min(kTgtKeyMax, b)) : (unsigned long long)kTgtKeyMax;
  cell[c] = c;
  if (n) atomicAdd(count, 1);
}

// body-pair count of the P2P list: sum over pairs of nbody(target) * nbody(source)
__global__ void k_p2p_bodypairs(const unsigned long long* __restrict__ pairs, long long n,
                                const int* __restrict__ nbody,
                                unsigned long long* __restrict__ out) {
  unsigned long long s = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    unsigned long long p = pairs[t];
    s += (unsigned long long)nbody[p >> 32] * (unsigned long long)nbody[pair_cell((unsigned)p)];
  }
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(out, s);
}

// (target << 32 | image << 27 | cell) <-> (target << (b + ib) | image << b | cell): sort keys
// of 2 b + ib bits (ib = 5 with periodic images, else 0)
__global__ void k_pack_pairs(unsigned long long* __restrict__ a, long long n, int b, int ib,
                             int pack) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const unsigned long long v = a[t];
    if (pack) {
      const unsigned src = (unsigned)v;
      a[t] = ((v >> 32) << (b + ib)) | ((unsigned long long)pair_img(src) << b) |
             (unsigned long long)pair_cell(src);
    } else {
      const unsigned long long src = ((v >> b) & ((1ULL << ib) - 1)) << kImgShift |
                                     (v & ((1ULL << b) - 1));
      a[t] = ((v >> (b + ib)) << 32) | src;
    }
  }
}

static int bits_for(int n) {
  int b = 1;
  while ((1LL << b) < (long long)n) b++;
  return b;
}

// group a list by target (k_seg_*): CSR offsets into off[0, ncells], pairs sorted within
// each target's range
// scratch: segcnt (ncells + 1 ints), keys (n), tmp (CUB scan scratch, or s.cub_tmp if null)
static void group_by_target(SolverBase& s, unsigned long long* lst, long long n, int b,
                            int* off, int* overflow, int* segcnt, unsigned* keys,
                            DevArr<char>* tmp) {
  const int TB = 256;
  FMM_CUDA(cudaMemsetAsync(segcnt, 0, (s.ncells + 1) * sizeof(int), s.stream));
  const int grid = (int)std::max(1LL, std::min<long long>(ceil_div(n, TB), 148 * 16));
  if (n > 0) {
    k_seg_count<<<grid, TB, 0, s.stream>>>(lst, n, segcnt);
    FMM_LAUNCH_CHECK();
  }
  exclusive_sum_int(s, segcnt, off, s.ncells + 1, tmp);
  if (n == 0) return;
  k_seg_scatter<<<grid, TB, 0, s.stream>>>(lst, n, off, segcnt, b, keys);
  FMM_LAUNCH_CHECK();
  k_seg_sort_warp<<<ceil_div(s.ncells, kSegWarps), 32 * kSegWarps, 0, s.stream>>>(s.ncells, off,
                                                                                 keys, b, lst);
  FMM_LAUNCH_CHECK();
  k_seg_sort_block<<<std::min(ceil_div(s.ncells, kSegBlock), 148), kSegBlock, 0, s.stream>>>(
      s.ncells, off, keys, b, lst, overflow);
  FMM_LAUNCH_CHECK();
}

// a whole list sorted on (target << (b + ib) | image << b | source), 2 b + ib key bits:
// the targets whose ranges were too long for k_seg_sort_block
static void global_sort_list(SolverBase& s, unsigned long long* lst, long long n, int b, int ib) {
  const int TB = 256;
  const int grid = (int)std::min<long long>(ceil_div(n, TB), 148 * 16);
  k_pack_pairs<<<grid, TB, 0, s.stream>>>(lst, n, b, ib, 1);
  FMM_LAUNCH_CHECK();
  sort_keys_u64(s, lst, s.list_tmp.p, (int)n, 2 * b + ib);
  k_pack_pairs<<<grid, TB, 0, s.stream>>>(s.list_tmp.p, n, b, ib, 0);
  FMM_LAUNCH_CHECK();
  FMM_CUDA(cudaMemcpyAsync(lst, s.list_tmp.p, 8 * (size_t)n, cudaMemcpyDeviceToDevice, s.stream));
}

// the mutual traversal applies to one tree with an open boundary, as in the reference (the
// image traversals and dualTreeTraversal(cells, jcells) run with mutual = false)
static int mutual_of(const SolverBase& s) {
  return s.cfg.mutual && s.cfg.images == 0 && !s.ij ? 1 : 0;
}

template <typename T> static void upload_roots(Solver<T>& s) {
  // one (root, root) pair per solve of the batch (lists never cross solves); with periodic
  // images one per shift of the source tree, in the reference's image order (:250-260)
  std::vector<int2> roots;
  if (s.ij) {
    // dualTreeTraversal(cells, jcells): the target root against the source root
    if (s.nroots == 2) roots.push_back(make_int2(s.root_cell[0], s.root_cell[1]));
  }
  for (int r = 0; r < s.nroots && !s.ij; r++) {
    if (s.cfg.images == 0) {
      roots.push_back(make_int2(s.root_cell[r], s.root_cell[r]));
      continue;
    }
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++)
        for (int iz = -1; iz <= 1; iz++)
          roots.push_back(make_int2(s.root_cell[r],
                                    s.root_cell[r] | (img_code(ix, iy, iz) << kImgShift)));
  }
  s.nfront0 = (int)roots.size();
  s.front.ensure(std::max(s.nfront0, 1));
  if (roots.empty()) return;
  if (roots.size() > s.roots_cap) {
    if (s.roots_host) s.roots_retired.push_back(s.roots_host);
    s.roots_host = nullptr;
    s.roots_cap = 0;
    const size_t cap = std::max<size_t>(2 * roots.size(), 64);
    FMM_CUDA(cudaMallocHost((void**)&s.roots_host, sizeof(int2) * cap));
    s.roots_cap = cap;
  }
  std::copy(roots.begin(), roots.end(), s.roots_host);
  FMM_CUDA(cudaMemcpyAsync(s.front.p, s.roots_host, sizeof(int2) * roots.size(),
                           cudaMemcpyHostToDevice, s.stream));
}

// Traversal with the sizes known up front: per step a count pass, one host read of the
// three totals, buffers grown to fit, then the write pass.  Returns the largest frontier.
template <typename T>
static long long counted_traversal(Solver<T>& s, long long& nm2l, long long& np2p) {
  const int TB = 256;
  unsigned long long* cnt = (unsigned long long*)s.scal.p;  // [0..2] counts, [3] body pairs
  unsigned long long* hc = (unsigned long long*)s.scal_host;
  upload_roots(s);
  long long nfront = s.nfront0, maxfront = s.nfront0;
  int steps = 0;
  nm2l = np2p = 0;
  // first sizes from typical list lengths per cell; grown below when they fall short
  s.m2l.ensure(std::max(1024LL, 64LL * s.ncells));
  s.p2p.ensure(std::max(1024LL, 16LL * s.ncells));
  while (nfront > 0) {
    FMM_CUDA(cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), s.stream));
    int grid = std::min(ceil_div(nfront, TB), 148 * 16);
    k_trav_count<T><<<grid, TB, 0, s.stream>>>(s.front.p, (int)nfront, s.cX.p, s.c_info.p,
                                               s.cfg.nspawn, (T)s.cfg.cycle,
                                               mutual_of(s), s.part_ptr(), cnt);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaMemcpyAsync(hc, cnt, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
    long long am = (long long)hc[0], ap = (long long)hc[1], an = (long long)hc[2];
    if (nm2l + am > (long long)s.m2l.cap) {
      DevArr<unsigned long long> t;
      t.ensure(std::max<size_t>(2 * s.m2l.cap, nm2l + am));
      if (nm2l) FMM_CUDA(cudaMemcpyAsync(t.p, s.m2l.p, nm2l * 8, cudaMemcpyDeviceToDevice, s.stream));
      FMM_CUDA(cudaStreamSynchronize(s.stream));
      retire_into(s.m2l, t);  // no cudaFree during a solve (DevArr)
      s.m2l = std::move(t);
    }
    if (np2p + ap > (long long)s.p2p.cap) {
      DevArr<unsigned long long> t;
      t.ensure(std::max<size_t>(2 * s.p2p.cap, np2p + ap));
      if (np2p) FMM_CUDA(cudaMemcpyAsync(t.p, s.p2p.p, np2p * 8, cudaMemcpyDeviceToDevice, s.stream));
      FMM_CUDA(cudaStreamSynchronize(s.stream));
      retire_into(s.p2p, t);  // no cudaFree during a solve (DevArr)
      s.p2p = std::move(t);
    }
    s.front2.ensure(std::max<long long>(an, 1));
    unsigned long long base[3] = {(unsigned long long)nm2l, (unsigned long long)np2p, 0};
    FMM_CUDA(cudaMemcpyAsync(cnt, base, sizeof(base), cudaMemcpyHostToDevice, s.stream));
    k_trav_write<T><<<grid, TB, 0, s.stream>>>(s.front.p, (int)nfront, s.cX.p, s.c_info.p,
                                               s.cfg.nspawn,
                                               (T)s.cfg.cycle, mutual_of(s), s.part_ptr(), cnt,
                                               s.m2l.p, s.p2p.p, s.front2.p);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaStreamSynchronize(s.stream));  // base[] lives on the host stack
    nm2l += am;
    np2p += ap;
    nfront = an;
    maxfront = std::max(maxfront, an);
    std::swap(s.front, s.front2);
    steps++;
  }
  s.trav_steps = steps;
  s.trav_maxlevel = s.maxlevel;
  return maxfront;
}

// Traversal on buffers sized by an earlier solve: a fixed number of steps, frontier sizes
// kept on the device, one host read at the end.  The steps: those of the handle's last
// traversal, two more per level that the tree has grown by since, and two to spare, at most
// enough for the deepest pair of cells.  Returns false, with the lists incomplete, when a
// buffer was too small or the steps did not reach the end.
template <typename T>
static bool fast_traversal(Solver<T>& s, long long& nm2l, long long& np2p) {
  const int TB = 256;
  const int bound = 2 * (s.maxlevel + 1) + 2;
  const int steps =
      s.trav_steps > 0
          ? std::min(bound, s.trav_steps + 2 * std::max(0, s.maxlevel - s.trav_maxlevel) + 2)
          : bound;
  // [0] M2L total, [1] P2P total, [2] invalid-index flag, [3 + l] frontier size of step l
  unsigned long long* ctr = (unsigned long long*)s.scal.p + 32;
  unsigned long long* hctr = (unsigned long long*)s.scal_host + 32;
  upload_roots(s);
  FMM_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * (4 + steps), s.stream));
  hctr[3] = (unsigned long long)s.nfront0;
  FMM_CUDA(cudaMemcpyAsync(ctr + 3, hctr + 3, sizeof(unsigned long long),
                           cudaMemcpyHostToDevice, s.stream));
  const unsigned long long fcap = std::min(s.front.cap, s.front2.cap);
  for (int l = 0; l < steps; l++) {
    DevArr<int2>& in = (l & 1) ? s.front2 : s.front;
    DevArr<int2>& out = (l & 1) ? s.front : s.front2;
    k_trav_step<T><<<148 * 8, TB, 0, s.stream>>>(
        in.p, ctr + 3 + l, fcap, s.cX.p, s.c_info.p,
        s.cfg.nspawn, (T)s.cfg.cycle, mutual_of(s), s.ncells, s.part_ptr(), ctr, ctr + 4 + l,
        s.m2l.p,
        s.m2l.cap, s.p2p.p,
        s.p2p.cap,
        out.p, fcap);
    FMM_LAUNCH_CHECK();
  }
  FMM_CUDA(cudaMemcpyAsync(hctr, ctr, sizeof(unsigned long long) * (4 + steps),
                           cudaMemcpyDeviceToHost, s.stream));
  FMM_CUDA(cudaStreamSynchronize(s.stream));
  if (hctr[2]) throw FmmError(FMM_ERR_DEVICE, "traversal read a cell index out of range");
  nm2l = (long long)hctr[0];
  np2p = (long long)hctr[1];
  if (hctr[0] > s.m2l.cap || hctr[1] > s.p2p.cap || hctr[3 + steps] != 0) return false;
  for (int l = 0; l <= steps; l++)
    if (hctr[3 + l] > fcap) return false;
  int used = 0;  // steps with a non-empty frontier
  while (used < steps && hctr[3 + used] != 0) used++;
  s.trav_steps = used;
  s.trav_maxlevel = s.maxlevel;
  return true;
}

// the P2P list of a build_lists(s, true): wait (on the host) for its grouping on the side
// stream, sort it globally if a target's range was too long for the blocks, and make the
// main stream wait for it
void finish_p2p_list(SolverBase& s) {
  if (!s.p2p_pending) return;
  s.p2p_pending = false;
  FMM_CUDA(cudaEventSynchronize(s.p2p_ready));
  const int* hflow = (const int*)((unsigned long long*)s.scal_host + 5);
  if (hflow[1]) {
    FMM_CUDA(cudaStreamWaitEvent(s.stream, s.p2p_ready, 0));
    global_sort_list(s, s.p2p.p, s.np2p, bits_for(s.ncells), s.cfg.images > 0 ? 5 : 0);
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  } else {
    FMM_CUDA(cudaStreamWaitEvent(s.stream, s.p2p_ready, 0));
  }
}

// P2P work of each leaf, as a descending sort key: its bodies times the bodies of its
// source leaves (0 without pairs)
__global__ void k_p2p_work(int nleaves, const int* __restrict__ leaves,
                           const int* __restrict__ off,
                           const unsigned long long* __restrict__ pairs,
                           const int* __restrict__ nbody, unsigned* __restrict__ key,
                           int* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaves) return;
  const int c = leaves[i];
  unsigned long long src = 0;
  for (int k = off[c]; k < off[c + 1]; k++) src += nbody[pair_cell((unsigned)pairs[k])];
  const unsigned long long w = src * (unsigned long long)nbody[c];
  key[i] = ~(unsigned)(w < 0xffffffffULL ? w : 0xffffffffULL);
  idx[i] = c;
}

// the leaves in the order of k_p2p_work's keys, on the solver's current stream
static void order_p2p_targets(SolverBase& s, DevArr<char>* tmp) {
  const int nl = s.nleaves;
  if (nl <= 0) return;
  s.p2p_wkey.ensure(nl);
  s.p2p_wkey2.ensure(nl);
  s.p2p_widx.ensure(nl);
  s.p2p_order.ensure(nl);
  k_p2p_work<<<ceil_div(nl, 256), 256, 0, s.stream>>>(nl, s.leaves.p, s.p2p_off.p, s.p2p.p,
                                                      s.c_nbody.p, s.p2p_wkey.p, s.p2p_widx.p);
  FMM_LAUNCH_CHECK();
  sort_pairs_u32(s, s.p2p_wkey.p, s.p2p_wkey2.p, s.p2p_widx.p, s.p2p_order.p, nl, 32, tmp);
  s.p2p_ordered = true;
}

template <typename T> void build_lists(Solver<T>& s, bool defer_p2p) {
  const int TB = 256;
  s.nm2l = s.np2p = s.p2p_body_pairs = 0;
  s.p2p_ordered = false;
  if (s.ncells == 0) return;
  if (s.ncells > (int)kCellMask)
    throw FmmError(FMM_ERR_NOT_SUPPORTED, "more than 2^27 - 1 cells (list pairs hold 27-bit cells)");
  unsigned long long* cnt = (unsigned long long*)s.scal.p;  // [0..2] counts, [3] body pairs
  unsigned long long* hc = (unsigned long long*)s.scal_host;
  long long nm2l = 0, np2p = 0;
  if (!s.trav_sized || !fast_traversal(s, nm2l, np2p)) {
    const long long maxfront = counted_traversal(s, nm2l, np2p);
    // size the buffers for the next solves of this handle (the 25% headroom of DevArr)
    s.front.ensure(maxfront);
    s.front2.ensure(maxfront);
    s.trav_sized = true;
  }
  s.nm2l = nm2l;
  s.np2p = np2p;
  const int b = bits_for(s.ncells), ib = s.cfg.images > 0 ? 5 : 0;
  if (std::max(nm2l, np2p) > (long long)INT_MAX)
    throw FmmError(FMM_ERR_NOT_SUPPORTED, "more than 2^31 - 1 pairs in an interaction list");
  s.list_tmp.ensure(std::max<long long>(std::max(nm2l, np2p), 1));
  s.m2l_off.ensure(s.ncells + 1);
  s.p2p_off.ensure(s.ncells + 1);
  s.seg_cnt.ensure(s.ncells + 1);
  int* overflow = (int*)(cnt + 5);  // per list: a target range too long for the blocks
  FMM_CUDA(cudaMemsetAsync(overflow, 0, 2 * sizeof(int), s.stream));
  group_by_target(s, s.m2l.p, nm2l, b, s.m2l_off.p, overflow, s.seg_cnt.p,
                  (unsigned*)s.list_tmp.p, nullptr);
  s.p2p_pending = defer_p2p && s.side != nullptr;
  if (s.p2p_pending) {
    // the P2P list is grouped on the side stream with scratch of its own, beside M2L; its
    // overflow flag reaches the host through the pinned mirror (finish_p2p_list)
    s.seg_cnt2.ensure(s.ncells + 1);
    s.seg_keys2.ensure(std::max<long long>(np2p, 1));
    if (!s.p2p_ready) FMM_CUDA(cudaEventCreateWithFlags(&s.p2p_ready, cudaEventDisableTiming));
    FMM_CUDA(cudaEventRecord(s.fork, s.stream));
    FMM_CUDA(cudaStreamWaitEvent(s.side, s.fork, 0));
    cudaStream_t main = s.stream;
    s.stream = s.side;
    try {
      group_by_target(s, s.p2p.p, np2p, b, s.p2p_off.p, overflow + 1, s.seg_cnt2.p,
                      s.seg_keys2.p, &s.cub_tmp2);
      order_p2p_targets(s, &s.cub_tmp2);
      FMM_CUDA(cudaMemcpyAsync((int*)(hc + 5) + 1, overflow + 1, sizeof(int),
                               cudaMemcpyDeviceToHost, s.stream));
      FMM_CUDA(cudaEventRecord(s.p2p_ready, s.stream));
    } catch (...) {
      s.stream = main;
      throw;
    }
    s.stream = main;
  } else {
    group_by_target(s, s.p2p.p, np2p, b, s.p2p_off.p, overflow + 1, s.seg_cnt.p,
                    (unsigned*)s.list_tmp.p, nullptr);
    order_p2p_targets(s, nullptr);
  }
  // M2L target order: by descending pair count in buckets (stable in cell index)
  {
    int* ntgt = (int*)(cnt + 4);
    FMM_CUDA(cudaMemsetAsync(ntgt, 0, sizeof(int), s.stream));
    s.keys.ensure(s.ncells);
    s.keys2.ensure(s.ncells);
    s.idx.ensure(s.ncells);
    s.m2l_tgt.ensure(s.ncells);
    k_m2l_targets<<<ceil_div(s.ncells, TB), TB, 0, s.stream>>>(
        s.ncells, s.m2l_off.p, s.cfg.basis == FMM_SPHERICAL ? 5 : 0, s.keys.p, s.idx.p, ntgt);
    FMM_LAUNCH_CHECK();
    sort_pairs_u64(s, s.keys.p, s.keys2.p, s.idx.p, s.m2l_tgt.p, s.ncells, kTgtKeyBits);
    FMM_CUDA(cudaMemcpyAsync(s.scal_host + 12, ntgt, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  }
  FMM_CUDA(cudaMemcpyAsync(hc + 3, cnt + 3, 2 * sizeof(unsigned long long) + sizeof(int),
                           cudaMemcpyDeviceToHost, s.stream));
  if (!s.p2p_pending)
    FMM_CUDA(cudaMemcpyAsync((int*)(hc + 5) + 1, overflow + 1, sizeof(int),
                             cudaMemcpyDeviceToHost, s.stream));
  FMM_CUDA(cudaStreamSynchronize(s.stream));
  const int* hflow = (const int*)(hc + 5);
  if (hflow[0] || (!s.p2p_pending && hflow[1])) {
    if (hflow[0]) global_sort_list(s, s.m2l.p, nm2l, b, ib);
    if (!s.p2p_pending && hflow[1]) global_sort_list(s, s.p2p.p, np2p, b, ib);
    FMM_CUDA(cudaStreamSynchronize(s.stream));
  }
  s.p2p_body_pairs = -1;  // counted when asked for (count_p2p_body_pairs)
  s.m2l_ntgt = s.scal_host[12];
}

// the body pairs of the P2P list, for the statistics (not needed by the solve itself)
long long count_p2p_body_pairs(SolverBase& s) {
  if (s.np2p == 0) return 0;
  const int TB = 256;
  unsigned long long* cnt = (unsigned long long*)s.scal.p;
  unsigned long long* hc = (unsigned long long*)s.scal_host;
  FMM_CUDA(cudaMemsetAsync(cnt + 3, 0, sizeof(unsigned long long), s.stream));
  k_p2p_bodypairs<<<std::max(1, std::min(ceil_div(s.np2p, TB), 148 * 8)), TB, 0, s.stream>>>(
      s.p2p.p, s.np2p, s.c_nbody.p, cnt + 3);
  FMM_LAUNCH_CHECK();
  FMM_CUDA(cudaMemcpyAsync(hc + 3, cnt + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           s.stream));
  FMM_CUDA(cudaStreamSynchronize(s.stream));
  return (long long)hc[3];
}

template void build_lists<float>(Solver<float>&, bool);
template void build_lists<double>(Solver<double>&, bool);

}  // namespace fmmb200
