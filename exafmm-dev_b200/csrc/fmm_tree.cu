// Adaptive octree build on the device, bit-exact with BuildTree (include/build_tree_tbb.h).
//
// The reference splits a node while it holds more than ncrit bodies (:172), scattering its
// bodies stably by octant (x > Xc) + 2 (y > Yc) + 4 (z > Zc) (:59, :101) around a centre
// that each level moves by +-R0 / 2^(level+1) (:199-203).  Here every body walks that same
// chain of centres once (k_keys), recording its octant at each of kMaxLevel levels as a
// 63-bit path key; a stable radix sort by key then lays the bodies out in octant order, and
// nodes are carved out of the sorted keys level by level (k_split / k_emit), each node's
// octant sub-ranges found by binary search.  Bodies inside a leaf keep their input order,
// as the stable partitions leave them, via a second stable sort by leaf-truncated key.
// Cells take the reference's layout (Nodes2cells :250-294): root first, the children of a
// cell contiguous, each child's subtree after the previous child's.
#include <cfloat>

#include <climits>

#include "fmm_solver.cuh"

namespace fmmb200 {

template <typename T> __device__ __forceinline__ T tmax();
template <> __device__ __forceinline__ float tmax<float>() { return FLT_MAX; }
template <> __device__ __forceinline__ double tmax<double>() { return DBL_MAX; }

// ---------------------------------------------------------------- bounds
// BoundBox::getBounds (include/bound_box.h:76-88): elementwise min / max of positions, per
// chunk of one root's bodies (one block per chunk), then per root (one block per root).
// Min and max are exact whatever the order in which values meet.

// the block's min / max of mn, mx (per thread) into thread 0's mn, mx
template <typename T> __device__ __forceinline__ void block_minmax(T* mn, T* mx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T a = __shfl_xor_sync(0xffffffffu, mn[d], o);
      T c = __shfl_xor_sync(0xffffffffu, mx[d], o);
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = c > mx[d] ? c : mx[d];
    }
  __shared__ T sh[32][6];
  int w = threadIdx.x >> 5;
  if (lane_id() == 0)
    for (int d = 0; d < 3; d++) sh[w][d] = mn[d], sh[w][3 + d] = mx[d];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 1; k < (int)(blockDim.x >> 5); k++)
      for (int d = 0; d < 3; d++) {
        mn[d] = sh[k][d] < mn[d] ? sh[k][d] : mn[d];
        mx[d] = sh[k][3 + d] > mx[d] ? sh[k][3 + d] : mx[d];
      }
}

template <typename T>
__global__ void k_minmax_chunks(const vec4<T>* __restrict__ b, const int* __restrict__ cb,
                                const int* __restrict__ ce, T* __restrict__ part) {
  T mn[3] = {tmax<T>(), tmax<T>(), tmax<T>()};
  T mx[3] = {-tmax<T>(), -tmax<T>(), -tmax<T>()};
  const int e = ce[blockIdx.x];
  for (int i = cb[blockIdx.x] + threadIdx.x; i < e; i += blockDim.x) {
    vec4<T> p = b[i];
    mn[0] = p.x < mn[0] ? p.x : mn[0];
    mn[1] = p.y < mn[1] ? p.y : mn[1];
    mn[2] = p.z < mn[2] ? p.z : mn[2];
    mx[0] = p.x > mx[0] ? p.x : mx[0];
    mx[1] = p.y > mx[1] ? p.y : mx[1];
    mx[2] = p.z > mx[2] ? p.z : mx[2];
  }
  block_minmax(mn, mx);
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; d++) part[6 * blockIdx.x + d] = mn[d], part[6 * blockIdx.x + 3 + d] = mx[d];
}

// BuildTree::bounds2box (include/build_tree_tbb.h:298-310), one block per root over the
// root's chunk bounds; box[16 r ..] = X0[3], R0, Xmin[3], Xmax[3]
template <typename T>
__global__ void k_box(int nroots, const int* __restrict__ chunk_lo, const T* __restrict__ part,
                      int shared, T* __restrict__ box) {
  const int r = blockIdx.x;
  if (r >= nroots) return;
  // shared: every root takes the box of the bounds of all bodies (BoundBox::getBounds of
  // the targets, then of the sources with those bounds, include/bound_box.h:91-97)
  const int c0 = shared ? chunk_lo[0] : chunk_lo[r], c1 = shared ? chunk_lo[nroots] : chunk_lo[r + 1];
  T mn[3] = {tmax<T>(), tmax<T>(), tmax<T>()};
  T mx[3] = {-tmax<T>(), -tmax<T>(), -tmax<T>()};
  for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x)
    for (int d = 0; d < 3; d++) {
      T a = part[6 * k + d], c = part[6 * k + 3 + d];
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = c > mx[d] ? c : mx[d];
    }
  block_minmax(mn, mx);
  if (threadIdx.x != 0) return;
  T X[3], R = 0;
  for (int d = 0; d < 3; d++) X[d] = div_rn(add_rn(mx[d], mn[d]), (T)2);
  for (int d = 0; d < 3; d++) {
    T a = sub_rn(X[d], mn[d]);
    R = R < a ? a : R;
    T c = sub_rn(mx[d], X[d]);
    R = R < c ? c : R;
  }
  T* bx = box + 16 * r;
  for (int d = 0; d < 3; d++) bx[d] = X[d], bx[4 + d] = mn[d], bx[7 + d] = mx[d];
  bx[3] = (T)__dmul_rn((double)R, 1.00001);
}

// ---------------------------------------------------------------- path keys
template <typename T>
__global__ void k_keys(const vec4<T>* __restrict__ b, int n, const T* __restrict__ box,
                       const int* __restrict__ root_first, int nroots,
                       unsigned long long* __restrict__ keys, int* __restrict__ idx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // root of body i: last r with root_first[r] <= i
  int lo = 0, hi = nroots - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (root_first[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  const T* bx = box + 16 * lo;
  vec4<T> p = b[i];
  T c0 = bx[0], c1 = bx[1], c2 = bx[2], R0 = bx[3];
  unsigned long long key = 0;
  T sc = T(0.5);  // 2^-(l+1), exact
  for (int l = 0; l < kMaxLevel; l++) {
    // R0 / 2^(l+1) as the product with 2^-(l+1): the same real number, so the same
    // rounding as the reference's division
    T r = mul_rn(R0, sc);
    sc = mul_rn(sc, T(0.5));
    int o = (p.x > c0) | ((p.y > c1) << 1) | ((p.z > c2) << 2);
    key = (key << 3) | (unsigned)o;
    c0 = add_rn(c0, (o & 1) ? r : -r);
    c1 = add_rn(c1, (o & 2) ? r : -r);
    c2 = add_rn(c2, (o & 4) ? r : -r);
  }
  keys[i] = key;
  idx[i] = i;
}

// forest sort helpers: root of each key-sorted body (binary search of its input index in
// the roots' first bodies), then a gather through the root-sorted permutation
__global__ void k_root_of(int n, const int* __restrict__ body, const int* __restrict__ root_first,
                          int nroots, unsigned* __restrict__ root, int* __restrict__ pos) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = body[i];
  int lo = 0, hi = nroots - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (root_first[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  root[i] = (unsigned)lo;
  pos[i] = i;
}

__global__ void k_gather_kv(int n, const int* __restrict__ perm,
                            const unsigned long long* __restrict__ kin,
                            const int* __restrict__ vin, unsigned long long* __restrict__ kout,
                            int* __restrict__ vout) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = perm[i];
  kout[i] = kin[j];
  vout[i] = vin[j];
}

__device__ __forceinline__ int digit_at(unsigned long long key, int level) {
  return (int)((key >> (3 * (kMaxLevel - 1 - level))) & 7ULL);
}

// one root node per non-empty solve, in solve order
template <typename T>
__global__ void k_roots(int nroots, const int* __restrict__ root_first, const T* __restrict__ box,
                        int* nbegin, int* ncount, int* nparent, int* nlevel, int* nsid, T* nX) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nroots) return;
  nbegin[r] = root_first[r];
  ncount[r] = root_first[r + 1] - root_first[r];
  nparent[r] = -1;
  nlevel[r] = 0;
  nsid[r] = r;
  for (int d = 0; d < 3; d++) nX[4 * r + d] = box[16 * r + d];
  nX[4 * r + 3] = 0;
}

// One level of BuildNodes (include/build_tree_tbb.h:165-218): a node with more than ncrit
// bodies gets one child per non-empty octant; octant boundaries by binary search.
// One warp per node: the 7 octant boundaries of its sorted key range are found together by
// 32-ary searches (32 samples per boundary and round, all loads of a round independent), so
// a node of c bodies needs log32(c) dependent rounds instead of the 7 log2(c) of a binary
// search per boundary.  Node w of the level (v = lo + w): child count into cnt[w], octant
// starts into starts[9 w ..].
__device__ __forceinline__ void split_node(int lane, int w, int v, int level, int ncrit,
                                           const unsigned long long* __restrict__ keys,
                                           const int* __restrict__ nbegin,
                                           const int* __restrict__ ncount,
                                           int* __restrict__ cnt, int* __restrict__ starts) {
  const int b = nbegin[v], c = ncount[v];
  int nch = 0;
  if (c > ncrit && level < kMaxLevel) {
    int* st = starts + 9 * w;
    int slo[8], shi[8];
#pragma unroll
    for (int o = 1; o < 8; o++) {
      slo[o] = b;
      shi[o] = b + c;
    }
    // invariant: the first index whose octant digit is >= o lies in [slo[o], shi[o]]
    for (;;) {
      bool open = false;
#pragma unroll
      for (int o = 1; o < 8; o++) open |= slo[o] < shi[o];
      if (!open) break;
      unsigned ball[8];
      int step[8];
#pragma unroll
      for (int o = 1; o < 8; o++) {
        const int len = shi[o] - slo[o];
        step[o] = len <= 32 ? 1 : (len + 31) / 32;
        const long long idx = slo[o] + (long long)lane * step[o];
        const bool pred = len > 0 && idx < shi[o] && digit_at(keys[idx], level) < o;
        ball[o] = __ballot_sync(0xffffffffu, pred);
      }
#pragma unroll
      for (int o = 1; o < 8; o++) {
        if (slo[o] >= shi[o]) continue;
        const int t = __popc(ball[o]);
        if (step[o] == 1) {
          slo[o] = shi[o] = slo[o] + t;
        } else if (t == 0) {
          shi[o] = slo[o];
        } else {
          const long long nlo = slo[o] + (long long)(t - 1) * step[o] + 1;
          const long long nhi = slo[o] + (long long)t * step[o];
          shi[o] = (int)(nhi < shi[o] ? nhi : shi[o]);
          slo[o] = (int)nlo;
        }
      }
    }
    if (lane == 0) {
      st[0] = b;
      st[8] = b + c;
#pragma unroll
      for (int o = 1; o < 8; o++) st[o] = slo[o];
    }
    int prev = b;
#pragma unroll
    for (int o = 1; o < 8; o++) {
      nch += slo[o] > prev;
      prev = slo[o];
    }
    nch += b + c > prev;
  }
  if (lane == 0) cnt[w] = nch;
}

__global__ void k_split(int lo, int hi, int level, int ncrit,
                        const unsigned long long* __restrict__ keys,
                        const int* __restrict__ nbegin, const int* __restrict__ ncount,
                        int* __restrict__ cnt, int* __restrict__ starts) {
  const int lane = lane_id();
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int m = hi - lo;
  if (w == m && lane == 0) cnt[m] = 0;
  if (w >= m) return;
  split_node(lane, (int)w, lo + (int)w, level, ncrit, keys, nbegin, ncount, cnt, starts);
}

// k_split with the level's node range read on the device (lvl[level], lvl[level + 1]) for
// the planned build: a grid-stride loop over the level's nodes.  The counts past them are
// zero (cnt is cleared before the first level, and k_emit_planned clears the counts it has
// used), as the scan over mcap + 1 entries that follows needs; a level of more than mcap
// nodes flags overflow and is not split.
__global__ void k_split_planned(const int* __restrict__ lvl, int level, int ncrit, int mcap,
                                const unsigned long long* __restrict__ keys,
                                const int* __restrict__ nbegin, const int* __restrict__ ncount,
                                int* __restrict__ cnt, int* __restrict__ starts,
                                int* __restrict__ overflow) {
  const int lane = lane_id();
  const int lo = lvl[level], m = lvl[level + 1] - lo;
  const int mm = m <= mcap ? m : 0;
  if (m > mcap && blockIdx.x == 0 && threadIdx.x == 0) atomicExch(overflow, 1);
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < mm; w += nw)
    split_node(lane, (int)w, lo + (int)w, level, ncrit, keys, nbegin, ncount, cnt, starts);
}

// the children of node t of the level (v = lo + t), from hi + coff[t] on
template <typename T>
__device__ __forceinline__ void emit_node(int t, int lo, int hi, int level,
                                          const int* __restrict__ cnt,
                                          const int* __restrict__ coff,
                                          const int* __restrict__ starts,
                                          const T* __restrict__ box, int* __restrict__ nbegin,
                                          int* __restrict__ ncount, int* __restrict__ nparent,
                                          int* __restrict__ nchildn, int* __restrict__ nfirst,
                                          int* __restrict__ nlevel, int* __restrict__ nsid,
                                          T* __restrict__ nX) {
  int v = lo + t;
  int nch = cnt[t];
  nchildn[v] = nch;
  if (nch == 0) {
    nfirst[v] = -1;
    return;
  }
  int first = hi + coff[t];
  nfirst[v] = first;
  const int* st = starts + 9 * t;
  const int root = nsid[v];
  T r = div_rn(box[16 * root + 3], (T)(1 << (level + 1)));
  T X0 = nX[4 * v], X1 = nX[4 * v + 1], X2 = nX[4 * v + 2];
  int k = 0;
  for (int o = 0; o < 8; o++) {
    if (st[o + 1] <= st[o]) continue;
    int u = first + k++;
    nbegin[u] = st[o];
    ncount[u] = st[o + 1] - st[o];
    nparent[u] = v;
    nlevel[u] = level + 1;
    nsid[u] = root;
    nX[4 * u] = add_rn(X0, (o & 1) ? r : -r);
    nX[4 * u + 1] = add_rn(X1, (o & 2) ? r : -r);
    nX[4 * u + 2] = add_rn(X2, (o & 4) ? r : -r);
    nX[4 * u + 3] = 0;
  }
}

template <typename T>
__global__ void k_emit(int lo, int hi, int level, const int* __restrict__ cnt,
                       const int* __restrict__ coff, const int* __restrict__ starts,
                       const T* __restrict__ box, int* __restrict__ nbegin,
                       int* __restrict__ ncount, int* __restrict__ nparent,
                       int* __restrict__ nchildn, int* __restrict__ nfirst,
                       int* __restrict__ nlevel, int* __restrict__ nsid, T* __restrict__ nX) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hi - lo) return;
  emit_node<T>(t, lo, hi, level, cnt, coff, starts, box, nbegin, ncount, nparent, nchildn,
               nfirst, nlevel, nsid, nX);
}

// k_emit of the planned build: the level's range and its child total (coff[m]) read on the
// device; the next level's end is written to lvl[level + 2]; children that would not fit
// the node arrays (ncap) flag overflow and are not emitted.
template <typename T>
__global__ void k_emit_planned(int* __restrict__ lvl, int level, int ncap,
                               int* __restrict__ cnt, const int* __restrict__ coff,
                               const int* __restrict__ starts, const T* __restrict__ box,
                               int* __restrict__ nbegin, int* __restrict__ ncount,
                               int* __restrict__ nparent, int* __restrict__ nchildn,
                               int* __restrict__ nfirst, int* __restrict__ nlevel,
                               int* __restrict__ nsid, T* __restrict__ nX,
                               int* __restrict__ overflow) {
  const int lo = lvl[level], hi = lvl[level + 1], m = hi - lo;
  const int total = m > 0 ? coff[m] : 0;
  const bool fits = (long long)hi + total <= ncap && *overflow == 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    lvl[level + 2] = fits ? hi + total : hi;
    if (!fits) atomicExch(overflow, 1);
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    if (fits)
      emit_node<T>(t, lo, hi, level, cnt, coff, starts, box, nbegin, ncount, nparent, nchildn,
                   nfirst, nlevel, nsid, nX);
    if (t < ncap) cnt[t] = 0;  // cleared for the next level's scan
  }
}

// leaf nodes: chain-less nodes at the deepest level of the last pass
__global__ void k_finish_level(int lo, int hi, int* nchildn, int* nfirst) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hi - lo) return;
  nchildn[lo + t] = 0;
  nfirst[lo + t] = -1;
}

// NNODE bottom-up (include/build_tree_tbb.h:215-217)
__global__ void k_nnode(int lo, int hi, const int* __restrict__ nchildn,
                        const int* __restrict__ nfirst, int* __restrict__ nnode) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hi - lo) return;
  int v = lo + t;
  int s = 1;
  for (int k = 0; k < nchildn[v]; k++) s += nnode[nfirst[v] + k];
  nnode[v] = s;
}

// Cell slots top-down (Nodes2cells, include/build_tree_tbb.h:272-286): children at CN,
// next free slot after the child block, each child's subtree after the previous child's.
__global__ void k_pos(int lo, int hi, const int* __restrict__ nchildn,
                      const int* __restrict__ nfirst, const int* __restrict__ nnode,
                      const int* __restrict__ cbase, int* __restrict__ npos,
                      int* __restrict__ ncb) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hi - lo) return;
  int v = lo + t;
  if (lo == 0) {  // roots: each root's cells start after the previous root's subtree
    npos[v] = cbase[v];
    ncb[v] = cbase[v] + 1;
  }
  int nch = nchildn[v];
  if (nch == 0) return;
  int cb = ncb[v];
  int acc = cb + nch;
  for (int k = 0; k < nch; k++) {
    int u = nfirst[v] + k;
    npos[u] = cb + k;
    ncb[u] = acc;
    acc += nnode[u] - 1;
  }
}

// (NCHILD, ICHILD, NBODY, IBODY) of every cell in one 16-byte record, for the traversal
__global__ void k_cell_info(int ncells, const int* __restrict__ nchild,
                            const int* __restrict__ ichild, const int* __restrict__ nbody,
                            const int* __restrict__ ibody, int4* __restrict__ info) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncells) info[c] = make_int4(nchild[c], ichild[c], nbody[c], ibody[c]);
}

// Cell records (Nodes2cells::operator(), include/build_tree_tbb.h:250-262) with the
// Morton index of getKey (:240-249) in 64-bit arithmetic.
template <typename T>
__global__ void k_cells(int nnodes, const T* __restrict__ boxes, const int* __restrict__ nbegin,
                        const int* __restrict__ ncount, const int* __restrict__ nparent,
                        const int* __restrict__ nchildn, const int* __restrict__ nlevel,
                        const int* __restrict__ nsid, const int* __restrict__ cbase,
                        const int* __restrict__ npos, const int* __restrict__ ncb,
                        const T* __restrict__ nX, int* iparent, int* ichild, int* nchild,
                        int* ibody, int* nbody, int* clevel, unsigned long long* icell,
                        vec4<T>* cX, int* croot) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nnodes) return;
  int c = npos[v];
  int lev = nlevel[v];
  const T* box = boxes + 16 * nsid[v];
  croot[c] = cbase[nsid[v]];
  T R0 = box[3];
  T R = div_rn(R0, (T)(1 << lev));
  T X[3] = {nX[4 * v], nX[4 * v + 1], nX[4 * v + 2]};
  iparent[c] = nparent[v] < 0 ? c : npos[nparent[v]];
  int nch = nchildn[v];
  nchild[c] = nch;
  ichild[c] = nch ? ncb[v] : 0;
  ibody[c] = nbegin[v];
  nbody[c] = ncount[v];
  clevel[c] = lev;
  T diam = mul_rn((T)2, R);
  int iX[3];
  for (int d = 0; d < 3; d++) iX[d] = (int)div_rn(sub_rn(X[d], sub_rn(box[d], R0)), diam);
  unsigned long long index = ((1ULL << (3 * lev)) - 1) / 7;
  for (int l = 0; l < lev; l++) {
    for (int d = 0; d < 3; d++) index += (unsigned long long)(iX[d] & 1) << (3 * l + d);
    for (int d = 0; d < 3; d++) iX[d] >>= 1;
  }
  icell[c] = index;
  cX[c] = make_v4<T>(X[0], X[1], X[2], R);
}

// leaf level of every sorted body (leaves only; ranges partition the bodies)
__global__ void k_leaf_levels(int nnodes, const int* __restrict__ nchildn,
                              const int* __restrict__ nbegin, const int* __restrict__ ncount,
                              const int* __restrict__ nlevel, int* __restrict__ blev) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nnodes || nchildn[v] != 0) return;
  int lev = nlevel[v];
  for (int b = nbegin[v]; b < nbegin[v] + ncount[v]; b++) blev[b] = lev;
}

// key truncated to the body's leaf, scattered back to input order
__global__ void k_tkey(int n, const unsigned long long* __restrict__ skeys,
                       const int* __restrict__ sidx, const int* __restrict__ blev,
                       unsigned long long* __restrict__ tkey, int* __restrict__ iota) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int lev = blev[b];
  unsigned long long mask = lev == 0 ? 0ULL : (~0ULL << (3 * (kMaxLevel - lev)));
  tkey[sidx[b]] = skeys[b] & mask;
  iota[b] = b;
}

// Input order inside every leaf of at most 64 bodies (warp per leaf node): the bodies'
// original indices, currently in full-key order, are ranked and written back ascending.
__global__ void k_leaf_reorder(int nnodes, const int* __restrict__ nchildn,
                               const int* __restrict__ nbegin, const int* __restrict__ ncount,
                               const int* __restrict__ sidx, int* __restrict__ order) {
  const int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = lane_id();
  if (v >= nnodes || nchildn[v] != 0) return;
  const int b0 = nbegin[v], n = ncount[v];
  const int a = lane < n ? sidx[b0 + lane] : 0x7fffffff;
  const int b = lane + 32 < n ? sidx[b0 + 32 + lane] : 0x7fffffff;
  int ra = 0, rb = 0;
  for (int k = 0; k < n; k++) {
    const int u = k < 32 ? __shfl_sync(0xffffffffu, a, k) : __shfl_sync(0xffffffffu, b, k - 32);
    ra += u < a;
    rb += u < b;
  }
  if (lane < n) order[b0 + ra] = a;
  if (lane + 32 < n) order[b0 + rb] = b;
}

template <typename T>
__global__ void k_permute(int n, const vec4<T>* __restrict__ in, const int* __restrict__ order,
                          vec4<T>* __restrict__ out) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) out[b] = in[order[b]];
}

__global__ void k_leaf_flags(int nnodes, const int* __restrict__ nchildn, int* __restrict__ f) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nnodes) f[v] = nchildn[v] == 0;
  if (v == nnodes) f[v] = 0;
}

__global__ void k_leaf_scatter(int nnodes, const int* __restrict__ nchildn,
                               const int* __restrict__ off, const int* __restrict__ npos,
                               int* __restrict__ leaves) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nnodes && nchildn[v] == 0) leaves[off[v]] = npos[v];
}

// grow a node array keeping its contents (the old buffer is retired, as DevArr::ensure does)
template <typename U> static void grow(SolverBase& s, DevArr<U>& a, size_t n) {
  if (n <= a.cap) return;
  DevArr<U> b;
  b.ensure(n > 2 * a.cap ? n : 2 * a.cap);
  if (a.p) FMM_CUDA(cudaMemcpyAsync(b.p, a.p, a.cap * sizeof(U), cudaMemcpyDeviceToDevice, s.stream));
  FMM_CUDA(cudaStreamSynchronize(s.stream));
  retire_into(a, b);
  a = std::move(b);
}

// Sort (key, body) pairs by (root, key), stable: one radix sort on the key over all roots,
// then a stable radix sort on the root id (least significant digit first), so the result is
// each root's range sorted on its own, as when the root is solved alone.  (CUB's segmented
// sort gives each segment one thread block, which is slow for a few large segments.)
template <typename T>
static void forest_sort(Solver<T>& s, const unsigned long long* kin, unsigned long long* kout,
                        const int* vin, int* vout, int n, int nroots, int end_bit,
                        int begin_bit = 0) {
  if (nroots == 1) {
    sort_pairs_u64(s, kin, kout, vin, vout, n, end_bit, begin_bit);
    return;
  }
  const int TB = 256;
  s.fs_keys.ensure(n);
  s.fs_idx.ensure(n);
  s.fs_root.ensure(n);
  s.fs_root2.ensure(n);
  s.fs_pos.ensure(n);
  s.fs_pos2.ensure(n);
  sort_pairs_u64(s, kin, s.fs_keys.p, vin, s.fs_idx.p, n, end_bit, begin_bit);
  k_root_of<<<ceil_div(n, TB), TB, 0, s.stream>>>(n, s.fs_idx.p, s.d_root_first.p, nroots,
                                                  s.fs_root.p, s.fs_pos.p);
  FMM_LAUNCH_CHECK();
  int bits = 1;
  while ((1LL << bits) < (long long)nroots) bits++;
  sort_pairs_u32(s, s.fs_root.p, s.fs_root2.p, s.fs_pos.p, s.fs_pos2.p, n, bits);
  k_gather_kv<<<ceil_div(n, TB), TB, 0, s.stream>>>(n, s.fs_pos2.p, s.fs_keys.p, s.fs_idx.p,
                                                    kout, vout);
  FMM_LAUNCH_CHECK();
}

// The levels of the node build without a host round trip per level, for a handle whose
// previous tree had s.tree_plan levels: tree_plan + 1 levels of k_split_planned, a scan of
// the counts and k_emit_planned run back to back with the level ranges kept on the device,
// then one read of the ranges.  Returns false (and the levels are built again level by
// level) if the node arrays overflowed or the tree went deeper than planned.
template <typename T>
static bool planned_levels(Solver<T>& s, int nroots, DevArr<int>** narr, int nnarr) {
  const int TB = 256;
  const int L = s.tree_plan + 1;
  size_t cap = s.nX.cap / 4;
  for (int i = 0; i < nnarr; i++) cap = std::min(cap, narr[i]->cap);
  const int ncap = (int)std::min<size_t>(cap, INT_MAX / 16);
  const int mcap = ncap;  // a level holds no more nodes than the arrays
  s.nsplit.ensure(9 * (size_t)(mcap + 1));
  s.coff.ensure((size_t)mcap + 2);
  s.idx.ensure(std::max((size_t)s.n, (size_t)mcap + 1));
  s.d_lvl.ensure(L + 2);
  int* cnt = s.idx.p;
  int* lvl = s.d_lvl.p;
  int* ovf = (int*)((unsigned long long*)s.scal.p + 6);
  int* hl = s.scal_host + 400;  // pinned: L + 2 level ends, then the overflow flag
  if (L + 3 > 512 - 400) return false;
  hl[0] = 0;
  hl[1] = nroots;
  FMM_CUDA(cudaMemcpyAsync(lvl, hl, 2 * sizeof(int), cudaMemcpyHostToDevice, s.stream));
  FMM_CUDA(cudaMemsetAsync(ovf, 0, sizeof(int), s.stream));
  FMM_CUDA(cudaMemsetAsync(cnt, 0, ((size_t)mcap + 1) * sizeof(int), s.stream));
  const int gs = (int)std::min<long long>(ceil_div(32LL * (mcap + 1), TB), 148 * 16);
  const int ge = (int)std::min<long long>(ceil_div((long long)mcap, TB), 148 * 8);
  for (int level = 0; level < L; level++) {
    k_split_planned<<<gs, TB, 0, s.stream>>>(lvl, level, s.cfg.ncrit, mcap, s.keys2.p,
                                              s.nbegin.p, s.ncount.p, cnt, s.nsplit.p, ovf);
    FMM_LAUNCH_CHECK();
    exclusive_sum_int(s, cnt, s.coff.p, mcap + 1);
    k_emit_planned<T><<<ge, TB, 0, s.stream>>>(lvl, level, ncap, cnt, s.coff.p, s.nsplit.p,
                                               s.box.p, s.nbegin.p, s.ncount.p, s.nparent.p,
                                               s.nchildn.p, s.nfirst.p, s.nlevel.p, s.nsid.p,
                                               s.nX.p, ovf);
    FMM_LAUNCH_CHECK();
  }
  FMM_CUDA(cudaMemcpyAsync(hl, lvl, (L + 2) * sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  FMM_CUDA(cudaMemcpyAsync(hl + L + 2, ovf, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  FMM_CUDA(cudaStreamSynchronize(s.stream));
  if (hl[L + 2] != 0 || hl[L + 1] != hl[L]) return false;
  // levels 0 .. d, d the first level without children
  int d = 0;
  while (hl[d + 2] != hl[d + 1]) d++;
  s.level_lo.assign(hl, hl + d + 2);
  return true;
}

// ---------------------------------------------------------------- uniform Morton tree
// BuildTree of include/build_tree_omp.h:214-262 (the builder of an OpenMP build without TBB,
// include/build_tree.h:12-13): every leaf at the depth `level` the host computes as the
// reference does (:218), bodies keyed by the interleaved bits of their grid cell at the
// leaf size d (getKey :36-57), stably sorted by key (radixSort :59-121), one leaf per run of
// equal keys (bodies2leafs :130-158), the parents of each level one per run of equal
// key / 8^l (leafs2cells :160-198), then the cell array reversed (reverseOrder :200-211):
// root first, each level in descending key order, children contiguous.  The cells are
// formed in the reference's construction order (leaves ascending, then each level above)
// and written at index ncells - 1 - c, with the reference's values throughout, including
// its root IPARENT (ncells - 1) and leaf ICHILD (ncells).
constexpr int kUniformMaxLevel = 10;  // the reference's `int id` holds 3 level bits (:45)

// the cell size of a level as getKey declares it: `float d = 2 * box.R / (1 << level)`
// evaluated in the working precision, then made a float (:38); a level above doubles it
// in float (:166)
template <typename T>
__device__ __forceinline__ float uniform_d(const T* __restrict__ box, int level) {
  return (float)div_rn(mul_rn(T(2), box[3]), (T)(1 << level));
}
// grid index along one axis: (X - Xmin) / d in the working precision (d promoted), truncated
template <typename T> __device__ __forceinline__ int uniform_ix(T x, T xmin, float d) {
  return (int)div_rn(sub_rn(x, xmin), (T)d);
}

template <typename T>
__global__ void k_ukeys(const vec4<T>* __restrict__ b, int n, const T* __restrict__ box,
                        int level, unsigned long long* __restrict__ key, int* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float d = uniform_d(box, level);
  const vec4<T> x = b[i];
  int ix = uniform_ix(x.x, box[4], d), iy = uniform_ix(x.y, box[5], d),
      iz = uniform_ix(x.z, box[6], d);
  int id = 0;
  for (int l = 0; l < level; l++) {
    id += (ix & 1) << (3 * l);
    id += (iy & 1) << (3 * l + 1);
    id += (iz & 1) << (3 * l + 2);
    ix >>= 1;
    iy >>= 1;
    iz >>= 1;
  }
  key[i] = (unsigned long long)id;
  idx[i] = i;
}

// run heads one level up: child c (construction index cb + c; its first body fb[cb + c], or
// the body c itself when fb is null) starts a new cell when its key shifted right by
// `shift` differs from its predecessor's; flags[m] = 0 closes the scan
__global__ void k_uheads(int m, int cb, const int* __restrict__ fb,
                         const unsigned long long* __restrict__ key, int shift,
                         int* __restrict__ flags) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > m) return;
  if (c == m) {
    flags[m] = 0;
    return;
  }
  const int b = fb ? fb[cb + c] : c;
  const int bp = c == 0 ? 0 : (fb ? fb[cb + c - 1] : c - 1);
  flags[c] = c == 0 || (key[b] >> shift) != (key[bp] >> shift);
}

// the cells of one level from the run heads of the level below (construction order: the new
// cells from ce on); body runs for the leaves (fb == null), cell runs above (ch0, par)
__global__ void k_uemit(int m, int cb, int ce, const int* __restrict__ flags,
                        const int* __restrict__ pos, int* __restrict__ fb,
                        int* __restrict__ ch0, int* __restrict__ par, bool leaves) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  const int r = pos[c] + flags[c] - 1;  // the new cell this child (or body) belongs to
  if (flags[c]) {
    fb[ce + r] = leaves ? c : fb[cb + c];
    ch0[ce + r] = leaves ? 0 : cb + c;
  }
  if (!leaves) par[cb + c] = ce + r;
}

struct UniformLevels {
  int begin[kUniformMaxLevel + 2];  // construction range of level l: [begin[l], end[l])
  int end[kUniformMaxLevel + 2];
};

// cell records at index ncells - 1 - c for construction index c (reverseOrder)
template <typename T>
__global__ void k_ucells(int nc, int n, int level, UniformLevels lv, const T* __restrict__ box,
                         const int* __restrict__ fb, const int* __restrict__ ch0,
                         const int* __restrict__ par, const unsigned long long* __restrict__ key,
                         const vec4<T>* __restrict__ bodies, int* __restrict__ iparent,
                         int* __restrict__ ichild, int* __restrict__ nchild,
                         int* __restrict__ ibody, int* __restrict__ nbody,
                         int* __restrict__ clevel, unsigned long long* __restrict__ icell,
                         vec4<T>* __restrict__ cX, int* __restrict__ croot) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  int L = level;
  while (c >= lv.end[L]) L--;  // levels are laid out leaves first
  const int f = nc - 1 - c;
  const int b = fb[c];
  const int nb = (c + 1 < lv.end[L] ? fb[c + 1] : n) - b;
  int nch = 0;
  if (L < level) nch = (c + 1 < lv.end[L] ? ch0[c + 1] : lv.end[L + 1]) - ch0[c];
  // reverseOrder: ICHILD = perm[ICHILD] - NCHILD + 1 (a leaf's ICHILD 0 goes to nc),
  // IPARENT = perm[IPARENT] (the root's IPARENT 0 goes to nc - 1)
  ichild[f] = (nc - 1 - (L < level ? ch0[c] : 0)) - nch + 1;
  iparent[f] = nc - 1 - (L > 0 ? par[c] : 0);
  nchild[f] = nch;
  ibody[f] = b;
  nbody[f] = nb;
  clevel[f] = L;
  icell[f] = key[b] >> (3 * (level - L));
  // centre and radius from the cell's first body at the level's cell size (:148-151,
  // :182-185): d (ix + .5) + Xmin in double, stored in the working precision
  float dl = uniform_d(box, level);
  for (int k = L; k < level; k++) dl *= 2.f;
  const vec4<T> x = bodies[b];
  const T xs[3] = {x.x, x.y, x.z};
  T X[3];
  for (int k = 0; k < 3; k++) {
    const int ik = uniform_ix(xs[k], box[4 + k], dl);
    X[k] = (T)__dadd_rn(__dmul_rn((double)dl, (double)ik + 0.5), (double)box[4 + k]);
  }
  cX[f] = make_v4<T>(X[0], X[1], X[2], (T)__dmul_rn((double)dl, 0.5));
  croot[f] = 0;
}

__global__ void k_iota(int n, int first, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = first + i;
}

// depth of the uniform tree for n bodies (include/build_tree_omp.h:218): host arithmetic,
// the reference's own expression (integer n / ncrit, libm log)
int uniform_level(int n, int ncrit) {
  return n >= ncrit ? 1 + int(log((double)(n / ncrit)) / M_LN2 / 3) : 0;
}

template <typename T> static void build_uniform(Solver<T>& s) {
  const int n = s.n, TB = 256;
  const int level = uniform_level(n, s.cfg.ncrit);
  if (level > kUniformMaxLevel)
    throw FmmError(FMM_ERR_NOT_SUPPORTED,
                   "uniform tree deeper than 10 levels (the reference's 32-bit Morton keys "
                   "overflow there)");
  // getKey, radixSort (stable, on the key's 3 level bits), permute
  s.keys.ensure(n);
  s.keys2.ensure(n);
  s.idx.ensure(n);
  s.idx2.ensure(n);
  k_ukeys<T><<<ceil_div(n, TB), TB, 0, s.stream>>>(s.bodies_in.p, n, s.box.p, level, s.keys.p,
                                                   s.idx.p);
  FMM_LAUNCH_CHECK();
  sort_pairs_u64(s, s.keys.p, s.keys2.p, s.idx.p, s.idx2.p, n, std::max(3 * level, 1));
  s.order.ensure(n);
  FMM_CUDA(cudaMemcpyAsync(s.order.p, s.idx2.p, sizeof(int) * n, cudaMemcpyDeviceToDevice,
                           s.stream));
  s.bodies.ensure(n);
  k_permute<T><<<ceil_div(n, TB), TB, 0, s.stream>>>(n, s.bodies_in.p, s.order.p, s.bodies.p);
  FMM_LAUNCH_CHECK();
  // cells in construction order, level by level from the leaves: first body (nbegin),
  // first child (nfirst), parent (nparent); run heads and their scan in nsplit / coff.
  // Level l holds at most min(n, 8^l) cells.
  size_t cap = 16;
  for (int L = 0; L <= level; L++) cap += std::min<size_t>((size_t)n, (size_t)1 << (3 * L));
  s.nbegin.ensure(cap);
  s.nfirst.ensure(cap);
  s.nparent.ensure(cap);
  s.nsplit.ensure((size_t)n + 1);
  s.coff.ensure((size_t)n + 1);
  UniformLevels lv{};
  int cb = 0, m = n, ce = 0;  // the level below: construction range [cb, cb + m)
  for (int L = level; L >= 0; L--) {
    const bool leaves = L == level;
    const int shift = 3 * (level - L);
    k_uheads<<<ceil_div(m + 1, TB), TB, 0, s.stream>>>(m, cb, leaves ? nullptr : s.nbegin.p,
                                                       s.keys2.p, shift, s.nsplit.p);
    FMM_LAUNCH_CHECK();
    exclusive_sum_int(s, s.nsplit.p, s.coff.p, m + 1);
    FMM_CUDA(cudaMemcpyAsync(s.scal_host, s.coff.p + m, sizeof(int), cudaMemcpyDeviceToHost,
                             s.stream));
    k_uemit<<<ceil_div(m, TB), TB, 0, s.stream>>>(m, cb, ce, s.nsplit.p, s.coff.p, s.nbegin.p,
                                                  s.nfirst.p, s.nparent.p, leaves);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaStreamSynchronize(s.stream));
    const int cnt = s.scal_host[0];
    lv.begin[L] = ce;
    lv.end[L] = ce + cnt;
    cb = ce;
    m = cnt;
    ce += cnt;
  }
  const int nc = ce;
  // reverseOrder into the reference's cell layout
  s.c_iparent.ensure(nc); s.c_ichild.ensure(nc); s.c_nchild.ensure(nc);
  s.c_ibody.ensure(nc); s.c_nbody.ensure(nc); s.c_level.ensure(nc);
  s.c_icell.ensure(nc);
  s.cX.ensure(nc);
  s.c_root.ensure(nc);
  k_ucells<T><<<ceil_div(nc, TB), TB, 0, s.stream>>>(
      nc, n, level, lv, s.box.p, s.nbegin.p, s.nfirst.p, s.nparent.p, s.keys2.p, s.bodies.p,
      s.c_iparent.p, s.c_ichild.p, s.c_nchild.p, s.c_ibody.p, s.c_nbody.p, s.c_level.p,
      s.c_icell.p, s.cX.p, s.c_root.p);
  FMM_LAUNCH_CHECK();
  s.c_info.ensure(nc);
  k_cell_info<<<ceil_div(nc, TB), TB, 0, s.stream>>>(nc, s.c_nchild.p, s.c_ichild.p,
                                                     s.c_nbody.p, s.c_ibody.p, s.c_info.p);
  FMM_LAUNCH_CHECK();
  // the level passes walk cells level by level: node v is cell v (npos the identity), the
  // cells of level l at [nc - end[l], nc - begin[l]); every leaf is on the deepest level
  s.npos.ensure(nc);
  k_iota<<<ceil_div(nc, TB), TB, 0, s.stream>>>(nc, 0, s.npos.p);
  FMM_LAUNCH_CHECK();
  const int nleaves = lv.end[level] - lv.begin[level];
  s.leaves.ensure(nleaves);
  k_iota<<<ceil_div(nleaves, TB), TB, 0, s.stream>>>(nleaves, nc - nleaves, s.leaves.p);
  FMM_LAUNCH_CHECK();
  s.level_lo.clear();
  for (int L = 0; L <= level; L++) s.level_lo.push_back(nc - lv.end[L]);
  s.level_lo.push_back(nc);
  s.cbase.ensure(2);
  FMM_CUDA(cudaMemsetAsync(s.cbase.p, 0, sizeof(int), s.stream));
  s.root_cell.assign(1, 0);
  s.maxlevel = level;
  s.ncells = nc;
  s.nleaves = nleaves;
  s.tree_plan = 0;
}

template <typename T> void build_tree(Solver<T>& s) {
  const int n = s.n;
  const int TB = 256;
  s.kc_valid = false;  // the host copies of the cells' index fields are stale
  s.p2p_ordered = false;  // so is the P2P target order of the last traversal
  s.level_lo.clear();
  s.ncells = s.maxlevel = s.nleaves = 0;
  // roots: non-empty solves in order
  const int nsolves = (int)s.seg.size() - 1;
  s.root_solve.clear();
  std::vector<int> rfirst;
  for (int q = 0; q < nsolves; q++)
    if (s.seg[q + 1] > s.seg[q]) {
      s.root_solve.push_back(q);
      rfirst.push_back(s.seg[q]);
    }
  rfirst.push_back(n);
  const int nroots = (int)s.root_solve.size();
  if (s.cfg.tree == FMM_TREE_UNIFORM && (nroots > 1 || s.ij))
    throw FmmError(FMM_ERR_NOT_SUPPORTED,
                   "the uniform tree builds one tree per call (no batches, no separate target "
                   "and source trees)");
  s.nroots = nroots;
  s.box.ensure(16 * (size_t)std::max(nroots, 1));
  if (nroots == 0) {
    FMM_CUDA(cudaMemsetAsync(s.box.p, 0, 16 * sizeof(T), s.stream));
    s.root_cell.clear();
    return;
  }
  // bounds per root over chunks of at most 4096 bodies (256 blocks at 2^20 bodies)
  const int CH = 4096;
  std::vector<int> hb, he, hlo{0};
  for (int r = 0; r < nroots; r++) {
    for (int b0 = rfirst[r]; b0 < rfirst[r + 1]; b0 += CH) {
      hb.push_back(b0);
      he.push_back(std::min(b0 + CH, rfirst[r + 1]));
    }
    hlo.push_back((int)hb.size());
  }
  const int nch = (int)hb.size();
  s.d_root_first.ensure(nroots + 1);
  s.d_seg.ensure(2 * (size_t)nch + nroots + 1);
  int* dcb = s.d_seg.p;
  int* dce = dcb + nch;
  int* dlo = dce + nch;
  FMM_CUDA(cudaMemcpyAsync(s.d_root_first.p, rfirst.data(), sizeof(int) * (nroots + 1),
                           cudaMemcpyHostToDevice, s.stream));
  FMM_CUDA(cudaMemcpyAsync(dcb, hb.data(), sizeof(int) * nch, cudaMemcpyHostToDevice, s.stream));
  FMM_CUDA(cudaMemcpyAsync(dce, he.data(), sizeof(int) * nch, cudaMemcpyHostToDevice, s.stream));
  FMM_CUDA(cudaMemcpyAsync(dlo, hlo.data(), sizeof(int) * (nroots + 1), cudaMemcpyHostToDevice,
                           s.stream));
  s.minmax_part.ensure(6 * (size_t)nch);
  k_minmax_chunks<T><<<nch, TB, 0, s.stream>>>(s.bodies_in.p, dcb, dce, s.minmax_part.p);
  FMM_LAUNCH_CHECK();
  k_box<T><<<nroots, TB, 0, s.stream>>>(nroots, dlo, s.minmax_part.p,
                                        s.ij && s.ij_common_box ? 1 : 0, s.box.p);
  FMM_LAUNCH_CHECK();
  phase_end(s, FMM_PHASE_BOUNDS);
  phase_begin(s, FMM_PHASE_TREE);
  if (s.cfg.tree == FMM_TREE_UNIFORM) {
    build_uniform(s);
    return;
  }
  // keys and first sort (within each root's range)
  s.keys.ensure(n);
  s.keys2.ensure(n);
  s.idx.ensure(n);
  s.idx2.ensure(n);
  // With a plan of L levels to split, the keys are sorted on their top L digits only: the
  // splits read no deeper digit, and the bodies of a leaf are put in input order afterwards
  // whatever the order of their deeper digits.  If the plan fails, they are sorted again on
  // every digit for the level-by-level build.
  const int plan_levels = s.tree_plan > 0 ? s.tree_plan + 1 : kMaxLevel;
  const int begin_bit = plan_levels < kMaxLevel ? 3 * (kMaxLevel - plan_levels) : 0;
  k_keys<T><<<ceil_div(n, TB), TB, 0, s.stream>>>(s.bodies_in.p, n, s.box.p, s.d_root_first.p,
                                                  nroots, s.keys.p, s.idx.p);
  FMM_LAUNCH_CHECK();
  forest_sort(s, s.keys.p, s.keys2.p, s.idx.p, s.idx2.p, n, nroots, 3 * kMaxLevel, begin_bit);
  // nodes, level by level
  size_t cap0 = (size_t)std::max(1024, 4 * (n / std::max(1, s.cfg.ncrit)) + 64 + nroots);
  DevArr<int>* narr[] = {&s.nbegin, &s.ncount, &s.nparent, &s.nchildn, &s.nfirst,
                         &s.nnode, &s.npos, &s.ncb, &s.nlevel, &s.nsid};
  for (auto* a : narr) a->ensure(cap0);
  s.nX.ensure(4 * cap0);
  k_roots<T><<<ceil_div(nroots, TB), TB, 0, s.stream>>>(nroots, s.d_root_first.p, s.box.p,
                                                        s.nbegin.p, s.ncount.p, s.nparent.p,
                                                        s.nlevel.p, s.nsid.p, s.nX.p);
  FMM_LAUNCH_CHECK();
  s.level_lo.push_back(0);
  s.level_lo.push_back(nroots);
  const bool planned = s.tree_plan > 0 && planned_levels(s, nroots, narr, sizeof(narr) / sizeof(*narr));
  if (!planned && begin_bit > 0) {
    k_keys<T><<<ceil_div(n, TB), TB, 0, s.stream>>>(s.bodies_in.p, n, s.box.p,
                                                    s.d_root_first.p, nroots, s.keys.p, s.idx.p);
    FMM_LAUNCH_CHECK();
    forest_sort(s, s.keys.p, s.keys2.p, s.idx.p, s.idx2.p, n, nroots, 3 * kMaxLevel);
    k_roots<T><<<ceil_div(nroots, TB), TB, 0, s.stream>>>(nroots, s.d_root_first.p, s.box.p,
                                                          s.nbegin.p, s.ncount.p, s.nparent.p,
                                                          s.nlevel.p, s.nsid.p, s.nX.p);
    FMM_LAUNCH_CHECK();
    s.level_lo.assign({0, nroots});
  }
  for (int level = 0; !planned; level++) {
    int lo = s.level_lo[level], hi = s.level_lo[level + 1];
    int m = hi - lo;
    s.nsplit.ensure(9 * (size_t)m);
    s.coff.ensure(m + 1);
    s.idx.ensure(std::max((size_t)n, (size_t)m + 1));
    int* cnt = s.idx.p;  // the input-order index array is free until the second sort
    k_split<<<ceil_div(32LL * (m + 1), TB), TB, 0, s.stream>>>(lo, hi, level, s.cfg.ncrit, s.keys2.p,
                                                       s.nbegin.p, s.ncount.p, cnt, s.nsplit.p);
    FMM_LAUNCH_CHECK();
    exclusive_sum_int(s, cnt, s.coff.p, m + 1);
    FMM_CUDA(cudaMemcpyAsync(s.scal_host, s.coff.p + m, sizeof(int), cudaMemcpyDeviceToHost,
                             s.stream));
    FMM_CUDA(cudaStreamSynchronize(s.stream));
    int total = s.scal_host[0];
    if (total == 0) {
      k_finish_level<<<ceil_div(m, TB), TB, 0, s.stream>>>(lo, hi, s.nchildn.p, s.nfirst.p);
      FMM_LAUNCH_CHECK();
      break;
    }
    size_t need = (size_t)hi + total;
    for (auto* a : narr) grow(s, *a, need);
    grow(s, s.nX, 4 * need);
    k_emit<T><<<ceil_div(m, TB), TB, 0, s.stream>>>(lo, hi, level, cnt, s.coff.p, s.nsplit.p,
                                                    s.box.p, s.nbegin.p, s.ncount.p,
                                                    s.nparent.p, s.nchildn.p, s.nfirst.p,
                                                    s.nlevel.p, s.nsid.p, s.nX.p);
    FMM_LAUNCH_CHECK();
    s.level_lo.push_back(hi + total);
  }
  const int nlev = (int)s.level_lo.size() - 1;
  const int nnodes = s.level_lo.back();
  s.tree_plan = nlev;
  s.maxlevel = nlev - 1;
  s.ncells = nnodes;
  for (int l = nlev - 1; l >= 0; l--) {
    int lo = s.level_lo[l], hi = s.level_lo[l + 1];
    k_nnode<<<ceil_div(hi - lo, TB), TB, 0, s.stream>>>(lo, hi, s.nchildn.p, s.nfirst.p,
                                                        s.nnode.p);
    FMM_LAUNCH_CHECK();
  }
  // first cell of each root: exclusive scan of the roots' subtree sizes
  s.cbase.ensure(nroots + 1);
  s.coff.ensure(nroots + 1);
  FMM_CUDA(cudaMemsetAsync(s.coff.p + nroots, 0, sizeof(int), s.stream));
  FMM_CUDA(cudaMemcpyAsync(s.coff.p, s.nnode.p, sizeof(int) * nroots, cudaMemcpyDeviceToDevice,
                           s.stream));
  exclusive_sum_int(s, s.coff.p, s.cbase.p, nroots + 1);
  for (int l = 0; l < nlev; l++) {
    int lo = s.level_lo[l], hi = s.level_lo[l + 1];
    k_pos<<<ceil_div(hi - lo, TB), TB, 0, s.stream>>>(lo, hi, s.nchildn.p, s.nfirst.p,
                                                      s.nnode.p, s.cbase.p, s.npos.p, s.ncb.p);
    FMM_LAUNCH_CHECK();
  }
  // cells
  s.c_iparent.ensure(nnodes); s.c_ichild.ensure(nnodes); s.c_nchild.ensure(nnodes);
  s.c_ibody.ensure(nnodes); s.c_nbody.ensure(nnodes); s.c_level.ensure(nnodes);
  s.c_icell.ensure(nnodes);
  s.cX.ensure(nnodes);
  s.c_root.ensure(nnodes);
  k_cells<T><<<ceil_div(nnodes, TB), TB, 0, s.stream>>>(
      nnodes, s.box.p, s.nbegin.p, s.ncount.p, s.nparent.p, s.nchildn.p, s.nlevel.p, s.nsid.p,
      s.cbase.p, s.npos.p, s.ncb.p, s.nX.p, s.c_iparent.p, s.c_ichild.p, s.c_nchild.p,
      s.c_ibody.p, s.c_nbody.p, s.c_level.p, s.c_icell.p, s.cX.p, s.c_root.p);
  FMM_LAUNCH_CHECK();
  s.c_info.ensure(nnodes);
  k_cell_info<<<ceil_div(nnodes, TB), TB, 0, s.stream>>>(nnodes, s.c_nchild.p, s.c_ichild.p,
                                                         s.c_nbody.p, s.c_ibody.p, s.c_info.p);
  FMM_LAUNCH_CHECK();
  // bodies inside a leaf in input order (the stable partitions of the reference keep it)
  s.order.ensure(n);
  if (s.cfg.ncrit <= 64 && s.maxlevel < kMaxLevel) {
    // every leaf holds at most ncrit <= 64 bodies: rank them per leaf
    k_leaf_reorder<<<ceil_div(32LL * nnodes, TB), TB, 0, s.stream>>>(
        nnodes, s.nchildn.p, s.nbegin.p, s.ncount.p, s.idx2.p, s.order.p);
    FMM_LAUNCH_CHECK();
  } else {
    // general case: stable sort by leaf-truncated key from input order
    int* blev = s.idx.p;
    k_leaf_levels<<<ceil_div(nnodes, TB), TB, 0, s.stream>>>(nnodes, s.nchildn.p, s.nbegin.p,
                                                             s.ncount.p, s.nlevel.p, blev);
    FMM_LAUNCH_CHECK();
    k_tkey<<<ceil_div(n, TB), TB, 0, s.stream>>>(n, s.keys2.p, s.idx2.p, blev, s.keys.p, s.order.p);
    FMM_LAUNCH_CHECK();
    // s.order holds 0..n-1 (input positions); sort them by truncated key within each root
    FMM_CUDA(cudaMemcpyAsync(s.idx.p, s.order.p, n * sizeof(int), cudaMemcpyDeviceToDevice,
                             s.stream));
    forest_sort(s, s.keys.p, s.keys2.p, s.idx.p, s.order.p, n, nroots, 3 * kMaxLevel);
  }
  s.bodies.ensure(n);
  k_permute<T><<<ceil_div(n, TB), TB, 0, s.stream>>>(n, s.bodies_in.p, s.order.p, s.bodies.p);
  FMM_LAUNCH_CHECK();
  // leaf cell list
  s.nsplit.ensure(nnodes + 1);
  int* flags = s.nsplit.p;
  s.coff.ensure(nnodes + 1);
  k_leaf_flags<<<ceil_div(nnodes + 1, TB), TB, 0, s.stream>>>(nnodes, s.nchildn.p, flags);
  FMM_LAUNCH_CHECK();
  exclusive_sum_int(s, flags, s.coff.p, nnodes + 1);
  FMM_CUDA(cudaMemcpyAsync(s.scal_host, s.coff.p + nnodes, sizeof(int), cudaMemcpyDeviceToHost,
                           s.stream));
  s.leaves.ensure(nnodes);
  k_leaf_scatter<<<ceil_div(nnodes, TB), TB, 0, s.stream>>>(nnodes, s.nchildn.p, s.coff.p,
                                                            s.npos.p, s.leaves.p);
  FMM_LAUNCH_CHECK();
  s.root_cell.resize(nroots);
  FMM_CUDA(cudaMemcpyAsync(s.root_cell.data(), s.cbase.p, sizeof(int) * nroots,
                           cudaMemcpyDeviceToHost, s.stream));
  FMM_CUDA(cudaStreamSynchronize(s.stream));
  s.nleaves = s.scal_host[0];
}

// The bodies of part `part` of nparts: [t0, t1) with t = floor(k n / nparts), each bound
// moved down to the first body of the leaf that holds it, so that every leaf belongs to one
// part.  One leaf holds each bound below n and writes it; the leaf that ends at n writes
// the bound n.
__global__ void k_part_range(int nleaves, const int* __restrict__ leaves,
                             const int* __restrict__ ibody, const int* __restrict__ nbody, int n,
                             int t0, int t1, int* __restrict__ range) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaves) return;
  const int c = leaves[i];
  const int b = ibody[c], e = b + nbody[c];
  if (b <= t0 && t0 < e) range[0] = b;
  if (b <= t1 && t1 < e) range[1] = b;
  if (t1 >= n && e == n) range[1] = n;
}

void partition_range(SolverBase& s) {
  if (s.nparts <= 1) return;
  if (s.nroots > 1 || s.ij)
    throw FmmError(FMM_ERR_NOT_SUPPORTED, "a partitioned solve is one solve of one tree");
  if (s.cfg.mutual && s.cfg.images == 0)
    throw FmmError(FMM_ERR_NOT_SUPPORTED, "a partitioned solve with the mutual traversal");
  s.part_range.ensure(2);
  if (s.n == 0 || s.nleaves == 0) return;
  const int t0 = (int)((long long)s.part * s.n / s.nparts);
  const int t1 = (int)((long long)(s.part + 1) * s.n / s.nparts);
  k_part_range<<<ceil_div(s.nleaves, 256), 256, 0, s.stream>>>(
      s.nleaves, s.leaves.p, s.c_ibody.p, s.c_nbody.p, s.n, t0, t1, s.part_range.p);
  FMM_LAUNCH_CHECK();
}

template void build_tree<float>(Solver<float>&);
template void build_tree<double>(Solver<double>&);

}  // namespace fmmb200
