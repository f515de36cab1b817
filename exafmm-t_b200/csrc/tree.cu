// tree.cu -- octree, interaction lists and M2L setup on the GPU.
//
// The reference builds its tree by a serial top-down recursion that stably
// partitions bodies by octant (include/build_tree.h:49-166), rebuilds it once more
// after a set-based 2:1 balance (build_tree.h:209-359), and numbers nodes in the
// order their 8-child blocks are allocated.  Here the same tree comes from keys and
// sorts, bit for bit:
//
//   1. bounds (min/max reduction) and x0, r0 exactly as get_bounds (build_tree.h:20-35)
//   2. per body, a 63-bit octant path key: at each of 21 levels the octant test
//      (x > cx) + 2(y > cy) + 4(z > cz) against centres advanced by the same FP64
//      operations as the reference (cx +- r/2, build_tree.h:151-157)
//   3. stable radix sort of the path keys; node body counts are then binary
//      searches over key prefixes, so the tree grows level-synchronously
//   4. balance: N_l = nonleaf keys u S, S = parents of in-bounds neighbours of
//      N_l, level by level from the deepest (build_tree.h:247-300) -- sorts + uniques
//   5. rebuild: a node at level 1..L-1 splits iff it is in N_l or holds > ncrit bodies
//      (the leaf-key rule of build_tree.h:95-103 after find_leaf_keys)
//   6. node idx = allocation order: children of the k-th split node in pre-order
//      occupy idx 1+8k .. 8+8k (build_tree.h:147-149); pre-order = stable sort of
//      split nodes by padded path key
//   7. body order = stable sort of the ORIGINAL body order by the start key of the
//      body's leaf (the successive stable partitions of the recursion)
//
// Lists follow build_list.h:16-197 node by node (count pass + fill pass).
#include <cub/cub.cuh>

#include <algorithm>
#include <numeric>

#include "xfmm_internal.h"

namespace xfmm {
namespace {

constexpr int TPB = 256;
inline int nblk(int64_t n, int t = TPB) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

// ---------------------------------------------------------------- CUB helper
struct CubTmp {
  DBuf<char> tmp;
  template <class F>
  void run(F&& f) {
    size_t bytes = 0;
    XCUDA(f((void*)nullptr, bytes));
    tmp.reserve(std::max<size_t>(bytes, 16));
    bytes = tmp.n;
    XCUDA(f((void*)tmp.p, bytes));
  }
};

// ---------------------------------------------------------------- bounds
__global__ void k_minmax(const double* __restrict__ xyz, int64_t n, double* part) {
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; d++) {
      double v = xyz[3 * i + d];
      mn[d] = v < mn[d] ? v : mn[d];
      mx[d] = v > mx[d] ? v : mx[d];
    }
  __shared__ double s[6][TPB];
  for (int d = 0; d < 3; d++) {
    s[d][threadIdx.x] = mn[d];
    s[3 + d][threadIdx.x] = mx[d];
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int d = 0; d < 3; d++) {
        double a = s[d][threadIdx.x + w], b = s[3 + d][threadIdx.x + w];
        s[d][threadIdx.x] = a < s[d][threadIdx.x] ? a : s[d][threadIdx.x];
        s[3 + d][threadIdx.x] = b > s[3 + d][threadIdx.x] ? b : s[3 + d][threadIdx.x];
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 6; d++) part[6 * blockIdx.x + d] = s[d][0];
}

// ---------------------------------------------------------------- keys
__global__ void k_path_keys(const double* __restrict__ xyz, int64_t n, double x0, double y0, double z0, double r0,
                            uint64_t* __restrict__ key, int* __restrict__ idx) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
  double cx = x0, cy = y0, cz = z0, r = r0;
  uint64_t k = 0;
  for (int l = 0; l < LMAX; l++) {
    const int o = (x > cx) | ((y > cy) << 1) | ((z > cz) << 2);
    k = (k << 3) | (uint64_t)o;
    r = r / 2;
    cx = (o & 1) ? cx + r : cx - r;
    cy = (o & 2) ? cy + r : cy - r;
    cz = (o & 4) ? cz + r : cz - r;
  }
  key[i] = k;
  idx[i] = (int)i;
}

__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t* a, int64_t n, uint64_t v) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (a[m] < v) lo = m + 1;
    else hi = m;
  }
  return lo;
}
__device__ __forceinline__ bool contains_u64(const uint64_t* a, int64_t n, uint64_t v) {
  int64_t i = lower_bound_u64(a, n, v);
  return i < n && a[i] == v;
}

// prefix at `level` -> integer cell coordinates (x digit bit 0, y bit 1, z bit 2)
__host__ __device__ __forceinline__ void deinterleave(uint64_t p, int level, int& ix, int& iy, int& iz) {
  ix = iy = iz = 0;
  for (int b = 0; b < level; b++) {
    ix |= (int)((p >> (3 * b)) & 1) << b;
    iy |= (int)((p >> (3 * b + 1)) & 1) << b;
    iz |= (int)((p >> (3 * b + 2)) & 1) << b;
  }
}
__host__ __device__ __forceinline__ uint64_t interleave(int ix, int iy, int iz, int level) {
  uint64_t p = 0;
  for (int b = 0; b < level; b++) {
    p |= (uint64_t)((ix >> b) & 1) << (3 * b);
    p |= (uint64_t)((iy >> b) & 1) << (3 * b + 1);
    p |= (uint64_t)((iz >> b) & 1) << (3 * b + 2);
  }
  return p;
}
// hilbert.h:15-17, 79-107 (EXAFMM_HILBERT == 0): z at bit 3l, y at 3l+1, x at 3l+2, plus level offset
__host__ __device__ __forceinline__ uint64_t ref_key(int ix, int iy, int iz, int level) {
  uint64_t k = 0;
  for (int b = 0; b < level; b++) {
    k |= (uint64_t)((iz >> b) & 1) << (3 * b);
    k |= (uint64_t)((iy >> b) & 1) << (3 * b + 1);
    k |= (uint64_t)((ix >> b) & 1) << (3 * b + 2);
  }
  return k + ((((uint64_t)1) << (3 * level)) - 1) / 7;
}

// ---------------------------------------------------------------- level-synchronous growth
enum { RULE_ADAPTIVE = 0, RULE_REBUILD = 1, RULE_UNIFORM = 2 };

__global__ void k_count_level(const uint64_t* __restrict__ pref, int n, int level, const uint64_t* __restrict__ skeys,
                              int64_t nsrc, const uint64_t* __restrict__ tkeys, int64_t ntrg, int rule, int ncrit,
                              int maxlevel, const uint64_t* __restrict__ nset, int64_t nset_n, int* __restrict__ ns,
                              int* __restrict__ nt, int* __restrict__ split) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sh = 3 * (LMAX - level);
  const uint64_t lo = level == 0 ? 0 : (pref[i] << sh);
  const uint64_t hi_pref = pref[i] + 1;
  // end of the prefix range (level 0 covers everything)
  int64_t s0 = lower_bound_u64(skeys, nsrc, lo), t0 = lower_bound_u64(tkeys, ntrg, lo);
  int64_t s1, t1;
  if (level == 0 || (hi_pref << sh) == 0 || hi_pref == ((uint64_t)1 << (3 * level))) {
    s1 = nsrc;
    t1 = ntrg;
  } else {
    s1 = lower_bound_u64(skeys, nsrc, hi_pref << sh);
    t1 = lower_bound_u64(tkeys, ntrg, hi_pref << sh);
  }
  const int a = (int)(s1 - s0), b = (int)(t1 - t0);
  ns[i] = a;
  nt[i] = b;
  int sp;
  if (rule == RULE_UNIFORM) {
    sp = (a + b > 0) && (level < maxlevel);
  } else if (rule == RULE_ADAPTIVE) {
    sp = (a > ncrit) || (b > ncrit);
  } else {
    if (level == 0) sp = 1;
    else if (level >= maxlevel) sp = 0;
    else sp = (a > ncrit) || (b > ncrit) || contains_u64(nset, nset_n, pref[i]);
  }
  split[i] = sp;
}

__global__ void k_make_children(const uint64_t* __restrict__ pref, const int* __restrict__ split,
                                const int* __restrict__ scan, int n, uint64_t* __restrict__ cpref,
                                int* __restrict__ cppos) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !split[i]) return;
  const int base = 8 * scan[i];
  for (int c = 0; c < 8; c++) {
    cpref[base + c] = pref[i] * 8 + (uint64_t)c;
    cppos[base + c] = i;
  }
}

struct Level {
  int n = 0;
  DBuf<uint64_t> pref;
  DBuf<int> ns, nt, split, scan, ppos;
  int nsplit = 0;
};

struct Sorted {
  DBuf<uint64_t> key_orig, key_sorted;
  DBuf<int> idx_orig, idx_sorted;
};

void grow(std::vector<Level>& L, const Sorted& S, const Sorted& T, int64_t ns, int64_t nt, int rule, int ncrit,
          int maxlevel, const std::vector<DBuf<uint64_t>>* nsets, const std::vector<int64_t>* nset_n, CubTmp& cub,
          cudaStream_t s) {
  L.clear();
  L.emplace_back();
  {
    Level& r = L.back();
    r.n = 1;
    std::vector<uint64_t> z(1, 0);
    r.pref.upload(z, s);
    std::vector<int> m(1, -1);
    r.ppos.upload(m, s);
  }
  DBuf<int> dcount(1);
  for (int l = 0;; l++) {
    Level& cur = L[l];
    cur.ns.alloc(cur.n);
    cur.nt.alloc(cur.n);
    cur.split.alloc(cur.n);
    cur.scan.alloc(cur.n);
    const uint64_t* nsp = nullptr;
    int64_t nsn = 0;
    if (nsets && l < (int)nsets->size()) {
      nsp = (*nsets)[l].p;
      nsn = (*nset_n)[l];
    }
    k_count_level<<<nblk(cur.n), TPB, 0, s>>>(cur.pref.p, cur.n, l, S.key_sorted.p, ns, T.key_sorted.p, nt, rule,
                                               ncrit, maxlevel, nsp, nsn, cur.ns.p, cur.nt.p, cur.split.p);
    XLAUNCH();
    cub.run([&](void* tp, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(tp, b, cur.split.p, cur.scan.p, cur.n, s);
    });
    int last_scan = 0, last_split = 0;
    XCUDA(cudaMemcpyAsync(&last_scan, cur.scan.p + cur.n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    XCUDA(cudaMemcpyAsync(&last_split, cur.split.p + cur.n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    XCUDA(cudaStreamSynchronize(s));
    cur.nsplit = last_scan + last_split;
    if (cur.nsplit == 0) break;
    XREQUIRE(l + 1 <= LMAX, XFMM_ERR_UNSUPPORTED,
             "tree deeper than 21 levels (coincident bodies beyond ncrit?)");
    Level nxt;
    nxt.n = 8 * cur.nsplit;
    nxt.pref.alloc(nxt.n);
    nxt.ppos.alloc(nxt.n);
    k_make_children<<<nblk(cur.n), TPB, 0, s>>>(cur.pref.p, cur.split.p, cur.scan.p, cur.n, nxt.pref.p,
                                                 nxt.ppos.p);
    XLAUNCH();
    L.push_back(std::move(nxt));
  }
}

// ---------------------------------------------------------------- balance (build_tree.h:247-300)
__global__ void k_select_split_pref(const uint64_t* pref, const int* split, const int* scan, int n, uint64_t* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && split[i]) out[scan[i]] = pref[i];
}
__global__ void k_neighbour_parents(const uint64_t* __restrict__ N, int64_t n, int level, uint64_t* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int ix, iy, iz;
  deinterleave(N[i], level, ix, iy, iz);
  const int lim = 1 << level;
  int w = 0;
  for (int m = -1; m <= 1; ++m)
    for (int nn = -1; nn <= 1; ++nn)
      for (int p = -1; p <= 1; ++p) {
        if (!(m || nn || p)) continue;
        const int a = ix + m, b = iy + nn, c = iz + p;
        uint64_t v = ~(uint64_t)0;
        if (a >= 0 && a < lim && b >= 0 && b < lim && c >= 0 && c < lim) v = interleave(a, b, c, level) >> 3;
        out[26 * i + w++] = v;
      }
}

// sort + unique in place; returns count (drops the all-ones sentinel)
int64_t sort_unique(DBuf<uint64_t>& a, int64_t n, CubTmp& cub, cudaStream_t s) {
  if (n == 0) return 0;
  DBuf<uint64_t> b(n);
  cub.run([&](void* tp, size_t& bytes) {
    return cub::DeviceRadixSort::SortKeys(tp, bytes, a.p, b.p, (int)n, 0, 64, s);
  });
  DBuf<int> cnt(1);
  cub.run([&](void* tp, size_t& bytes) { return cub::DeviceSelect::Unique(tp, bytes, b.p, a.p, cnt.p, (int)n, s); });
  int m = 0;
  XCUDA(cudaMemcpyAsync(&m, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  uint64_t last = 0;
  XCUDA(cudaStreamSynchronize(s));
  if (m > 0) {
    XCUDA(cudaMemcpyAsync(&last, a.p + m - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    XCUDA(cudaStreamSynchronize(s));
    if (last == ~(uint64_t)0) m--;
  }
  return m;
}


// ---------------------------------------------------------------- numbering (build_tree.h:86, 147-149)
// padded path key of every split node, concatenated level by level (ascending level), so that a
// stable sort by padded key yields the pre-order (ancestors before descendants on ties)
__global__ void k_split_padded(const uint64_t* pref, const int* split, const int* scan, int n, int level, int base,
                               uint64_t* padded, int* sid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !split[i]) return;
  padded[base + scan[i]] = pref[i] << (3 * (LMAX - level));
  sid[base + scan[i]] = base + scan[i];
}
__global__ void k_rank(const int* sid_sorted, int n, int* rank, int* nonleaf_sid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rank[sid_sorted[i]] = i;
  nonleaf_sid[i] = sid_sorted[i];
}

struct NodeOut {
  int *lv, *isl, *nsr, *ntr, *par, *oct, *ch0;
  double4* ctr;
  uint64_t* key;
  int4* ixyz;       // cell coordinates + level
  uint64_t* start;  // padded start key
};

// idx and node fields of all nodes of one level; children of split parent k (in split order at
// level-1) are positions 8k..8k+7 of this level, so the parent's split id is sbase_prev + i/8
__global__ void k_fill_level(const uint64_t* __restrict__ pref, const int* __restrict__ ns, const int* __restrict__ nt,
                             const int* __restrict__ split, const int* __restrict__ scan,
                             const int* __restrict__ ppos, int n, int level, int sbase, int sbase_prev,
                             const int* __restrict__ rank, const int* __restrict__ prev_idx, int* __restrict__ idx,
                             double x0, double y0, double z0, double r0, NodeOut o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int id = 0, par = -1, oc = 0;
  if (level > 0) {
    id = 1 + 8 * rank[sbase_prev + i / 8] + (i & 7);
    par = prev_idx[ppos[i]];
    oc = (int)(pref[i] & 7);
  }
  idx[i] = id;
  o.lv[id] = level;
  o.isl[id] = split[i] ? 0 : 1;
  o.nsr[id] = ns[i];
  o.ntr[id] = nt[i];
  o.par[id] = par;
  o.oct[id] = oc;
  o.ch0[id] = split[i] ? 1 + 8 * rank[sbase + scan[i]] : -1;
  // centre by the reference's sequence of FP64 operations from the root (build_tree.h:151-157)
  double cx = x0, cy = y0, cz = z0, r = r0;
  for (int l = level - 1; l >= 0; l--) {
    const int d = (int)((pref[i] >> (3 * l)) & 7);
    r = r / 2;
    cx = (d & 1) ? cx + r : cx - r;
    cy = (d & 2) ? cy + r : cy - r;
    cz = (d & 4) ? cz + r : cz - r;
  }
  o.ctr[id] = make_double4(cx, cy, cz, r);
  int ix, iy, iz;
  deinterleave(pref[i], level, ix, iy, iz);
  o.key[id] = ref_key(ix, iy, iz, level);
  o.ixyz[id] = make_int4(ix, iy, iz, level);
  o.start[id] = level == 0 ? 0 : (pref[i] << (3 * (LMAX - level)));
}

// masked key = start key of the body's leaf (last leaf start <= body key)
__global__ void k_mask_keys(const uint64_t* __restrict__ key, int64_t n, const uint64_t* __restrict__ lstart, int nl,
                            uint64_t* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = key[i];
  int lo = 0, hi = nl;  // upper_bound
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (lstart[m] <= k) lo = m + 1;
    else hi = m;
  }
  out[i] = lstart[lo - 1];
}
__global__ void k_node_ranges(const uint64_t* __restrict__ start, int nn, const uint64_t* __restrict__ skeys,
                              int64_t nsrc, const uint64_t* __restrict__ tkeys, int64_t ntrg, int64_t* sbeg,
                              int64_t* tbeg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  sbeg[i] = lower_bound_u64(skeys, nsrc, start[i]);
  tbeg[i] = lower_bound_u64(tkeys, ntrg, start[i]);
}
__global__ void k_gather_bodies(const double* __restrict__ xyz, const int* __restrict__ perm, int64_t n,
                                double4* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = perm[i];
  out[i] = make_double4(xyz[3 * (int64_t)j], xyz[3 * (int64_t)j + 1], xyz[3 * (int64_t)j + 2], 0.0);
}

void sort_bodies(const double* xyz, int64_t n, const double* x0, double r0, Sorted& S, CubTmp& cub, cudaStream_t s) {
  S.key_orig.alloc(n);
  S.key_sorted.alloc(n);
  S.idx_orig.alloc(n);
  S.idx_sorted.alloc(n);
  k_path_keys<<<nblk(n), TPB, 0, s>>>(xyz, n, x0[0], x0[1], x0[2], r0, S.key_orig.p, S.idx_orig.p);
  XLAUNCH();
  cub.run([&](void* tp, size_t& b) {
    return cub::DeviceRadixSort::SortPairs(tp, b, S.key_orig.p, S.key_sorted.p, S.idx_orig.p, S.idx_sorted.p,
                                           (int)n, 0, 63, s);
  });
}

}  // namespace

// ================================================================= build_tree
void build_tree(Fmm& fmm, Tree& t, const double* src, const double* trg, int nonadaptive_depth, cudaStream_t s) {
  const int64_t ns = t.nsrc, nt = t.ntrg;
  XREQUIRE(ns > 0 && nt > 0, XFMM_ERR_ARG, "build_tree needs at least one source and one target");
  XREQUIRE(ns < (1ll << 31) && nt < (1ll << 31), XFMM_ERR_UNSUPPORTED, "more than 2^31-1 bodies");
  CubTmp cub;
  // 1. bounds (build_tree.h:20-35)
  const int nb = 128;
  DBuf<double> part(2 * 6 * nb);
  k_minmax<<<nb, TPB, 0, s>>>(src, ns, part.p);
  XLAUNCH();
  k_minmax<<<nb, TPB, 0, s>>>(trg, nt, part.p + 6 * nb);
  XLAUNCH();
  std::vector<double> hp = part.download(s);
  double mn[3], mx[3];
  for (int d = 0; d < 3; d++) {
    mn[d] = hp[d];
    mx[d] = hp[3 + d];
  }
  for (int b = 0; b < 2 * nb; b++)
    for (int d = 0; d < 3; d++) {
      mn[d] = hp[6 * b + d] < mn[d] ? hp[6 * b + d] : mn[d];
      mx[d] = hp[6 * b + 3 + d] > mx[d] ? hp[6 * b + 3 + d] : mx[d];
    }
  for (int d = 0; d < 3; d++)
    XREQUIRE(std::isfinite(mn[d]) && std::isfinite(mx[d]), XFMM_ERR_NUMERIC, "non-finite body coordinates");
  double x0[3];
  for (int d = 0; d < 3; d++) x0[d] = (mx[d] + mn[d]) / 2;
  double a = x0[0] - mn[0], b = mx[0] - x0[0];
  for (int d = 1; d < 3; d++) {
    a = a > x0[d] - mn[d] ? a : x0[d] - mn[d];
    b = b > mx[d] - x0[d] ? b : mx[d] - x0[d];
  }
  double r0 = std::fmax(a, b);
  r0 *= 1.00001;
  XREQUIRE(r0 > 0, XFMM_ERR_ARG, "all bodies coincide (zero-size bounding box)");
  for (int d = 0; d < 3; d++) t.x0[d] = fmm.x0[d] = x0[d];
  t.r0 = fmm.r0 = r0;
  t.ncrit = fmm.ncrit;
  t.nonadaptive = nonadaptive_depth >= 0;

  // 2-3. path keys + stable sort
  Sorted S, T;
  sort_bodies(src, ns, x0, r0, S, cub, s);
  sort_bodies(trg, nt, x0, r0, T, cub, s);

  // 4-5. levels
  std::vector<Level> L;
  int depth;
  if (nonadaptive_depth >= 0) {
    XREQUIRE(nonadaptive_depth <= LMAX, XFMM_ERR_UNSUPPORTED, "uniform depth above 21");
    grow(L, S, T, ns, nt, RULE_UNIFORM, fmm.ncrit, nonadaptive_depth, nullptr, nullptr, cub, s);
    depth = nonadaptive_depth;
  } else {
    grow(L, S, T, ns, nt, RULE_ADAPTIVE, fmm.ncrit, LMAX, nullptr, nullptr, cub, s);
    const int maxlevel = (int)L.size() - 1;
    depth = maxlevel;
    if (maxlevel > 0) {
      std::vector<DBuf<uint64_t>> Nset(maxlevel + 1);
      std::vector<int64_t> Nn(maxlevel + 1, 0);
      DBuf<uint64_t> Sset;
      int64_t Sn = 0;
      for (int l = maxlevel; l > 0; --l) {
        Level& lv = L[l];
        const int64_t nn = lv.nsplit + Sn;
        DBuf<uint64_t> N(std::max<int64_t>(nn, 1));
        if (lv.nsplit) {
          k_select_split_pref<<<nblk(lv.n), TPB, 0, s>>>(lv.pref.p, lv.split.p, lv.scan.p, lv.n, N.p);
          XLAUNCH();
        }
        if (Sn) XCUDA(cudaMemcpyAsync(N.p + lv.nsplit, Sset.p, Sn * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        const int64_t m = sort_unique(N, nn, cub, s);
        // S <- parents of the in-bounds neighbours of N (build_tree.h:262-284)
        if (m) {
          DBuf<uint64_t> P(26 * m);
          k_neighbour_parents<<<nblk(m), TPB, 0, s>>>(N.p, m, l, P.p);
          XLAUNCH();
          Sn = sort_unique(P, 26 * m, cub, s);
          Sset = std::move(P);
        } else {
          Sn = 0;
        }
        Nset[l] = std::move(N);
        Nn[l] = m;
      }
      grow(L, S, T, ns, nt, RULE_REBUILD, fmm.ncrit, maxlevel, &Nset, &Nn, cub, s);
      XREQUIRE((int)L.size() - 1 == maxlevel, XFMM_ERR_STATE, "balanced rebuild changed the tree depth");
    }
  }
  t.depth = fmm.depth = depth;

  // 6. numbering
  const int nlev = (int)L.size();
  std::vector<int> sbase(nlev + 1, 0);
  for (int l = 0; l < nlev; l++) sbase[l + 1] = sbase[l] + L[l].nsplit;
  const int nsplit = sbase[nlev];
  const int nnodes = 1 + 8 * nsplit;
  t.nnodes = nnodes;
  t.nnonleafs = nsplit;
  DBuf<int> rank(std::max(nsplit, 1)), nonleaf_sid(std::max(nsplit, 1));
  if (nsplit) {
    DBuf<uint64_t> padded(nsplit), padded_sorted(nsplit);
    DBuf<int> sid(nsplit), sid_sorted(nsplit);
    for (int l = 0; l < nlev; l++)
      if (L[l].nsplit) {
        k_split_padded<<<nblk(L[l].n), TPB, 0, s>>>(L[l].pref.p, L[l].split.p, L[l].scan.p, L[l].n, l, sbase[l],
                                                     padded.p, sid.p);
        XLAUNCH();
      }
    cub.run([&](void* tp, size_t& bb) {
      return cub::DeviceRadixSort::SortPairs(tp, bb, padded.p, padded_sorted.p, sid.p, sid_sorted.p, nsplit, 0, 63,
                                             s);
    });
    k_rank<<<nblk(nsplit), TPB, 0, s>>>(sid_sorted.p, nsplit, rank.p, nonleaf_sid.p);
    XLAUNCH();
  }
  t.level.alloc(nnodes);
  t.is_leaf.alloc(nnodes);
  t.nsrcs.alloc(nnodes);
  t.ntrgs.alloc(nnodes);
  t.parent.alloc(nnodes);
  t.octant.alloc(nnodes);
  t.child0.alloc(nnodes);
  t.center.alloc(nnodes);
  t.key.alloc(nnodes);
  DBuf<int4> ixyz(nnodes);
  DBuf<uint64_t> start(nnodes);
  NodeOut o{t.level.p, t.is_leaf.p, t.nsrcs.p, t.ntrgs.p, t.parent.p, t.octant.p, t.child0.p,
            t.center.p, t.key.p, ixyz.p, start.p};
  std::vector<DBuf<int>> lidx(nlev);
  for (int l = 0; l < nlev; l++) {
    lidx[l].alloc(L[l].n);
    k_fill_level<<<nblk(L[l].n), TPB, 0, s>>>(L[l].pref.p, L[l].ns.p, L[l].nt.p, L[l].split.p, L[l].scan.p,
                                               L[l].ppos.p, L[l].n, l, sbase[l], l > 0 ? sbase[l - 1] : 0, rank.p,
                                               l > 0 ? lidx[l - 1].p : nullptr, lidx[l].p, x0[0], x0[1], x0[2], r0,
                                               o);
    XLAUNCH();
  }
  // nonleafs in pre-order: node idx of split node with rank k is the idx of that split node
  {
    std::vector<int> h_sid = nonleaf_sid.download(s, nsplit);
    std::vector<int> split_node(nsplit);
    for (int l = 0; l < nlev; l++) {
      if (!L[l].nsplit) continue;
      std::vector<int> sp = L[l].split.download(s), sc = L[l].scan.download(s), id = lidx[l].download(s);
      for (int i = 0; i < L[l].n; i++)
        if (sp[i]) split_node[sbase[l] + sc[i]] = id[i];
    }
    t.h_nonleafs.resize(nsplit);
    for (int k = 0; k < nsplit; k++) t.h_nonleafs[k] = split_node[h_sid[k]];
    t.nonleafs.upload(t.h_nonleafs, s);
  }
  // 7. leaves (all, incl. empty) by start key; body order
  t.h_level = t.level.download(s);
  t.h_is_leaf = t.is_leaf.download(s);
  t.h_child0 = t.child0.download(s);
  t.h_nsrcs = t.nsrcs.download(s);
  t.h_ntrgs = t.ntrgs.download(s);
  std::vector<uint64_t> h_start = start.download(s);
  std::vector<int> all_leaves;
  for (int i = 0; i < nnodes; i++)
    if (t.h_is_leaf[i]) all_leaves.push_back(i);
  std::sort(all_leaves.begin(), all_leaves.end(), [&](int x, int y) { return h_start[x] < h_start[y]; });
  std::vector<uint64_t> lstart(all_leaves.size());
  t.h_leafs.clear();
  for (size_t k = 0; k < all_leaves.size(); k++) {
    lstart[k] = h_start[all_leaves[k]];
    if (t.h_nsrcs[all_leaves[k]] || t.h_ntrgs[all_leaves[k]]) t.h_leafs.push_back(all_leaves[k]);
  }
  t.nleafs = (int)t.h_leafs.size();
  t.leafs.upload(t.h_leafs, s);
  DBuf<uint64_t> dlstart;
  dlstart.upload(lstart, s);
  for (int w = 0; w < 2; w++) {
    Sorted& B = w ? T : S;
    const int64_t n = w ? nt : ns;
    DBuf<uint64_t> masked(n), masked_sorted(n);
    k_mask_keys<<<nblk(n), TPB, 0, s>>>(B.key_orig.p, n, dlstart.p, (int)lstart.size(), masked.p);
    XLAUNCH();
    DBuf<int>& perm = w ? t.trg_perm : t.src_perm;
    perm.alloc(n);
    cub.run([&](void* tp, size_t& bb) {
      return cub::DeviceRadixSort::SortPairs(tp, bb, masked.p, masked_sorted.p, B.idx_orig.p, perm.p, (int)n, 0, 63,
                                             s);
    });
    DBuf<double4>& bod = w ? t.trg4 : t.src4;
    bod.alloc(n);
    k_gather_bodies<<<nblk(n), TPB, 0, s>>>(w ? trg : src, perm.p, n, bod.p);
    XLAUNCH();
  }
  t.src_qim.alloc(ns);
  XCUDA(cudaMemsetAsync(t.src_qim.p, 0, ns * sizeof(double), s));
  t.sbeg.alloc(nnodes);
  t.tbeg.alloc(nnodes);
  k_node_ranges<<<nblk(nnodes), TPB, 0, s>>>(start.p, nnodes, S.key_sorted.p, ns, T.key_sorted.p, nt, t.sbeg.p,
                                             t.tbeg.p);
  XLAUNCH();
  XCUDA(cudaStreamSynchronize(s));
  t.lists_built = false;
  t.m2l_ready = false;
}

// ================================================================= lists (build_list.h)
namespace {

// membership in the relative-position tables of init_rel_coord(max_r, min_r, step) (geometry.h:156-173)
__device__ __forceinline__ bool in_table(int max_r, int min_r, int step, int a, int b, int c) {
  const int v[3] = {a, b, c};
  bool big = false;
  for (int d = 0; d < 3; d++) {
    if (v[d] < -max_r || v[d] > max_r || ((v[d] + max_r) % step) != 0) return false;
    if (abs(v[d]) >= min_r) big = true;
  }
  return big;
}
// index into the 26 M2L slots (M2L_Type: max 1, min 1, step 1; (0,0,0) excluded)
__device__ __forceinline__ int m2l_slot(int a, int b, int c) {
  if (a < -1 || a > 1 || b < -1 || b > 1 || c < -1 || c > 1) return -1;
  const int pos = (c + 1) * 9 + (b + 1) * 3 + (a + 1);
  return pos == 13 ? -1 : (pos < 13 ? pos : pos - 1);
}

__global__ void k_colleagues(const int4* __restrict__ ixyz, int nn, const uint64_t* __restrict__ skey,
                             const int* __restrict__ sidx, int* __restrict__ col) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int4 c = ixyz[i];
  const int lim = 1 << c.w;
  for (int k = 0; k < 27; k++) {
    const int a = c.x + (k % 3) - 1, b = c.y + ((k / 3) % 3) - 1, d = c.z + ((k / 9) % 3) - 1;
    int r = -1;
    if (a >= 0 && a < lim && b >= 0 && b < lim && d >= 0 && d < lim) {
      const uint64_t key = ref_key(a, b, d, c.w);
      const int64_t j = lower_bound_u64(skey, nn, key);
      if (j < nn && skey[j] == key) r = sidx[j];
    }
    col[27 * (int64_t)i + k] = r;
  }
}

struct ListArgs {
  const int *col, *is_leaf, *parent, *octant, *child0, *ntrgs, *nsrcs;
  int nsurf, nonadaptive;
};

// One node's lists in the reference's push order; counts only when the outputs are null.
__device__ void node_lists(const ListArgs& A, int n, int* p2p, int* m2p, int* p2l, int* m2l, int& np, int& nm,
                           int& nx) {
  np = nm = nx = 0;
  const bool leaf = A.is_leaf[n];
  // build_list_parent_level (build_list.h:16-43)
  const int par = A.parent[n];
  if (par >= 0) {
    const int oc = A.octant[n];
    for (int i = 0; i < 27; i++) {
      const int pc = A.col[27 * (int64_t)par + i];
      if (pc >= 0 && A.is_leaf[pc]) {
        const int a = (i % 3) * 4 - 4 - ((oc & 1) ? 2 : 0) + 1;
        const int b = ((i / 3) % 3) * 4 - 4 - ((oc & 2) ? 2 : 0) + 1;
        const int c = ((i / 9) % 3) * 4 - 4 - ((oc & 4) ? 2 : 0) + 1;
        if (leaf && in_table(3, 3, 2, a, b, c)) {  // P2P0
          if (p2p) p2p[np] = pc;
          np++;
        }
        if (in_table(5, 5, 2, a, b, c)) {  // P2L
          if (leaf && A.ntrgs[n] <= A.nsurf) {
            if (p2p) p2p[np] = pc;
            np++;
          } else {
            if (p2l) p2l[nx] = pc;
            nx++;
          }
        }
      }
    }
  }
  // build_list_current_level (build_list.h:52-74)
  for (int i = 0; i < 27; i++) {
    const int c = A.col[27 * (int64_t)n + i];
    if (c < 0) continue;
    const int a = (i % 3) - 1, b = ((i / 3) % 3) - 1, d = ((i / 9) % 3) - 1;
    const bool cl = A.is_leaf[c];
    if (cl && leaf) {
      if (in_table(1, 0, 1, a, b, d)) {  // P2P1
        if (p2p) p2p[np] = c;
        np++;
      }
    } else if (!cl && !leaf) {
      const int slot = m2l_slot(a, b, d);
      if (slot >= 0 && m2l) m2l[slot] = c;
    }
  }
  // build_list_child_level (build_list.h:84-114); NON_ADAPTIVE gates it on ntrgs (131-136)
  if (leaf && (!A.nonadaptive || A.ntrgs[n])) {
    for (int i = 0; i < 27; i++) {
      const int c = A.col[27 * (int64_t)n + i];
      if (c < 0 || A.is_leaf[c]) continue;
      for (int j = 0; j < 8; j++) {
        const int cc = A.child0[c] + j;
        const int a = (i % 3) * 4 - 4 + ((j & 1) ? 2 : 0) - 1;
        const int b = ((i / 3) % 3) * 4 - 4 + ((j & 2) ? 2 : 0) - 1;
        const int d = ((i / 9) % 3) * 4 - 4 + ((j & 4) ? 2 : 0) - 1;
        if (in_table(3, 3, 2, a, b, d)) {  // P2P2
          if (p2p) p2p[np] = cc;
          np++;
        }
        if (in_table(5, 5, 2, a, b, d)) {  // M2P
          if (A.is_leaf[cc] && A.nsrcs[cc] <= A.nsurf) {
            if (p2p) p2p[np] = cc;
            np++;
          } else {
            if (m2p) m2p[nm] = cc;
            nm++;
          }
        }
      }
    }
  }
}

__global__ void k_list_count(ListArgs A, int nn, int64_t* cp, int64_t* cm, int64_t* cx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  int a, b, c;
  node_lists(A, i, nullptr, nullptr, nullptr, nullptr, a, b, c);
  cp[i] = a;
  cm[i] = b;
  cx[i] = c;
}
__global__ void k_list_fill(ListArgs A, int nn, const int64_t* op, const int64_t* om, const int64_t* ox, int* p2p,
                            int* m2p, int* p2l, int* m2l) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  int* m = m2l + 26 * (int64_t)i;
  for (int k = 0; k < 26; k++) m[k] = -1;
  int a, b, c;
  node_lists(A, i, p2p + op[i], m2p + om[i], p2l + ox[i], m, a, b, c);
}

void exclusive_scan_i64(DBuf<int64_t>& cnt, int nn, DBuf<int64_t>& off, CubTmp& cub, cudaStream_t s,
                        int64_t& total) {
  off.alloc(nn + 1);
  cub.run([&](void* tp, size_t& b) { return cub::DeviceScan::ExclusiveSum(tp, b, cnt.p, off.p, nn + 1, s); });
  XCUDA(cudaMemcpyAsync(&total, off.p + nn, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  XCUDA(cudaStreamSynchronize(s));
}

}  // namespace

void build_lists(Fmm& fmm, Tree& t, cudaStream_t s) {
  XREQUIRE(t.nnodes > 0, XFMM_ERR_STATE, "build_list before build_tree");
  CubTmp cub;
  const int nn = t.nnodes;
  // cell coordinates from the reference keys (get3DIndex, hilbert.h:115-195)
  std::vector<uint64_t> hkey = t.key.download(s);
  std::vector<int4> hix(nn);
  for (int i = 0; i < nn; i++) {
    const int lv = t.h_level[i];
    uint64_t k = hkey[i] - ((((uint64_t)1) << (3 * lv)) - 1) / 7;
    int ix = 0, iy = 0, iz = 0;
    for (int b = 0; b < lv; b++) {
      iz |= (int)((k >> (3 * b)) & 1) << b;
      iy |= (int)((k >> (3 * b + 1)) & 1) << b;
      ix |= (int)((k >> (3 * b + 2)) & 1) << b;
    }
    hix[i] = make_int4(ix, iy, iz, lv);
  }
  DBuf<int4> ixyz;
  ixyz.upload(hix, s);
  DBuf<uint64_t> skey(nn);
  DBuf<int> iota(nn), sidx(nn);
  {
    std::vector<int> h(nn);
    std::iota(h.begin(), h.end(), 0);
    iota.upload(h, s);
  }
  cub.run([&](void* tp, size_t& b) {
    return cub::DeviceRadixSort::SortPairs(tp, b, t.key.p, skey.p, iota.p, sidx.p, nn, 0, 64, s);
  });
  t.colleagues.alloc(27 * (size_t)nn);
  k_colleagues<<<nblk(nn), TPB, 0, s>>>(ixyz.p, nn, skey.p, sidx.p, t.colleagues.p);
  XLAUNCH();
  ListArgs A{t.colleagues.p, t.is_leaf.p, t.parent.p, t.octant.p, t.child0.p, t.ntrgs.p, t.nsrcs.p, fmm.nsurf,
             t.nonadaptive};
  t.nsurf_lists = fmm.nsurf;
  DBuf<int64_t> cp(nn + 1), cm(nn + 1), cx(nn + 1);
  XCUDA(cudaMemsetAsync(cp.p + nn, 0, sizeof(int64_t), s));
  XCUDA(cudaMemsetAsync(cm.p + nn, 0, sizeof(int64_t), s));
  XCUDA(cudaMemsetAsync(cx.p + nn, 0, sizeof(int64_t), s));
  k_list_count<<<nblk(nn), TPB, 0, s>>>(A, nn, cp.p, cm.p, cx.p);
  XLAUNCH();
  exclusive_scan_i64(cp, nn, t.p2p_off, cub, s, t.np2p);
  exclusive_scan_i64(cm, nn, t.m2p_off, cub, s, t.nm2p);
  exclusive_scan_i64(cx, nn, t.p2l_off, cub, s, t.np2l);
  t.p2p.alloc(std::max<int64_t>(t.np2p, 1));
  t.m2p.alloc(std::max<int64_t>(t.nm2p, 1));
  t.p2l.alloc(std::max<int64_t>(t.np2l, 1));
  t.m2l.alloc(26 * (size_t)nn);
  k_list_fill<<<nblk(nn), TPB, 0, s>>>(A, nn, t.p2p_off.p, t.m2p_off.p, t.p2l_off.p, t.p2p.p, t.m2p.p, t.p2l.p,
                                       t.m2l.p);
  XLAUNCH();

  // schedules for the passes
  std::vector<int64_t> hp_off = t.p2p_off.download(s), hm_off = t.m2p_off.download(s), hx_off = t.p2l_off.download(s);
  std::vector<int> hp2p = t.p2p.download(s, t.np2p), hm2p = t.m2p.download(s, t.nm2p);
  t.nl_level_off.assign(t.depth + 2, 0);
  std::vector<int> nl_sorted;
  for (int l = 0; l <= t.depth; l++) {
    t.nl_level_off[l] = (int)nl_sorted.size();
    for (int k : t.h_nonleafs)
      if (t.h_level[k] == l) nl_sorted.push_back(k);
  }
  t.nl_level_off[t.depth + 1] = (int)nl_sorted.size();
  t.nl_by_level.upload(nl_sorted, s);
  std::vector<int> ev;
  std::vector<int64_t> work;  // near-field pairs per evaluated leaf
  std::vector<float> sc;
  std::vector<double> sc64;
  t.p2p_pairs = t.m2p_pairs = t.l2p_pairs = 0;
  for (int k = 0; k < t.nleafs; k++) {
    const int n = t.h_leafs[k];
    sc.push_back((float)std::pow(0.5, t.h_level[n]));
    sc64.push_back(std::pow(0.5, t.h_level[n]));
    if (t.h_ntrgs[n] > 0) {
      ev.push_back(k);
      int64_t srcs = 0;
      for (int64_t j = hp_off[n]; j < hp_off[n + 1]; j++) srcs += t.h_nsrcs[hp2p[j]];
      t.p2p_pairs += srcs * t.h_ntrgs[n];
      work.push_back(srcs * t.h_ntrgs[n]);
      t.m2p_pairs += (hm_off[n + 1] - hm_off[n]) * (int64_t)fmm.nsurf * t.h_ntrgs[n];
      t.l2p_pairs += (int64_t)fmm.nsurf * t.h_ntrgs[n];
    }
  }
#ifndef XFMM_SORT_EVAL
#define XFMM_SORT_EVAL 1
#endif
  if (XFMM_SORT_EVAL) {
    // evaluate the heaviest leaves first: one warp per leaf, so the grid's tail is made of small leaves
    std::vector<int> order(ev.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::vector<int> sorted(ev.size());
    for (size_t i = 0; i < order.size(); i++) sorted[i] = ev[order[i]];
    ev.swap(sorted);
  }
  t.n_eval_leafs = (int)ev.size();
  t.eval_leafs.upload(ev, s);
  t.leaf_scale.upload(sc, s);
  t.leaf_scale64.upload(sc64, s);
  std::vector<int> px;
  for (int i = 0; i < nn; i++)
    if (hx_off[i + 1] > hx_off[i]) px.push_back(i);
  t.n_p2l_nodes = (int)px.size();
  t.p2l_nodes.upload(px, s);
  XCUDA(cudaStreamSynchronize(s));
  t.lists_built = true;
  t.m2l_ready = false;
}

// ================================================================= M2L setup
void m2l_setup(Fmm& fmm, Tree& t, cudaStream_t s) {
  XREQUIRE(t.lists_built, XFMM_ERR_STATE, "M2L_setup before build_list");
  std::vector<int> hm2l = t.m2l.download(s);
  const bool per_level = fmm.kernel != XFMM_LAPLACE;
  t.m2l_grouped_by_level = per_level;
  const int ngroups = per_level ? std::max(t.depth, 1) : 1;
  std::vector<int> src, trg, tab;
  std::vector<float> scale;
  std::vector<double> scale64;
  t.m2l_src_off.assign(ngroups + 1, 0);
  t.m2l_trg_off.assign(ngroups + 1, 0);
  std::vector<int> slot(t.nnodes, -1);
  t.m2l_pairs = 0;
  for (int g = 0; g < ngroups; g++) {
    t.m2l_src_off[g] = (int)src.size();
    t.m2l_trg_off[g] = (int)trg.size();
    std::vector<int> tg;
    for (int k : t.h_nonleafs)
      if (!per_level || t.h_level[k] == g) tg.push_back(k);
    // unique M2L sources of this group, in node (pointer) order as std::set<Node*> (fmm_scale_invariant.h:283-296)
    std::vector<char> mark(t.nnodes, 0);
    for (int k : tg)
      for (int j = 0; j < 26; j++)
        if (hm2l[26 * (size_t)k + j] >= 0) mark[hm2l[26 * (size_t)k + j]] = 1;
    int cnt = 0;
    for (int i = 0; i < t.nnodes; i++)
      if (mark[i]) {
        slot[i] = cnt++;
        src.push_back(i);
      }
    for (int k : tg) {
      trg.push_back(k);
      for (int j = 0; j < 26; j++) {
        const int sn = hm2l[26 * (size_t)k + j];
        tab.push_back(sn >= 0 ? slot[sn] : -1);
        t.m2l_pairs += sn >= 0;
      }
      scale.push_back(per_level ? 1.0f : (float)std::pow(2.0, t.h_level[k] + 1));
      scale64.push_back(per_level ? 1.0 : std::pow(2.0, t.h_level[k] + 1));
    }
  }
  t.m2l_src_off[ngroups] = (int)src.size();
  t.m2l_trg_off[ngroups] = (int)trg.size();
  t.n_m2l_src = (int)src.size();
  t.n_m2l_trg = (int)trg.size();
  t.m2l_src.upload(src, s);
  t.m2l_trg.upload(trg, s);
  t.h_m2l_trg = trg;
  t.m2l_tab.upload(tab, s);
  t.h_m2l_tab = tab;
  t.m2l_scale.upload(scale, s);
  t.m2l_scale64.upload(scale64, s);
  XCUDA(cudaStreamSynchronize(s));
  t.m2l_ready = true;
}

}  // namespace xfmm
