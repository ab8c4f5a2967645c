// Octree construction on the B200, bit-exact with the reference's recursive
// FP64 octant partition.
//
// Reference: periodic unwrap tree_pm_coupling.cpp:94-218; Morton ordering
// tree_ordering.cpp:13-171; TreeGravitySolver::build tree_gravity.cpp:343-524,
// buildNodeRecursive :1081-1206 (octantForParticle :50-61), accumulateMultipoles
// :1208-1380.
//
// The reference builds the octree recursively: starting from Morton order it
// stably partitions each node's particles by (x >= cx, y >= cy, z >= cz)
// against FP64 centres obtained by repeated centre +- half/2, stopping at
// count <= leaf or half <= 1e-12. The same tree is produced here in parallel:
//  1. unwrap each axis (largest circular gap of the canonical coordinates):
//     per-bucket {min, max} over about n/8 buckets find it when no bucket's
//     own extent can hide it, else the axis is sorted;
//  2. Morton keys per particle (they order particles within a leaf);
//  3. per particle, the geometric octant path (3 bits/level, 21 levels per
//     64-bit word) by the same FP64 centre recurrence; stable sort by path,
//     resolving first only the levels the previous tree needed;
//  4. nodes = maximal runs of equal path prefix whose parent run has more
//     than `leaf` particles; they are enumerated in preorder from the
//     common-prefix lengths of neighbouring sorted paths (node ends and
//     parents by nearest-smaller queries on block minima of those lengths);
//  5. within each leaf, particles ranked by (Morton key, row): the
//     reference's order (a leaf above 1024 particles takes a stable sort of
//     the Morton order by leaf instead);
//  6. FP64 multipoles bottom-up, each parent reduced once, children in octant
//     order, by the last child to finish.
#include <cuda_runtime.h>

#include <climits>

#include <cmath>
#include <algorithm>
#include <cstring>
#include <vector>

#include "context.cuh"

namespace chui {
namespace {

inline unsigned gridFor(size_t n, int block) {
  size_t b = (n + block - 1) / block;
  if (b > 148u * 64u) b = 148u * 64u;
  return static_cast<unsigned>(b ? b : 1);
}

__device__ __forceinline__ unsigned long long dbits(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v));
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double(static_cast<long long>(b));
}

// ---------------------------------------------------------------- unwrap

// unwrapPeriodicAxis (tree_pm_coupling.cpp:94-218): canonical wrap, the
// coordinates sorted by their non-negative IEEE bits, the largest circular gap
// between neighbours, and one box added below the value after it.
//
// The canonical periodic coordinate (tree_pm_coupling.cpp:166-183), one
// compiled copy (not inlined, so that no caller's contraction changes its
// bits).
__device__ __noinline__ double canonicalCoordinate(double x, double box, int canonical) {
  double v = canonical ? x : x - box * floor(x / box);
  if (v >= box) {
    v = 0.0;
  } else if (v < 0.0) {
    v += box;
  }
  if (v == 0.0) v = 0.0;
  return v;
}

// Gap bucket of a canonical coordinate: floor(v * nb / L), clamped. The map is
// monotone in v (a product with a positive factor and a truncation both
// keep order), so every value of bucket k is <= every value of bucket k+1.
__device__ __forceinline__ uint32_t gapBucket(double v, double scale, uint32_t nb) {
  const double f = v * scale;
  if (!(f > 0.0)) return 0u;
  return f >= static_cast<double>(nb) ? nb - 1u : static_cast<uint32_t>(f);
}

// The canonical coordinate of every particle, and per gap bucket the
// smallest and largest value, as bits (non-negative doubles order like their
// bits). A plain read first skips the atomics that cannot change the bucket
// (a stale read only ever asks for an atomic that was not needed): particles
// in row order often share a bucket across a warp.
__global__ void canonicalBucketsKernel(int64_t n, const double* __restrict__ in, double box, int canonical,
                                       double* out, double scale, uint32_t nb, unsigned long long* bmin,
                                       unsigned long long* bmax) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = canonicalCoordinate(in[i], box, canonical);
    out[i] = v;
    const uint32_t k = gapBucket(v, scale, nb);
    const unsigned long long b = dbits(v);
    if (b < bmin[k]) atomicMin(bmin + k, b);
    if (b > bmax[k]) atomicMax(bmax + k, b);
  }
}

// flag[k] = 1 for a non-empty bucket (flag[nb] = 0: the scan's total slot)
__global__ void bucketFlagsKernel(uint32_t nb, const unsigned long long* __restrict__ bmin, uint32_t* flag) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k <= nb;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    flag[k] = k < nb && bmin[k] != ~0ull ? 1u : 0u;
  }
}

// The non-empty buckets' {min, max}, in bucket (= value) order.
__global__ void bucketCompactKernel(uint32_t nb, const unsigned long long* __restrict__ bmin,
                                    const unsigned long long* __restrict__ bmax, const uint32_t* __restrict__ off,
                                    unsigned long long* cmin, unsigned long long* cmax) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nb;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long lo = bmin[k];
    if (lo == ~0ull) continue;
    const uint32_t j = off[k];
    if (j < nb) {  // always true; a guard on the computed index
      cmin[j] = lo;
      cmax[j] = bmax[k];
    }
  }
}

// Circular gaps between consecutive runs of sorted coordinates: run i holds
// values lo[i] .. hi[i], gap_i = lo[i+1] - hi[i], and lo[0] + L - hi[m-1]
// around the box (tree_pm_coupling.cpp:189-207). With the fully sorted
// coordinates every run is one value (lo == hi); with gap buckets a run is a
// bucket, and a bucket whose own extent hi - lo is not below the largest gap
// found could hide a larger or equal gap inside it: pass 1 then raises
// *suspect and the axis is sorted instead. Pass 0 finds the largest gap (gaps
// are >= 0, so their bits order like the values; one atomic per block); pass
// 1 takes the smallest value after a gap equal to it as the anchor. The run
// count is m, or *m_dev when given.
__global__ void __launch_bounds__(256) runGapKernel(int64_t m, const uint32_t* __restrict__ m_dev,
                                                    const unsigned long long* __restrict__ lo,
                                                    const unsigned long long* __restrict__ hi, double box,
                                                    unsigned long long* best_gap, int pass,
                                                    unsigned long long* best_anchor, unsigned long long* suspect) {
  if (m_dev) m = *m_dev;
  unsigned long long local = 0ull;
  const unsigned long long target = pass == 0 ? 0ull : *best_gap;
  bool hidden = false;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double cur = bitsd(hi[i]);
    const bool around = i + 1 == m;
    const unsigned long long after = around ? lo[0] : lo[i + 1];
    const double cand = bitsd(after);
    const double next = around ? cand + box : cand;
    const double gap = next - cur;
    if (pass == 0) {
      const unsigned long long g = dbits(gap);
      local = g > local ? g : local;
    } else {
      if (dbits(gap) == target) atomicMin(best_anchor, after);
      if (suspect && lo[i] != hi[i] && dbits(cur - bitsd(lo[i])) >= target) hidden = true;
    }
  }
  if (pass != 0) {
    if (hidden) atomicOr(suspect, 1ull);
    return;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, local, off);
    local = o > local ? o : local;
  }
  __shared__ unsigned long long warp_max[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_max[warp] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long v = 0ull;
    for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) v = warp_max[k] > v ? warp_max[k] : v;
    if (v != 0ull) atomicMax(best_gap, v);
  }
}

// u += L below the anchor; skipped while the axis's bucket gaps are suspect.
__global__ void applyAnchorKernel(int64_t n, double* u, double box, const unsigned long long* anchor_bits,
                                  const unsigned long long* suspect) {
  if (suspect && *suspect) return;
  const double anchor = bitsd(*anchor_bits);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (u[i] < anchor) u[i] += box;
  }
}


// ------------------------------------------------------------- bounds

__global__ void boundsKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, unsigned long long* out /* 6 */) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double p[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], p[a]);
      hi[a] = fmax(hi[a], p[a]);
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(out + a, orderedBits(lo[a]));
      atomicMax(out + 3 + a, orderedBits(hi[a]));
    }
  }
}

// ------------------------------------------------------------- Morton

// expandBits21 / morton3D (tree_ordering.cpp:73-85).
__device__ __forceinline__ unsigned long long spread21(unsigned v) {
  unsigned long long x = v & 0x1FFFFFu;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// std::llround for a finite value in [0, 2^21): round half away from zero.
__device__ __forceinline__ unsigned roundHalfAway(double v) {
  const double t = trunc(v);
  const double frac = __dsub_rn(v, t);
  return static_cast<unsigned>(t) + (frac >= 0.5 ? 1u : 0u);
}

// buildMortonOrderingInPlace (tree_ordering.cpp:152-168).
__global__ void mortonKernel(int64_t n, const double* __restrict__ ux, const double* __restrict__ uy,
                             const double* __restrict__ uz, double lo0, double lo1, double lo2,
                             double extent, unsigned long long* keys, uint32_t* idx) {
  const double grid = static_cast<double>((1u << 21) - 1u);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v[3] = {__ddiv_rn(__dsub_rn(ux[i], lo0), extent), __ddiv_rn(__dsub_rn(uy[i], lo1), extent),
                         __ddiv_rn(__dsub_rn(uz[i], lo2), extent)};
    unsigned q[3];
    for (int a = 0; a < 3; ++a) {
      const double c = v[a] < 0.0 ? 0.0 : (v[a] > 1.0 ? 1.0 : v[a]);
      q[a] = roundHalfAway(__dmul_rn(c, grid));
    }
    keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    idx[i] = static_cast<uint32_t>(i);
  }
}

// ------------------------------------------------------------ paths

// Octant path of each particle (row order, or perm[j] for entry j) by the reference's centre
// recurrence: digit d compares against the level-(d-1) centre, then
// centre += +-half/2 (tree_gravity.cpp:50-61, :1181-1185). Word w holds levels
// 21w+1 .. 21w+21, level 1 in the top digit.
__global__ void pathKernel(int64_t n, int words, const uint32_t* __restrict__ perm,
                           const double* __restrict__ ux, const double* __restrict__ uy,
                           const double* __restrict__ uz, double cx0, double cy0, double cz0,
                           double half0, unsigned long long mask0, unsigned long long* path /* words * n */) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t p = perm ? perm[j] : static_cast<uint32_t>(j);
    const double px = ux[p], py = uy[p], pz = uz[p];
    double cx = cx0, cy = cy0, cz = cz0, h = half0;
    for (int w = 0; w < words; ++w) {
      unsigned long long word = 0;
      for (int k = 0; k < kLevelsPerWord; ++k) {
        const unsigned o = (px >= cx ? 4u : 0u) | (py >= cy ? 2u : 0u) | (pz >= cz ? 1u : 0u);
        word = (word << 3) | o;
        const double ch = 0.5 * h;
        cx = __dadd_rn(cx, (o & 4u) ? ch : -ch);
        cy = __dadd_rn(cy, (o & 2u) ? ch : -ch);
        cz = __dadd_rn(cz, (o & 1u) ? ch : -ch);
        h = ch;
      }
      path[static_cast<size_t>(w) * n + j] = w == 0 ? word & mask0 : word;
    }
  }
}

__global__ void gatherU64Kernel(int64_t n, const unsigned long long* __restrict__ src,
                                const uint32_t* __restrict__ idx, unsigned long long* dst) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    dst[i] = src[idx[i]];
  }
}

__device__ __forceinline__ unsigned digitAt(const unsigned long long* path, int64_t n, int64_t i, int level) {
  // level >= 1
  const int w = (level - 1) / kLevelsPerWord;
  const int k = (level - 1) % kLevelsPerWord;
  return static_cast<unsigned>((path[static_cast<size_t>(w) * n + i] >> (3 * (kLevelsPerWord - 1 - k))) & 7ull);
}

// Number of leading equal digits of the paths at sorted positions i-1, i.
__global__ void commonPrefixKernel(int64_t n, int words, int levels, const unsigned long long* __restrict__ path,
                                   int* cp) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (i == 0) {
      cp[0] = -1;
      continue;
    }
    int c = levels;  // equal through every resolved level
    for (int w = 0; w < words; ++w) {
      const unsigned long long x = path[static_cast<size_t>(w) * n + i - 1] ^ path[static_cast<size_t>(w) * n + i];
      if (x != 0) {
        c = kLevelsPerWord * w + (__clzll(static_cast<long long>(x)) - 1) / 3;
        break;
      }
    }
    cp[i] = c;
  }
}

struct NodePlan {
  int64_t n;
  int leaf;        // max_leaf_size
  int depth_half;  // first depth whose half size <= 1e-12
  int depth_max;   // resolvable depth = 21 * words
};

// Leaf depth of the chain of nodes started at sorted position i, or -1 when i
// starts no node. A node (d, i) exists when its parent run is internal
// (size > leaf and half > 1e-12, tree_gravity.cpp:1136); it is a leaf when
// its own run has at most `leaf` particles or d reaches depth_half.
__device__ int chainLeafDepth(const NodePlan& p, const int* __restrict__ cp, int64_t i, uint32_t* status) {
  const int ci = cp[i];
  const int64_t n = p.n;
  if (ci >= p.depth_max) return -1;  // identical to the previous path through all resolved levels
  if (i > 0) {
    // parent run at level ci containing i-1 and i
    if (ci >= p.depth_half) return -1;
    int64_t s = -1, r = -1;
    for (int64_t k = i - 1; k >= 0 && k >= i - p.leaf; --k) {
      if (cp[k] < ci) {
        s = k;
        break;
      }
    }
    for (int64_t k = i + 1; k < n && k <= i + p.leaf; ++k) {
      if (cp[k] < ci) {
        r = k;
        break;
      }
    }
    if (r < 0 && i + p.leaf >= n) r = n;
    if (s >= 0 && r >= 0 && r - s <= p.leaf) return -1;  // parent is a leaf
  }
  int m = -1;  // min common prefix in the forward window; -1 when the array ends inside it
  if (i + p.leaf < n) {
    m = 1 << 30;
    for (int64_t k = i + 1; k <= i + p.leaf; ++k) m = min(m, cp[k]);
  }
  int l = max(ci + 1, min(m + 1, p.depth_half));
  if (l > p.depth_max) {
    atomicOr(status, kStatusNeedMorePathWords);
    l = p.depth_max;
  }
  if (l > kMaxDepth) atomicOr(status, kStatusDepthExceeded);
  return l;
}

__global__ void nodeCountKernel(NodePlan p, const int* __restrict__ cp, uint32_t* counts, uint32_t* status) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i <= p.n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (i == p.n) {
      counts[i] = 0;
      continue;
    }
    const int l = chainLeafDepth(p, cp, i, status);
    counts[i] = l < 0 ? 0u : static_cast<uint32_t>(l - cp[i]);
  }
}

// Block minima of the common-prefix lengths: level 0 is cp itself, entry b of
// level L+1 the minimum of entries 32b .. 32b+31 of level L. Node ends and
// run starts are then nearest-smaller queries that scan at most 32 entries
// per level up and down instead of searching the path words.
constexpr int kCpLevels = 7;
struct CpLevels {
  const int* lv[kCpLevels];
  int64_t len[kCpLevels];
  int count;  // levels in use; the top one is scanned whole
};

__global__ void cpBlockMinKernel(int64_t len, const int* __restrict__ in, int* out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t whole = (len + 31) / 32 * 32;  // whole warps: every lane takes part in the reduction
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < whole; i += stride) {
    const int v = i < len ? in[i] : INT_MAX;
    const int m = __reduce_min_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0) out[i >> 5] = m;
  }
}

// First position k > i with cp[k] < t, or n.
__device__ int64_t nextBelow(const CpLevels& c, int64_t i, int t) {
  int64_t k = i + 1;
  int level = 0;
  for (;;) {
    const int64_t len = c.len[level];
    const int64_t end = level + 1 == c.count ? len : ((k >> 5) + 1) << 5;
    const int64_t stop = end < len ? end : len;
    for (; k < stop; ++k)
      if (c.lv[level][k] < t) goto found;
    if (stop >= len) return c.len[0];
    k = stop >> 5;
    ++level;
  }
found:
  while (level > 0) {
    --level;
    const int64_t b = k << 5;
    const int64_t e = b + 32 < c.len[level] ? b + 32 : c.len[level];
    for (k = b; k < e; ++k)
      if (c.lv[level][k] < t) break;
  }
  return k;
}

// Last position k <= i with cp[k] < t, or -1.
__device__ int64_t prevBelow(const CpLevels& c, int64_t i, int t) {
  int64_t k = i;
  int level = 0;
  for (;;) {
    const int64_t beg = level + 1 == c.count ? 0 : (k >> 5) << 5;
    for (; k >= beg; --k)
      if (c.lv[level][k] < t) goto found;
    if (beg == 0) return -1;
    k = (beg >> 5) - 1;
    ++level;
  }
found:
  while (level > 0) {
    --level;
    const int64_t b = k << 5;
    const int64_t e = b + 32 < c.len[level] ? b + 32 : c.len[level];
    for (k = e - 1; k >= b; --k)
      if (c.lv[level][k] < t) break;
  }
  return k;
}

struct NodeOut {
  double4* geom;
  uint4* range;      // begin, count, child_count (filled later), subtree_end
  uint32_t* parent;
  uint32_t* depth;
  uint32_t* child;   // 8 per node
  uint32_t* leaf_of_pos;
};

// Emit the chain of nodes started at each sorted position, in preorder.
// The sorted positions that start a chain of nodes (counts[i] > 0), listed in
// order: starts[pos_off[i]] = i. The emission then runs one thread per chain
// instead of one per position (most positions start none).
__global__ void chainFlagsKernel(int64_t n, const uint32_t* __restrict__ counts, uint32_t* flag) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i <= n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    flag[i] = i < n && counts[i] > 0u ? 1u : 0u;
}

__global__ void chainListKernel(int64_t n, const uint32_t* __restrict__ counts, const uint32_t* __restrict__ pos_off,
                                uint32_t* starts) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (counts[i] > 0u) starts[pos_off[i]] = static_cast<uint32_t>(i);
}

__global__ void nodeEmitKernel(NodePlan p, int words, const unsigned long long* __restrict__ path,
                               const int* __restrict__ cp, const uint32_t* __restrict__ counts,
                               const uint32_t* __restrict__ offset, const uint32_t* __restrict__ starts,
                               const uint32_t* __restrict__ chains, CpLevels lv, double cx0, double cy0,
                               double cz0, double half0, uint32_t total_nodes, NodeOut out, uint32_t* status) {
  const int64_t n = p.n;
  const int64_t m = *chains;  // chain starts
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < m;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = starts[j];
    const uint32_t cnt = i < n ? counts[i] : 0u;
    if (cnt == 0) {
      atomicOr(status, kStatusIndexRange);
      return;
    }
    const int ci = cp[i];
    const int d0 = ci + 1;
    const int l = d0 + static_cast<int>(cnt) - 1;
    // replay the centre recurrence down to depth d0 - 1
    double cx = cx0, cy = cy0, cz = cz0, h = half0;
    for (int d = 1; d < d0; ++d) {
      const unsigned o = digitAt(path, n, i, d);
      const double ch = 0.5 * h;
      cx = __dadd_rn(cx, (o & 4u) ? ch : -ch);
      cy = __dadd_rn(cy, (o & 2u) ? ch : -ch);
      cz = __dadd_rn(cz, (o & 1u) ? ch : -ch);
      h = ch;
    }
    for (int d = d0; d <= l; ++d) {
      if (d > 0) {
        const unsigned o = digitAt(path, n, i, d);
        const double ch = 0.5 * h;
        cx = __dadd_rn(cx, (o & 4u) ? ch : -ch);
        cy = __dadd_rn(cy, (o & 2u) ? ch : -ch);
        cz = __dadd_rn(cz, (o & 1u) ? ch : -ch);
        h = ch;
      }
      const uint32_t node = offset[i] + static_cast<uint32_t>(d - d0);
      // the run of the d-digit prefix ends where the common prefix drops below d
      const int64_t end = (d == 0) ? n : nextBelow(lv, i, d);
      if (node >= total_nodes || end > n || end <= i) {
        atomicOr(status, kStatusIndexRange);
        return;
      }
      const uint32_t count = static_cast<uint32_t>(end - i);
      out.geom[node] = make_double4(cx, cy, cz, h);
      out.range[node] = make_uint4(static_cast<uint32_t>(i), count, 0u, offset[end]);
      out.depth[node] = static_cast<uint32_t>(d);
      if (d == 0) {
        out.parent[node] = kInvalid;
      } else {
        uint32_t parent;
        if (d > d0) {
          parent = node - 1;
        } else {
          // the parent's run starts at the last position whose prefix differs within d - 1 digits
          const int64_t s = prevBelow(lv, i, d - 1);
          if (s < 0) {
            atomicOr(status, kStatusIndexRange);
            return;
          }
          parent = offset[s] + static_cast<uint32_t>((d - 1) - (cp[s] + 1));
        }
        if (parent >= total_nodes) {
          atomicOr(status, kStatusIndexRange);
          return;
        }
        out.parent[node] = parent;
        out.child[8 * static_cast<size_t>(parent) + digitAt(path, n, i, d)] = node;
      }
      if (d == l) {
        for (int64_t k = i; k < end; ++k) out.leaf_of_pos[k] = node;
        if (count > kLeafOrderMax) atomicOr(status, kStatusLargeLeaf);
      }
    }
  }
}

__global__ void childCountKernel(int64_t nodes, const uint32_t* __restrict__ child, uint4* range) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nodes;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t c = 0;
    for (int o = 0; o < 8; ++o) c += child[8 * k + o] != kInvalid ? 1u : 0u;
    range[k].z = c;
  }
}

__global__ void invertKernel(int64_t n, const uint32_t* __restrict__ perm, uint32_t* inv) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    inv[perm[i]] = static_cast<uint32_t>(i);
  }
}

// Within-leaf order. The reference partitions the Morton-sorted particles
// into octants, so a leaf's particles keep their Morton order (key, then row:
// the radix sort is stable over rows; tree_gravity.cpp:1081-1206,
// tree_ordering.cpp:13-71). Here the octant paths are sorted directly, and
// each particle's place in its leaf is its rank by (Morton key, row) among
// the leaf's particles: positions [begin, begin + count) of the path order.
__global__ void leafOrderKernel(int64_t n, const uint32_t* __restrict__ leaf_of_pos, const uint4* __restrict__ range,
                                const uint32_t* __restrict__ row_of_pos, const unsigned long long* __restrict__ key_of_pos,
                                uint32_t* sorted_index, uint32_t* status) {
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint4 r = range[leaf_of_pos[p]];
    if (r.y > static_cast<uint32_t>(kLeafOrderMax) || p < r.x || p >= static_cast<int64_t>(r.x) + r.y ||
        static_cast<int64_t>(r.x) + r.y > n) {
      atomicOr(status, kStatusIndexRange);
      continue;
    }
    const unsigned long long k = key_of_pos[p];
    const uint32_t row = row_of_pos[p];
    uint32_t rank = 0u;
    for (uint32_t q = r.x; q < r.x + r.y; ++q) {
      const unsigned long long kq = key_of_pos[q];
      rank += (kq < k || (kq == k && row_of_pos[q] < row)) ? 1u : 0u;
    }
    sorted_index[r.x + rank] = row;
  }
}

// Leaf of each particle in Morton order (the large-leaf path: a stable sort
// of the Morton order by leaf gives the same order).
__global__ void leafKeyKernel(int64_t n, const uint32_t* __restrict__ perm_m, const uint32_t* __restrict__ pos_of_particle,
                              const uint32_t* __restrict__ leaf_of_pos, uint32_t* key) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    key[j] = leaf_of_pos[pos_of_particle[perm_m[j]]];
  }
}

struct MomentIn {
  const double4* u4;  // tree-ordered tree-frame positions and masses
  int quadrupole;
  const double* eps;  // tree-ordered source softening (nullable: uniform)
  double2* soft;      // per node {min, max} source softening (when eps is given)
};

// Source softening range of a node (accumulateMultipoles,
// tree_gravity.cpp:1215-1240, 1320-1323): leaves over their sources, parents
// over their children; a node without sources keeps {+inf, 0}.
__device__ __forceinline__ double2 leafSoftening(const MomentIn& in, const uint4 r) {
  double lo = INFINITY, hi = 0.0;
  for (uint32_t t = r.x; t < r.x + r.y; ++t) {
    const double e = in.eps[t];
    lo = fmin(lo, e);
    hi = fmax(hi, e);
  }
  return make_double2(lo, hi);
}

__device__ void leafMoments(int64_t node, const MomentIn& in, const double4 g, const uint4 r,
                            double4* com_out, double* quad_out) {
  double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
  for (uint32_t t = r.x; t < r.x + r.y; ++t) {
    const double4 p = in.u4[t];
    const double ms = p.w;
    total += ms;
    wx += ms * p.x;
    wy += ms * p.y;
    wz += ms * p.z;
  }
  double cx = g.x, cy = g.y, cz = g.z;
  if (total > 0.0) {
    cx = wx / total;
    cy = wy / total;
    cz = wz / total;
  }
  double q[7] = {0, 0, 0, 0, 0, 0, 0};
  if (in.quadrupole && total > 0.0) {
    double ixx = 0, ixy = 0, ixz = 0, iyy = 0, iyz = 0, izz = 0;
    for (uint32_t t = r.x; t < r.x + r.y; ++t) {
      const double4 p = in.u4[t];
      const double ms = p.w;
      const double rx = p.x - cx, ry = p.y - cy, rz = p.z - cz;
      ixx += ms * rx * rx;
      ixy += ms * rx * ry;
      ixz += ms * rx * rz;
      iyy += ms * ry * ry;
      iyz += ms * ry * rz;
      izz += ms * rz * rz;
    }
    const double tr = ixx + iyy + izz;
    q[0] = 3.0 * ixx - tr;
    q[1] = 3.0 * ixy;
    q[2] = 3.0 * ixz;
    q[3] = 3.0 * iyy - tr;
    q[4] = 3.0 * iyz;
    q[5] = 3.0 * izz - tr;
    q[6] = tr;
  }
  *com_out = make_double4(cx, cy, cz, total);
  const double ox = g.x - cx, oy = g.y - cy, oz = g.z - cz;
  for (int k = 0; k < 7; ++k) quad_out[k] = q[k];
  quad_out[7] = sqrt(ox * ox + oy * oy + oz * oz);
  (void)node;
}

__device__ __forceinline__ double4 ldcg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = __ldcg(q), b = __ldcg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ void internalMoments(int64_t node, const double4 g, const uint32_t* __restrict__ child,
                                const double4* com, const double* quad, int quadrupole,
                                double4* com_out, double* quad_out) {
  double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
  for (int o = 0; o < 8; ++o) {
    const uint32_t c = __ldcg(child + 8 * node + o);
    if (c == kInvalid) continue;
    const double4 cc = ldcg4(com + c);
    total += cc.w;
    wx += cc.w * cc.x;
    wy += cc.w * cc.y;
    wz += cc.w * cc.z;
  }
  double cx = g.x, cy = g.y, cz = g.z;
  if (total > 0.0) {
    cx = wx / total;
    cy = wy / total;
    cz = wz / total;
  }
  double q[7] = {0, 0, 0, 0, 0, 0, 0};
  if (quadrupole && total > 0.0) {
    for (int o = 0; o < 8; ++o) {
      const uint32_t c = __ldcg(child + 8 * node + o);
      if (c == kInvalid) continue;
      const double4 cc = ldcg4(com + c);
      const double dx = cc.x - cx, dy = cc.y - cy, dz = cc.z - cz;
      const double m = cc.w;
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double* qc = quad + 8 * static_cast<size_t>(c);
      q[0] += __ldcg(qc + 0) + m * (3.0 * dx * dx - d2);
      q[1] += __ldcg(qc + 1) + m * (3.0 * dx * dy);
      q[2] += __ldcg(qc + 2) + m * (3.0 * dx * dz);
      q[3] += __ldcg(qc + 3) + m * (3.0 * dy * dy - d2);
      q[4] += __ldcg(qc + 4) + m * (3.0 * dy * dz);
      q[5] += __ldcg(qc + 5) + m * (3.0 * dz * dz - d2);
      q[6] += __ldcg(qc + 6) + m * d2;
    }
  }
  *com_out = make_double4(cx, cy, cz, total);
  const double ox = g.x - cx, oy = g.y - cy, oz = g.z - cz;
  for (int k = 0; k < 7; ++k) quad_out[k] = q[k];
  quad_out[7] = sqrt(ox * ox + oy * oy + oz * oz);
}

// Bottom-up moments: each leaf computes itself, then the last child to finish
// a parent computes it from its children in octant order (deterministic).
__global__ void momentsKernel(int64_t nodes, MomentIn in, const double4* __restrict__ geom,
                              const uint4* __restrict__ range, const uint32_t* __restrict__ parent,
                              const uint32_t* __restrict__ child, uint32_t* counter, double4* com,
                              double* quad) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nodes;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint4 r = range[k];
    if (r.z != 0) continue;  // internal
    double4 cm;
    double q[8];
    leafMoments(k, in, geom[k], r, &cm, q);
    com[k] = cm;
    for (int t = 0; t < 8; ++t) quad[8 * k + t] = q[t];
    if (in.eps) in.soft[k] = leafSoftening(in, r);
    int64_t node = k;
    while (true) {
      __threadfence();
      const uint32_t p = parent[node];
      if (p == kInvalid) break;
      const uint32_t done = atomicAdd(counter + p, 1u);
      if (done + 1 != range[p].z) break;
      __threadfence();
      internalMoments(p, geom[p], child, com, quad, in.quadrupole, &cm, q);
      com[p] = cm;
      for (int t = 0; t < 8; ++t) quad[8 * static_cast<size_t>(p) + t] = q[t];
      if (in.eps) {
        double lo = INFINITY, hi = 0.0;
        for (int o = 0; o < 8; ++o) {
          const uint32_t ch = __ldcg(child + 8 * static_cast<size_t>(p) + o);
          if (ch == kInvalid) continue;
          const double2 cs = __ldcg(in.soft + ch);
          lo = fmin(lo, cs.x);
          hi = fmax(hi, cs.y);
        }
        in.soft[p] = make_double2(lo, hi);
      }
      node = p;
    }
  }
}

// FP32 COM offset from the node centre and |centre - COM| for the walk's
// single-precision acceptance tests.
__global__ void nodeFrameKernel(int64_t nodes, const double4* __restrict__ geom, const double4* __restrict__ com,
                                const double* __restrict__ quad, float4* f4, float4* mq) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nodes;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double4 g = geom[k], c = com[k];
    const double* q = quad + 8 * k;
    f4[k] = make_float4(static_cast<float>(c.x - g.x), static_cast<float>(c.y - g.y), static_cast<float>(c.z - g.z),
                        static_cast<float>(q[7]));
    // the screened-quadrupole tensor M = (Q + tr I) / 3 of the multipole force
    const double tr = q[6];
    mq[2 * k] = make_float4(static_cast<float>(c.w), static_cast<float>((q[0] + tr) / 3.0),
                            static_cast<float>(q[1] / 3.0), static_cast<float>(q[2] / 3.0));
    mq[2 * k + 1] = make_float4(static_cast<float>((q[3] + tr) / 3.0), static_cast<float>(q[4] / 3.0),
                                static_cast<float>((q[5] + tr) / 3.0), static_cast<float>(tr));
  }
}

__global__ void nodeBoundsKernel(int64_t nodes, const double4* __restrict__ geom,
                                 const double4* __restrict__ com, unsigned long long* out) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nodes;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double4 g = geom[k], c = com[k];
    const double a[3] = {g.x, g.y, g.z}, b[3] = {c.x, c.y, c.z};
    for (int t = 0; t < 3; ++t) {
      lo[t] = fmin(lo[t], fmin(a[t], b[t]));
      hi[t] = fmax(hi[t], fmax(a[t], b[t]));
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(out + a, orderedBits(lo[a]));
      atomicMax(out + 3 + a, orderedBits(hi[a]));
    }
  }
}

// Tree-ordered source records (the reference's source lanes,
// tree_pm_coupling.cpp:3736-3800), written from row order: each row's caller
// position, tree-frame position (the unwrapped coordinates), mass and
// softening are read contiguously and its records are scattered to its tree
// position (whole 32-byte records: no partial sectors).
__global__ void scatterSourcesKernel(int64_t n, const uint32_t* __restrict__ pos_of_row,
                                     const double* __restrict__ x, const double* __restrict__ y,
                                     const double* __restrict__ z, const double* __restrict__ ux,
                                     const double* __restrict__ uy, const double* __restrict__ uz,
                                     const double* __restrict__ m, double uniform_mass, double4* d4, double4* u4,
                                     const double* __restrict__ eps_rows, double* eps_tree) {
  for (int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; s < n;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t t = pos_of_row[s];
    const double ms = m ? m[s] : uniform_mass;
    d4[t] = make_double4(x[s], y[s], z[s], ms);
    u4[t] = make_double4(ux[s], uy[s], uz[s], ms);
    if (eps_rows) eps_tree[t] = eps_rows[s];
  }
}

// Mixed precision: each source's FP32 offset from its leaf's FP64 centre, in
// tree order (a leaf's sources are consecutive).
__global__ void leafOffsetsKernel(int64_t n, const uint32_t* __restrict__ leaf_of_pos,
                                  const double4* __restrict__ geom, const double4* __restrict__ u4, float4* f4) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double4 u = u4[t];
    const double4 g = geom[leaf_of_pos[t]];
    f4[t] = make_float4(static_cast<float>(u.x - g.x), static_cast<float>(u.y - g.y), static_cast<float>(u.z - g.z),
                        static_cast<float>(u.w));
  }
}

__global__ void targetKeyKernel(int64_t nt, const uint32_t* __restrict__ active, int64_t n,
                                const uint32_t* __restrict__ pos_of_row, int explicit_targets,
                                uint32_t* key, uint32_t* slot) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nt;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t row = active ? active[k] : static_cast<uint32_t>(k);
    key[k] = (row < n) ? pos_of_row[row] : 0xFFFFFFFFu;
    (void)explicit_targets;
    slot[k] = static_cast<uint32_t>(k);
  }
}

__global__ void iotaKernel(int64_t n, uint32_t* v) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    v[i] = static_cast<uint32_t>(i);
  }
}

int bitsFor(uint64_t maxval) {
  int b = 1;
  while (b < 32 && (1ull << b) <= maxval) ++b;
  return b;
}

}  // namespace

#ifndef CHUI_GAP_BUCKET_DIV
#define CHUI_GAP_BUCKET_DIV 8  // about n / 8 gap buckets per axis (n / 4: 9.3 ms tree build at 256^3, n / 8: 8.8)
#endif

// Unwrap the axes into `out` (tree frame), returning each axis's anchor. Per
// axis, the canonical coordinates go into about n/8 gap buckets (min and max
// per bucket), the non-empty buckets are listed in order, and the largest
// circular gap is taken between consecutive buckets. When every bucket's own
// extent is below that gap no gap inside a bucket can reach it, so it is the
// largest gap of the sorted coordinates and the anchor is theirs. Otherwise
// (few particles, or a bucket holding the largest gap) the axis's
// coordinates are sorted and the gaps taken between consecutive values, as
// the reference does.
static int unwrapAxes(Context& c, int64_t n, int axes, const int* axis, const double* const* in, const double* box,
                      const int* canonical, double* const* out, double* anchor, cudaStream_t s) {
  if (n == 0 || axes == 0) {
    for (int k = 0; k < axes; ++k) anchor[axis[k]] = 0.0;
    return 0;
  }
  uint32_t nb = 1;
  while (nb < static_cast<uint64_t>(n) / CHUI_GAP_BUCKET_DIV && nb < (1u << 30)) nb <<= 1;
  if (ensure(c.bucket_min, static_cast<size_t>(nb) * 8) || ensure(c.bucket_max, static_cast<size_t>(nb) * 8) ||
      ensure(c.gap_min, static_cast<size_t>(nb) * 8) || ensure(c.gap_max, static_cast<size_t>(nb) * 8) ||
      ensure(c.gap_flag, (static_cast<size_t>(nb) + 1) * 4) || ensure(c.gap_off, (static_cast<size_t>(nb) + 1) * 4))
    return CHUI_TREEPM_ENOMEM;
  auto* sc = c.scalars.as<unsigned long long>();
  unsigned long long* suspect = sc + 16;  // one flag per axis slot
  unsigned long long init[6] = {0ull, ~0ull, 0ull, ~0ull, 0ull, ~0ull};
  cudaMemcpyAsync(sc, init, sizeof(init), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(suspect, 0, 3 * 8, s);
  unsigned long long* bmin = c.bucket_min.as<unsigned long long>();
  unsigned long long* bmax = c.bucket_max.as<unsigned long long>();
  uint32_t* flag = c.gap_flag.as<uint32_t>();
  uint32_t* off = c.gap_off.as<uint32_t>();
  for (int k = 0; k < axes; ++k) {
    const int a = axis[k];
    unsigned long long* g = sc + 2 * k;
    cudaMemsetAsync(bmin, 0xFF, static_cast<size_t>(nb) * 8, s);
    cudaMemsetAsync(bmax, 0, static_cast<size_t>(nb) * 8, s);
    const double scale = static_cast<double>(nb) / box[a];
    { noteLaunch(); canonicalBucketsKernel<<<gridFor(n, 256), 256, 0, s>>>(n, in[a], box[a], canonical[a], out[a], scale,
                                                                       nb, bmin, bmax); }
    { noteLaunch(); bucketFlagsKernel<<<gridFor(static_cast<size_t>(nb) + 1, 256), 256, 0, s>>>(nb, bmin, flag); }
    if (int rc = exclusiveScanU32(c, flag, off, static_cast<int64_t>(nb) + 1, s)) return rc;
    { noteLaunch(); bucketCompactKernel<<<gridFor(nb, 256), 256, 0, s>>>(nb, bmin, bmax, off, c.gap_min.as<unsigned long long>(),
                                                                     c.gap_max.as<unsigned long long>()); }
    for (int pass = 0; pass < 2; ++pass) {
      noteLaunch();
      runGapKernel<<<gridFor(nb, 256), 256, 0, s>>>(nb, off + nb, c.gap_min.as<unsigned long long>(),
                                                    c.gap_max.as<unsigned long long>(), box[a], g, pass, g + 1,
                                                    suspect + k);
    }
    { noteLaunch(); applyAnchorKernel<<<gridFor(n, 256), 256, 0, s>>>(n, out[a], box[a], g + 1, suspect + k); }
  }
  unsigned long long ab[6], sus[3];
  cudaMemcpyAsync(ab, sc, sizeof(ab), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(sus, suspect, sizeof(sus), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  bool resorted = false;
  for (int k = 0; k < axes; ++k) {
    if (!sus[k]) continue;
    // out[a] still holds the canonical coordinates (the anchor was skipped)
    const int a = axis[k];
    if (ensure(c.keys_b, static_cast<size_t>(n) * 8)) return CHUI_TREEPM_ENOMEM;
    const unsigned long long* kin = reinterpret_cast<const unsigned long long*>(out[a]);
    unsigned long long* sorted = c.keys_b.as<unsigned long long>();
    // canonical coordinates are non-negative: bit 63 is zero
    if (int rc = radixSortKeysU64(c, 1, &kin, &sorted, n, 63, s)) return rc;
    unsigned long long* g = sc + 2 * k;
    const unsigned long long reset[2] = {0ull, ~0ull};
    cudaMemcpyAsync(g, reset, sizeof(reset), cudaMemcpyHostToDevice, s);
    for (int pass = 0; pass < 2; ++pass) {
      noteLaunch();
      runGapKernel<<<gridFor(n, 256), 256, 0, s>>>(n, nullptr, sorted, sorted, box[a], g, pass, g + 1, nullptr);
    }
    { noteLaunch(); applyAnchorKernel<<<gridFor(n, 256), 256, 0, s>>>(n, out[a], box[a], g + 1, nullptr); }
    cudaMemcpyAsync(&ab[2 * k], g, 16, cudaMemcpyDeviceToHost, s);
    resorted = true;
  }
  if (resorted && cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  c.unwrap_sorted_axes = 0;
  for (int k = 0; k < axes; ++k) {
    std::memcpy(&anchor[axis[k]], &ab[2 * k + 1], 8);
    if (sus[k]) c.unwrap_sorted_axes |= 1 << axis[k];
  }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

int treeBuild(Context& c, int64_t n, const double* x, const double* y, const double* z,
              const double* m, double uniform_mass, const double src_lo[3], const double src_hi[3],
              cudaStream_t s) {
  c.n_nodes = 0;
  c.max_depth = 0;
  c.unwrap_sorted_axes = 0;
  c.large_leaf = 0;
  c.path_levels_retried = 0;
  if (n == 0) return 0;
  const double box[3] = {c.cfg.box_x, c.cfg.box_y, c.cfg.box_z};
  if (ensure(c.ux, n * 8) || ensure(c.uy, n * 8) || ensure(c.uz, n * 8)) return CHUI_TREEPM_ENOMEM;
  const double* in[3] = {x, y, z};
  double* u[3] = {c.ux.as<double>(), c.uy.as<double>(), c.uz.as<double>()};
  double anchors[3];
  int canonical[3], axis[3], axes = 0;
  for (int a = 0; a < 3; ++a) {
    // canonical flag as tree_pm_coupling.cpp:3183-3194
    canonical[a] = src_lo[a] >= 0.0 && src_hi[a] < box[a];
    if (c.cfg.boundary_condition != CHUI_TREEPM_BOUNDARY_PERIODIC) {
      // isolated/open: the tree takes the caller's coordinates (tree_pm_coupling.cpp:3179-3196)
      cudaMemcpyAsync(u[a], in[a], static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
      anchors[a] = 0.0;
      continue;
    }
    axis[axes++] = a;
  }
  if (int rc = unwrapAxes(c, n, axes, axis, in, box, canonical, u, anchors, s)) return rc;
  // bounds of the unwrapped frame
  auto* sc = c.scalars.as<unsigned long long>();
  unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
  cudaMemcpyAsync(sc, init, sizeof(init), cudaMemcpyHostToDevice, s);
  { noteLaunch(); boundsKernel<<<std::min(gridFor(n, 256), kReduceBlocks), 256, 0, s>>>(n, u[0], u[1], u[2], sc); }
  unsigned long long hb[6];
  cudaMemcpyAsync(hb, sc, sizeof(hb), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = fromOrderedBits(hb[a]);
    hi[a] = fromOrderedBits(hb[3 + a]);
  }
  const double max_extent = std::fmax(hi[0] - lo[0], std::fmax(hi[1] - lo[1], hi[2] - lo[2]));

  // Morton keys (tree_ordering.cpp:152-172). The reference sorts them and
  // partitions the sorted list into octants; here the octant paths are sorted
  // directly and the Morton keys only order each leaf's particles.
  const double extent = std::fmax(max_extent, 1.0e-12);
  if (ensure(c.keys_a, n * 8) || ensure(c.keys_b, n * 8) || ensure(c.idx_a, n * 4) || ensure(c.idx_b, n * 4) ||
      ensure(c.idx_c, (n + 1) * 4) || ensure(c.idx_d, (n + 1) * 4) || ensure(c.morton_keys, n * 8))
    return CHUI_TREEPM_ENOMEM;
  unsigned long long* morton = c.morton_keys.as<unsigned long long>();
  { noteLaunch(); mortonKernel<<<gridFor(n, 256), 256, 0, s>>>(n, u[0], u[1], u[2], lo[0], lo[1], lo[2], extent,
                                               morton, c.idx_a.as<uint32_t>()); }
  int rc = 0;

  // root (tree_gravity.cpp:448-452)
  const double mext = std::fmax(max_extent, 1.0e-10);
  const double cx0 = 0.5 * (lo[0] + hi[0]);
  const double cy0 = 0.5 * (lo[1] + hi[1]);
  const double cz0 = 0.5 * (lo[2] + hi[2]);
  const double half0 = 0.5 * mext * (1.0 + 1.0e-8);
  int depth_half = 0;
  for (double h = half0; !(h <= 1.0e-12) && depth_half < 4 * kMaxDepth; h *= 0.5) ++depth_half;

  if (ensure(c.common_prefix, n * 4) || ensure(c.node_count_per_pos, (n + 1) * 4) ||
      ensure(c.node_offset, (n + 1) * 4) || ensure(c.inv_pos, n * 4) || ensure(c.leaf_of_pos, n * 4) ||
      ensure(c.sorted_index, n * 4) || ensure(c.pos_of_row, n * 4))
    return CHUI_TREEPM_ENOMEM;
  uint32_t* status = c.status.as<uint32_t>();
  int* cp = c.common_prefix.as<int>();
  uint32_t* counts = c.node_count_per_pos.as<uint32_t>();
  uint32_t* offset = c.node_offset.as<uint32_t>();
  unsigned long long* path = nullptr;
  uint32_t* row_of_pos = nullptr;
  uint32_t total_nodes = 0;
  int words = 1;
  NodePlan plan;
  plan.n = n;
  plan.leaf = static_cast<int>(c.cfg.max_leaf_size);
  plan.depth_half = depth_half;
  // The first attempt resolves only the levels the previous tree of this
  // context needed (plus one): the lower digits of the path word are zeroed,
  // so the sort skips them. A node that needs a deeper level raises the
  // same status as a missing path word, and the build repeats with every
  // level of the word.
  int masked_levels = kLevelsPerWord;
  if (c.prev_tree_depth > 0) {
    const int need = c.prev_tree_depth + 1 < kLevelsPerWord ? c.prev_tree_depth + 1 : kLevelsPerWord;
    const int zero_digits = (3 * kLevelsPerWord - 3 * need) / 8;  // whole 8-bit digits below the kept levels
    masked_levels = (3 * kLevelsPerWord - 8 * zero_digits) / 3;
  }
  for (;; ++words) {
    if (words > kMaxPathWords) {
      c.last_error = "Tree gravity maximum depth contract exceeded";
      return CHUI_TREEPM_ERANGE;
    }
    // bucket_max is the sorted-key scratch here; the periodic unwrap sizes it
    // as well, but isolated/open boundaries skip the unwrap
    if (ensure(c.path_words, static_cast<size_t>(words) * n * 8) ||
        ensure(c.keys_a, static_cast<size_t>(words) * n * 8) || ensure(c.bucket_max, static_cast<size_t>(n) * 8))
      return CHUI_TREEPM_ENOMEM;
    path = c.path_words.as<unsigned long long>();
    unsigned long long* by_row = c.keys_a.as<unsigned long long>();
    unsigned long long* key_cur = c.keys_b.as<unsigned long long>();
    unsigned long long* key_sorted = c.bucket_max.as<unsigned long long>();
    const bool masked = words == 1 && masked_levels < kLevelsPerWord;
    const int levels = masked ? masked_levels : kLevelsPerWord * words;
    const unsigned long long mask0 = masked ? ~((1ull << (3 * (kLevelsPerWord - masked_levels))) - 1ull) : ~0ull;
    { noteLaunch(); pathKernel<<<gridFor(n, 256), 256, 0, s>>>(n, words, nullptr, u[0], u[1], u[2], cx0, cy0, cz0, half0,
                                               mask0, by_row); }
    uint32_t* rank_in = c.idx_c.as<uint32_t>();
    uint32_t* rank_out = c.idx_d.as<uint32_t>();
    { noteLaunch(); iotaKernel<<<gridFor(n, 256), 256, 0, s>>>(n, rank_in); }
    // LSD over path words, each pass a stable sort; the first pass reads the
    // words in row order and the last writes the sorted first word in place
    for (int w = words - 1; w >= 0; --w) {
      const unsigned long long* key_in = by_row + static_cast<size_t>(w) * n;
      if (w != words - 1) {
        noteLaunch();
        gatherU64Kernel<<<gridFor(n, 256), 256, 0, s>>>(n, key_in, rank_in, key_cur);
        key_in = key_cur;
      }
      rc = radixSortPairsU64(c, key_in, w == 0 ? path : key_sorted, rank_in, rank_out, n, 63, s);
      if (rc) return rc;
      uint32_t* t = rank_in;
      rank_in = rank_out;
      rank_out = t;
    }
    // rank_in: path position -> row
    row_of_pos = rank_in;
    for (int w = 1; w < words; ++w)
      { noteLaunch(); gatherU64Kernel<<<gridFor(n, 256), 256, 0, s>>>(n, by_row + static_cast<size_t>(w) * n, rank_in,
                                                      path + static_cast<size_t>(w) * n); }
    { noteLaunch(); commonPrefixKernel<<<gridFor(n, 256), 256, 0, s>>>(n, words, levels, path, cp); }
    plan.depth_max = levels;
    cudaMemsetAsync(status, 0, 4, s);
    { noteLaunch(); nodeCountKernel<<<gridFor(n + 1, 256), 256, 0, s>>>(plan, cp, counts, status); }
    if ((rc = exclusiveScanU32(c, counts, offset, n + 1, s))) return rc;
    uint32_t hs[2];
    cudaMemcpyAsync(&hs[0], status, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hs[1], offset + n, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      c.last_error = "tree node enumeration failed";
      return CHUI_TREEPM_EDEVICE;
    }
    if (hs[0] & kStatusNeedMorePathWords) {
      if (masked) {
        masked_levels = kLevelsPerWord;  // the same word count with every level
        c.path_levels_retried = 1;
        --words;
      }
      continue;
    }
    if (hs[0] & kStatusDepthExceeded) {
      c.last_error = "Tree gravity maximum depth contract exceeded";
      return CHUI_TREEPM_ERANGE;
    }
    total_nodes = hs[1];
    break;
  }
  c.path_words_used = words;
  c.n_nodes = total_nodes;
  if (ensure(c.node_geom, total_nodes * sizeof(double4)) || ensure(c.node_com, total_nodes * sizeof(double4)) ||
      ensure(c.node_quad, total_nodes * 8 * sizeof(double)) || ensure(c.node_child, total_nodes * 8 * 4) ||
      ensure(c.node_range, total_nodes * sizeof(uint4)) || ensure(c.node_parent, total_nodes * 4) ||
      ensure(c.node_depth, total_nodes * 4) || ensure(c.node_counter, total_nodes * 4))
    return CHUI_TREEPM_ENOMEM;
  NodeOut out;
  out.geom = c.node_geom.as<double4>();
  out.range = c.node_range.as<uint4>();
  out.parent = c.node_parent.as<uint32_t>();
  out.depth = c.node_depth.as<uint32_t>();
  out.child = c.node_child.as<uint32_t>();
  out.leaf_of_pos = c.leaf_of_pos.as<uint32_t>();
  cudaMemsetAsync(out.leaf_of_pos, 0, n * 4, s);
  cudaMemsetAsync(out.child, 0xFF, static_cast<size_t>(total_nodes) * 8 * 4, s);  // all slots empty
  cudaMemsetAsync(status, 0, 4, s);
  bool large_leaf = false;
  // block minima of the common-prefix lengths for the run queries
  CpLevels lv{};
  {
    size_t total = 0;
    int64_t len = n;
    lv.lv[0] = cp;
    lv.len[0] = n;
    lv.count = 1;
    while (len > 32 && lv.count < kCpLevels) {
      len = (len + 31) / 32;
      lv.len[lv.count++] = len;
      total += static_cast<size_t>(len);
    }
    if (ensure(c.cp_levels, (total + 1) * sizeof(int))) return CHUI_TREEPM_ENOMEM;
    int* dst = c.cp_levels.as<int>();
    for (int l = 1; l < lv.count; ++l) {
      noteLaunch();
      cpBlockMinKernel<<<gridFor(lv.len[l - 1], 256), 256, 0, s>>>(lv.len[l - 1], lv.lv[l - 1], dst);
      lv.lv[l] = dst;
      dst += lv.len[l];
    }
  }
  // the chain starts, listed (at most one per node)
  if (ensure(c.idx_a, (n + 1) * 4) || ensure(c.idx_b, (n + 1) * 4) || ensure(c.inv_pos, n * 4))
    return CHUI_TREEPM_ENOMEM;
  uint32_t* chain_flag = c.idx_b.as<uint32_t>();
  uint32_t* chain_off = c.idx_a.as<uint32_t>();
  uint32_t* chain_start = c.inv_pos.as<uint32_t>();
  { noteLaunch(); chainFlagsKernel<<<gridFor(n + 1, 256), 256, 0, s>>>(n, counts, chain_flag); }
  if ((rc = exclusiveScanU32(c, chain_flag, chain_off, n + 1, s))) return rc;
  { noteLaunch(); chainListKernel<<<gridFor(n, 256), 256, 0, s>>>(n, counts, chain_off, chain_start); }
  { noteLaunch(); nodeEmitKernel<<<gridFor(total_nodes, 128), 128, 0, s>>>(plan, words, path, cp, counts, offset,
                                                 chain_start, chain_off + n, lv, cx0, cy0, cz0, half0, total_nodes,
                                                 out, status); }
  {
    uint32_t est = 0;
    cudaMemcpyAsync(&est, status, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
    if (est & ~static_cast<uint32_t>(kStatusLargeLeaf)) {
      c.last_error = "tree node enumeration produced an inconsistent node range";
      return CHUI_TREEPM_EDEVICE;
    }
    large_leaf = (est & kStatusLargeLeaf) != 0;
    c.large_leaf = large_leaf ? 1 : 0;
  }
  { noteLaunch(); childCountKernel<<<gridFor(total_nodes, 256), 256, 0, s>>>(total_nodes, out.child, out.range); }
  // final order: each leaf's particles in Morton order
  if (!large_leaf) {
    unsigned long long* key_of_pos = c.keys_b.as<unsigned long long>();
    { noteLaunch(); gatherU64Kernel<<<gridFor(n, 256), 256, 0, s>>>(n, morton, row_of_pos, key_of_pos); }
    { noteLaunch(); leafOrderKernel<<<gridFor(n, 256), 256, 0, s>>>(n, out.leaf_of_pos, out.range, row_of_pos, key_of_pos,
                                                    c.sorted_index.as<uint32_t>(), status); }
  } else {
    // a leaf above the in-place limit (particles at the depth limit): the
    // stable Morton sort, then a stable sort of that order by leaf
    { noteLaunch(); iotaKernel<<<gridFor(n, 256), 256, 0, s>>>(n, c.idx_a.as<uint32_t>()); }
    rc = radixSortPairsU64(c, morton, c.keys_b.as<unsigned long long>(), c.idx_a.as<uint32_t>(),
                           c.idx_b.as<uint32_t>(), n, 63, s);
    if (rc) return rc;
    const uint32_t* perm_m = c.idx_b.as<uint32_t>();
    { noteLaunch(); invertKernel<<<gridFor(n, 256), 256, 0, s>>>(n, row_of_pos, c.inv_pos.as<uint32_t>()); }
    uint32_t* leaf_key = c.idx_a.as<uint32_t>();
    { noteLaunch(); leafKeyKernel<<<gridFor(n, 256), 256, 0, s>>>(n, perm_m, c.inv_pos.as<uint32_t>(), out.leaf_of_pos,
                                                  leaf_key); }
    // row_of_pos may share idx_d with the sort's key output: it is not read again
    rc = radixSortPairsU32(c, leaf_key, c.idx_d.as<uint32_t>(), perm_m, c.sorted_index.as<uint32_t>(), n,
                           bitsFor(total_nodes), s);
    if (rc) return rc;
  }
  // tree-ordered source records
  const bool mixed = c.cfg.precision == CHUI_TREEPM_MIXED;
  if (mixed) {
    if (ensure(c.src_f4, n * sizeof(float4))) return CHUI_TREEPM_ENOMEM;
  }
  if (ensure(c.src_d4, n * sizeof(double4))) return CHUI_TREEPM_ENOMEM;
  if (ensure(c.src_u4, n * sizeof(double4))) return CHUI_TREEPM_ENOMEM;
  if (c.soft_rows && (ensure(c.src_eps, n * sizeof(double)) || ensure(c.node_soft, total_nodes * sizeof(double2))))
    return CHUI_TREEPM_ENOMEM;
  // tree position of each row, then the records scattered from row order
  { noteLaunch(); invertKernel<<<gridFor(n, 256), 256, 0, s>>>(n, c.sorted_index.as<uint32_t>(), c.pos_of_row.as<uint32_t>()); }
  { noteLaunch(); scatterSourcesKernel<<<gridFor(n, 256), 256, 0, s>>>(n, c.pos_of_row.as<uint32_t>(), x, y, z, u[0], u[1],
                                                       u[2], m, uniform_mass, c.src_d4.as<double4>(),
                                                       c.src_u4.as<double4>(), c.soft_rows,
                                                       c.soft_rows ? c.src_eps.as<double>() : nullptr); }
  if (mixed)
    { noteLaunch(); leafOffsetsKernel<<<gridFor(n, 256), 256, 0, s>>>(n, out.leaf_of_pos, out.geom, c.src_u4.as<double4>(),
                                                      c.src_f4.as<float4>()); }
  // moments (leaves read the tree-ordered records written above)
  cudaMemsetAsync(c.node_counter.ptr, 0, total_nodes * 4, s);
  MomentIn mi;
  mi.u4 = c.src_u4.as<double4>();
  mi.quadrupole = c.cfg.multipole_order == 2 ? 1 : 0;
  mi.eps = c.soft_rows ? c.src_eps.as<double>() : nullptr;
  mi.soft = c.soft_rows ? c.node_soft.as<double2>() : nullptr;
  { noteLaunch(); momentsKernel<<<gridFor(total_nodes, 128), 128, 0, s>>>(total_nodes, mi, out.geom, out.range, out.parent,
                                                          out.child, c.node_counter.as<uint32_t>(),
                                                          c.node_com.as<double4>(), c.node_quad.as<double>()); }
  if (ensure(c.node_f4, total_nodes * sizeof(float4)) || ensure(c.node_mq, total_nodes * 2 * sizeof(float4)))
    return CHUI_TREEPM_ENOMEM;
  { noteLaunch(); nodeFrameKernel<<<gridFor(total_nodes, 256), 256, 0, s>>>(total_nodes, out.geom, c.node_com.as<double4>(),
                                                            c.node_quad.as<double>(), c.node_f4.as<float4>(),
                                                            c.node_mq.as<float4>()); }
  // maximum depth (for stack sizing and stats); the status of the
  // within-leaf ordering is read at the same synchronisation
  {
    uint32_t hd = 0, est = 0;
    cudaMemcpyAsync(&est, status, 4, cudaMemcpyDeviceToHost, s);
    if (maxU32(c, out.depth, total_nodes, &hd, s)) {
      c.last_error = "tree build kernels failed";
      return CHUI_TREEPM_EDEVICE;
    }
    if (est & ~static_cast<uint32_t>(kStatusLargeLeaf)) {
      c.last_error = "tree leaf ordering produced an inconsistent index";
      return CHUI_TREEPM_EDEVICE;
    }
    c.max_depth = hd;
    c.prev_tree_depth = static_cast<int>(hd);
  }
  c.tree_anchor[0] = anchors[0];
  c.tree_anchor[1] = anchors[1];
  c.tree_anchor[2] = anchors[2];
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

int treeNodeBounds(Context& c, double lo[3], double hi[3], cudaStream_t s) {
  auto* sc = c.scalars.as<unsigned long long>();
  unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
  cudaMemcpyAsync(sc, init, sizeof(init), cudaMemcpyHostToDevice, s);
  if (c.n_nodes > 0)
    { noteLaunch(); nodeBoundsKernel<<<std::min(gridFor(c.n_nodes, 256), kReduceBlocks), 256, 0, s>>>(c.n_nodes, c.node_geom.as<double4>(),
                                                              c.node_com.as<double4>(), sc); }
  unsigned long long hb[6];
  cudaMemcpyAsync(hb, sc, sizeof(hb), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  for (int a = 0; a < 3; ++a) {
    lo[a] = c.n_nodes > 0 ? fromOrderedBits(hb[a]) : INFINITY;
    hi[a] = c.n_nodes > 0 ? fromOrderedBits(hb[3 + a]) : -INFINITY;
  }
  return 0;
}

// Visit order: active slots sorted by the tree position of their row
// (tree_pm_coupling.cpp:3808-3838); slots without a local source go last.
int treeOrderTargets(Context& c, int64_t nt, const uint32_t* active, int explicit_targets, int64_t n,
                     cudaStream_t s) {
  if (nt == 0) return 0;
  if (ensure(c.target_order, nt * 4) || ensure(c.idx_a, std::max<int64_t>(nt, n) * 4) ||
      ensure(c.idx_c, (std::max<int64_t>(nt, n) + 1) * 4) || ensure(c.idx_d, (std::max<int64_t>(nt, n) + 1) * 4))
    return CHUI_TREEPM_ENOMEM;
  if (!active && !explicit_targets && nt == n) {
    // every source is a target: the visit order is the tree order itself
    cudaMemcpyAsync(c.target_order.ptr, c.sorted_index.ptr, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToDevice, s);
    return 0;
  }
  uint32_t* key = c.idx_c.as<uint32_t>();
  uint32_t* slot = c.idx_a.as<uint32_t>();
  { noteLaunch(); targetKeyKernel<<<gridFor(nt, 256), 256, 0, s>>>(nt, active, n, c.pos_of_row.as<uint32_t>(), explicit_targets,
                                                   key, slot); }
  return radixSortPairsU32(c, key, c.idx_d.as<uint32_t>(), slot, c.target_order.as<uint32_t>(), nt, 32, s);
}

}  // namespace chui
