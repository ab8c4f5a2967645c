// Stable LSD radix sort, exclusive scan and maximum for the tree build.
//
// The reference orders particles with a stable least-significant-digit radix
// sort of 8-bit digits (radixSortMortonOrdering, tree_ordering.cpp:13-71; the
// unwrap's radixSortNonNegativeDoubleBits, tree_pm_coupling.cpp:94-140). Any
// stable sort by the full key yields the same order, which is what the tree
// needs bit for bit; this one is built for the B200:
//
//  - one pass over the keys counts all eight digits at once, and digits that
//    are equal for every key are skipped (a pass over them keeps the order);
//  - each remaining pass is three launches with no waiting between blocks:
//    upsweep (per-tile digit counts), a per-digit exclusive scan over tiles,
//    and a downsweep that ranks each tile stably and writes it out;
//  - the downsweep ranks 32 consecutive keys at a time per warp with
//    __match_any_sync (lanes of a digit are ranked by lane order, rounds in
//    key order, warps in tile order), places the tile in shared memory sorted
//    by digit, and writes each digit's run to consecutive addresses.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "context.cuh"

namespace chui {
namespace {

// grid-stride launches: up to 64 blocks per SM of the 148
inline unsigned gridFor(size_t n, int block) {
  size_t b = (n + block - 1) / block;
  if (b > 148u * 64u) b = 148u * 64u;
  return static_cast<unsigned>(b ? b : 1);
}

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
#ifndef CHUI_SORT_ITEMS
#define CHUI_SORT_ITEMS 16  // keys per thread of a tile
#endif
#ifndef CHUI_SORT_MIN_BLOCKS
#define CHUI_SORT_MIN_BLOCKS 0  // resident downsweep blocks per SM to size registers for (0: the compiler's choice)
#endif
#if CHUI_SORT_MIN_BLOCKS > 0
#define CHUI_SORT_BOUNDS __launch_bounds__(kSortThreads, CHUI_SORT_MIN_BLOCKS)
#else
#define CHUI_SORT_BOUNDS __launch_bounds__(kSortThreads)
#endif
constexpr int kItemsPerThread = CHUI_SORT_ITEMS;
constexpr int kTile = kSortThreads * kItemsPerThread;  // 4096 keys per tile
constexpr int kWarpItems = kTile / kSortWarps;          // 512 consecutive keys per warp
constexpr int kRounds = kWarpItems / 32;                // 16 rounds of 32
constexpr int kMaxBatch = 3;                            // independent sorts per launch (blockIdx.y)

// Up to kMaxBatch sorts of n keys each, one per blockIdx.y (the periodic
// unwrap sorts its three axes together).
struct SortJob {
  const void* kin[kMaxBatch];
  void* kout[kMaxBatch];
  const uint32_t* vin[kMaxBatch];
  uint32_t* vout[kMaxBatch];
};

// One of a job's pointers by blockIdx.y with constant indices (a dynamic index
// into the kernel's parameter block would copy it to local memory).
template <class T>
__device__ __forceinline__ T pick(const T (&p)[kMaxBatch], int y) {
  return y == 0 ? p[0] : (y == 1 ? p[1] : p[2]);
}

template <class K>
__device__ __forceinline__ uint32_t digitOf(K key, int shift) {
  return static_cast<uint32_t>(key >> shift) & 0xFFu;
}

// All digit histograms of every sort's keys in one pass: hist[(y * 8 + d) * 256 + v].
template <class K>
__global__ void __launch_bounds__(kSortThreads) digitHistogramKernel(int64_t n, SortJob job, int digits,
                                                                   uint32_t* hist) {
  __shared__ uint32_t h[8][256];
  const K* __restrict__ keys = static_cast<const K*>(pick(job.kin, blockIdx.y));
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0u;
  __syncthreads();
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const K k = keys[i];
    for (int d = 0; d < digits; ++d) atomicAdd(&h[d][digitOf(k, 8 * d)], 1u);
  }
  __syncthreads();
  uint32_t* out = hist + static_cast<size_t>(blockIdx.y) * 8 * 256;
  for (int i = threadIdx.x; i < digits * 256; i += blockDim.x) {
    const uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(out + i, v);
  }
}

// Per-tile counts of one digit: counts[(y * 256 + v) * tiles + tile].
template <class K>
__global__ void __launch_bounds__(kSortThreads) upsweepKernel(int64_t n, SortJob job, int shift, int64_t tiles,
                                                            uint32_t* counts) {
  __shared__ uint32_t h[256];
  const K* __restrict__ keys = static_cast<const K*>(pick(job.kin, blockIdx.y));
  h[threadIdx.x] = 0u;
  __syncthreads();
  const int64_t base = blockIdx.x * static_cast<int64_t>(kTile);
  for (int i = threadIdx.x; i < kTile; i += kSortThreads) {
    const int64_t k = base + i;
    if (k < n) atomicAdd(&h[digitOf(keys[k], shift)], 1u);
  }
  __syncthreads();
  counts[(static_cast<int64_t>(blockIdx.y) * 256 + threadIdx.x) * tiles + blockIdx.x] = h[threadIdx.x];
}

// Block-wide exclusive scan of one value per thread (256 threads); returns
// the exclusive prefix and writes the total to *total.
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* warp_sums, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < kSortWarps ? warp_sums[lane] : 0u;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, off);
      if (lane >= off) s += y;
    }
    if (lane < kSortWarps) warp_sums[lane] = s;  // inclusive warp totals
  }
  __syncthreads();
  const uint32_t before = warp == 0 ? 0u : warp_sums[warp - 1];
  *total = warp_sums[kSortWarps - 1];
  __syncthreads();
  return before + x - v;
}

// For each digit of each sort (block (v, y)): exclusive prefix over tiles in
// place and the digit's total. The row is staged through shared memory in
// coalesced chunks of kScanRow; each thread scans a run of consecutive
// entries there.
constexpr int kScanRow = 4096;
__global__ void __launch_bounds__(kSortThreads) tileScanKernel(int64_t tiles, uint32_t* counts, uint32_t* totals) {
  __shared__ uint32_t warp_sums[kSortWarps];
  __shared__ uint32_t row_sm[kScanRow + kScanRow / 32];  // one pad word per 32: no bank conflicts
  const int64_t row = static_cast<int64_t>(blockIdx.y) * 256 + blockIdx.x;
  uint32_t* c = counts + row * tiles;
  constexpr int kPer = kScanRow / kSortThreads;  // 16 entries per thread
  uint32_t carry = 0u;
  for (int64_t b = 0; b < tiles; b += kScanRow) {
    const int len = tiles - b < kScanRow ? static_cast<int>(tiles - b) : kScanRow;
    for (int i = threadIdx.x; i < kScanRow; i += kSortThreads) row_sm[i + i / 32] = i < len ? c[b + i] : 0u;
    __syncthreads();
    uint32_t sum = 0u;
    for (int i = 0; i < kPer; ++i) {
      const int q = threadIdx.x * kPer + i;
      sum += row_sm[q + q / 32];
    }
    uint32_t total;
    uint32_t run = carry + blockExclusiveScan(sum, warp_sums, &total);
    for (int i = 0; i < kPer; ++i) {
      const int q = threadIdx.x * kPer + i;
      const uint32_t v = row_sm[q + q / 32];
      row_sm[q + q / 32] = run;
      run += v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < len; i += kSortThreads) c[b + i] = row_sm[i + i / 32];
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[row] = carry;
}

// Dynamic shared memory of the downsweep: the staged tile (keys, values).
template <class K, bool kValues>
constexpr size_t downsweepSmem() {
  return static_cast<size_t>(kTile) * sizeof(K) + (kValues ? static_cast<size_t>(kTile) * sizeof(uint32_t) : 0);
}

// Rank, stage and scatter one tile for one digit.
template <class K, bool kValues>
__global__ void CHUI_SORT_BOUNDS downsweepKernel(int64_t n, SortJob job, SortJob dst, int shift,
                                                              int64_t tiles, const uint32_t* __restrict__ counts,
                                                              const uint32_t* __restrict__ totals) {
  __shared__ uint32_t wcount[kSortWarps][256];  // per-warp digit counts, then prefixes
  __shared__ uint32_t tile_start[256];           // digit start within the tile
  __shared__ uint32_t gbase[256];                // digit start in the output for this tile
  __shared__ uint32_t warp_sums[kSortWarps];
  extern __shared__ __align__(16) unsigned char stage[];
  K* skeys = reinterpret_cast<K*>(stage);
  uint32_t* svals = reinterpret_cast<uint32_t*>(stage + static_cast<size_t>(kTile) * sizeof(K));
  const int y = blockIdx.y;
  const K* __restrict__ kin = static_cast<const K*>(pick(job.kin, y));
  K* __restrict__ kout = static_cast<K*>(pick(dst.kout, y));
  const uint32_t* __restrict__ vin = kValues ? pick(job.vin, y) : nullptr;
  uint32_t* __restrict__ vout = kValues ? pick(dst.vout, y) : nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int w = 0; w < kSortWarps; ++w) wcount[w][threadIdx.x] = 0u;
  // the digit's output start: all smaller digits' totals plus this tile's prefix
  {
    uint32_t all;
    const int64_t row = static_cast<int64_t>(y) * 256 + threadIdx.x;
    const uint32_t before = blockExclusiveScan(totals[row], warp_sums, &all);
    gbase[threadIdx.x] = before + counts[row * tiles + blockIdx.x];
  }
  __syncthreads();
  const int64_t base = blockIdx.x * static_cast<int64_t>(kTile) + warp * kWarpItems;
  K key[kRounds];
  uint32_t val[kRounds], rank[kRounds];
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    const int64_t i = base + r * 32 + lane;
    key[r] = i < n ? kin[i] : K(0);
    if constexpr (kValues) val[r] = i < n ? vin[i] : 0u;
  }
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    const bool ok = base + r * 32 + lane < n;
    const uint32_t d = ok ? digitOf(key[r], shift) : 256u;  // out-of-range lanes form their own group
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t before = __popc(peers & ((1u << lane) - 1u));
    const uint32_t cur = ok ? wcount[warp][d] : 0u;
    __syncwarp();
    if (ok) {
      rank[r] = cur + before;
      if (before == 0) wcount[warp][d] = cur + __popc(peers);  // the group's first lane advances the count
    }
    __syncwarp();
  }
  __syncthreads();
  // per digit: warps' prefixes (warp order is key order) and the digit's tile total
  {
    const int d = threadIdx.x;
    uint32_t run = 0u;
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = wcount[w][d];
      wcount[w][d] = run;
      run += c;
    }
    uint32_t all;
    tile_start[d] = blockExclusiveScan(run, warp_sums, &all);
  }
  __syncthreads();
  // stage the tile sorted by digit
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    if (base + r * 32 + lane < n) {
      const uint32_t d = digitOf(key[r], shift);
      const uint32_t t = tile_start[d] + wcount[warp][d] + rank[r];
      if (t < static_cast<uint32_t>(kTile)) {  // always true; a guard on the computed index
        skeys[t] = key[r];
        if constexpr (kValues) svals[t] = val[r];
      }
    }
  }
  __syncthreads();
  // consecutive staged keys of one digit go to consecutive output addresses
  const int64_t tile_n = n - blockIdx.x * static_cast<int64_t>(kTile);
  const int count = tile_n < kTile ? static_cast<int>(tile_n) : kTile;
  for (int t = threadIdx.x; t < count; t += kSortThreads) {
    const K k = skeys[t];
    const uint32_t d = digitOf(k, shift);
    const int64_t o = static_cast<int64_t>(gbase[d]) + (t - static_cast<int64_t>(tile_start[d]));
    if (o >= 0 && o < n) {  // always true; a guard on the computed index
      kout[o] = k;
      if constexpr (kValues) vout[o] = svals[t];
    }
  }
}

// batch sorts of n keys each; every sort takes the passes of the digits that
// vary in any of them (a pass over a constant digit keeps the order)
template <class K>
int radixSortBatch(Context& c, int batch, const K* const* kin, K* const* kout, const uint32_t* const* vin,
                   uint32_t* const* vout, int64_t n, int end_bit, cudaStream_t s) {
  if (n <= 0) return 0;
  if (n > 0xFFFFFFFFll || batch < 1 || batch > kMaxBatch) return CHUI_TREEPM_ERANGE;
  const int digits = (end_bit + 7) / 8;
  const int64_t tiles = (n + kTile - 1) / kTile;
  const bool values = vin != nullptr;
  if (ensure(c.sort_hist, kMaxBatch * 8 * 256 * sizeof(uint32_t)) ||
      ensure(c.sort_counts, static_cast<size_t>(batch) * 256 * tiles * sizeof(uint32_t)) ||
      ensure(c.sort_totals, kMaxBatch * 256 * sizeof(uint32_t)) ||
      ensure(c.sort_keys, static_cast<size_t>(batch) * n * sizeof(K)) ||
      (values && ensure(c.sort_vals, static_cast<size_t>(batch) * n * sizeof(uint32_t))))
    return CHUI_TREEPM_ENOMEM;
  SortJob src{}, out{}, tmp{};
  for (int y = 0; y < batch; ++y) {
    src.kin[y] = kin[y];
    out.kout[y] = kout[y];
    tmp.kout[y] = c.sort_keys.as<K>() + static_cast<size_t>(y) * n;
    if (values) {
      src.vin[y] = vin[y];
      out.vout[y] = vout[y];
      tmp.vout[y] = c.sort_vals.as<uint32_t>() + static_cast<size_t>(y) * n;
    }
  }
  // which digits vary
  uint32_t* hist = c.sort_hist.as<uint32_t>();
  cudaMemsetAsync(hist, 0, kMaxBatch * 8 * 256 * sizeof(uint32_t), s);
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (n + kSortThreads - 1) / kSortThreads;
    const unsigned blocks = static_cast<unsigned>(want < 4 * sms ? want : 4 * sms);
    noteLaunch();
    digitHistogramKernel<K><<<dim3(blocks, batch), kSortThreads, 0, s>>>(n, src, digits, hist);
  }
  std::vector<uint32_t> h(static_cast<size_t>(batch) * 8 * 256);
  cudaMemcpyAsync(h.data(), hist, h.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  std::vector<int> shifts;
  for (int d = 0; d < digits; ++d) {
    bool varies = false;
    for (int y = 0; y < batch; ++y) {
      bool constant = false;
      for (int v = 0; v < 256; ++v)
        if (h[(static_cast<size_t>(y) * 8 + d) * 256 + v] == static_cast<uint32_t>(n)) constant = true;
      varies = varies || !constant;
    }
    if (varies) shifts.push_back(8 * d);
  }
  const int passes = static_cast<int>(shifts.size());
  if (passes == 0) {
    for (int y = 0; y < batch; ++y) {
      cudaMemcpyAsync(kout[y], kin[y], n * sizeof(K), cudaMemcpyDeviceToDevice, s);
      if (values) cudaMemcpyAsync(vout[y], vin[y], n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
  }
  const size_t smem = values ? downsweepSmem<K, true>() : downsweepSmem<K, false>();
  if (values) cudaFuncSetAttribute(downsweepKernel<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  else cudaFuncSetAttribute(downsweepKernel<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  uint32_t* counts = c.sort_counts.as<uint32_t>();
  uint32_t* totals = c.sort_totals.as<uint32_t>();
  const dim3 grid(static_cast<unsigned>(tiles), batch);
  SortJob cur = src;
  for (int p = 0; p < passes; ++p) {
    // ping-pong so that the last pass writes the output
    const SortJob& dst = ((passes - 1 - p) % 2) == 0 ? out : tmp;
    const int shift = shifts[p];
    { noteLaunch(); upsweepKernel<K><<<grid, kSortThreads, 0, s>>>(n, cur, shift, tiles, counts); }
    { noteLaunch(); tileScanKernel<<<dim3(256, batch), kSortThreads, 0, s>>>(tiles, counts, totals); }
    noteLaunch();
    if (values) downsweepKernel<K, true><<<grid, kSortThreads, smem, s>>>(n, cur, dst, shift, tiles, counts, totals);
    else downsweepKernel<K, false><<<grid, kSortThreads, smem, s>>>(n, cur, dst, shift, tiles, counts, totals);
    // the next pass reads what this one wrote
    for (int y = 0; y < batch; ++y) {
      cur.kin[y] = dst.kout[y];
      cur.vin[y] = values ? dst.vout[y] : nullptr;
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

// ---- exclusive scan of uint32 counts (the node emission plan) --------------

constexpr int kScanItems = 8;
constexpr int kScanTile = kSortThreads * kScanItems;

// Per tile: exclusive scan in place and the tile's sum.
__global__ void __launch_bounds__(kSortThreads) scanTilesKernel(int64_t n, const uint32_t* __restrict__ in,
                                                              uint32_t* out, uint32_t* tile_sums) {
  __shared__ uint32_t warp_sums[kSortWarps];
  const int64_t base = blockIdx.x * static_cast<int64_t>(kScanTile) + threadIdx.x * kScanItems;
  uint32_t v[kScanItems], sum = 0u;
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0u;
    sum += v[k];
  }
  uint32_t total;
  uint32_t run = blockExclusiveScan(sum, warp_sums, &total);
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums in place.
__global__ void __launch_bounds__(kSortThreads) scanSumsKernel(int64_t tiles, uint32_t* sums) {
  __shared__ uint32_t warp_sums[kSortWarps];
  uint32_t carry = 0u;
  for (int64_t b = 0; b < tiles; b += kSortThreads) {
    const int64_t i = b + threadIdx.x;
    const uint32_t v = i < tiles ? sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = blockExclusiveScan(v, warp_sums, &total);
    if (i < tiles) sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void scanAddKernel(int64_t n, uint32_t* out, const uint32_t* __restrict__ tile_sums) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] += tile_sums[i / kScanTile];
}

__global__ void maxKernel(int64_t n, const uint32_t* __restrict__ in, uint32_t* out) {
  uint32_t m = 0u;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    m = max(m, in[i]);
  for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace

int radixSortPairsU64(Context& c, const unsigned long long* kin, unsigned long long* kout, const uint32_t* vin,
                      uint32_t* vout, int64_t n, int end_bit, cudaStream_t s) {
  return radixSortBatch<unsigned long long>(c, 1, &kin, &kout, &vin, &vout, n, end_bit, s);
}

int radixSortKeysU64(Context& c, int batch, const unsigned long long* const* kin, unsigned long long* const* kout,
                     int64_t n, int end_bit, cudaStream_t s) {
  return radixSortBatch<unsigned long long>(c, batch, kin, kout, nullptr, nullptr, n, end_bit, s);
}

int radixSortPairsU32(Context& c, const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout,
                      int64_t n, int end_bit, cudaStream_t s) {
  return radixSortBatch<uint32_t>(c, 1, &kin, &kout, &vin, &vout, n, end_bit, s);
}

int exclusiveScanU32(Context& c, const uint32_t* in, uint32_t* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return 0;
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (ensure(c.sort_totals, (tiles > 256 ? tiles : 256) * sizeof(uint32_t))) return CHUI_TREEPM_ENOMEM;
  uint32_t* sums = c.sort_totals.as<uint32_t>();
  { noteLaunch(); scanTilesKernel<<<static_cast<unsigned>(tiles), kSortThreads, 0, s>>>(n, in, out, sums); }
  { noteLaunch(); scanSumsKernel<<<1, kSortThreads, 0, s>>>(tiles, sums); }
  { noteLaunch(); scanAddKernel<<<gridFor(n, 256), 256, 0, s>>>(n, out, sums); }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

int maxU32(Context& c, const uint32_t* in, int64_t n, uint32_t* result, cudaStream_t s) {
  *result = 0u;
  if (n <= 0) return 0;
  uint32_t* d = reinterpret_cast<uint32_t*>(c.scalars.as<unsigned long long>() + 14);
  cudaMemsetAsync(d, 0, 4, s);
  { noteLaunch(); maxKernel<<<std::min(gridFor(n, 256), kReduceBlocks), 256, 0, s>>>(n, in, d); }
  cudaMemcpyAsync(result, d, 4, cudaMemcpyDeviceToHost, s);
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

}  // namespace chui
