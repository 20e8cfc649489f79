// Report compaction: LSD radix sort of 64-bit report keys (offset << 32 | id)
// followed by duplicate removal and conversion to the reference's packed form
// (id << 32 | offset). Replaces the host sort/unique of the reference
// (code/src/ngap/ngap.cu:1890-1932, order of compareResult ngap.cu:19-30).
//
// Each pass sorts one 4-bit digit: per-tile digit histograms, one exclusive
// scan over the digit-major histogram table, then a stable scatter in which
// each thread owns kSortItems consecutive keys of the tile. Digits that are
// constant over all keys (bits above the largest offset and id) are skipped
// by the host. The key count is read from device memory (*d_n, clamped to
// cap), so the whole pipeline runs without a host round trip; grids stride
// over tiles.
#pragma once

#include <cstdint>

namespace ngap {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
constexpr int kScanThreads = 1024;

__device__ __forceinline__ uint64_t dev_count(const unsigned long long* d_n, uint64_t cap) {
  uint64_t n = *d_n;
  return n < cap ? n : cap;
}

__device__ __forceinline__ uint32_t num_tiles(uint64_t n) {
  return (uint32_t)((n + kSortTile - 1) / kSortTile);
}

// hist[d * ntiles + tile] = number of keys of the tile whose digit is d.
__global__ void __launch_bounds__(kSortThreads) radix_hist(const uint64_t* __restrict__ keys,
                                                           const unsigned long long* d_n,
                                                           uint64_t cap, int shift,
                                                           uint32_t* __restrict__ hist) {
  __shared__ uint32_t cnt[16];
  const uint64_t n = dev_count(d_n, cap);
  const uint32_t ntiles = num_tiles(n);
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (threadIdx.x < 16) cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)tile * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
      uint64_t g = base + (uint64_t)i;
      if (g < n) atomicAdd(&cnt[(keys[g] >> shift) & 15u], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 16) hist[(uint64_t)threadIdx.x * ntiles + tile] = cnt[threadIdx.x];
    __syncthreads();
  }
}

// In-place exclusive scan of a[0 .. mult * ntiles(*d_n)) with one block.
// Writes the total to *total when non-null.
__global__ void __launch_bounds__(kScanThreads) scan_exclusive_1block(uint32_t* a,
                                                                      const unsigned long long* d_n,
                                                                      uint64_t cap, uint32_t mult,
                                                                      unsigned long long* total) {
  __shared__ uint32_t part[kScanThreads];
  const uint32_t n = mult * num_tiles(dev_count(d_n, cap));
  const uint32_t per = (n + kScanThreads - 1) / kScanThreads;
  const uint32_t b = min(threadIdx.x * per, n), e = min(b + per, n);
  uint32_t s = 0;
  for (uint32_t i = b; i < e; i++) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {  // Hillis-Steele inclusive scan
    uint32_t y = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0u;
    __syncthreads();
    part[threadIdx.x] += y;
    __syncthreads();
  }
  uint32_t run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0u;
  for (uint32_t i = b; i < e; i++) {
    uint32_t x = a[i];
    a[i] = run;
    run += x;
  }
  if (total && n > 0 && threadIdx.x == kScanThreads - 1) *total = part[kScanThreads - 1];
}

// Stable scatter of one digit pass. offs = scanned hist (digit-major).
__global__ void __launch_bounds__(kSortThreads) radix_scatter(const uint64_t* __restrict__ in,
                                                              uint64_t* __restrict__ out,
                                                              const unsigned long long* d_n,
                                                              uint64_t cap, int shift,
                                                              const uint32_t* __restrict__ offs) {
  __shared__ uint64_t tile_keys[kSortTile];
  __shared__ uint32_t cnt[16][kSortThreads];
  const uint64_t n = dev_count(d_n, cap);
  const uint32_t ntiles = num_tiles(n);
  const int t = threadIdx.x;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t base = (uint64_t)tile * kSortTile;
    for (int i = t; i < kSortTile; i += kSortThreads) {
      uint64_t g = base + (uint64_t)i;
      tile_keys[i] = g < n ? in[g] : 0ull;
    }
    __syncthreads();
    uint32_t c[16];
#pragma unroll
    for (int d = 0; d < 16; d++) c[d] = 0;
    uint64_t mine[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      const int i = t * kSortItems + k;
      mine[k] = tile_keys[i];
      if (base + (uint64_t)i < n) c[(mine[k] >> shift) & 15u]++;
    }
#pragma unroll
    for (int d = 0; d < 16; d++) cnt[d][t] = c[d];
    __syncthreads();
    {  // exclusive scan of each digit row over threads: warp w scans rows 2w, 2w+1
      const int warp = t >> 5, lane = t & 31;
      for (int d = warp * 2; d < warp * 2 + 2; d++) {
        uint32_t run = 0;
        for (int c0 = 0; c0 < kSortThreads; c0 += 32) {
          uint32_t x = cnt[d][c0 + lane];
          uint32_t incl = x;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
          }
          cnt[d][c0 + lane] = run + incl - x;
          run += __shfl_sync(0xffffffffu, incl, 31);
        }
      }
    }
    __syncthreads();
    uint32_t pos[16];
#pragma unroll
    for (int d = 0; d < 16; d++) pos[d] = offs[(uint64_t)d * ntiles + tile] + cnt[d][t];
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      const int i = t * kSortItems + k;
      if (base + (uint64_t)i < n) {
        const uint32_t d = (mine[k] >> shift) & 15u;
        uint32_t dst = 0;
#pragma unroll
        for (int dd = 0; dd < 16; dd++)
          if (dd == (int)d) dst = pos[dd]++;
        out[dst] = mine[k];
      }
    }
    __syncthreads();
  }
}

// Per tile: number of keys that differ from their predecessor.
__global__ void __launch_bounds__(kSortThreads) unique_count(const uint64_t* __restrict__ keys,
                                                             const unsigned long long* d_n,
                                                             uint64_t cap,
                                                             uint32_t* __restrict__ cnt) {
  __shared__ uint32_t s;
  const uint64_t n = dev_count(d_n, cap);
  const uint32_t ntiles = num_tiles(n);
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)tile * kSortTile;
    uint32_t mine = 0;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
      uint64_t g = base + (uint64_t)i;
      if (g < n && (g == 0 || keys[g] != keys[g - 1])) mine++;
    }
    atomicAdd(&s, mine);
    __syncthreads();
    if (threadIdx.x == 0) cnt[tile] = s;
    __syncthreads();
  }
}

// Writes the first key of every run of equal keys, in order, converted from
// (offset << 32 | id) to the reference's (id << 32 | offset).
__global__ void __launch_bounds__(kSortThreads) unique_write(const uint64_t* __restrict__ keys,
                                                             const unsigned long long* d_n,
                                                             uint64_t cap,
                                                             const uint32_t* __restrict__ offs,
                                                             uint64_t* __restrict__ out) {
  __shared__ uint32_t wsum[kSortThreads / 32];
  const uint64_t n = dev_count(d_n, cap);
  const uint32_t ntiles = num_tiles(n);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t base = (uint64_t)tile * kSortTile;
    uint32_t flags = 0, c = 0;
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      uint64_t g = base + (uint64_t)t * kSortItems + k;
      bool f = g < n && (g == 0 || keys[g] != keys[g - 1]);
      flags |= (uint32_t)f << k;
      c += f;
    }
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int i = 0; i < warp; i++) before += wsum[i];
    uint32_t pos = offs[tile] + before + incl - c;
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      if (flags & (1u << k)) {
        uint64_t key = keys[base + (uint64_t)t * kSortItems + k];
        out[pos++] = (key << 32) | (key >> 32);
      }
    }
    __syncthreads();
  }
}

// Batched form of unique_write: keys are stream << sshift | offset << oshift |
// id; writes the reference encoding (id << 32 | offset, offset local to the
// stream) and the stream index of each unique report.
__global__ void __launch_bounds__(kSortThreads) unique_write_fields(
    const uint64_t* __restrict__ keys, const unsigned long long* d_n, uint64_t cap,
    const uint32_t* __restrict__ offs, int oshift, int sshift, uint64_t* __restrict__ out,
    uint32_t* __restrict__ out_stream) {
  __shared__ uint32_t wsum[kSortThreads / 32];
  const uint64_t n = dev_count(d_n, cap);
  const uint32_t ntiles = num_tiles(n);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t id_mask = (1ull << oshift) - 1, off_mask = (1ull << (sshift - oshift)) - 1;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t base = (uint64_t)tile * kSortTile;
    uint32_t flags = 0, c = 0;
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      uint64_t g = base + (uint64_t)t * kSortItems + k;
      bool f = g < n && (g == 0 || keys[g] != keys[g - 1]);
      flags |= (uint32_t)f << k;
      c += f;
    }
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int i = 0; i < warp; i++) before += wsum[i];
    uint32_t pos = offs[tile] + before + incl - c;
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
      if (flags & (1u << k)) {
        const uint64_t key = keys[base + (uint64_t)t * kSortItems + k];
        const uint64_t id = key & id_mask, off = (key >> oshift) & off_mask;
        out[pos] = (id << 32) | off;
        out_stream[pos] = sshift < 64 ? (uint32_t)(key >> sshift) : 0u;
        pos++;
      }
    }
    __syncthreads();
  }
}

// Small report sets: one CTA sorts and deduplicates up to kSmallSort keys in
// shared memory (bitonic sort over the next power of two, padded with
// all-ones keys, which sort last), then writes the unique reports like
// unique_write (MODE 0) or unique_write_fields (MODE 1). It stores in
// *radix_n the key count the radix pipeline still has to sort: 0 when the
// keys were handled here (the pipeline's kernels then find no tiles), n
// otherwise; launched from a graph, it also sets the condition of the
// conditional node that holds the pipeline.
constexpr int kSmallSort = 8192;
constexpr int kSmallThreads = 1024;
constexpr int kSmallSortSmem = kSmallSort * 8;

template <int MODE>
__global__ void __launch_bounds__(kSmallThreads) small_sort_unique(
    const uint64_t* __restrict__ keys, const unsigned long long* d_n, uint64_t cap,
    unsigned long long* radix_n, unsigned long long* d_unique_n, int oshift, int sshift,
    uint64_t* __restrict__ out, uint32_t* __restrict__ out_stream, cudaGraphConditionalHandle cond,
    int set_cond) {
  extern __shared__ __align__(16) uint64_t sk[];
  __shared__ uint32_t wsum[kSmallThreads / 32];
  const uint64_t n = dev_count(d_n, cap);
  const bool big = n > (uint64_t)kSmallSort;
  if (threadIdx.x == 0) {
    *radix_n = big ? n : 0ull;
    if (set_cond) cudaGraphSetConditional(cond, big ? 1u : 0u);  // graph launches only
  }
  if (big) return;
  const uint32_t nn = (uint32_t)n;
  uint32_t m = 1;
  while (m < nn) m <<= 1;
  for (uint32_t i = threadIdx.x; i < m; i += kSmallThreads) sk[i] = i < nn ? keys[i] : ~0ull;
  __syncthreads();
  for (uint32_t k = 2; k <= m; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < m; i += kSmallThreads) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const uint64_t a = sk[i], b = sk[l];
          if ((a > b) == ((i & k) == 0)) {
            sk[i] = b;
            sk[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  // first key of every run, compacted in order: thread t owns [b, e)
  const uint32_t per = (nn + kSmallThreads - 1) / kSmallThreads;
  const uint32_t b = min(threadIdx.x * per, nn), e = min(b + per, nn);
  uint32_t c = 0;
  for (uint32_t i = b; i < e; i++) c += (i == 0 || sk[i] != sk[i - 1]) ? 1u : 0u;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  uint32_t pos = incl - c;
  for (int i = 0; i < warp; i++) pos += wsum[i];
  for (uint32_t i = b; i < e; i++) {
    if (!(i == 0 || sk[i] != sk[i - 1])) continue;
    const uint64_t key = sk[i];
    if (MODE == 0) {
      out[pos] = (key << 32) | (key >> 32);
    } else {
      const uint64_t id = key & ((1ull << oshift) - 1);
      const uint64_t off = (key >> oshift) & ((1ull << (sshift - oshift)) - 1);
      out[pos] = (id << 32) | off;
      out_stream[pos] = sshift < 64 ? (uint32_t)(key >> sshift) : 0u;
    }
    pos++;
  }
  if (threadIdx.x == kSmallThreads - 1) *d_unique_n = pos;
}

}  // namespace ngap
