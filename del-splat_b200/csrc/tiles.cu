// tiles.cu -- tile-pair construction: device scan, stable LSD radix sort,
// rank-ordered pair emission and per-tile range finding.
//
// Reference counterpart: del-splat-cudarc/src/splat_gauss.rs:96-195 (count ->
// two exclusive scans -> D2H read of the pair total -> fill_index_info ->
// radix_sort_by_key_u64_u32 on 64-bit (tile << 32 | depth bits) keys), with
// scan and sort taken from the absent del-cudarc-sys crate.
//
// Design here (same result, fewer bytes moved):
//   1. depth sort: the N per-point depth keys are sorted once (stable, so
//      equal depths stay in point-index order) -> a rank per point;
//   2. pairs are emitted in rank order (exclusive scan of the per-point
//      counts taken in rank order gives each point's output run);
//   3. a stable LSD sort of the pairs by tile id alone (8-bit digits over
//      ceil(log2(#tiles)) bits) -- stability keeps rank order inside a tile.
// The result is the reference's order, (tile, depth bits, point index)
// ascending, i.e. the same tile2idx / idx2pnt bit for bit, while the P-sized
// sort touches 8 bytes per pair per pass over ~2 passes instead of 12 bytes
// over 5-7 passes.
#include "common.cuh"

namespace dsplat {

// ---------------------------------------------------------------------------
// Exclusive scan of u32 (three kernels; any length).
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Block-wide exclusive scan of one value per thread; returns the prefix and
// writes the block total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  uint32_t inc = warp_incl_scan(x, lane);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nwarps ? warp_sums[lane] : 0u;
    uint32_t si = warp_incl_scan(s, lane);
    if (lane < nwarps) warp_sums[lane] = si - s;
    if (lane == nwarps - 1) *total = si;
  }
  __syncthreads();
  uint32_t r = warp_sums[warp] + inc - x;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ in, size_t n,
                                                              uint32_t* __restrict__ sums) {
  const size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) s += in[base + i];
  __shared__ uint32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// single block: exclusive scan of the block sums, any count
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t* sums, uint32_t nb) {
  __shared__ uint32_t carry_s;
  __shared__ uint32_t tot;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += kScanThreads) {
    const uint32_t i = base + threadIdx.x;
    uint32_t x = i < nb ? sums[i] : 0u;
    uint32_t p = block_excl_scan(x, &tot);
    const uint32_t c = carry_s;
    if (i < nb) sums[i] = c + p;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = c + tot;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t* __restrict__ in,
                                                             uint32_t* __restrict__ out, size_t n,
                                                             const uint32_t* __restrict__ sums) {
  const size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < n ? in[base + i] : 0u;
    s += v[i];
  }
  __shared__ uint32_t tot;
  uint32_t p = block_excl_scan(s, &tot) + sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = p;
    p += v[i];
  }
}

size_t scan_tmp_words(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

cudaError_t exclusive_scan(cudaStream_t st, const uint32_t* in, uint32_t* out, size_t n, uint32_t* tmp) {
  if (n == 0) return cudaSuccess;
  const uint32_t nb = uint32_t((n + kScanTile - 1) / kScanTile);
  k_scan_reduce<<<nb, kScanThreads, 0, st>>>(in, n, tmp); count_launch();
  k_scan_sums<<<1, kScanThreads, 0, st>>>(tmp, nb); count_launch();
  k_scan_apply<<<nb, kScanThreads, 0, st>>>(in, out, n, tmp); count_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (u32 key, u32 value), 8-bit digits.
// Each block owns a tile of 4096 consecutive elements (8 warps x 16 rounds x
// 32 lanes, in index order).  Segmented form: with nb_seg blocks per segment
// the histogram is laid out (segment, digit, block) so that one exclusive scan
// yields every element's destination and segments never mix.
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsRounds = 16;
constexpr int kRsTile = kRsThreads * kRsRounds;  // 4096

__device__ __forceinline__ uint32_t live_count(size_t n, const uint32_t* count_ptr) {
  if (!count_ptr) return uint32_t(n);
  const uint32_t c = *count_ptr;
  return c < n ? c : uint32_t(n);
}

__global__ void __launch_bounds__(kRsThreads) k_radix_upsweep(const uint32_t* __restrict__ keys, size_t n,
                                                              const uint32_t* __restrict__ count_ptr, int shift,
                                                              uint32_t nb_seg, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t cnt = live_count(n, count_ptr);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t base = size_t(blockIdx.x) * kRsTile + size_t(warp) * (kRsRounds * 32);
#pragma unroll 4
  for (int r = 0; r < kRsRounds; ++r) {
    const size_t idx = base + r * 32 + lane;
    const bool valid = idx < cnt;
    const uint32_t d = valid ? (keys[idx] >> shift) & 255u : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(&h[d], __popc(peers));
  }
  __syncthreads();
  const uint32_t seg = blockIdx.x / nb_seg, b = blockIdx.x % nb_seg;
  hist[(size_t(seg) * 256 + threadIdx.x) * nb_seg + b] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads) k_radix_downsweep(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, size_t n, const uint32_t* __restrict__ count_ptr, int shift, uint32_t nb_seg,
    const uint32_t* __restrict__ offs) {
  __shared__ uint32_t wc[kRsWarps][256];
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) wc[w][threadIdx.x] = 0;
  __syncthreads();
  const uint32_t cnt = live_count(n, count_ptr);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const size_t base = size_t(blockIdx.x) * kRsTile + size_t(warp) * (kRsRounds * 32);
  uint32_t k[kRsRounds], v[kRsRounds];
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const size_t idx = base + r * 32 + lane;
    if (idx < cnt) {
      k[r] = kin[idx];
      v[r] = vin[idx];
    } else {
      k[r] = 0;
      v[r] = 0;
    }
  }
  // phase 1: per-warp digit counts
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const bool valid = base + r * 32 + lane < cnt;
    const uint32_t d = valid ? (k[r] >> shift) & 255u : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (valid && lane == __ffs(peers) - 1) wc[warp][d] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // phase 2: warp bases = block offset of the digit + earlier warps
  {
    const uint32_t d = threadIdx.x;
    const uint32_t seg = blockIdx.x / nb_seg, b = blockIdx.x % nb_seg;
    uint32_t run = offs[(size_t(seg) * 256 + d) * nb_seg + b];
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) {
      const uint32_t t = wc[w][d];
      wc[w][d] = run;
      run += t;
    }
  }
  __syncthreads();
  // phase 3: stable scatter
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const bool valid = base + r * 32 + lane < cnt;
    const uint32_t d = valid ? (k[r] >> shift) & 255u : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rb = valid ? wc[warp][d] : 0u;
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wc[warp][d] = rb + __popc(peers);
    __syncwarp();
    if (valid) {
      const uint32_t pos = rb + __popc(peers & lt);
      kout[pos] = k[r];
      vout[pos] = v[r];
    }
  }
}

size_t radix_hist_words(size_t n) { return ((n + kRsTile - 1) / kRsTile) * 256; }

// Sorts (ka, va) by bits [0, nbits) of the key, ping-ponging with (kb, vb).
// Returns in *result_in_b whether the sorted data ended in the b buffers.
// n must be a multiple of 4096 per segment when nseg > 1.
cudaError_t radix_sort(cudaStream_t st, uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, size_t n,
                       const uint32_t* count_ptr, int nbits, uint32_t nseg, uint32_t* hist, uint32_t* scan_tmp,
                       bool* result_in_b) {
  const uint32_t nblocks = uint32_t((n + kRsTile - 1) / kRsTile);
  const uint32_t nb_seg = nblocks / nseg;
  const size_t hw = size_t(nblocks) * 256;
  bool in_b = false;
  if (n == 0) {
    *result_in_b = false;
    return cudaSuccess;
  }
  for (int shift = 0; shift < nbits; shift += 8) {
    const uint32_t* ki = in_b ? kb : ka;
    const uint32_t* vi = in_b ? vb : va;
    uint32_t* ko = in_b ? ka : kb;
    uint32_t* vo = in_b ? va : vb;
    k_radix_upsweep<<<nblocks, kRsThreads, 0, st>>>(ki, n, count_ptr, shift, nb_seg, hist); count_launch();
    cudaError_t e = exclusive_scan(st, hist, hist, hw, scan_tmp);
    if (e != cudaSuccess) return e;
    k_radix_downsweep<<<nblocks, kRsThreads, 0, st>>>(ki, vi, ko, vo, n, count_ptr, shift, nb_seg, hist); count_launch();
    in_b = !in_b;
  }
  *result_in_b = in_b;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Pair emission in rank order.
// ---------------------------------------------------------------------------
__global__ void k_iota_pad(uint32_t* __restrict__ vals, uint32_t* __restrict__ keys, uint32_t n, uint32_t npad,
                           uint32_t nseg) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= size_t(npad) * nseg) return;
  const uint32_t r = uint32_t(i % npad);
  vals[i] = r < n ? r : 0xffffffffu;
  if (r >= n) keys[i] = 0xffffffffu;
}

// counts in rank order: cs[v*npad + r] = cnt[v*n + order[v*npad + r]]
__global__ void k_gather_counts(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cnt, uint32_t n,
                                uint32_t npad, uint32_t nseg, uint32_t* __restrict__ cs) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i > size_t(npad) * nseg) return;
  if (i == size_t(npad) * nseg) {
    cs[i] = 0;
    return;
  }
  const uint32_t v = uint32_t(i / npad);
  const uint32_t g = order[i];
  cs[i] = g < n ? cnt[size_t(v) * n + g] : 0u;
}

__global__ void k_emit_pairs(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cs,
                             const uint32_t* __restrict__ off, const uint2* __restrict__ rect, uint32_t n,
                             uint32_t npad, uint32_t nseg, const ViewBatch b, uint64_t capacity,
                             uint32_t* __restrict__ pkey, uint32_t* __restrict__ pval, uint32_t* __restrict__ flags) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= size_t(npad) * nseg) return;
  const uint32_t c = cs[i];
  if (c == 0) return;
  const uint32_t v = uint32_t(i / npad);
  const uint32_t g = order[i];
  const uint64_t o = off[i];
  if (o + c > capacity) {
    set_flag(flags, kFlagPairOverflow);
    for (uint64_t j = o; j < capacity; ++j) pkey[j] = 0xffffffffu;
    return;
  }
  const uint2 rc = rect[size_t(v) * n + g];
  const int x0 = rc.x & 0xffff, y0 = rc.x >> 16, x1 = rc.y & 0xffff, y1 = rc.y >> 16;
  const uint32_t tw = uint32_t(b.v[v].tile_w), base = b.v[v].item_base;
  uint32_t j = uint32_t(o);
  // tile_acceleration.h:34-50 order: ix outer, iy inner
  for (int ix = x0; ix < x1; ++ix)
    for (int iy = y0; iy < y1; ++iy) {
      pkey[j] = base + uint32_t(iy) * tw + uint32_t(ix);
      pval[j] = g;
      ++j;
    }
}

// item_start[j] for j in [0, I] from the tile-sorted keys (boundary detection;
// empty items take the start of the next non-empty one).  Keys >= I (overflow
// sentinels) count as I.
__global__ void k_item_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ count_ptr,
                              uint64_t capacity, uint32_t num_items, uint32_t* __restrict__ item_start) {
  uint32_t cnt = *count_ptr;
  if (cnt > capacity) cnt = uint32_t(capacity);
  auto eff = [&](size_t q) -> int64_t {
    const uint32_t k = keys[q];
    return k < num_items ? int64_t(k) : int64_t(num_items);
  };
  for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p <= cnt; p += size_t(gridDim.x) * blockDim.x) {
    const int64_t k = p < cnt ? eff(p) : int64_t(num_items);
    const int64_t kp = p > 0 ? eff(p - 1) : -1;
    for (int64_t j = kp + 1; j <= k; ++j) item_start[j] = uint32_t(p);
  }
}

__global__ void k_copy_total(const uint32_t* __restrict__ off, size_t idx, uint32_t* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = off[idx];
}

// keys for the drop-in API: idx2tiledepth = (tile << 32) | depth bits, the
// depth bits recomputed from pnt2pixxydepth (the key buffer is sorted by now)
__global__ void k_make_keys64(const uint32_t* __restrict__ tkey, const uint32_t* __restrict__ tval,
                              const float* __restrict__ xyd, const uint32_t* __restrict__ count_ptr,
                              uint64_t capacity, uint64_t* __restrict__ out) {
  uint32_t cnt = *count_ptr;
  if (cnt > capacity) cnt = uint32_t(capacity);
  for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < cnt; p += size_t(gridDim.x) * blockDim.x)
    out[p] = (uint64_t(tkey[p]) << 32) | depth_bits(xyd[3 * size_t(tval[p]) + 2]);
}

}  // namespace dsplat
