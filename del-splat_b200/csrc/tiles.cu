// tiles.cu -- tile-pair construction: device scan, stable LSD radix sort,
// rank-ordered pair emission and per-tile range finding.
//
// Reference counterpart: del-splat-cudarc/src/splat_gauss.rs:96-195 (count ->
// two exclusive scans -> D2H read of the pair total -> fill_index_info ->
// radix_sort_by_key_u64_u32 on 64-bit (tile << 32 | depth bits) keys), with
// scan and sort taken from the absent del-cudarc-sys crate.
//
// Design here (same result, fewer bytes moved):
//   1. depth sort: each view's N depth keys are sorted once by a stable
//      segmented LSD radix sort (equal depths stay in point-index order) ->
//      the points of every view in rank order;
//   2. stage 1: a stable multisplit of that rank sequence into superblock
//      lists (square blocks of 1, 2, 4 or 8 tiles per side, chosen per view):
//      per (chunk, superblock) counts, one exclusive scan, then a scatter
//      whose in-warp slots come from ballots; an entry is (point, its tile
//      span clipped to the superblock).  The batched rasteriser walks these
//      lists directly, filtering by tile;
//   3. stage 2 (reference-format output only): one CTA per superblock splits
//      its list into per-tile lists with ballot ranking -> tile2idx/idx2pnt.
// Filtering a rank-ordered superblock list by tile keeps rank order, so every
// tile list is the reference's order, (tile, depth bits, point index)
// ascending, bit for bit; no 64-bit pair key is sorted.
#include "common.cuh"

namespace dsplat {

// ---------------------------------------------------------------------------
// Exclusive scan of u32 (two kernels: block totals, then each block adds the
// earlier blocks' totals to its own scan; any length).
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
  // the earlier blocks' totals, summed by every block itself (a few hundred
  // words for the scans here, so no separate pass scans them)
  uint32_t part = 0;
  for (uint32_t i = threadIdx.x; i < blockIdx.x; i += kScanThreads) part += sums[i];
  __shared__ uint32_t carry, tot;
  block_excl_scan(part, &carry);
  uint32_t p = block_excl_scan(s, &tot) + carry;
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
  k_scan_apply<<<nb, kScanThreads, 0, st>>>(in, out, n, tmp); count_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (u32 key, u32 value), 8-bit digits.
// Each block owns a tile of 4096 consecutive elements.  Segmented form: with
// nb_seg blocks per segment the histogram is laid out (segment, digit, block)
// so that one exclusive scan yields every block's output offset per digit and
// segments never mix.
//   upsweep:   16-byte key loads, per-warp shared histograms;
//   downsweep: warp w ranks its 512 elements (16 rounds of 32, in index
//              order) with match_any; the block turns the per-warp counts
//              into local digit offsets, scatters (key, value) into shared
//              memory in digit order, and writes each digit's run to its
//              global offset with consecutive threads on consecutive
//              addresses.
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsRounds = 16;
constexpr int kRsTile = kRsThreads * kRsRounds;  // 4096

__global__ void __launch_bounds__(kRsThreads) k_radix_upsweep(const uint32_t* __restrict__ keys, int shift,
                                                              uint32_t nb_seg, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[kRsWarps][256];
  for (int i = threadIdx.x; i < kRsWarps * 256; i += kRsThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  const uint4* k4 = reinterpret_cast<const uint4*>(keys + size_t(blockIdx.x) * kRsTile);
#pragma unroll
  for (int r = 0; r < kRsTile / 4 / kRsThreads; ++r) {
    const uint4 q = k4[r * kRsThreads + threadIdx.x];
    atomicAdd(&h[warp][(q.x >> shift) & 255u], 1u);
    atomicAdd(&h[warp][(q.y >> shift) & 255u], 1u);
    atomicAdd(&h[warp][(q.z >> shift) & 255u], 1u);
    atomicAdd(&h[warp][(q.w >> shift) & 255u], 1u);
  }
  __syncthreads();
  uint32_t sum = 0;
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) sum += h[w][threadIdx.x];
  const uint32_t seg = blockIdx.x / nb_seg, b = blockIdx.x % nb_seg;
  hist[(size_t(seg) * 256 + threadIdx.x) * nb_seg + b] = sum;
}

// lanes of the warp whose 8-bit digit equals this lane's (one ballot per bit)
__device__ __forceinline__ uint32_t peers_of_digit(uint32_t d) {
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int bit = 0; bit < 8; ++bit) {
    const uint32_t b = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
    m &= ((d >> bit) & 1u) ? b : ~b;
  }
  return m;
}

__global__ void __launch_bounds__(kRsThreads) k_radix_downsweep(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, int shift, uint32_t nb_seg, const uint32_t* __restrict__ offs, int write_keys,
    const uint2* __restrict__ gather_src, uint32_t gather_n, uint2* __restrict__ gather_dst, uint32_t iota_n) {
  __shared__ uint32_t wc[kRsWarps][256];
  __shared__ uint32_t dstart[256];
  __shared__ uint32_t goff[256];
  __shared__ uint32_t sk[kRsTile];
  __shared__ uint32_t sv[kRsTile];
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) wc[w][threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const size_t base = size_t(blockIdx.x) * kRsTile + size_t(warp) * (kRsRounds * 32);
  uint32_t k[kRsRounds], v[kRsRounds];
  // vin null (first pass of a sort of the identity permutation): an
  // element's value is its index in its segment, 0xffffffff from iota_n on
  if (vin) {
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
      k[r] = kin[base + r * 32 + lane];
      v[r] = vin[base + r * 32 + lane];
    }
  } else {
    const uint32_t local0 = (blockIdx.x % nb_seg) * kRsTile + uint32_t(warp) * (kRsRounds * 32) + uint32_t(lane);
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
      k[r] = kin[base + r * 32 + lane];
      const uint32_t local = local0 + uint32_t(r) * 32u;
      v[r] = local < iota_n ? local : 0xffffffffu;
    }
  }
  // phase 1: per-warp digit counts (the peer masks are kept for phase 3)
  uint32_t pm[kRsRounds];
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const uint32_t d = (k[r] >> shift) & 255u;
    pm[r] = peers_of_digit(d);
    if (lane == __ffs(pm[r]) - 1) wc[warp][d] += __popc(pm[r]);
    __syncwarp();
  }
  __syncthreads();
  // phase 2: block-local digit starts, warp bases, global digit offsets
  {
    const uint32_t d = threadIdx.x;
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) tot += wc[w][d];
    uint32_t all;
    uint32_t run = block_excl_scan(tot, &all);
    dstart[d] = run;
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) {
      const uint32_t t = wc[w][d];
      wc[w][d] = run;
      run += t;
    }
    const uint32_t seg = blockIdx.x / nb_seg, b = blockIdx.x % nb_seg;
    goff[d] = offs[(size_t(seg) * 256 + d) * nb_seg + b];
  }
  __syncthreads();
  // phase 3: stable scatter into shared memory, digit-major
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const uint32_t d = (k[r] >> shift) & 255u;
    const uint32_t peers = pm[r];
    const uint32_t rb = wc[warp][d];
    __syncwarp();
    if (lane == __ffs(peers) - 1) wc[warp][d] = rb + __popc(peers);
    __syncwarp();
    const uint32_t lp = rb + __popc(peers & lt);
    sk[lp] = k[r];
    sv[lp] = v[r];
  }
  __syncthreads();
  // phase 4: digit runs to their global offsets
#pragma unroll 4
  for (int i = threadIdx.x; i < kRsTile; i += kRsThreads) {
    const uint32_t key = sk[i];
    const uint32_t d = (key >> shift) & 255u;
    const uint32_t pos = goff[d] + (uint32_t(i) - dstart[d]);
    const uint32_t val = sv[i];
    if (write_keys) kout[pos] = key;
    vout[pos] = val;
    // optional: the value's record gathered into sorted order (segment-major
    // source, one row of gather_n records per segment; values >= gather_n
    // are padding and get an empty record)
    if (gather_dst) {
      const uint32_t seg = blockIdx.x / nb_seg;
      gather_dst[pos] = val < gather_n ? gather_src[size_t(seg) * gather_n + val] : make_uint2(0u, 0u);
    }
  }
}

size_t radix_hist_words(size_t n) { return ((n + kRsTile - 1) / kRsTile) * 256; }

// Sorts (ka, va) by bits [0, nbits) of the key, ping-ponging with (kb, vb).
// Returns in *result_in_b whether the sorted values ended in the b buffers;
// the keys of the last pass are not written (callers use the values only).
// n must be a multiple of 4096 (per segment when nseg > 1); count_ptr must be
// null (every element takes part).
// gather_dst (nullable): the last pass also writes, per sorted position,
// gather_src[segment * gather_n + value] (an empty record for padding).
// iota_values: the values are the identity permutation (each segment's
// element indices, 0xffffffff from iota_n on); va is not read, the first pass
// forms them.
cudaError_t radix_sort(cudaStream_t st, uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, size_t n,
                       const uint32_t* count_ptr, int nbits, uint32_t nseg, uint32_t* hist, uint32_t* scan_tmp,
                       bool* result_in_b, const uint2* gather_src, uint32_t gather_n, uint2* gather_dst,
                       bool iota_values, uint32_t iota_n) {
  if (n % kRsTile != 0 || count_ptr != nullptr || nseg == 0 || (n / kRsTile) % nseg != 0)
    return cudaErrorInvalidValue;
  const uint32_t nblocks = uint32_t(n / kRsTile);
  const uint32_t nb_seg = nblocks / nseg;
  const size_t hw = size_t(nblocks) * 256;
  bool in_b = false;
  if (n == 0) {
    *result_in_b = false;
    return cudaSuccess;
  }
  for (int shift = 0; shift < nbits; shift += 8) {
    const uint32_t* ki = in_b ? kb : ka;
    const uint32_t* vi = iota_values && shift == 0 ? nullptr : in_b ? vb : va;
    uint32_t* ko = in_b ? ka : kb;
    uint32_t* vo = in_b ? va : vb;
    k_radix_upsweep<<<nblocks, kRsThreads, 0, st>>>(ki, shift, nb_seg, hist); count_launch();
    cudaError_t e = exclusive_scan(st, hist, hist, hw, scan_tmp);
    if (e != cudaSuccess) return e;
    const int last = shift + 8 >= nbits;
    k_radix_downsweep<<<nblocks, kRsThreads, 0, st>>>(ki, vi, ko, vo, shift, nb_seg, hist, last ? 0 : 1,
                                                       gather_src, gather_n, last ? gather_dst : nullptr, iota_n);
    count_launch();
    in_b = !in_b;
  }
  *result_in_b = in_b;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Rank order helpers
// ---------------------------------------------------------------------------
// Keys of the padding elements [n, npad) of every segment: 0xffffffff (they
// sort last; their values are formed by the sort's first pass).
__global__ void k_pad_keys(uint32_t* __restrict__ keys, uint32_t n, uint32_t npad, uint32_t nseg) {
  const uint32_t pad = npad - n;
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= size_t(pad) * nseg) return;
  keys[size_t(i / pad) * npad + n + uint32_t(i % pad)] = 0xffffffffu;
}

// superblock span of a tile span (superblocks of 1 << sl tiles per side);
// empty if no tile
__device__ __forceinline__ bool sb_span(uint2 rc, int sl, int* sx0, int* sy0, int* sx1, int* sy1) {
  const int x0 = rc.x & 0xffff, y0 = rc.x >> 16, x1 = rc.y & 0xffff, y1 = rc.y >> 16;
  if (x1 <= x0 || y1 <= y0) return false;
  *sx0 = x0 >> sl;
  *sy0 = y0 >> sl;
  *sx1 = ((x1 - 1) >> sl) + 1;
  *sy1 = ((y1 - 1) >> sl) + 1;
  return true;
}

// tile span clipped to superblock (sx, sy), in local tile coordinates
// 0..(1 << sl): x0 | y0 << 4 | x1 << 8 | y1 << 12
__device__ __forceinline__ uint32_t local_rect(uint2 rc, int sl, int sx, int sy) {
  const int side = 1 << sl, bx = sx << sl, by = sy << sl;
  const int x0 = max(int(rc.x & 0xffff), bx) - bx, x1 = min(int(rc.y & 0xffff), bx + side) - bx;
  const int y0 = max(int(rc.x >> 16), by) - by, y1 = min(int(rc.y >> 16), by + side) - by;
  return uint32_t(x0) | uint32_t(y0) << 4 | uint32_t(x1) << 8 | uint32_t(y1) << 12;
}

constexpr int kMsThreads = 256;
constexpr int kMsWarps = kMsThreads / 32;
constexpr int kMsRounds = 16;
constexpr int kMsChunk = kMsThreads * kMsRounds;  // 4096 ranks per chunk

// ---------------------------------------------------------------------------
// Stage 1a: per (chunk, superblock) counts.  Block = one chunk of 4096 ranks
// of one view.  Output layout cnt[(sb_base[v] + s) * nchunk + c] so that an
// exclusive scan in index order yields (view, superblock, rank) positions.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kMsThreads) k_sb_count(const uint32_t* __restrict__ order,
                                                         const uint2* __restrict__ srect, uint32_t n, uint32_t npad,
                                                         const ViewBatch b,
                                                         uint32_t* __restrict__ cnt,
                                                         unsigned long long* __restrict__ totals) {
  extern __shared__ uint32_t hist[];
  const uint32_t nchunk = npad / kMsChunk;
  const uint32_t v = blockIdx.x / nchunk, c = blockIdx.x % nchunk;
  const ViewDev& vd = b.v[v];
  const int sl = vd.sb_log2, sbw = sb_cols(vd), sbh = sb_rows(vd);
  const int nsb = sbw * sbh;
  for (int i = threadIdx.x; i < nsb; i += kMsThreads) hist[i] = 0;
  __syncthreads();
  const size_t base = size_t(v) * npad + size_t(c) * kMsChunk;
  unsigned long long pairs = 0, entries = 0;
  for (int i = threadIdx.x; i < kMsChunk; i += kMsThreads) {
    const uint2 rc = srect[base + i];
    int sx0, sy0, sx1, sy1;
    if (!sb_span(rc, sl, &sx0, &sy0, &sx1, &sy1)) continue;
    pairs += (unsigned long long)((rc.y & 0xffff) - (rc.x & 0xffff)) * ((rc.y >> 16) - (rc.x >> 16));
    entries += (unsigned long long)(sx1 - sx0) * (sy1 - sy0);
    for (int sy = sy0; sy < sy1; ++sy)
      for (int sx = sx0; sx < sx1; ++sx) atomicAdd(&hist[sy * sbw + sx], 1u);
  }
  // exact 64-bit totals of tile pairs (tile-span areas) and superblock
  // entries, known even when a later stage overflows or a 32-bit list offset
  // wraps
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    entries += __shfl_xor_sync(0xffffffffu, entries, o);
  }
  if ((threadIdx.x & 31) == 0 && entries) {
    atomicAdd(&totals[0], pairs);
    atomicAdd(&totals[1], entries);
  }
  __syncthreads();
  const uint32_t sb0 = vd.sb_base;
  for (int i = threadIdx.x; i < nsb; i += kMsThreads) cnt[(size_t(sb0) + i) * nchunk + c] = hist[i];
}

// ---------------------------------------------------------------------------
// Stage 1b: stable scatter of point indices into superblock lists.  Warp w
// owns ranks [w*512, w*512+512) of the chunk in 16 rounds of 32.  In a round,
// each lane sets its bit in a shared mask per superblock column and row its
// span covers; the lanes covering superblock (x, y) are then
// colmask[x] & rowmask[y], and a lane's slot is its popcount among them.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kMsThreads) k_sb_scatter(const uint32_t* __restrict__ order,
                                                           const uint2* __restrict__ srect, uint32_t n, uint32_t npad,
                                                           const ViewBatch b,
                                                           const uint32_t* __restrict__ off, uint64_t capacity,
                                                           uint2* __restrict__ list1, uint32_t* __restrict__ flags) {
  extern __shared__ uint32_t smem_ms[];  // [kMsWarps][nsb] counters, then [kMsWarps][2 * side] masks
  const uint32_t nchunk = npad / kMsChunk;
  const uint32_t v = blockIdx.x / nchunk, c = blockIdx.x % nchunk;
  const ViewDev& vd = b.v[v];
  const int sl = vd.sb_log2, sbw = sb_cols(vd), sbh = sb_rows(vd);
  const int nsb = sbw * sbh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t* wc = smem_ms;
  const uint32_t side = b.max_sb_side;
  uint32_t* colmask = smem_ms + kMsWarps * b.max_sb + warp * 2 * side;
  uint32_t* rowmask = colmask + side;
  for (int i = threadIdx.x; i < kMsWarps * nsb; i += kMsThreads) wc[i] = 0;
  __syncthreads();
  const size_t base = size_t(v) * npad + size_t(c) * kMsChunk + size_t(warp) * (kMsRounds * 32);
  uint32_t* my = wc + warp * nsb;
  // phase 1: per-warp counts
  for (int r = 0; r < kMsRounds; ++r) {
    int sx0, sy0, sx1, sy1;
    if (sb_span(srect[base + r * 32 + lane], sl, &sx0, &sy0, &sx1, &sy1))
      for (int sy = sy0; sy < sy1; ++sy)
        for (int sx = sx0; sx < sx1; ++sx) atomicAdd(&my[sy * sbw + sx], 1u);
  }
  __syncthreads();
  // phase 2: warp bases = chunk offset + earlier warps
  const uint32_t sb0 = vd.sb_base;
  for (int i = threadIdx.x; i < nsb; i += kMsThreads) {
    uint32_t run = off[(size_t(sb0) + i) * nchunk + c];
    for (int w = 0; w < kMsWarps; ++w) {
      const uint32_t t = wc[w * nsb + i];
      wc[w * nsb + i] = run;
      run += t;
    }
  }
  __syncthreads();
  // phase 3: stable scatter, round by round
  for (int r = 0; r < kMsRounds; ++r) {
    const uint32_t g = order[base + r * 32 + lane];
    int sx0 = 0, sy0 = 0, sx1 = 0, sy1 = 0;
    const uint2 rc = srect[base + r * 32 + lane];
    const bool has = sb_span(rc, sl, &sx0, &sy0, &sx1, &sy1);
    // the round's column / row coverage masks: every lane clears, then sets
    // its bit in, the entries of the columns and rows its span covers
    if (has) {
      for (int x = sx0; x < sx1; ++x) colmask[x] = 0u;
      for (int y = sy0; y < sy1; ++y) rowmask[y] = 0u;
    }
    __syncwarp();
    if (has) {
      for (int x = sx0; x < sx1; ++x) atomicOr(&colmask[x], 1u << lane);
      for (int y = sy0; y < sy1; ++y) atomicOr(&rowmask[y], 1u << lane);
    }
    __syncwarp();
    for (int sy = sy0; sy < sy1; ++sy) {
      const uint32_t rm = rowmask[sy];
      for (int sx = sx0; sx < sx1; ++sx) {
        const uint32_t m = colmask[sx] & rm;
        const uint32_t dst = my[sy * sbw + sx] + uint32_t(__popc(m & lt));
        if (dst < capacity) list1[dst] = make_uint2(g, local_rect(rc, sl, sx, sy));
        else set_flag(flags, kFlagPairOverflow);
      }
    }
    __syncwarp();
    // the highest lane covering a superblock advances the warp's counter
    for (int sy = sy0; sy < sy1; ++sy) {
      const uint32_t rm = rowmask[sy];
      for (int sx = sx0; sx < sx1; ++sx) {
        const uint32_t m = colmask[sx] & rm;
        if ((m >> lane) == 1u) my[sy * sbw + sx] += uint32_t(__popc(m));
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Stage 1b, staged: the same result as k_sb_scatter with coalesced stores.
// The chunk is processed in sub-passes of kSubRanks consecutive ranks (each
// warp takes kSubRanks / 8 consecutive ranks of the sub-pass).  A sub-pass's
// entries are ranked per superblock (per-warp counts, one block-wide scan)
// into a shared-memory stage ordered by superblock, then each superblock's
// run is written to its contiguous range of the superblock list (the block's
// cursor for that superblock advances sub-pass by sub-pass).  A sub-pass
// with more entries than the stage holds writes the same slots directly.
// Shared memory (words): counters [8][max_sb], cursors [max_sb], stage
// bases [max_sb + 2] (one spare word keeps the stage 8-byte aligned), masks
// [8][2 * max_sb_side] (superblock columns, then rows), then the stage
// (uint2[qcap]) and its superblock ids (u16[qcap]).
// ---------------------------------------------------------------------------
constexpr int kSubRounds = 2;
constexpr int kSubRanks = kMsThreads * kSubRounds;  // 512 ranks per sub-pass

size_t sb_scatter_staged_smem(uint32_t max_sb, uint32_t max_side, uint32_t qcap) {
  return (size_t(kMsWarps) * max_sb + 2 * size_t(max_sb) + 2 + size_t(kMsWarps) * 2 * max_side) * 4 +
         size_t(qcap) * 8 +
         ((size_t(qcap) + 1) / 2) * 4;
}

__global__ void __launch_bounds__(kMsThreads) k_sb_scatter_staged(const uint32_t* __restrict__ order,
                                                                  const uint2* __restrict__ srect, uint32_t n,
                                                                  uint32_t npad, const ViewBatch b,
                                                                  const uint32_t* __restrict__ off, uint64_t capacity,
                                                                  uint2* __restrict__ list1,
                                                                  uint32_t* __restrict__ flags, uint32_t qcap) {
  extern __shared__ uint32_t smem_ms[];
  __shared__ uint32_t sub_total;
  const uint32_t nchunk = npad / kMsChunk;
  const uint32_t v = blockIdx.x / nchunk, c = blockIdx.x % nchunk;
  const ViewDev& vd = b.v[v];
  const int sl = vd.sb_log2, sbw = sb_cols(vd), sbh = sb_rows(vd);
  const int nsb = sbw * sbh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t M = b.max_sb;
  uint32_t* wc = smem_ms;                     // [kMsWarps][nsb]
  uint32_t* cur = wc + kMsWarps * M;          // [nsb]
  uint32_t* sbase = cur + M;                  // [nsb + 1]
  const uint32_t side = b.max_sb_side;
  uint32_t* colmask = sbase + M + 2 + warp * 2 * side;
  uint32_t* rowmask = colmask + side;
  uint2* stage = reinterpret_cast<uint2*>(sbase + M + 2 + kMsWarps * 2 * side);  // 10 M + 2 + 16 side words: 8-byte aligned
  uint16_t* stage_sb = reinterpret_cast<uint16_t*>(stage + qcap);
  uint32_t* my = wc + warp * nsb;
  const uint32_t sb0 = vd.sb_base;
  for (int i = threadIdx.x; i < nsb; i += kMsThreads) cur[i] = off[(size_t(sb0) + i) * nchunk + c];
  const int seg = (nsb + kMsThreads - 1) / kMsThreads;
  const int s_lo = min(nsb, int(threadIdx.x) * seg), s_hi = min(nsb, s_lo + seg);
  for (int sub = 0; sub < kMsChunk / kSubRanks; ++sub) {
    for (int i = threadIdx.x; i < kMsWarps * nsb; i += kMsThreads) wc[i] = 0;
    __syncthreads();
    const size_t base = size_t(v) * npad + size_t(c) * kMsChunk + size_t(sub) * kSubRanks +
                        size_t(warp) * (kSubRounds * 32);
    // per-warp counts of the sub-pass
    for (int r = 0; r < kSubRounds; ++r) {
      int sx0, sy0, sx1, sy1;
      if (sb_span(srect[base + r * 32 + lane], sl, &sx0, &sy0, &sx1, &sy1))
        for (int sy = sy0; sy < sy1; ++sy)
          for (int sx = sx0; sx < sx1; ++sx) atomicAdd(&my[sy * sbw + sx], 1u);
    }
    __syncthreads();
    // stage layout: superblock-major, then warp (= rank order)
    uint32_t loc = 0;
    for (int sb = s_lo; sb < s_hi; ++sb)
#pragma unroll
      for (int w = 0; w < kMsWarps; ++w) loc += wc[w * nsb + sb];
    uint32_t run = block_excl_scan(loc, &sub_total);
    for (int sb = s_lo; sb < s_hi; ++sb) {
      sbase[sb] = run;
#pragma unroll
      for (int w = 0; w < kMsWarps; ++w) {
        const uint32_t t = wc[w * nsb + sb];
        wc[w * nsb + sb] = run;
        run += t;
      }
    }
    if (threadIdx.x == 0) sbase[nsb] = sub_total;
    __syncthreads();
    const uint32_t total = sub_total;
    const bool staged = total <= qcap;
    for (int r = 0; r < kSubRounds; ++r) {
      const uint32_t g = order[base + r * 32 + lane];
      int sx0 = 0, sy0 = 0, sx1 = 0, sy1 = 0;
      const uint2 rc = srect[base + r * 32 + lane];
      const bool has = sb_span(rc, sl, &sx0, &sy0, &sx1, &sy1);
      if (has) {
        for (int x = sx0; x < sx1; ++x) colmask[x] = 0u;
        for (int y = sy0; y < sy1; ++y) rowmask[y] = 0u;
      }
      __syncwarp();
      if (has) {
        for (int x = sx0; x < sx1; ++x) atomicOr(&colmask[x], 1u << lane);
        for (int y = sy0; y < sy1; ++y) atomicOr(&rowmask[y], 1u << lane);
      }
      __syncwarp();
      for (int sy = sy0; sy < sy1; ++sy) {
        const uint32_t rm = rowmask[sy];
        for (int sx = sx0; sx < sx1; ++sx) {
          const int sb = sy * sbw + sx;
          const uint32_t sp = my[sb] + uint32_t(__popc(colmask[sx] & rm & lt));
          const uint2 en = make_uint2(g, local_rect(rc, sl, sx, sy));
          if (staged) {
            stage[sp] = en;
            stage_sb[sp] = uint16_t(sb);
          } else {
            const uint64_t dst = uint64_t(cur[sb]) + (sp - sbase[sb]);
            if (dst < capacity) list1[dst] = en;
            else set_flag(flags, kFlagPairOverflow);
          }
        }
      }
      __syncwarp();
      for (int sy = sy0; sy < sy1; ++sy) {
        const uint32_t rm = rowmask[sy];
        for (int sx = sx0; sx < sx1; ++sx) {
          const uint32_t m = colmask[sx] & rm;
          if ((m >> lane) == 1u) my[sy * sbw + sx] += uint32_t(__popc(m));
        }
      }
      __syncwarp();
    }
    __syncthreads();
    if (staged) {
      for (uint32_t i = threadIdx.x; i < total; i += kMsThreads) {
        const int sb = stage_sb[i];
        const uint64_t dst = uint64_t(cur[sb]) + (i - sbase[sb]);
        if (dst < capacity) list1[dst] = stage[i];
        else set_flag(flags, kFlagPairOverflow);
      }
    }
    __syncthreads();
    for (int sb = threadIdx.x; sb < nsb; sb += kMsThreads) cur[sb] += sbase[sb + 1] - sbase[sb];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Stage 2a: per-tile pair counts, one CTA per superblock walking its list.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int view_of_sb(const ViewBatch& b, uint32_t sb) {
  int v = 0;
  for (int k = 1; k < b.num_views; ++k)
    if (sb >= b.v[k].sb_base) v = k;
  return v;
}

__global__ void __launch_bounds__(kMsThreads) k_tile_count(const uint2* __restrict__ list1,
                                                           const uint32_t* __restrict__ off1, uint32_t nchunk,
                                                           uint64_t capacity, const ViewBatch b,
                                                           uint32_t* __restrict__ tcnt) {
  __shared__ uint32_t h[64];
  const uint32_t sb = blockIdx.x;
  const int v = view_of_sb(b, sb);
  const ViewDev& vd = b.v[v];
  const int sl = vd.sb_log2, side = 1 << sl, sbw = sb_cols(vd);
  const uint32_t ls = sb - vd.sb_base;
  const int tx0 = int(ls % uint32_t(sbw)) << sl, ty0 = int(ls / uint32_t(sbw)) << sl;
  if (threadIdx.x < 64) h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t s = min(uint64_t(off1[size_t(sb) * nchunk]), capacity);
  const uint64_t e = min(uint64_t(off1[size_t(sb + 1) * nchunk]), capacity);
  for (uint64_t i = s + threadIdx.x; i < e; i += kMsThreads) {
    const uint32_t lr = list1[i].y;
    const int x0 = lr & 15, y0 = (lr >> 4) & 15, x1 = (lr >> 8) & 15, y1 = (lr >> 12) & 15;
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) atomicAdd(&h[y * 8 + x], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 64 && int(threadIdx.x & 7) < side && int(threadIdx.x >> 3) < side) {
    const int x = tx0 + (threadIdx.x & 7), y = ty0 + (threadIdx.x >> 3);
    if (x < vd.tile_w && y < vd.tile_h) tcnt[vd.item_base + uint32_t(y) * vd.tile_w + x] = h[threadIdx.x];
  }
}

// ---------------------------------------------------------------------------
// Stage 2b: stable scatter into tile lists.  Chunks of 256 list entries, one
// per thread in order; for each of the 64 tiles a warp ballot says which lanes
// cover it, and popcounts of the ballots give every pair its slot:
//   slot = tile start + earlier chunks + earlier warps + lower lanes.
// out_tile (nullable) receives each pair's item id.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kMsThreads) k_tile_scatter(const uint2* __restrict__ list1,
                                                             const uint32_t* __restrict__ off1, uint32_t nchunk,
                                                             uint64_t capacity, const ViewBatch b,
                                                               const uint32_t* __restrict__ item_start,
                                                             uint32_t* __restrict__ idx2pnt,
                                                             uint32_t* __restrict__ out_tile,
                                                             uint32_t* __restrict__ flags) {
  __shared__ uint32_t run[64];
  __shared__ uint32_t tot[64];
  __shared__ uint32_t masks[kMsWarps][64];
  __shared__ uint32_t pre[kMsWarps][64];
  const uint32_t sb = blockIdx.x;
  const int v = view_of_sb(b, sb);
  const ViewDev& vd = b.v[v];
  const int sl = vd.sb_log2, side = 1 << sl, sbw = sb_cols(vd);
  const uint32_t ls = sb - vd.sb_base;
  const int tx0 = int(ls % uint32_t(sbw)) << sl, ty0 = int(ls / uint32_t(sbw)) << sl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  if (threadIdx.x < 64) {
    const int x = tx0 + (threadIdx.x & 7), y = ty0 + (threadIdx.x >> 3);
    const bool in = int(threadIdx.x & 7) < side && int(threadIdx.x >> 3) < side && x < vd.tile_w && y < vd.tile_h;
    run[threadIdx.x] = in ? item_start[vd.item_base + uint32_t(y) * vd.tile_w + x] : 0u;
  }
  __syncthreads();
  const uint64_t s = min(uint64_t(off1[size_t(sb) * nchunk]), capacity);
  const uint64_t e = min(uint64_t(off1[size_t(sb + 1) * nchunk]), capacity);
  for (uint64_t c0 = s; c0 < e; c0 += kMsThreads) {
    const uint64_t i = c0 + threadIdx.x;
    uint32_t g = 0;
    int x0 = 0, x1 = 0, y0 = 0, y1 = 0;
    if (i < e) {
      const uint2 en = list1[i];
      g = en.x;
      x0 = en.y & 15;
      y0 = (en.y >> 4) & 15;
      x1 = (en.y >> 8) & 15;
      y1 = (en.y >> 12) & 15;
    }
#pragma unroll
    for (int k = 0; k < 64; ++k) {
      const int kx = k & 7, ky = k >> 3;
      if (kx >= side || ky >= side) continue;  // outside a smaller superblock
      const uint32_t m = __ballot_sync(0xffffffffu, kx >= x0 && kx < x1 && ky >= y0 && ky < y1);
      if ((k & 31) == lane) masks[warp][k] = m;
    }
    __syncthreads();
    if (threadIdx.x < 64) {
      uint32_t acc = 0;
#pragma unroll
      for (int w = 0; w < kMsWarps; ++w) {
        pre[w][threadIdx.x] = acc;
        acc += __popc(masks[w][threadIdx.x]);
      }
      tot[threadIdx.x] = acc;
    }
    __syncthreads();
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) {
        const int k = y * 8 + x;
        const uint32_t slot = run[k] + pre[warp][k] + __popc(masks[warp][k] & lt);
        if (slot < capacity) {
          idx2pnt[slot] = g;
          if (out_tile) out_tile[slot] = vd.item_base + uint32_t(ty0 + y) * vd.tile_w + uint32_t(tx0 + x);
        } else {
          set_flag(flags, kFlagPairOverflow);
        }
      }
    __syncthreads();
    if (threadIdx.x < 64) run[threadIdx.x] += tot[threadIdx.x];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Longest-first task order for the rasteriser: items bucketed by floor(log2)
// of their cost, heaviest bucket first, so the tail of the persistent launch
// is made of short tasks.  The cost is the number of list positions the last
// forward walked for the item (measured, kept in the workspace) or, where
// none is recorded yet, its superblock-list length.  Only the schedule
// depends on it, never the results.  sched[0..32] counts, [40..72] cursors.
// ---------------------------------------------------------------------------
// Longest-first bucket of an item (0 = longest): clz of the list positions
// its task walked in the previous forward (cost[item]), else of its
// superblock's list length.  With nt > 1 adjacent tiles per task (8x8
// tiles) only a group's leading tile leads a task and carries its cost; the
// other tiles lead none (their tasks return at once) and go last.
__device__ __forceinline__ uint32_t item_cost_bucket(const ViewBatch& b, uint32_t item, const uint32_t* off1,
                                                     uint32_t nchunk, const uint32_t* cost, int nt) {
  int v = 0;
  for (int k = 1; k < b.num_views; ++k)
    if (item >= b.v[k].item_base) v = k;
  const ViewDev& vd = b.v[v];
  const uint32_t t = item - vd.item_base;
  const uint32_t tx = t % uint32_t(vd.tile_w), ty = t / uint32_t(vd.tile_w);
  if (nt > 1 && tx % min(uint32_t(nt), 1u << vd.sb_log2)) return 31u;
  const uint32_t measured = cost ? cost[item] : 0u;
  if (measured) return uint32_t(__clz(measured));
  const uint32_t sb = vd.sb_base + (ty >> vd.sb_log2) * uint32_t(sb_cols(vd)) + (tx >> vd.sb_log2);
  const uint32_t len = off1[size_t(sb + 1) * nchunk] - off1[size_t(sb) * nchunk];
  return len ? uint32_t(__clz(len)) : 32u;
}

__global__ void k_order_hist(const ViewBatch b, const uint32_t* __restrict__ off1, uint32_t nchunk,
                             const uint32_t* __restrict__ cost, int nt, uint32_t* __restrict__ sched) {
  __shared__ uint32_t h[33];
  if (threadIdx.x < 33) h[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.num_items; i += gridDim.x * blockDim.x)
    atomicAdd(&h[item_cost_bucket(b, i, off1, nchunk, cost, nt)], 1u);
  __syncthreads();
  if (threadIdx.x < 33 && h[threadIdx.x]) atomicAdd(&sched[threadIdx.x], h[threadIdx.x]);
}

// Scatter into bucket order: each block ranks its items in shared memory and
// takes one range per bucket from the global cursors (one global atomic per
// bucket and block instead of one per item on 33 hot counters).  sched[0..33)
// holds the bucket counts, sched[40..73) the cursors (zero at the start);
// every block forms the buckets' starts from the counts itself.
__global__ void k_order_scatter(const ViewBatch b, const uint32_t* __restrict__ off1, uint32_t nchunk,
                                const uint32_t* __restrict__ cost, int nt, uint32_t* __restrict__ sched,
                                uint32_t* __restrict__ order) {
  __shared__ uint32_t cnt[33], base[33], start[33];
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = 0; k < 33; ++k) {
      start[k] = run;
      run += sched[k];
    }
  }
  __syncthreads();
  const uint32_t per_block = (b.num_items + gridDim.x - 1) / gridDim.x;
  const uint32_t lo = blockIdx.x * per_block, hi = min(b.num_items, lo + per_block);
  for (uint32_t i0 = lo; i0 < hi; i0 += blockDim.x) {
    if (threadIdx.x < 33) cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = i0 + threadIdx.x;
    uint32_t bucket = 0, slot = 0;
    if (i < hi) {
      bucket = item_cost_bucket(b, i, off1, nchunk, cost, nt);
      slot = atomicAdd(&cnt[bucket], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 33 && cnt[threadIdx.x])
      base[threadIdx.x] = start[threadIdx.x] + atomicAdd(&sched[40 + threadIdx.x], cnt[threadIdx.x]);
    __syncthreads();
    if (i < hi) order[base[bucket] + slot] = i;
    __syncthreads();
  }
}


// Clamp tile ranges to the pair capacity after an overflow so that readers
// stay in bounds (the results are then invalid and the flag is set).
__global__ void k_clamp_ranges(uint32_t* __restrict__ item_start, uint32_t num_items, uint64_t capacity,
                               uint32_t* __restrict__ flags) {
  const uint32_t total = item_start[num_items];
  if (total <= capacity) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) set_flag(flags, kFlagPairOverflow);
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i <= num_items; i += size_t(gridDim.x) * blockDim.x)
    if (item_start[i] > capacity) item_start[i] = uint32_t(capacity);
}

// Flags a capacity overflow when the superblock lists need more entries than
// the capacity (the 64-bit total also catches a wrapped 32-bit offset scan).
__global__ void k_check_capacity(const unsigned long long* __restrict__ entries, uint64_t capacity,
                                 uint32_t* __restrict__ flags) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && *entries > capacity) set_flag(flags, kFlagPairOverflow);
}

// keys for the drop-in API: idx2tiledepth = (tile << 32) | depth bits of the
// point, recomputed from pnt2pixxydepth
__global__ void k_make_keys64(const uint32_t* __restrict__ tile, const uint32_t* __restrict__ pnt,
                              const float* __restrict__ xyd, const unsigned long long* __restrict__ count_ptr,
                              uint64_t capacity, uint64_t* __restrict__ out) {
  const uint64_t cnt = *count_ptr < capacity ? uint64_t(*count_ptr) : capacity;
  for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < cnt; p += size_t(gridDim.x) * blockDim.x)
    out[p] = (uint64_t(tile[p]) << 32) | depth_bits(xyd[3 * size_t(pnt[p]) + 2]);
}

}  // namespace dsplat
