// Steps 2-4 of the rasterizer: the stable (tile, depth, index) ordering of all splat-tile pairs.
//
// The reference duplicates one 64-bit key (tile << 32 | depth bits) per pair in Gaussian-index order
// and radix-sorts all of them over bits [0, 32 + bits(tiles)) (gpu_render.cu:148-161, 324-345).
// A stable LSD sort handles the low (depth) digits first, and duplication commutes with a stable
// sort on a key every copy of a Gaussian shares, so the same order is produced here with less
// traffic:
//   1. the preprocess kernel writes every entry's depth key (a sentinel when culled);
//   2. four 8-bit LSD passes sort the V visible (depth bits, entry) pairs -- V, not P, items;
//      the first pass reads all N keys in entry order and drops the culled ones as it ranks;
//   3. a pair-offset scan over those V, then an expansion, in depth order, into P (tile, entry)
//      pairs with the same number of pairs per block (the nearest splats own thousands of tiles);
//   4. ceil(bits(tiles) / 8) LSD passes (or / 9 with 9-bit digits allowed, each pass 8 bits wide
//      unless 9 are needed) stably sort the pairs by tile;
//   5. tile ranges as gpu_render.cu:164-177.
// A frame of at most kBinMaxTiles tiles replaces 4 and 5 by one stable counting pass over the
// whole tile id (the one-pass tile binning below): two kernels where the LSD passes and the
// ranges take five or six.
// Each tile's run ends up ordered by (depth bits, entry index), exactly the reference's order, so
// keys, values and ranges are bit-identical to the reference's for the same projection.
//
// Every LSD pass is reduce-then-scan over a fixed number of spans (contiguous runs of 2048-item
// blocks, one span per CTA, four CTAs per SM): an upsweep counts each span's digits (in a small
// frame the preprocess and the expansion count the first depth and tile passes as they write the
// keys, and those passes have no upsweep), one CTA per digit scans that digit's counts over the
// spans, and a downsweep re-reads each block, ranks it within each warp (ballots on the
// latency-bound passes of at most 4M items; match_any in 512-thread CTAs over 4096-item chunks on
// the large passes of a batch, whose longer digit runs fill more of each written sector), and
// scatters it through shared memory so global writes are contiguous per digit.
// No CTA ever waits on another, so there is no spin loop anywhere in the sort; item counts that
// are known only on the device (visible entries, pairs) are read from the control block, and the
// grids are sized for the capacity.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 8;
constexpr int kBlockItems = kThreads * kItems;  // items one CTA ranks at a time
constexpr int kMaxSpans = 4 * 148;
constexpr int kMaxRadixBits = 9;  // digit widths: 8 or 9 bits
constexpr unsigned kBallotRankMax = 1u << 22;  // passes up to this many items rank with ballots
constexpr int kScanItems = 4;
constexpr int kScanBlock = kThreads * kScanItems;
constexpr int kExpandItems = 8;
constexpr int kExpandChunk = kThreads * kExpandItems;  // pairs per expansion CTA
constexpr unsigned kBinMaxTiles = 4096;                 // global tiles of a frame the one-pass tile binning takes
constexpr unsigned kBinMaxPairs = 1u << 24;             // and its pair capacity (the count matrix grows with it)
static_assert(kBlockItems == kSortBlockItems, "an LSD block is kSortBlockItems items");
static_assert(kExpandChunk == kSortBlockItems, "an expansion CTA writes exactly one LSD block of pairs");

// Clears the control block, `zero_words` words at `zero` (the first pass's digit counts) and
// `ranges` tile ranges (a tile without pairs keeps [0, 0)). Clearing the ranges here rather than
// with a memset ahead of the frame keeps one more operation off the frame's critical path.
__global__ void frame_begin_kernel(Ctrl* ctrl, unsigned* __restrict__ zero, unsigned zero_words,
                                   uint2* __restrict__ range, unsigned ranges) {
    chain_entry();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctrl->sticky_flags |= ctrl->flags;
        if (ctrl->pair_total > ctrl->max_pair_total) ctrl->max_pair_total = ctrl->pair_total;
        ctrl->pair_total = 0;
        ctrl->vis_count = 0;
        ctrl->flags = 0;
        ctrl->sort_barrier = 0;
    }
    const unsigned stride = gridDim.x * blockDim.x, first = blockIdx.x * blockDim.x + threadIdx.x;
    for (unsigned i = first; i < zero_words; i += stride) zero[i] = 0;  // at most 512 x 592 words
    // 64-bit index: a tile count within one stride of 2^32 must not wrap the loop.
    for (unsigned long long i = first; i < ranges; i += stride) range[i] = make_uint2(0u, 0u);
}

// Copies `words` 32-bit words of a frame's tables from page-locked host memory (read through the
// device's mapping, uncached, so that a staging buffer rewritten between launches or graph replays
// is read afresh) into device memory: the frame's first chained kernel, where a host-to-device copy
// would be one more non-kernel operation between two frames' kernels.
__global__ void upload_kernel(const unsigned* __restrict__ src, unsigned* __restrict__ dst, unsigned words) {
    chain_entry();
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < words) dst[i] = __ldcv(src + i);
}

// upload_kernel and frame_begin_kernel as one launch (the frame's first): threads copy the tables
// and clear the control block, the counts and the ranges side by side. One kernel fewer at the
// head of every frame's chain.
__global__ void frame_start_kernel(const unsigned* __restrict__ src, unsigned* __restrict__ dst, unsigned words,
                                   Ctrl* ctrl, unsigned* __restrict__ zero, unsigned zero_words,
                                   uint2* __restrict__ range, unsigned ranges) {
    chain_entry();
    const unsigned stride = gridDim.x * blockDim.x, first = blockIdx.x * blockDim.x + threadIdx.x;
    for (unsigned i = first; i < words; i += stride) dst[i] = __ldcv(src + i);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctrl->sticky_flags |= ctrl->flags;
        if (ctrl->pair_total > ctrl->max_pair_total) ctrl->max_pair_total = ctrl->pair_total;
        ctrl->pair_total = 0;
        ctrl->vis_count = 0;
        ctrl->flags = 0;
        ctrl->sort_barrier = 0;
    }
    for (unsigned i = first; i < zero_words; i += stride) zero[i] = 0;
    for (unsigned long long i = first; i < ranges; i += stride) range[i] = make_uint2(0u, 0u);
}

// Copies the control block into `host` (page-locked host memory this device maps) and clears its
// flags, so that the next frame_begin does not fold flags the host has already read into the
// sticky ones. One chained launch where a device-to-host copy and a memset would be two
// operations after the frame's last kernel.
__global__ void publish_ctrl_kernel(Ctrl* ctrl, Ctrl* host) {
    chain_entry();
    *host = *ctrl;
    ctrl->flags = 0;
}

// Items of this frame's pass; false when the frame overflowed (nothing after duplication runs).
__device__ __forceinline__ bool pass_items(const Ctrl* ctrl, SortCount src, unsigned fixed, unsigned capacity,
                                           unsigned& n) {
    if (ctrl->flags & kFlagOverflow) return false;
    if (src == SortCount::kFixed) {
        n = fixed;
    } else if (src == SortCount::kVisible) {
        n = ctrl->vis_count;
    } else {
        const unsigned long long p = ctrl->pair_total;
        if (p > capacity) return false;
        n = static_cast<unsigned>(p);
    }
    return true;
}

// Blocks [t0, t1) of the n items that span b of `spans` covers.
__device__ __forceinline__ void span_blocks(unsigned n, unsigned spans, unsigned b, unsigned& t0, unsigned& t1) {
    const unsigned long long T = (static_cast<unsigned long long>(n) + kBlockItems - 1) / kBlockItems;
    t0 = static_cast<unsigned>(T * b / spans);
    t1 = static_cast<unsigned>(T * (b + 1) / spans);
}

// Block t: lane `lane` of warp `warp` holds items base + warp*kItems*32 + k*32 + lane, so (k, lane)
// order within a warp is ascending position. fetch_block issues the loads of the keys (and values
// with kVals, unless kMasked: there the value is the position); block_digits then gives each item
// its digit dg (R digits), or R for no item. The two are apart so that a kernel walking several
// blocks can issue the next block's loads while it still works on the current one.
template <bool kMasked, bool kVals>
__device__ __forceinline__ void fetch_block(const unsigned* __restrict__ keys_in, const unsigned* __restrict__ vals_in,
                                            unsigned t, unsigned n, int warp, int lane, unsigned (&key)[kItems],
                                            unsigned (&val)[kItems]) {
    const unsigned long long wbase = static_cast<unsigned long long>(t) * kBlockItems + warp * (kItems * 32) + lane;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const unsigned long long idx = wbase + k * 32;
        const bool valid = idx < n;
        key[k] = valid ? keys_in[idx] : 0u;
        if (!kMasked && kVals) val[k] = valid ? vals_in[idx] : 0u;
    }
}

template <int R, bool kMasked>
__device__ __forceinline__ void block_digits(unsigned t, unsigned n, int shift, int warp, int lane,
                                             const unsigned (&key)[kItems], unsigned (&val)[kItems],
                                             unsigned (&dg)[kItems]) {
    const unsigned long long wbase = static_cast<unsigned long long>(t) * kBlockItems + warp * (kItems * 32) + lane;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const unsigned long long idx = wbase + k * 32;
        bool valid = idx < n;
        if (kMasked) {
            valid = valid && key[k] != kCulledKey;
            val[k] = static_cast<unsigned>(idx);
        }
        dg[k] = valid ? ((key[k] >> shift) & (R - 1)) : R;
    }
}

// Digit counts of each span: counts[d * spans + b]. Counting needs no ranks, so each warp adds
// into its own shared histogram with plain atomics (lanes of one warp that share a digit are
// serialised by the hardware, which costs less than resolving peers first).
template <int BITS, bool kMasked>
__global__ void __launch_bounds__(kThreads) upsweep_kernel(const unsigned* __restrict__ keys_in, SortCount src,
                                                           unsigned fixed, unsigned capacity, int shift,
                                                           unsigned spans, unsigned* __restrict__ counts,
                                                           const Ctrl* __restrict__ ctrl) {
    chain_entry();
    constexpr int R = 1 << BITS;
    __shared__ unsigned s_h[kWarps][R];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned n;
    if (!pass_items(ctrl, src, fixed, capacity, n)) return;
    unsigned t0, t1;
    span_blocks(n, spans, blockIdx.x, t0, t1);
    unsigned key[kItems], val[kItems], dg[kItems];
    if (t0 < t1) fetch_block<kMasked, false>(keys_in, nullptr, t0, n, warp, lane, key, val);
    for (int d = tid; d < R; d += kThreads)
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s_h[w][d] = 0;
    __syncthreads();
    for (unsigned t = t0; t < t1; ++t) {
        block_digits<R, kMasked>(t, n, shift, warp, lane, key, val, dg);
        if (t + 1 < t1) fetch_block<kMasked, false>(keys_in, nullptr, t + 1, n, warp, lane, key, val);  // in flight
#pragma unroll
        for (int k = 0; k < kItems; ++k)
            if (dg[k] < R) atomicAdd(&s_h[warp][dg[k]], 1u);
    }
    __syncthreads();
    for (int d = tid; d < R; d += kThreads) {
        unsigned c = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) c += s_h[w][d];
        counts[static_cast<size_t>(d) * spans + blockIdx.x] = c;
    }
}

// One CTA per digit: exclusive scan of the digit's counts over the spans, in place, and its total.
// All CTAs together also clear `zero_words` words at `zero`: the next pass's counts, which the
// downsweep after this kernel accumulates (their previous reader, the downsweep before, is done).
__global__ void __launch_bounds__(kThreads) span_scan_kernel(unsigned* __restrict__ counts, unsigned* __restrict__ totals,
                                                             unsigned spans, SortCount src, unsigned fixed,
                                                             unsigned capacity, const Ctrl* __restrict__ ctrl,
                                                             unsigned* __restrict__ zero, unsigned zero_words) {
    chain_entry();
    __shared__ unsigned s_tmp[kWarps];
    for (unsigned i = blockIdx.x * kThreads + threadIdx.x; i < zero_words; i += gridDim.x * kThreads) zero[i] = 0;
    unsigned n;
    if (!pass_items(ctrl, src, fixed, capacity, n)) return;
    unsigned* row = counts + static_cast<size_t>(blockIdx.x) * spans;
    unsigned carry = 0;
    for (unsigned b0 = 0; b0 < spans; b0 += kThreads) {  // spans <= kMaxSpans: at most 3 rounds
        const unsigned b = b0 + threadIdx.x;
        const unsigned c = b < spans ? row[b] : 0u;
        unsigned tot;
        const unsigned ex = block_excl_scan<kThreads>(c, s_tmp, tot);
        if (b < spans) row[b] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// The downsweep of a pass of at most kBallotRankMax items (larger ones take downsweep_wide_kernel):
// ranks, scatters and writes each block of the span. The masked pass publishes the visible count.
// Thread tid owns digits [tid * DPT, tid * DPT + DPT) in the per-digit phases, so a block scan over
// the threads' sums is a scan in digit order. Four CTAs per SM (64 registers). A lane's peers (the
// lanes holding the same digit) come from BITS + 1 ballots (one per digit bit, one for validity):
// more instructions than __match_any_sync but a shorter dependent chain, which wins where a pass
// is latency-bound (0.336 -> 0.330 ms per 740k frame).
template <int BITS, bool kMasked, bool kKeysOut>
__global__ void __launch_bounds__(kThreads, 4) downsweep_kernel(const unsigned* __restrict__ keys_in,
                                                                const unsigned* __restrict__ vals_in,
                                                                unsigned* __restrict__ keys_out,
                                                                unsigned* __restrict__ vals_out, SortCount src,
                                                                unsigned fixed, unsigned capacity, int shift,
                                                                unsigned spans, const unsigned* __restrict__ counts,
                                                                const unsigned* __restrict__ totals, Ctrl* ctrl) {
    chain_entry();
    constexpr int R = 1 << BITS;
    constexpr int DPT = R / kThreads;  // digits per thread: 1 (8-bit digits) or 2 (9-bit)
    static_assert(DPT * kThreads == R, "digit count must be a multiple of the block size");
    __shared__ unsigned s_keys[kBlockItems];
    __shared__ unsigned s_vals[kBlockItems];
    __shared__ unsigned s_wh[kWarps][R];
    __shared__ unsigned s_dstart[R];
    __shared__ unsigned s_gbase[R];
    __shared__ unsigned s_tmp[kWarps];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned n;
    if (!pass_items(ctrl, src, fixed, capacity, n)) return;
    unsigned t0, t1;
    span_blocks(n, spans, blockIdx.x, t0, t1);
    if (t0 == t1 && !(kMasked && blockIdx.x == 0)) return;  // an empty span (span 0 publishes the count)
    const int d0 = tid * DPT;
    unsigned run[DPT];  // next global output position of each of this thread's digits
    {
        unsigned tot[DPT], sum = 0;
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
            tot[j] = totals[d0 + j];
            sum += tot[j];
        }
        unsigned all;
        unsigned g = block_excl_scan<kThreads>(sum, s_tmp, all);
        if (kMasked && blockIdx.x == 0 && tid == 0) ctrl->vis_count = all;
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
            run[j] = g + counts[static_cast<size_t>(d0 + j) * spans + blockIdx.x];
            g += tot[j];
        }
    }
    const unsigned lt = lanemask_lt();

    for (unsigned t = t0; t < t1; ++t) {
#pragma unroll
        for (int j = 0; j < DPT; ++j)
#pragma unroll
            for (int w = 0; w < kWarps; ++w) s_wh[w][d0 + j] = 0;
        unsigned key[kItems], val[kItems], dg[kItems];
        fetch_block<kMasked, true>(keys_in, vals_in, t, n, warp, lane, key, val);
        block_digits<R, kMasked>(t, n, shift, warp, lane, key, val, dg);
        __syncthreads();
        // Warp-level stable ranking: items in (k, lane) order, i.e. ascending position.
        unsigned rank[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            unsigned peers = 0xFFFFFFFFu;
#pragma unroll
            for (int b = 0; b <= BITS; ++b) {
                const bool bit = (dg[k] >> b) & 1u;
                const unsigned vb = __ballot_sync(0xFFFFFFFFu, bit);
                peers &= bit ? vb : ~vb;
            }
            const unsigned cnt = dg[k] < R ? s_wh[warp][dg[k]] : 0u;
            rank[k] = cnt + __popc(peers & lt);
            __syncwarp();
            if (dg[k] < R && lane == 31 - __clz(peers)) s_wh[warp][dg[k]] = cnt + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // Per digit: the offset of each warp's run, the block's digit count and the block-local start.
        unsigned cnt[DPT], sum = 0;
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
            cnt[j] = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const unsigned c = s_wh[w][d0 + j];
                s_wh[w][d0 + j] = cnt[j];
                cnt[j] += c;
            }
            sum += cnt[j];
        }
        unsigned block_total;
        unsigned dstart = block_excl_scan<kThreads>(sum, s_tmp, block_total);
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
            s_dstart[d0 + j] = dstart;
            s_gbase[d0 + j] = run[j] - dstart;
            run[j] += cnt[j];
            dstart += cnt[j];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (dg[k] < R) {
                const unsigned pos = s_dstart[dg[k]] + s_wh[warp][dg[k]] + rank[k];
                s_keys[pos] = key[k];
                s_vals[pos] = val[k];
            }
        }
        __syncthreads();
        for (unsigned p = tid; p < block_total; p += kThreads) {
            const unsigned k = s_keys[p];
            const unsigned g = s_gbase[(k >> shift) & (R - 1)] + p;
            if (kKeysOut) keys_out[g] = k;
            vals_out[g] = s_vals[p];
        }
        __syncthreads();
    }
}

// The downsweep of a large pass (match_any ranking) in 512-thread CTAs over chunks of
// kWideItems = 4096 items: the same span, digit offsets and stable order as downsweep_kernel,
// with each chunk's digit runs twice as long (fuller 32-byte sectors in the scattered writes) and
// half the barriers per item. Thread tid owns digit tid in the per-digit phases (threads past R
// own none). Shared memory (dynamic): the chunk's keys and values, the warps' digit counts, the
// digits' chunk starts and global bases.
constexpr int kWideThreads = 512;
constexpr int kWideWarps = kWideThreads / 32;
constexpr int kWideItems = kWideThreads * kItems;

__host__ __device__ constexpr size_t wide_smem_bytes(int bits) {
    return (2 * static_cast<size_t>(kWideItems) + (kWideWarps + 2) * (static_cast<size_t>(1) << bits)) *
           sizeof(unsigned);
}

template <int BITS, bool kMasked, bool kKeysOut>
__global__ void __launch_bounds__(kWideThreads, 2) downsweep_wide_kernel(const unsigned* __restrict__ keys_in,
                                                                         const unsigned* __restrict__ vals_in,
                                                                         unsigned* __restrict__ keys_out,
                                                                         unsigned* __restrict__ vals_out, SortCount src,
                                                                         unsigned fixed, unsigned capacity, int shift,
                                                                         unsigned spans,
                                                                         const unsigned* __restrict__ counts,
                                                                         const unsigned* __restrict__ totals, Ctrl* ctrl) {
    chain_entry();
    constexpr int R = 1 << BITS;
    static_assert(R <= kWideThreads, "one digit per thread at most");
    extern __shared__ unsigned s_dyn[];
    unsigned* s_keys = s_dyn;                   // [kWideItems]
    unsigned* s_vals = s_keys + kWideItems;     // [kWideItems]
    unsigned* s_wh = s_vals + kWideItems;       // [kWideWarps][R]
    unsigned* s_dstart = s_wh + kWideWarps * R; // [R]
    unsigned* s_gbase = s_dstart + R;           // [R]
    __shared__ unsigned s_tmp[kWideWarps];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned n;
    if (!pass_items(ctrl, src, fixed, capacity, n)) return;
    unsigned t0, t1;
    span_blocks(n, spans, blockIdx.x, t0, t1);
    if (t0 == t1 && !(kMasked && blockIdx.x == 0)) return;  // an empty span (span 0 publishes the count)
    // The span's items: [i0, i1).
    const unsigned long long i0 = static_cast<unsigned long long>(t0) * kBlockItems;
    const unsigned long long i1 = min(static_cast<unsigned long long>(t1) * kBlockItems,
                                      static_cast<unsigned long long>(n));
    const bool own = tid < R;
    unsigned run = 0;  // next global output position of the thread's digit
    {
        const unsigned tot = own ? totals[tid] : 0u;
        unsigned all;
        const unsigned g = block_excl_scan<kWideThreads>(tot, s_tmp, all);
        if (kMasked && blockIdx.x == 0 && tid == 0) ctrl->vis_count = all;
        if (own) run = g + counts[static_cast<size_t>(tid) * spans + blockIdx.x];
    }
    const unsigned lt = lanemask_lt();

    unsigned key[kItems], val[kItems], dg[kItems];
    // Item (warp, k, lane) of the chunk at c: c + warp * kItems * 32 + k * 32 + lane.
    const auto fetch = [&](unsigned long long c) {
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned long long idx = c + warp * (kItems * 32) + k * 32 + lane;
            const bool valid = idx < i1;
            key[k] = valid ? keys_in[idx] : 0u;
            if (!kMasked) val[k] = valid ? vals_in[idx] : 0u;
        }
    };
    if (i0 < i1) fetch(i0);
    for (unsigned long long c = i0; c < i1; c += kWideItems) {
        for (int i = tid; i < kWideWarps * R; i += kWideThreads) s_wh[i] = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned long long idx = c + warp * (kItems * 32) + k * 32 + lane;
            bool valid = idx < i1;
            if (kMasked) {
                valid = valid && key[k] != kCulledKey;
                val[k] = static_cast<unsigned>(idx);
            }
            dg[k] = valid ? ((key[k] >> shift) & (R - 1)) : R;
        }
        __syncthreads();
        unsigned rank[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, dg[k]);
            const unsigned cnt = dg[k] < R ? s_wh[warp * R + dg[k]] : 0u;
            rank[k] = cnt + __popc(peers & lt);
            __syncwarp();
            if (dg[k] < R && lane == 31 - __clz(peers)) s_wh[warp * R + dg[k]] = cnt + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        unsigned cnt = 0;
        if (own)
#pragma unroll
            for (int w = 0; w < kWideWarps; ++w) {
                const unsigned c2 = s_wh[w * R + tid];
                s_wh[w * R + tid] = cnt;
                cnt += c2;
            }
        unsigned chunk_total;
        const unsigned dstart = block_excl_scan<kWideThreads>(cnt, s_tmp, chunk_total);
        if (own) {
            s_dstart[tid] = dstart;
            s_gbase[tid] = run - dstart;
            run += cnt;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (dg[k] < R) {
                const unsigned pos = s_dstart[dg[k]] + s_wh[warp * R + dg[k]] + rank[k];
                s_keys[pos] = key[k];
                s_vals[pos] = val[k];
            }
        }
        __syncthreads();
        if (c + kWideItems < i1) fetch(c + kWideItems);  // in flight while this chunk is written out
        for (unsigned p = tid; p < chunk_total; p += kWideThreads) {
            const unsigned k = s_keys[p];
            const unsigned g = s_gbase[(k >> shift) & (R - 1)] + p;
            if (kKeysOut) keys_out[g] = k;
            vals_out[g] = s_vals[p];
        }
        __syncthreads();
    }
}

__device__ __forceinline__ unsigned rect_area(unsigned long long r) {
    const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu, y1 = r >> 48;
    return (x1 - x0 + 1) * (y1 - y0 + 1);
}

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v, unsigned long long* s_tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) s_tmp[warp] = v;
    __syncthreads();
    unsigned long long s = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += s_tmp[w];
    __syncthreads();
    return s;
}

// Entries [V b / spans, V (b+1) / spans) of the depth-sorted list: gathers each one's rectangle
// into sorted order, records its sorted position (for the adjoint; rank may be NULL), and sums
// its tile counts. The gathers are random, so each thread keeps kGather of them in flight.
constexpr int kGather = 8;
__global__ void __launch_bounds__(kThreads) pair_count_kernel(const unsigned* __restrict__ sorted_idx,
                                                              const unsigned long long* __restrict__ rect16,
                                                              const Ctrl* __restrict__ ctrl, unsigned spans,
                                                              unsigned* __restrict__ rank,
                                                              unsigned long long* __restrict__ rect_sorted,
                                                              unsigned long long* __restrict__ span_sum) {
    chain_entry();
    __shared__ unsigned long long s_tmp[kWarps];
    const unsigned long long V = ctrl->vis_count;
    const unsigned lo = static_cast<unsigned>(V * blockIdx.x / spans);
    const unsigned hi = static_cast<unsigned>(V * (blockIdx.x + 1) / spans);
    unsigned long long sum = 0;
    for (unsigned j0 = lo + threadIdx.x; j0 < hi; j0 += kThreads * kGather) {
        unsigned g[kGather];
        unsigned long long r[kGather];
#pragma unroll
        for (int k = 0; k < kGather; ++k) {
            const unsigned j = j0 + k * kThreads;
            g[k] = j < hi ? sorted_idx[j] : 0u;
        }
#pragma unroll
        for (int k = 0; k < kGather; ++k) {
            const unsigned j = j0 + k * kThreads;
            r[k] = j < hi ? rect16[g[k]] : 0ull;
        }
#pragma unroll
        for (int k = 0; k < kGather; ++k) {
            const unsigned j = j0 + k * kThreads;
            if (j < hi) {
                if (rank) rank[g[k]] = j;
                rect_sorted[j] = r[k];
                sum += rect_area(r[k]);
            }
        }
    }
    sum = block_sum_u64(sum, s_tmp);
    if (threadIdx.x == 0) span_sum[blockIdx.x] = sum;
}

// Exclusive pair offset of every depth-sorted entry, and, for every chunk of kExpandChunk pairs,
// the entry that holds the chunk's first pair. The last span stores the frame's pair total and
// flags an overflow of the pair capacity.
__global__ void __launch_bounds__(kThreads) pair_offsets_kernel(const unsigned long long* __restrict__ rect_sorted,
                                                                Ctrl* ctrl, unsigned spans, unsigned capacity,
                                                                const unsigned long long* __restrict__ span_sum,
                                                                unsigned* __restrict__ offs,
                                                                unsigned* __restrict__ chunk_start) {
    chain_entry();
    __shared__ unsigned long long s_tmp64[kWarps];
    __shared__ unsigned s_tmp[kWarps];
    const unsigned b = blockIdx.x;
    unsigned long long before = 0;
    for (unsigned k = threadIdx.x; k < b; k += kThreads) before += span_sum[k];
    unsigned long long base = block_sum_u64(before, s_tmp64);
    if (b == spans - 1 && threadIdx.x == 0) {
        const unsigned long long P = base + span_sum[b];
        ctrl->pair_total = P;
        if (P > capacity) atomicOr(&ctrl->flags, kFlagOverflow);
    }
    if (base > capacity) return;  // the frame overflows: nothing reads these offsets
    const unsigned long long V = ctrl->vis_count;
    const unsigned lo = static_cast<unsigned>(V * b / spans);
    const unsigned hi = static_cast<unsigned>(V * (b + 1) / spans);
    const unsigned long long last_chunk = (static_cast<unsigned long long>(capacity) + kExpandChunk - 1) / kExpandChunk;
    for (unsigned j0 = lo; j0 < hi; j0 += kScanBlock) {
        unsigned cnt[kScanItems];
        unsigned thread_total = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const unsigned j = j0 + threadIdx.x * kScanItems + k;
            cnt[k] = j < hi ? rect_area(rect_sorted[j]) : 0u;
            thread_total += cnt[k];
        }
        unsigned tile_total;
        const unsigned ex = block_excl_scan<kThreads>(thread_total, s_tmp, tile_total);
        unsigned long long o = base + ex;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const unsigned j = j0 + threadIdx.x * kScanItems + k;
            if (j < hi && o <= capacity) {
                offs[j] = static_cast<unsigned>(o);
                for (unsigned long long c = (o + kExpandChunk - 1) / kExpandChunk;
                     c * kExpandChunk < o + cnt[k] && c <= last_chunk; ++c)
                    chunk_start[c] = j;
            }
            o += cnt[k];
        }
        base += tile_total;
    }
}

// The kExpandItems pairs from position p0 (< P) of one expansion CTA (the CTA's entries staged in
// shared memory); hist: also counts each pair's digit there.
__device__ __forceinline__ void expand_run(unsigned p0, unsigned P, unsigned G, const unsigned* s_off,
                                           const unsigned* s_idx, const unsigned* s_org, const unsigned short* s_w,
                                           const unsigned short* s_tx, unsigned* __restrict__ pair_key,
                                           unsigned* __restrict__ pair_val, unsigned* hist, unsigned shift,
                                           unsigned mask) {
    unsigned lo = 0, hi = G - 1;  // last k with s_off[k] <= p0
    while (lo < hi) {
        const unsigned mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= p0) lo = mid;
        else hi = mid - 1;
    }
    unsigned w = s_w[lo], tx = s_tx[lo], org = s_org[lo], idx = s_idx[lo], next = s_off[lo + 1];
    const unsigned kk = p0 - s_off[lo];
    unsigned row = kk / w, col = kk - row * w;
    unsigned key[kExpandItems], val[kExpandItems];
#pragma unroll
    for (int i = 0; i < kExpandItems; ++i) {
        const unsigned p = p0 + i;
        key[i] = org + row * tx + col;
        val[i] = idx;
        if (p + 1 == next && p + 1 < P) {  // the next pair starts the next entry
            ++lo;
            w = s_w[lo];
            tx = s_tx[lo];
            org = s_org[lo];
            idx = s_idx[lo];
            next = s_off[lo + 1];
            row = 0;
            col = 0;
        } else if (++col == w) {
            col = 0;
            ++row;
        }
    }
    if (p0 + kExpandItems <= P) {
        uint4* k4 = reinterpret_cast<uint4*>(pair_key + p0);
        uint4* v4 = reinterpret_cast<uint4*>(pair_val + p0);
        k4[0] = make_uint4(key[0], key[1], key[2], key[3]);
        k4[1] = make_uint4(key[4], key[5], key[6], key[7]);
        v4[0] = make_uint4(val[0], val[1], val[2], val[3]);
        v4[1] = make_uint4(val[4], val[5], val[6], val[7]);
    } else {
#pragma unroll
        for (int i = 0; i < kExpandItems; ++i)
            if (p0 + i < P) {
                pair_key[p0 + i] = key[i];
                pair_val[p0 + i] = val[i];
            }
    }
    if (hist)
#pragma unroll
        for (int i = 0; i < kExpandItems; ++i)
            if (p0 + i < P) atomicAdd(&hist[(key[i] >> shift) & mask], 1u);
}

// Expands the depth-sorted list into (tile, entry) pairs: CTA b writes pairs
// [b * kExpandChunk, (b + 1) * kExpandChunk), each thread kExpandItems consecutive ones (one
// search for its first pair, then a walk), row-major over each rectangle as gpu_render.cu:155-160
// does. Tile ids are global over the batch. With first.counts set, the CTA also adds its pairs'
// digits to the first tile pass's counts: its pairs are exactly LSD block b, all in one span, so
// it counts them in shared memory and adds each non-zero digit count once. With bin_counts set
// instead (the one-pass tile binning), it counts its pairs per tile and writes row b of the
// (block, tile) matrix, bin_tiles words, zeros included. The counts live in dynamic shared memory.
__global__ void __launch_bounds__(kThreads) expand_kernel(const unsigned* __restrict__ sorted_idx,
                                                          const unsigned long long* __restrict__ rect_sorted,
                                                          const unsigned* __restrict__ offs,
                                                          const unsigned* __restrict__ chunk_start,
                                                          const Ctrl* __restrict__ ctrl, unsigned capacity,
                                                          BatchTables tables, unsigned* __restrict__ pair_key,
                                                          unsigned* __restrict__ pair_val, PassCounts first,
                                                          unsigned* __restrict__ bin_counts, unsigned bin_tiles) {
    chain_entry();
    __shared__ unsigned s_off[kExpandChunk + 2];
    __shared__ unsigned s_idx[kExpandChunk + 1];
    __shared__ unsigned s_org[kExpandChunk + 1];       // global tile of the rectangle's corner
    __shared__ unsigned short s_w[kExpandChunk + 1];   // rectangle width in tiles
    __shared__ unsigned short s_tx[kExpandChunk + 1];  // tiles per row of the entry's view
    extern __shared__ unsigned s_hist[];               // digit (or tile) counts: launched with their size
    const int tid = threadIdx.x;
    if (ctrl->flags & kFlagOverflow) return;
    const unsigned long long P64 = ctrl->pair_total;
    if (P64 > capacity) return;
    const unsigned P = static_cast<unsigned>(P64);
    const unsigned base = blockIdx.x * kExpandChunk;
    if (base >= P) return;
    const unsigned V = ctrl->vis_count;
    const unsigned j0 = chunk_start[blockIdx.x];
    const unsigned j1 = base + kExpandChunk < P ? chunk_start[blockIdx.x + 1] : V - 1;
    const unsigned G = j1 - j0 + 1;  // <= kExpandChunk + 1: every entry owns at least one pair
    for (unsigned k = tid; k < G; k += kThreads) {
        const unsigned long long r = rect_sorted[j0 + k];
        const unsigned e = sorted_idx[j0 + k];
        const unsigned v = find_segment(tables.entry_base, tables.n_views, e);
        const unsigned tx = tables.tiles_x[v];
        const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu;
        s_off[k] = offs[j0 + k];
        s_idx[k] = e;
        s_org[k] = tables.tile_base[v] + y0 * tx + x0;
        s_w[k] = static_cast<unsigned short>(x1 - x0 + 1);
        s_tx[k] = static_cast<unsigned short>(tx);
    }
    if (tid == 0) s_off[G] = j1 + 1 < V ? offs[j1 + 1] : P;
    const bool bins = bin_counts != nullptr;
    const bool count = first.counts != nullptr || bins;
    const unsigned hist_words = bins ? bin_tiles : first.mask + 1;
    if (count)
        for (unsigned d = tid; d < hist_words; d += kThreads) s_hist[d] = 0;
    __syncthreads();

    const unsigned p0 = base + tid * kExpandItems;
    if (p0 < P) expand_run(p0, P, G, s_off, s_idx, s_org, s_w, s_tx, pair_key, pair_val, count ? s_hist : nullptr,
                           bins ? 0u : first.shift, bins ? 0xFFFFFFFFu : first.mask);
    if (!count) return;
    __syncthreads();
    if (bins) {  // this block's row of the (block, tile) count matrix, every cell written
        unsigned* row = bin_counts + static_cast<size_t>(blockIdx.x) * bin_tiles;
        for (unsigned t = tid; t < bin_tiles; t += kThreads) row[t] = s_hist[t];
        return;
    }
    const unsigned span = span_of(base, first.spans, (P + kSortBlockItems - 1) / kSortBlockItems);
    for (unsigned d = tid; d <= first.mask; d += kThreads)
        if (s_hist[d]) atomicAdd(&first.counts[d * first.digit_stride + span * first.span_stride], s_hist[d]);
}

// ranges[tile] = [first, last + 1) over the sorted tile keys; four keys per thread and step.
__global__ void __launch_bounds__(kThreads) ranges_kernel(const unsigned* __restrict__ keys,
                                                          const Ctrl* __restrict__ ctrl, unsigned capacity,
                                                          uint2* __restrict__ ranges) {
    chain_entry();
    if (ctrl->flags & kFlagOverflow) return;
    const unsigned long long pt = ctrl->pair_total;
    if (pt > capacity) return;
    const unsigned P = static_cast<unsigned>(pt);
    for (unsigned long long g = static_cast<unsigned long long>(blockIdx.x) * kThreads + threadIdx.x; g * 4 < P;
         g += static_cast<unsigned long long>(gridDim.x) * kThreads) {
        const unsigned i0 = static_cast<unsigned>(g * 4);
        unsigned k[4];
        if (i0 + 4 <= P) {
            const uint4 q = *reinterpret_cast<const uint4*>(keys + i0);
            k[0] = q.x;
            k[1] = q.y;
            k[2] = q.z;
            k[3] = q.w;
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) k[i] = i0 + i < P ? keys[i0 + i] : 0u;
        }
        unsigned prev = i0 > 0 ? keys[i0 - 1] : 0u;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const unsigned idx = i0 + i;
            if (idx >= P) break;
            const unsigned tile = k[i];
            if (idx == 0) {
                ranges[tile].x = 0;
            } else if (prev != tile) {
                ranges[prev].y = idx;
                ranges[tile].x = idx;
            }
            if (idx == P - 1) ranges[tile].y = P;
            prev = tile;
        }
    }
}

// ---- one-pass tile binning --------------------------------------------------------------------
// Where a frame has at most kBinMaxTiles global tiles, the tile order is made in one stable
// counting pass over the tile id instead of LSD passes over its digits: the expansion writes the
// pairs in depth order and each block's per-tile counts (one row of a blocks x tiles matrix);
// bin_scan turns every tile's column into the blocks' offsets within the tile and, in its last
// CTA, the tiles' starts and ranges; bin_scatter sorts each block by tile in shared memory (two
// stable 6-bit passes) and writes every pair to its tile's start + its block's offset + its rank in
// the block. Stability at both levels keeps each tile's pairs in depth order: the reference's
// order, as the LSD passes give it.
constexpr int kBinLocalBits = 6;
constexpr int kBinLocalR = 1 << kBinLocalBits;
constexpr int kBinScanThreads = 1024;
constexpr int kBinScanGroups = kBinScanThreads / 32;  // row groups per 32-tile column strip

__device__ __forceinline__ bool frame_pairs(const Ctrl* ctrl, unsigned capacity, unsigned& P) {
    if (ctrl->flags & kFlagOverflow) return false;
    const unsigned long long pt = ctrl->pair_total;
    if (pt > capacity) return false;
    P = static_cast<unsigned>(pt);
    return true;
}

// CTA c owns tiles [32 c, 32 c + 32): 32 groups of warps each sum a contiguous run of the blocks'
// rows (one coalesced 128-byte read per row), the group sums are scanned, and each group writes
// its rows' exclusive running sums back in place. The tiles' totals go to tile_start; the last CTA
// to finish (a ticket on the control block: no CTA waits for another) scans them into the tiles'
// starts and writes every tile's range ([0, 0) for a tile without pairs, as the reference's
// cleared ranges are). (Eight-tile strips of 512 threads, every row load of a group in flight at
// once, measured slower in the frame: 0.122 against 0.119 ms of sort.)
__global__ void __launch_bounds__(kBinScanThreads) bin_scan_kernel(unsigned* __restrict__ counts, unsigned tiles,
                                                                   unsigned* __restrict__ tile_start,
                                                                   uint2* __restrict__ ranges, Ctrl* ctrl,
                                                                   unsigned capacity) {
    chain_entry();
    __shared__ unsigned s_part[kBinScanGroups][33];
    __shared__ unsigned s_tmp[kBinScanThreads / 32];
    __shared__ unsigned s_last;
    unsigned P;
    if (!frame_pairs(ctrl, capacity, P)) return;
    const unsigned blocks = (P + kBlockItems - 1) / kBlockItems;
    const int tid = threadIdx.x, lane = tid & 31, g = tid >> 5;
    const unsigned t = blockIdx.x * 32 + lane;
    const unsigned r0 = static_cast<unsigned>(static_cast<unsigned long long>(blocks) * g / kBinScanGroups);
    const unsigned r1 = static_cast<unsigned>(static_cast<unsigned long long>(blocks) * (g + 1) / kBinScanGroups);
    unsigned sum = 0;
    if (t < tiles)
#pragma unroll 8
        for (unsigned r = r0; r < r1; ++r) sum += counts[static_cast<size_t>(r) * tiles + t];
    s_part[g][lane] = sum;
    __syncthreads();
    unsigned run = 0;
    for (int k = 0; k < g; ++k) run += s_part[k][lane];
    if (t < tiles) {
        if (g == kBinScanGroups - 1) tile_start[t] = run + sum;  // the tile's total, for the last CTA
#pragma unroll 8
        for (unsigned r = r0; r < r1; ++r) {
            unsigned* cell = counts + static_cast<size_t>(r) * tiles + t;
            const unsigned c = *cell;
            *cell = run;
            run += c;
        }
    }
    // Every thread's fence, not only the writers' of tile_start: measured 1 us faster per frame.
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(&ctrl->sort_barrier, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // The last CTA: tiles <= kBinMaxTiles = 4 per thread, in order.
    constexpr int kPer = kBinMaxTiles / kBinScanThreads;
    unsigned tot[kPer], own = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const unsigned tt = tid * kPer + k;
        tot[k] = tt < tiles ? __ldcg(tile_start + tt) : 0u;
        own += tot[k];
    }
    unsigned all;
    unsigned start = block_excl_scan<kBinScanThreads>(own, s_tmp, all);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const unsigned tt = tid * kPer + k;
        if (tt < tiles) {
            tile_start[tt] = start;
            ranges[tt] = tot[k] ? make_uint2(start, start + tot[k]) : make_uint2(0u, 0u);
        }
        start += tot[k];
    }
}

// Block b (kBlockItems pairs of the depth-ordered list) sorted stably by tile in shared memory and
// written out in tile order. bits: bits of the largest tile id (1..12); one local pass for up to 6,
// else two (low 6 bits, then the rest). A lane ranks its item among the warp's with ballots on the
// digit's bits (the items of a warp are in position order (k, lane)), warps in order, as the LSD
// downsweep does.
__global__ void __launch_bounds__(kThreads, 4) bin_scatter_kernel(const unsigned* __restrict__ keys_in,
                                                                  const unsigned* __restrict__ vals_in,
                                                                  unsigned* __restrict__ keys_out,
                                                                  unsigned* __restrict__ vals_out,
                                                                  const unsigned* __restrict__ counts, unsigned tiles,
                                                                  int bits, const unsigned* __restrict__ tile_start,
                                                                  const Ctrl* ctrl, unsigned capacity) {
    chain_entry();
    __shared__ unsigned short s_key[kBlockItems];
    __shared__ unsigned s_val[kBlockItems];
    __shared__ unsigned short s_first[kBinMaxTiles];  // first local position of each tile in the block
    __shared__ unsigned s_wh[kWarps][kBinLocalR];
    __shared__ unsigned s_dstart[kBinLocalR];
    __shared__ unsigned s_tmp[kWarps];
    unsigned P;
    if (!frame_pairs(ctrl, capacity, P)) return;
    const unsigned b = blockIdx.x;
    if (static_cast<unsigned long long>(b) * kBlockItems >= P) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    unsigned key[kItems], val[kItems];
    const unsigned long long wbase = static_cast<unsigned long long>(b) * kBlockItems + warp * (kItems * 32) + lane;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const unsigned long long idx = wbase + k * 32;
        key[k] = idx < P ? keys_in[idx] : kBinMaxTiles;  // kBinMaxTiles: no item
        val[k] = idx < P ? vals_in[idx] : 0u;
    }
    const int passes = bits > kBinLocalBits ? 2 : 1;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = pass * kBinLocalBits;
        unsigned dg[kItems], rank[kItems];
        if (tid < kBinLocalR)
#pragma unroll
            for (int w = 0; w < kWarps; ++w) s_wh[w][tid] = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k)
            dg[k] = key[k] < kBinMaxTiles ? (key[k] >> shift) & (kBinLocalR - 1) : kBinLocalR;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            unsigned peers = 0xFFFFFFFFu;
#pragma unroll
            for (int bb = 0; bb <= kBinLocalBits; ++bb) {
                const bool bit = (dg[k] >> bb) & 1u;
                const unsigned vb = __ballot_sync(0xFFFFFFFFu, bit);
                peers &= bit ? vb : ~vb;
            }
            const unsigned cnt = dg[k] < kBinLocalR ? s_wh[warp][dg[k]] : 0u;
            rank[k] = cnt + __popc(peers & lt);
            __syncwarp();
            if (dg[k] < kBinLocalR && lane == 31 - __clz(peers)) s_wh[warp][dg[k]] = cnt + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        unsigned digit_count = 0;
        if (tid < kBinLocalR)
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const unsigned c = s_wh[w][tid];
                s_wh[w][tid] = digit_count;
                digit_count += c;
            }
        unsigned total;
        const unsigned dstart = block_excl_scan<kThreads>(digit_count, s_tmp, total);
        if (tid < kBinLocalR) s_dstart[tid] = dstart;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kItems; ++k)
            if (dg[k] < kBinLocalR) {
                const unsigned pos = s_dstart[dg[k]] + s_wh[warp][dg[k]] + rank[k];
                s_key[pos] = static_cast<unsigned short>(key[k]);
                s_val[pos] = val[k];
            }
        __syncthreads();
        // Reload in (k, lane) order: the next pass ranks the items in their new order.
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned pos = warp * (kItems * 32) + k * 32 + lane;
            const bool valid = static_cast<unsigned long long>(b) * kBlockItems + pos < P;
            key[k] = valid ? s_key[pos] : kBinMaxTiles;
            val[k] = valid ? s_val[pos] : 0u;
        }
        __syncthreads();
    }
    // key[k] is now the tile of local position pos (sorted); record each tile's first position.
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const unsigned pos = warp * (kItems * 32) + k * 32 + lane;
        if (key[k] < kBinMaxTiles && (pos == 0 || s_key[pos - 1] != key[k]))
            s_first[key[k]] = static_cast<unsigned short>(pos);
    }
    __syncthreads();
    const unsigned* row = counts + static_cast<size_t>(b) * tiles;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (key[k] >= kBinMaxTiles) continue;
        const unsigned pos = warp * (kItems * 32) + k * 32 + lane;
        const unsigned g = __ldg(tile_start + key[k]) + __ldg(row + key[k]) + (pos - s_first[key[k]]);
        keys_out[g] = key[k];
        vals_out[g] = val[k];
    }
}

// Depth keys (kCulledKey when tiles_touched is 0; else the depth's bits less key_base) and
// rectangles of a projection given in the reference kernel's layout -- what the preprocess kernel
// writes for its own.
__global__ void __launch_bounds__(kThreads) projection_keys_kernel(int64_t n, const unsigned* __restrict__ tiles_touched,
                                                                   const float* __restrict__ depth,
                                                                   const uint4* __restrict__ rect,
                                                                   unsigned* __restrict__ depth_key,
                                                                   unsigned long long* __restrict__ rect16,
                                                                   unsigned key_base) {
    chain_entry();
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
    if (i >= n) return;
    unsigned key = kCulledKey;
    if (tiles_touched[i]) {
        key = __float_as_uint(depth[i]) - key_base;
        const uint4 r = rect[i];
        rect16[i] = static_cast<unsigned long long>(r.x) | (static_cast<unsigned long long>(r.y) << 16) |
                    (static_cast<unsigned long long>(r.z) << 32) | (static_cast<unsigned long long>(r.w) << 48);
    }
    depth_key[i] = key;
}

int bits_of(unsigned v) {  // bits needed to hold v
    int b = 0;
    while (b < 32 && (v >> b) != 0) ++b;
    return b;
}

unsigned spans_for(uint64_t max_items) {
    const uint64_t blocks = (max_items + kBlockItems - 1) / kBlockItems;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(blocks, kMaxSpans)));
}

}  // namespace

void launch_upload(const unsigned* src_mapped, unsigned* dst, unsigned words, cudaStream_t stream) {
    const unsigned blocks = std::max(1u, (words + kThreads - 1) / kThreads);
    launch_chained(upload_kernel, dim3(blocks), dim3(kThreads), stream, src_mapped, dst, words);
}

void launch_frame_start(const unsigned* src_mapped, unsigned* dst, unsigned words, Ctrl* ctrl, unsigned* zero,
                        unsigned zero_words, uint2* ranges, unsigned tiles, cudaStream_t stream) {
    const unsigned most = std::max(std::max(zero_words, tiles), words);
    const unsigned blocks = std::max(1u, std::min((most + kThreads * 4 - 1) / (kThreads * 4), 148u));
    launch_chained(frame_start_kernel, dim3(blocks), dim3(kThreads), stream, src_mapped, dst, words, ctrl, zero,
                   zero_words, ranges, tiles);
}

void launch_publish_ctrl(Ctrl* ctrl, Ctrl* host, cudaStream_t stream) {
    launch_chained(publish_ctrl_kernel, dim3(1), dim3(1), stream, ctrl, host);
}

void launch_frame_begin(Ctrl* ctrl, cudaStream_t stream) {
    launch_chained(frame_begin_kernel, dim3(1), dim3(1), stream, ctrl, static_cast<unsigned*>(nullptr), 0u,
                   static_cast<uint2*>(nullptr), 0u);
}

void launch_frame_begin(Ctrl* ctrl, unsigned* zero, unsigned zero_words, uint2* ranges, unsigned tiles,
                        cudaStream_t stream) {
    const unsigned most = std::max(zero_words, tiles);
    const unsigned blocks = std::max(1u, std::min((most + kThreads * 4 - 1) / (kThreads * 4), 148u));
    launch_chained(frame_begin_kernel, dim3(blocks), dim3(kThreads), stream, ctrl, zero, zero_words, ranges, tiles);
}

size_t sort_scratch_words() { return static_cast<size_t>(1 << kMaxRadixBits) * (kMaxSpans + 1); }
size_t sort_count_words() { return static_cast<size_t>(1 << kMaxRadixBits) * kMaxSpans; }
size_t sort_span_sums() { return kMaxSpans; }
unsigned sort_spans(uint64_t max_items) { return spans_for(max_items); }
unsigned expand_chunk_pairs() { return kExpandChunk; }
bool radix_bits_supported(int bits) { return bits == 8 || bits == 9; }

namespace {
template <int BITS>
void count_pass(const unsigned* keys_in, bool masked, SortCount src, unsigned fixed, unsigned capacity, int shift,
                unsigned* counts, Ctrl* ctrl, cudaStream_t stream) {
    const unsigned spans = spans_for(src == SortCount::kFixed ? fixed : capacity);
    const dim3 grid(spans), block(kThreads);
    if (masked)
        launch_chained(upsweep_kernel<BITS, true>, grid, block, stream, keys_in, src, fixed, capacity, shift, spans,
                       counts, ctrl);
    else
        launch_chained(upsweep_kernel<BITS, false>, grid, block, stream, keys_in, src, fixed, capacity, shift, spans,
                       counts, ctrl);
}

// Launches the wide downsweep, raising its dynamic shared memory limit once per device first.
template <int BITS, bool kMasked, bool kKeysOut>
void launch_wide(dim3 grid, cudaStream_t stream, const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out,
                 unsigned* vals_out, SortCount src, unsigned fixed, unsigned capacity, int shift, unsigned spans,
                 unsigned* counts, unsigned* totals, Ctrl* ctrl) {
    constexpr int kDevices = 64;
    static bool raised[kDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kDevices && !raised[dev]) {
        if (cudaFuncSetAttribute(downsweep_wide_kernel<BITS, kMasked, kKeysOut>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(wide_smem_bytes(BITS))) == cudaSuccess)
            raised[dev] = true;
    }
    cudaGetLastError();  // a failed raise shows up as the launch's error
    launch_chained_smem(downsweep_wide_kernel<BITS, kMasked, kKeysOut>, grid, dim3(kWideThreads),
                        wide_smem_bytes(BITS), stream, keys_in, vals_in, keys_out, vals_out, src, fixed, capacity,
                        shift, spans, static_cast<const unsigned*>(counts), static_cast<const unsigned*>(totals), ctrl);
}

template <int BITS>
void scatter_pass(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out, bool masked,
                  SortCount src, unsigned fixed, unsigned capacity, int shift, unsigned* counts, unsigned* totals,
                  unsigned* zero, unsigned zero_words, Ctrl* ctrl, cudaStream_t stream) {
    constexpr int R = 1 << BITS;
    const unsigned spans = spans_for(src == SortCount::kFixed ? fixed : capacity);
    const dim3 grid(spans), block(kThreads);
    launch_chained(span_scan_kernel, dim3(R), block, stream, counts, totals, spans, src, fixed, capacity, ctrl, zero,
                   zero_words);
    const bool small = (src == SortCount::kFixed ? fixed : capacity) <= kBallotRankMax;
    if (!small) {  // a large pass: the wide downsweep
        if (masked)
            launch_wide<BITS, true, true>(grid, stream, keys_in, vals_in, keys_out, vals_out, src, fixed, capacity,
                                          shift, spans, counts, totals, ctrl);
        else if (keys_out)
            launch_wide<BITS, false, true>(grid, stream, keys_in, vals_in, keys_out, vals_out, src, fixed, capacity,
                                           shift, spans, counts, totals, ctrl);
        else
            launch_wide<BITS, false, false>(grid, stream, keys_in, vals_in, keys_out, vals_out, src, fixed, capacity,
                                            shift, spans, counts, totals, ctrl);
        return;
    }
    if (masked)
        launch_chained(downsweep_kernel<BITS, true, true>, grid, block, stream, keys_in, vals_in, keys_out, vals_out,
                       src, fixed, capacity, shift, spans, counts, totals, ctrl);
    else if (keys_out)
        launch_chained(downsweep_kernel<BITS, false, true>, grid, block, stream, keys_in, vals_in, keys_out, vals_out,
                       src, fixed, capacity, shift, spans, counts, totals, ctrl);
    else
        launch_chained(downsweep_kernel<BITS, false, false>, grid, block, stream, keys_in, vals_in, keys_out, vals_out,
                       src, fixed, capacity, shift, spans, counts, totals, ctrl);
}
}  // namespace

void launch_radix_pass(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                       bool masked, SortCount src, unsigned fixed, unsigned capacity, int shift, int bits,
                       unsigned* scratch, Ctrl* ctrl, cudaStream_t stream) {
    unsigned* totals = scratch + sort_count_words();
    launch_radix_count(keys_in, masked, src, fixed, capacity, shift, bits, scratch, ctrl, stream);
    launch_radix_scatter(keys_in, vals_in, keys_out, vals_out, masked, src, fixed, capacity, shift, bits, scratch,
                         totals, nullptr, 0, ctrl, stream);
}

void launch_radix_count(const unsigned* keys_in, bool masked, SortCount src, unsigned fixed, unsigned capacity,
                        int shift, int bits, unsigned* counts, Ctrl* ctrl, cudaStream_t stream) {
    if (bits == 9) count_pass<9>(keys_in, masked, src, fixed, capacity, shift, counts, ctrl, stream);
    else count_pass<8>(keys_in, masked, src, fixed, capacity, shift, counts, ctrl, stream);
}

void launch_radix_scatter(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                          bool masked, SortCount src, unsigned fixed, unsigned capacity, int shift, int bits,
                          unsigned* counts, unsigned* totals, unsigned* zero, unsigned zero_words, Ctrl* ctrl,
                          cudaStream_t stream) {
    if (bits == 9)
        scatter_pass<9>(keys_in, vals_in, keys_out, vals_out, masked, src, fixed, capacity, shift, counts, totals, zero,
                        zero_words, ctrl, stream);
    else
        scatter_pass<8>(keys_in, vals_in, keys_out, vals_out, masked, src, fixed, capacity, shift, counts, totals, zero,
                        zero_words, ctrl, stream);
}

namespace {
// The expansion's counts live in dynamic shared memory; with the 16 KB of a tile-bin row it goes
// past the 48 KB a kernel gets without asking (once per device).
constexpr int kMaxDevices = 64;
bool g_expand_smem_set[kMaxDevices];

void allow_expand_smem() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return;
    }
    if (g_expand_smem_set[dev]) return;
    if (cudaFuncSetAttribute(expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kBinMaxTiles * sizeof(unsigned))) == cudaSuccess)
        g_expand_smem_set[dev] = true;
    else
        cudaGetLastError();
}
}  // namespace

unsigned bin_max_tiles() { return kBinMaxTiles; }
unsigned bin_max_pairs() { return kBinMaxPairs; }
size_t bin_count_words(unsigned capacity, unsigned tiles) {
    return static_cast<size_t>((capacity + kBlockItems - 1) / kBlockItems) * tiles;
}

void launch_duplicate(const unsigned* sorted_idx, const unsigned long long* rect16, Ctrl* ctrl, unsigned capacity,
                      unsigned max_visible, const BatchTables& tables, const DupBuffers& buf, unsigned* pair_key,
                      unsigned* pair_val, cudaStream_t stream, const PassCounts& first, unsigned* bin_counts,
                      unsigned bin_tiles) {
    if (max_visible == 0) return;
    const unsigned spans = spans_for(max_visible);
    launch_chained(pair_count_kernel, dim3(spans), dim3(kThreads), stream, sorted_idx, rect16, ctrl, spans, buf.rank,
                   buf.rect_sorted, buf.span_sum);
    launch_chained(pair_offsets_kernel, dim3(spans), dim3(kThreads), stream, buf.rect_sorted, ctrl, spans, capacity,
                   buf.span_sum, buf.offs, buf.chunk_start);
    // At least one CTA: with capacity 0 (a count-only call) the frame overflows and the CTA leaves.
    const unsigned expand_blocks = std::max(1u, (capacity + kExpandChunk - 1) / kExpandChunk);
    const unsigned hist_words = bin_counts ? bin_tiles : first.counts ? first.mask + 1 : 0u;
    if (bin_counts) allow_expand_smem();
    launch_chained_smem(expand_kernel, dim3(expand_blocks), dim3(kThreads), hist_words * sizeof(unsigned), stream,
                        sorted_idx, buf.rect_sorted, buf.offs, buf.chunk_start, ctrl, capacity, tables, pair_key,
                        pair_val, first, bin_counts, bin_tiles);
}

void launch_tile_bins(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                      unsigned* counts, unsigned tiles, unsigned* tile_start, uint2* ranges, Ctrl* ctrl,
                      unsigned capacity, cudaStream_t stream) {
    const int bits = std::max(1, bits_of(tiles > 0 ? tiles - 1 : 0));
    launch_chained(bin_scan_kernel, dim3(std::max(1u, (tiles + 31) / 32)), dim3(kBinScanThreads), stream, counts,
                   tiles, tile_start, ranges, ctrl, capacity);
    const unsigned blocks = std::max(1u, (capacity + kBlockItems - 1) / kBlockItems);
    launch_chained(bin_scatter_kernel, dim3(blocks), dim3(kThreads), stream, keys_in, vals_in, keys_out, vals_out,
                   static_cast<const unsigned*>(counts), tiles, bits, static_cast<const unsigned*>(tile_start),
                   static_cast<const Ctrl*>(ctrl), capacity);
}

void launch_ranges(const unsigned* sorted_keys, const Ctrl* ctrl, unsigned capacity, uint2* ranges,
                   cudaStream_t stream) {
    const unsigned groups = (capacity + 4u * kThreads - 1) / (4u * kThreads);
    const unsigned blocks = std::max(1u, std::min(groups, 148u * 8u));
    launch_chained(ranges_kernel, dim3(blocks), dim3(kThreads), stream, sorted_keys, ctrl, capacity, ranges);
}

void launch_projection_keys(int64_t n, const unsigned* tiles_touched, const float* depth, const uint4* rect,
                            unsigned* depth_key, unsigned long long* rect16, cudaStream_t stream, unsigned key_base) {
    const unsigned blocks = static_cast<unsigned>((n + kThreads - 1) / kThreads);
    if (blocks == 0) return;
    launch_chained(projection_keys_kernel, dim3(blocks), dim3(kThreads), stream, n, tiles_touched, depth, rect,
                   depth_key, rect16, key_base);
}

}  // namespace ab2
