// Steps 2-4 of the rasterizer: the stable (tile, depth, index) ordering of all splat-tile pairs.
//
// The reference duplicates one 64-bit key (tile << 32 | depth bits) per pair in Gaussian-index order
// and radix-sorts all of them over bits [0, 32 + bits(tiles)) (gpu_render.cu:148-161, 324-345).
// A stable LSD sort handles the low (depth) digits first, and duplication commutes with a stable
// sort on a key every copy of a Gaussian shares, so the same order is produced here with less
// traffic:
//   1. the preprocess kernel writes every Gaussian's depth key (a sentinel when culled);
//   2. four 8-bit onesweep passes sort the V visible (depth bits, index) pairs -- V, not P, items;
//      the first pass reads all N keys in index order and drops the culled ones as it ranks;
//   3. a pair-offset scan over those V, then an expansion, in depth order, into P (tile, index)
//      pairs with the same number of pairs per block (the nearest splats own thousands of tiles);
//   4. ceil(bits(tiles) / 8) onesweep passes stably sort the pairs by tile;
//   5. tile ranges as gpu_render.cu:164-177.
// Each tile's run ends up ordered by (depth bits, Gaussian index), exactly the reference's order,
// so keys, values and ranges are bit-identical to the reference's for the same projection.
//
// The onesweep pass follows the single-pass LSD scheme of Adinets & Merrill (2022): a block ranks
// a chunk of keys with warp-level match_any, publishes its per-digit counts, looks back over the
// preceding chunks (decoupled look-back, bounded waits) for each digit's running offset, and
// scatters through shared memory so global writes are contiguous per digit.
#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

constexpr int kOsThreads = 256;
constexpr int kOsItems = 8;
constexpr int kOsChunk = kOsThreads * kOsItems;
constexpr int kScanItems = 4;
constexpr int kScanChunk = 256 * kScanItems;
constexpr int kExpandChunk = 1024;

__global__ void frame_begin_kernel(Ctrl* ctrl) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        ctrl->sticky_flags |= ctrl->flags;
        if (ctrl->pair_total > ctrl->max_pair_total) ctrl->max_pair_total = ctrl->pair_total;
        ctrl->pair_total = 0;
        ctrl->vis_count = 0;
        ctrl->flags = 0;
        unsigned e = (ctrl->epoch + 1u) & 0x3FFFFFFFu;
        ctrl->epoch = e == 0 ? 1u : e;
    }
    if (tid < 16) ctrl->chunk_ctr[tid] = 0;
    for (int k = tid; k < kMaxPasses * kRadix; k += blockDim.x) {
        ctrl->depth_hist[k] = 0;
        ctrl->tile_hist[k] = 0;
    }
}

// One stable LSD pass over a chunk of kOsThreads * ITEMS (key, value) pairs.
//   masked_count > 0: the input is every Gaussian's depth key (kCulledKey = culled), values are the
//                     indices themselves (vals_in unused); culled keys are dropped, so this pass
//                     also compacts the visible list. The pass publishes the visible count.
//   masked_count = 0: the input holds exactly as many items as this digit's histogram counts.
template <int ITEMS>
__global__ void __launch_bounds__(kOsThreads) onesweep_kernel(const unsigned* __restrict__ keys_in,
                                                               const unsigned* __restrict__ vals_in,
                                                               unsigned* __restrict__ keys_out,
                                                               unsigned* __restrict__ vals_out, unsigned masked_count,
                                                               int shift, const unsigned* __restrict__ hist,
                                                               unsigned long long* status, unsigned* chunk_ctr,
                                                               Ctrl* ctrl) {
    constexpr int CH = kOsThreads * ITEMS;
    constexpr int NW = kOsThreads / 32;
    __shared__ unsigned s_keys[CH];
    __shared__ unsigned s_vals[CH];
    __shared__ unsigned s_wh[NW][kRadix];
    __shared__ unsigned s_dstart[kRadix];
    __shared__ unsigned s_gbase[kRadix];
    __shared__ unsigned s_tmp[NW];
    __shared__ unsigned s_chunk;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (ctrl->flags & kFlagOverflow) return;
    if (tid == 0) s_chunk = atomicAdd(chunk_ctr, 1u);
    for (int k = tid; k < NW * kRadix; k += kOsThreads) (&s_wh[0][0])[k] = 0;
    const unsigned d = tid;  // this thread's digit in the per-digit phases
    unsigned hist_total;
    const unsigned gstart = block_excl_scan<kOsThreads>(hist[d], s_tmp, hist_total);
    const unsigned chunk = s_chunk;
    const bool masked = masked_count > 0;
    const unsigned count = masked ? masked_count : hist_total;
    if (masked && chunk == 0 && tid == 0) ctrl->vis_count = hist_total;
    const unsigned base = chunk * CH;
    if (base >= count) return;

    unsigned key[ITEMS], val[ITEMS], rank[ITEMS];
    const unsigned wbase = base + warp * (ITEMS * 32) + lane;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned idx = wbase + k * 32;
        bool valid = idx < count;
        key[k] = valid ? keys_in[idx] : 0u;
        if (masked) {
            valid = valid && key[k] != kCulledKey;
            val[k] = idx;
        } else {
            val[k] = valid ? vals_in[idx] : 0u;
        }
        rank[k] = valid ? ((key[k] >> shift) & (kRadix - 1)) : kRadix;  // digit; kRadix = not an item
    }
    // Warp-level stable ranking: items in (k, lane) order, i.e. ascending position.
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned dg = rank[k];
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, dg);
        const unsigned cnt = dg < kRadix ? s_wh[warp][dg] : 0u;
        const unsigned r = cnt + __popc(peers & lt);
        __syncwarp();
        if (dg < kRadix && lane == 31 - __clz(peers)) s_wh[warp][dg] = cnt + __popc(peers);
        __syncwarp();
        rank[k] = dg < kRadix ? r : 0xFFFFFFFFu;
    }
    __syncthreads();

    // Per digit: offsets of each warp's run, the block's digit total and the block-local start.
    unsigned run = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const unsigned c = s_wh[w][d];
        s_wh[w][d] = run;
        run += c;
    }
    unsigned block_total;
    const unsigned dstart = block_excl_scan<kOsThreads>(run, s_tmp, block_total);
    s_dstart[d] = dstart;

    // Decoupled look-back for digit d over the preceding chunks. Each round trip loads the status
    // of kLookback predecessors at once, so a block whose predecessors have only published their
    // own counts (all blocks finish ranking together when the chunks fit on the GPU at once) sums
    // kLookback of them per L2 latency instead of one.
    const unsigned epoch = ctrl->epoch;
    unsigned long long* my = status + static_cast<size_t>(chunk) * kRadix + d;
    st_store(my, st_make(epoch, chunk == 0 ? kStInc : kStAgg, run));
    unsigned excl = 0;
    if (chunk > 0) {
        constexpr unsigned kLookback = 8;
        unsigned c = chunk, spins = 0;  // predecessors still to add: c-1, c-2, ...
        bool found = false;
        while (!found && c > 0) {
            const unsigned k_count = min(kLookback, c);
            unsigned long long sv[kLookback];
#pragma unroll
            for (unsigned k = 0; k < kLookback; ++k)
                sv[k] = k < k_count ? st_load(status + static_cast<size_t>(c - 1 - k) * kRadix + d) : 0ull;
            unsigned used = 0;
#pragma unroll
            for (unsigned k = 0; k < kLookback; ++k) {
                if (k >= k_count || found) break;
                const unsigned f = st_flag(sv[k], epoch);
                if (f == 0) break;  // not published yet: reload from here
                excl += static_cast<unsigned>(sv[k]);
                used = k + 1;
                if (f == kStInc) found = true;
            }
            c -= used;
            if (!found && used < k_count && ++spins > kSpinLimit) {
                atomicOr(&ctrl->flags, kFlagTimeout);
                break;
            }
        }
        st_store(my, st_make(epoch, kStInc, excl + run));
    }
    s_gbase[d] = gstart + excl - dstart;
    __syncthreads();

    // Scatter into shared memory in block-sorted order, then write out contiguously per digit.
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (rank[k] != 0xFFFFFFFFu) {
            const unsigned dd = (key[k] >> shift) & (kRadix - 1);
            const unsigned pos = s_dstart[dd] + s_wh[warp][dd] + rank[k];
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();
    for (unsigned p = tid; p < block_total; p += kOsThreads) {
        const unsigned k = s_keys[p];
        const unsigned g = s_gbase[(k >> shift) & (kRadix - 1)] + p;
        if (keys_out) keys_out[g] = k;
        vals_out[g] = s_vals[p];
    }
}

// Pair offsets of the depth-sorted visible list: an exclusive scan of each Gaussian's tile count
// (single pass, decoupled look-back), written with its rectangle in sorted order. For every chunk
// of kExpandChunk pairs it also records the Gaussian that holds the chunk's first pair, so the
// expansion can give every block the same number of pairs. The last block stores the frame's
// pair total and flags an overflow of the pair capacity.
__global__ void __launch_bounds__(256) pair_scan_kernel(const unsigned* __restrict__ sorted_idx,
                                                        const unsigned long long* __restrict__ rect16, Ctrl* ctrl,
                                                        unsigned capacity, unsigned* __restrict__ offs,
                                                        unsigned* __restrict__ rank,
                                                        unsigned long long* __restrict__ rect_sorted,
                                                        unsigned* __restrict__ chunk_start,
                                                        unsigned long long* status) {
    __shared__ unsigned s_tmp[8];
    __shared__ unsigned s_chunk, s_base;
    const int tid = threadIdx.x;
    if (tid == 0) s_chunk = atomicAdd(&ctrl->chunk_ctr[kCtrDup], 1u);
    __syncthreads();
    const unsigned chunk = s_chunk;
    const unsigned V = ctrl->vis_count;
    const unsigned first = chunk * kScanChunk;
    if (first >= V) return;

    unsigned cnt[kScanItems];
    unsigned long long rect[kScanItems];
    unsigned thread_total = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const unsigned j = first + tid * kScanItems + k;
        unsigned c = 0;
        unsigned long long r = 0;
        if (j < V) {
            const unsigned g = sorted_idx[j];
            rank[g] = j;
            r = rect16[g];
            const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu, y1 = r >> 48;
            c = (x1 - x0 + 1) * (y1 - y0 + 1);
        }
        cnt[k] = c;
        rect[k] = r;
        thread_total += c;
    }
    unsigned block_total;
    const unsigned thread_base = block_excl_scan<256>(thread_total, s_tmp, block_total);
    if (tid < 32) {
        const unsigned b = lookback_warp(status, chunk, block_total, ctrl->epoch, &ctrl->flags);
        if (tid == 0) {
            s_base = b;
            if (first + kScanChunk >= V) {  // the last chunk: the frame's pair total
                const unsigned long long P = static_cast<unsigned long long>(b) + block_total;
                ctrl->pair_total = P;
                if (P > capacity) atomicOr(&ctrl->flags, kFlagOverflow);
            }
        }
    }
    __syncthreads();
    const unsigned last_chunk = (capacity + kExpandChunk - 1) / kExpandChunk;
    unsigned long long o = static_cast<unsigned long long>(s_base) + thread_base;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const unsigned j = first + tid * kScanItems + k;
        if (j < V) {
            offs[j] = static_cast<unsigned>(o);
            rect_sorted[j] = rect[k];
            for (unsigned long long c = (o + kExpandChunk - 1) / kExpandChunk;
                 c * kExpandChunk < o + cnt[k] && c <= last_chunk; ++c)
                chunk_start[c] = j;
        }
        o += cnt[k];
    }
}

// Expands the depth-sorted list into (tile, Gaussian) pairs: block b writes pairs
// [b * kExpandChunk, (b + 1) * kExpandChunk), row-major over each rectangle as
// gpu_render.cu:155-160 does, and builds the tile-digit histograms of the onesweep passes.
__global__ void __launch_bounds__(256) expand_kernel(const unsigned* __restrict__ sorted_idx,
                                                     const unsigned long long* __restrict__ rect_sorted,
                                                     const unsigned* __restrict__ offs,
                                                     const unsigned* __restrict__ chunk_start, Ctrl* ctrl,
                                                     unsigned capacity, BatchTables tables, int tile_passes,
                                                     unsigned* __restrict__ pair_key,
                                                     unsigned* __restrict__ pair_val) {
    __shared__ unsigned s_off[kExpandChunk + 1];
    __shared__ unsigned s_idx[kExpandChunk + 1];
    __shared__ unsigned long long s_rect[kExpandChunk + 1];
    __shared__ unsigned s_tbase[kExpandChunk + 1];  // global tile of (0, 0) of the entry's view
    __shared__ unsigned short s_tx[kExpandChunk + 1];  // tiles per row of the entry's view
    __shared__ unsigned s_hist[kMaxPasses * kRadix];
    const int tid = threadIdx.x;
    if (ctrl->flags & kFlagOverflow) return;
    const unsigned long long P = ctrl->pair_total;
    if (P > capacity) return;
    const unsigned base = blockIdx.x * kExpandChunk;
    if (base >= P) return;
    for (int k = tid; k < kMaxPasses * kRadix; k += 256) s_hist[k] = 0;
    const unsigned V = ctrl->vis_count;
    const unsigned j0 = chunk_start[blockIdx.x];
    const unsigned j1 = base + kExpandChunk < P ? chunk_start[blockIdx.x + 1] : V - 1;
    const unsigned G = j1 - j0 + 1;  // <= kExpandChunk + 1: every Gaussian owns at least one pair
    for (unsigned k = tid; k < G; k += 256) {
        s_off[k] = offs[j0 + k];
        const unsigned e = sorted_idx[j0 + k];
        s_idx[k] = e;
        s_rect[k] = rect_sorted[j0 + k];
        const unsigned v = find_segment(tables.entry_base, tables.n_views, e);
        s_tbase[k] = tables.tile_base[v];
        s_tx[k] = static_cast<unsigned short>(tables.tiles_x[v]);
    }
    __syncthreads();
    const unsigned n_here = static_cast<unsigned>(min(static_cast<unsigned long long>(kExpandChunk), P - base));
    const int lane = tid & 31;
    for (unsigned q0 = 0; q0 < n_here; q0 += 256) {  // uniform trip count: whole warps vote below
        const unsigned q = q0 + tid;
        unsigned tile = 0;
        const bool valid = q < n_here;
        if (valid) {
            const unsigned p = base + q;
            unsigned lo = 0, hi = G - 1;  // last k with s_off[k] <= p
            while (lo < hi) {
                const unsigned mid = (lo + hi + 1) >> 1;
                if (s_off[mid] <= p) lo = mid;
                else hi = mid - 1;
            }
            const unsigned k = p - s_off[lo];
            const unsigned long long r = s_rect[lo];
            const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu;
            const unsigned w = x1 - x0 + 1;
            const unsigned row = k / w;
            tile = s_tbase[lo] + (y0 + row) * static_cast<unsigned>(s_tx[lo]) + x0 + (k - row * w);
            pair_key[p] = tile;
            pair_val[p] = s_idx[lo];
            atomicAdd(&s_hist[tile & (kRadix - 1)], 1u);  // low digit: neighbours differ, few conflicts
        }
        // Higher digits repeat along a warp (neighbouring tiles share them): one add per distinct digit.
        for (int ps = 1; ps < tile_passes; ++ps) {
            const unsigned dg = valid ? (tile >> (ps * kRadixBits)) & (kRadix - 1) : kRadix;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, dg);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&s_hist[ps * kRadix + dg], __popc(peers));
        }
    }
    __syncthreads();
    for (int k = tid; k < tile_passes * kRadix; k += 256)
        if (s_hist[k]) atomicAdd(&ctrl->tile_hist[k], s_hist[k]);
}

__global__ void ranges_kernel(const unsigned* __restrict__ keys, const Ctrl* ctrl, unsigned capacity,
                              uint2* __restrict__ ranges) {
    if (ctrl->flags & kFlagOverflow) return;
    const unsigned long long pt = ctrl->pair_total;
    if (pt > capacity) return;
    const unsigned P = static_cast<unsigned>(pt);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        const unsigned tile = keys[i];
        if (i == 0) ranges[tile].x = 0;
        else {
            const unsigned prev = keys[i - 1];
            if (prev != tile) {
                ranges[prev].y = i;
                ranges[tile].x = i;
            }
        }
        if (i == P - 1) ranges[tile].y = P;
    }
}

// Depth keys (kCulledKey when tiles_touched is 0), rectangles and depth histograms of a projection
// given in the reference kernel's layout -- what the preprocess kernel writes for its own.
__global__ void __launch_bounds__(256) projection_keys_kernel(int64_t n, const unsigned* __restrict__ tiles_touched,
                                                              const float* __restrict__ depth,
                                                              const uint4* __restrict__ rect, Ctrl* ctrl,
                                                              unsigned* __restrict__ depth_key,
                                                              unsigned long long* __restrict__ rect16) {
    __shared__ unsigned s_hist[kMaxPasses * kRadix];
    const int tid = threadIdx.x;
    for (int k = tid; k < kMaxPasses * kRadix; k += 256) s_hist[k] = 0;
    __syncthreads();
    const int64_t i = static_cast<int64_t>(blockIdx.x) * 256 + tid;
    if (i < n) {
        unsigned key = kCulledKey;
        if (tiles_touched[i]) {
            key = __float_as_uint(depth[i]);
            const uint4 r = rect[i];
            rect16[i] = static_cast<unsigned long long>(r.x) | (static_cast<unsigned long long>(r.y) << 16) |
                        (static_cast<unsigned long long>(r.z) << 32) | (static_cast<unsigned long long>(r.w) << 48);
#pragma unroll
            for (int p = 0; p < kMaxPasses; ++p)
                atomicAdd(&s_hist[p * kRadix + ((key >> (p * kRadixBits)) & (kRadix - 1))], 1u);
        }
        depth_key[i] = key;
    }
    __syncthreads();
    for (int k = tid; k < kMaxPasses * kRadix; k += 256)
        if (s_hist[k]) atomicAdd(&ctrl->depth_hist[k], s_hist[k]);
}

}  // namespace

void launch_frame_begin(Ctrl* ctrl, cudaStream_t stream) { frame_begin_kernel<<<1, 256, 0, stream>>>(ctrl); }

int onesweep_items_per_thread() { return kOsItems; }
unsigned onesweep_chunk_items() { return kOsChunk; }

void launch_onesweep(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                     unsigned masked_count, unsigned capacity, int shift, const unsigned* hist,
                     unsigned long long* status, unsigned* chunk_ctr, Ctrl* ctrl, cudaStream_t stream) {
    const unsigned blocks = (capacity + kOsChunk - 1) / kOsChunk;
    if (blocks == 0) return;
    onesweep_kernel<kOsItems><<<blocks, kOsThreads, 0, stream>>>(keys_in, vals_in, keys_out, vals_out, masked_count,
                                                                 shift, hist, status, chunk_ctr, ctrl);
}

unsigned pair_scan_chunk_items() { return kScanChunk; }
unsigned expand_chunk_pairs() { return kExpandChunk; }

void launch_duplicate(const unsigned* sorted_idx, const unsigned long long* rect16, Ctrl* ctrl, unsigned capacity,
                      unsigned max_visible, const BatchTables& tables, int tile_passes, const DupBuffers& buf,
                      unsigned* pair_key,
                      unsigned* pair_val, unsigned long long* status, cudaStream_t stream) {
    const unsigned scan_blocks = (max_visible + kScanChunk - 1) / kScanChunk;
    if (scan_blocks == 0) return;
    pair_scan_kernel<<<scan_blocks, 256, 0, stream>>>(sorted_idx, rect16, ctrl, capacity, buf.offs, buf.rank,
                                                      buf.rect_sorted, buf.chunk_start, status);
    const unsigned expand_blocks = (capacity + kExpandChunk - 1) / kExpandChunk;
    expand_kernel<<<expand_blocks, 256, 0, stream>>>(sorted_idx, buf.rect_sorted, buf.offs, buf.chunk_start, ctrl,
                                                     capacity, tables, tile_passes, pair_key, pair_val);
}

void launch_ranges(const unsigned* sorted_keys, const Ctrl* ctrl, unsigned capacity, uint2* ranges,
                   cudaStream_t stream) {
    ranges_kernel<<<148 * 4, 256, 0, stream>>>(sorted_keys, ctrl, capacity, ranges);
}

void launch_projection_keys(int64_t n, const unsigned* tiles_touched, const float* depth, const uint4* rect,
                            Ctrl* ctrl, unsigned* depth_key, unsigned long long* rect16, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    if (blocks == 0) return;
    projection_keys_kernel<<<blocks, 256, 0, stream>>>(n, tiles_touched, depth, rect, ctrl, depth_key, rect16);
}

}  // namespace ab2
