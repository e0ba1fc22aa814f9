// Steps 2-4 of the rasterizer: the stable (tile, depth, index) ordering of all splat-tile pairs.
//
// The reference duplicates one 64-bit key (tile << 32 | depth bits) per pair in Gaussian-index order
// and radix-sorts all of them over bits [0, 32 + bits(tiles)) (gpu_render.cu:148-161, 324-345).
// A stable LSD sort handles the low (depth) digits first, and duplication commutes with a stable
// sort on a key every copy of a Gaussian shares, so the same order is produced here with less
// traffic:
//   1. the preprocess kernel compacts the V visible Gaussians in index order;
//   2. four 8-bit onesweep passes sort those V (depth bits, index) pairs -- V, not P, items;
//   3. duplicate expands them, in depth order, into P (tile, index) pairs (load-balanced: each
//      block writes a contiguous run of pairs found by binary search over its scan);
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
constexpr int kOsItems = 16;
constexpr int kOsChunk = kOsThreads * kOsItems;
constexpr int kDupItems = 4;
constexpr int kDupChunk = 256 * kDupItems;

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

__device__ __forceinline__ unsigned frame_count(const unsigned* count32, const unsigned long long* count64,
                                                unsigned capacity) {
    if (count32) return *count32;
    const unsigned long long c = *count64;
    return c > capacity ? 0u : static_cast<unsigned>(c);
}

template <int ITEMS>
__global__ void __launch_bounds__(kOsThreads) onesweep_kernel(const unsigned* __restrict__ keys_in,
                                                               const unsigned* __restrict__ vals_in,
                                                               unsigned* __restrict__ keys_out,
                                                               unsigned* __restrict__ vals_out,
                                                               const unsigned* count32,
                                                               const unsigned long long* count64, unsigned capacity,
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
    const unsigned count = frame_count(count32, count64, capacity);
    if (tid == 0) s_chunk = atomicAdd(chunk_ctr, 1u);
    for (int k = tid; k < NW * kRadix; k += kOsThreads) (&s_wh[0][0])[k] = 0;
    __syncthreads();
    const unsigned chunk = s_chunk;
    const unsigned base = chunk * CH;
    if (base >= count) return;

    unsigned key[ITEMS], val[ITEMS], rank[ITEMS];
    const unsigned wbase = base + warp * (ITEMS * 32) + lane;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned idx = wbase + k * 32;
        const bool valid = idx < count;
        key[k] = valid ? keys_in[idx] : 0u;
        val[k] = valid ? vals_in[idx] : 0u;
        rank[k] = valid ? ((key[k] >> shift) & (kRadix - 1)) : kRadix;  // digit, kRadix = padding
    }
    // Warp-level stable ranking: items in (k, lane) order, i.e. ascending position.
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned d = rank[k];
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
        const unsigned cnt = d < kRadix ? s_wh[warp][d] : 0u;
        rank[k] = cnt + __popc(peers & lt);
        __syncwarp();
        if (d < kRadix && lane == 31 - __clz(peers)) s_wh[warp][d] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // Per digit: offsets of each warp's run, the block's digit total and the block-local start.
    const unsigned d = tid;
    unsigned run = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const unsigned c = s_wh[w][d];
        s_wh[w][d] = run;
        run += c;
    }
    unsigned block_total;
    const unsigned dstart = block_excl_scan<kOsThreads>(run, s_tmp, block_total);
    unsigned hist_total;
    const unsigned gstart = block_excl_scan<kOsThreads>(hist[d], s_tmp, hist_total);
    s_dstart[d] = dstart;

    // Decoupled look-back for digit d over the preceding chunks.
    const unsigned epoch = ctrl->epoch;
    unsigned long long* my = status + static_cast<size_t>(chunk) * kRadix + d;
    st_store(my, st_make(epoch, chunk == 0 ? kStInc : kStAgg, run));
    unsigned excl = 0;
    if (chunk > 0) {
        unsigned c = chunk - 1, spins = 0;
        while (true) {
            const unsigned long long s = st_load(status + static_cast<size_t>(c) * kRadix + d);
            const unsigned f = st_flag(s, epoch);
            if (f == 0) {
                if (++spins > kSpinLimit) {
                    atomicOr(&ctrl->flags, kFlagTimeout);
                    break;
                }
                continue;
            }
            excl += static_cast<unsigned>(s);
            if (f == kStInc || c == 0) break;
            --c;
        }
        st_store(my, st_make(epoch, kStInc, excl + run));
    }
    s_gbase[d] = gstart + excl - dstart;
    __syncthreads();

    // Scatter into shared memory in block-sorted order, then write out contiguously per digit.
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned idx = wbase + k * 32;
        if (idx < count) {
            const unsigned dd = (key[k] >> shift) & (kRadix - 1);
            const unsigned pos = s_dstart[dd] + s_wh[warp][dd] + rank[k];
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();
    const unsigned nvalid = min(static_cast<unsigned>(CH), count - base);
    for (unsigned p = tid; p < nvalid; p += kOsThreads) {
        const unsigned k = s_keys[p];
        const unsigned g = s_gbase[(k >> shift) & (kRadix - 1)] + p;
        if (keys_out) keys_out[g] = k;
        vals_out[g] = s_vals[p];
    }
}

__global__ void __launch_bounds__(256) duplicate_kernel(const unsigned* __restrict__ sorted_idx,
                                                        const unsigned long long* __restrict__ rect16,
                                                        Ctrl* ctrl, unsigned capacity, int tiles_x, int tile_passes,
                                                        unsigned* __restrict__ pair_key,
                                                        unsigned* __restrict__ pair_val,
                                                        unsigned long long* status) {
    __shared__ unsigned s_incl[kDupChunk];
    __shared__ unsigned s_idx[kDupChunk];
    __shared__ unsigned long long s_rect[kDupChunk];
    __shared__ unsigned s_hist[kMaxPasses * kRadix];
    __shared__ unsigned s_tmp[8];
    __shared__ unsigned s_chunk, s_base;
    const int tid = threadIdx.x;
    if (tid == 0) s_chunk = atomicAdd(&ctrl->chunk_ctr[kCtrDup], 1u);
    for (int k = tid; k < kMaxPasses * kRadix; k += 256) s_hist[k] = 0;
    __syncthreads();
    const unsigned chunk = s_chunk;
    const unsigned V = ctrl->vis_count;
    if (ctrl->pair_total > capacity) {
        if (chunk == 0 && tid == 0) atomicOr(&ctrl->flags, kFlagOverflow);
        return;
    }
    const unsigned first = chunk * kDupChunk;
    if (first >= V) return;

    unsigned cnt[kDupItems];
    unsigned thread_total = 0;
#pragma unroll
    for (int k = 0; k < kDupItems; ++k) {
        const unsigned j = first + tid * kDupItems + k;
        unsigned g = 0;
        unsigned long long r = 0;
        unsigned c = 0;
        if (j < V) {
            g = sorted_idx[j];
            r = rect16[g];
            const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu, y1 = r >> 48;
            c = (x1 - x0 + 1) * (y1 - y0 + 1);
        }
        s_idx[tid * kDupItems + k] = g;
        s_rect[tid * kDupItems + k] = r;
        cnt[k] = c;
        thread_total += c;
    }
    unsigned block_total;
    unsigned run = block_excl_scan<256>(thread_total, s_tmp, block_total);
#pragma unroll
    for (int k = 0; k < kDupItems; ++k) {
        run += cnt[k];
        s_incl[tid * kDupItems + k] = run;
    }
    if (tid < 32) {
        const unsigned b = lookback_warp(status, chunk, block_total, ctrl->epoch, &ctrl->flags);
        if (tid == 0) s_base = b;
    }
    __syncthreads();
    const unsigned pbase = s_base;
    for (unsigned q = tid; q < block_total; q += 256) {
        int lo = 0, hi = kDupChunk - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s_incl[mid] > q) hi = mid;
            else lo = mid + 1;
        }
        const unsigned start = lo ? s_incl[lo - 1] : 0u;
        const unsigned k = q - start;
        const unsigned long long r = s_rect[lo];
        const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu;
        const unsigned w = x1 - x0 + 1;
        const unsigned row = k / w;
        const unsigned tile = (y0 + row) * static_cast<unsigned>(tiles_x) + x0 + (k - row * w);
        pair_key[pbase + q] = tile;
        pair_val[pbase + q] = s_idx[lo];
        for (int p = 0; p < tile_passes; ++p)
            atomicAdd(&s_hist[p * kRadix + ((tile >> (p * kRadixBits)) & (kRadix - 1))], 1u);
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

__global__ void __launch_bounds__(256) compact_kernel(int64_t n, const unsigned* __restrict__ tiles_touched,
                                                      const float* __restrict__ depth, const uint4* __restrict__ rect,
                                                      Ctrl* ctrl, unsigned* __restrict__ vis_key,
                                                      unsigned* __restrict__ vis_idx,
                                                      unsigned long long* __restrict__ rect16,
                                                      unsigned long long* status) {
    __shared__ unsigned s_chunk, s_base;
    __shared__ unsigned s_tmp[8];
    __shared__ unsigned s_hist[kMaxPasses * kRadix];
    const int tid = threadIdx.x;
    for (int k = tid; k < kMaxPasses * kRadix; k += 256) s_hist[k] = 0;
    if (tid == 0) s_chunk = atomicAdd(&ctrl->chunk_ctr[kCtrCompact], 1u);
    __syncthreads();
    const unsigned chunk = s_chunk;
    const int64_t i = static_cast<int64_t>(chunk) * 256 + tid;
    unsigned count = 0, bits = 0;
    if (i < n) {
        count = tiles_touched[i];
        if (count) {
            bits = __float_as_uint(depth[i]);
            const uint4 r = rect[i];
            rect16[i] = static_cast<unsigned long long>(r.x) | (static_cast<unsigned long long>(r.y) << 16) |
                        (static_cast<unsigned long long>(r.z) << 32) | (static_cast<unsigned long long>(r.w) << 48);
#pragma unroll
            for (int p = 0; p < kMaxPasses; ++p)
                atomicAdd(&s_hist[p * kRadix + ((bits >> (p * kRadixBits)) & (kRadix - 1))], 1u);
        }
    }
    unsigned total;
    const unsigned local = block_excl_scan<256>(count ? 1u : 0u, s_tmp, total);
    unsigned pairs;
    block_excl_scan<256>(count, s_tmp, pairs);
    if (tid < 32) {
        const unsigned b = lookback_warp(status, chunk, total, ctrl->epoch, &ctrl->flags);
        if (tid == 0) {
            s_base = b;
            if (total) atomicAdd(&ctrl->vis_count, total);
            if (pairs) atomicAdd(&ctrl->pair_total, static_cast<unsigned long long>(pairs));
        }
    }
    __syncthreads();
    if (count) {
        vis_key[s_base + local] = bits;
        vis_idx[s_base + local] = static_cast<unsigned>(i);
    }
    for (int k = tid; k < kMaxPasses * kRadix; k += 256)
        if (s_hist[k]) atomicAdd(&ctrl->depth_hist[k], s_hist[k]);
}

}  // namespace

void launch_frame_begin(Ctrl* ctrl, cudaStream_t stream) { frame_begin_kernel<<<1, 256, 0, stream>>>(ctrl); }

int onesweep_items_per_thread() { return kOsItems; }
unsigned onesweep_chunk_items() { return kOsChunk; }

void launch_onesweep(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                     const unsigned* count, const unsigned long long* count64, unsigned capacity, int shift,
                     const unsigned* hist, unsigned long long* status, unsigned* chunk_ctr, Ctrl* ctrl,
                     cudaStream_t stream) {
    const unsigned blocks = (capacity + kOsChunk - 1) / kOsChunk;
    if (blocks == 0) return;
    onesweep_kernel<kOsItems><<<blocks, kOsThreads, 0, stream>>>(keys_in, vals_in, keys_out, vals_out, count,
                                                                 count64, capacity, shift, hist, status, chunk_ctr,
                                                                 ctrl);
}

unsigned duplicate_chunk_items() { return kDupChunk; }

void launch_duplicate(const unsigned* sorted_idx, const unsigned long long* rect16, Ctrl* ctrl, unsigned capacity,
                      unsigned max_visible, int tiles_x, int tile_passes, unsigned* pair_key, unsigned* pair_val,
                      unsigned long long* status, cudaStream_t stream) {
    const unsigned blocks = (max_visible + kDupChunk - 1) / kDupChunk;
    if (blocks == 0) return;
    duplicate_kernel<<<blocks, 256, 0, stream>>>(sorted_idx, rect16, ctrl, capacity, tiles_x, tile_passes, pair_key,
                                                 pair_val, status);
}

void launch_ranges(const unsigned* sorted_keys, const Ctrl* ctrl, unsigned capacity, uint2* ranges,
                   cudaStream_t stream) {
    ranges_kernel<<<148 * 4, 256, 0, stream>>>(sorted_keys, ctrl, capacity, ranges);
}

void launch_compact_projection(int64_t n, const unsigned* tiles_touched, const float* depth, const uint4* rect,
                               Ctrl* ctrl, unsigned* vis_key, unsigned* vis_idx, unsigned long long* rect16,
                               unsigned long long* status, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    if (blocks == 0) return;
    compact_kernel<<<blocks, 256, 0, stream>>>(n, tiles_touched, depth, rect, ctrl, vis_key, vis_idx, rect16, status);
}

}  // namespace ab2
