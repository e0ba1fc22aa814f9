// Steps 2-4 of the rasterizer in ONE cooperative launch: the stable (tile, depth, index) ordering
// of all splat-tile pairs and the tile ranges, with the same algorithm and the same outputs as the
// multi-kernel sequence of sort.cu (depth-sorted visible list, pair expansion in depth order, tile
// passes, ranges; the reference's order, gpu_render.cu:148-177, 324-345, bit for bit).
//
// Why one launch: at the working size (740k Gaussians, ~325k visible, ~1.6M pairs at 1280x720)
// every pass of the multi-kernel sort is a few microseconds of work spread over three launches, and
// the ~19 launches of a frame's sort cost more in launch and drain latency than in memory traffic
// (the whole working set sits in L2). Here one 1024-thread CTA per SM runs every phase, and the
// phases are separated by grid barriers: a CTA arrives with one atomic add on a counter and polls
// it with acquire loads. The cooperative launch guarantees every CTA is resident, so a barrier
// cannot wait on a CTA that never runs; every wait is nevertheless bounded (kSpinLimit polls),
// after which the frame is marked void (kFlagWaitTimeout | kFlagOverflow: nothing downstream uses
// it) and every CTA returns -- no wait can hang the device.
//
// Measured, it is the slower sort, so it is opt-in (ANISO_B200_SORT=persistent): 0.169 against
// 0.125 ms per 740k 1280x720 frame. ncu: one 1024-thread CTA per SM (64 registers), half the warp
// slots active, 35% issue-active, and the top stall is the block barrier: each scatter round is a
// chain of about nine __syncthreads around a few instructions of work per thread, and a phase
// cannot end before its slowest CTA, where the multi-kernel sequence overlaps one kernel's tail
// with the next one's launch.
//
// Phases (one CTA = one contiguous chunk of each pass's items: blocks [T c / G, T (c + 1) / G) of
// kSortBlockItems, the chunking the producers' digit counts use):
//   depth pass 0 (8-bit, compacting): counts from the preprocess (or a counting phase), then
//     scan + scatter;  depth passes 1-3: count | barrier | scan + scatter | barrier
//   pair count: rectangles gathered into depth order, each CTA's pair total | barrier
//   pair offsets: each sorted entry's first pair, the entry holding each CTA's first pair | barrier
//   expansion: each CTA writes exactly its chunk of the pairs and counts their first tile digit
//     | barrier
//   tile passes: (count | barrier |) scan + scatter | barrier;  tile ranges.
// "scan" is each CTA reading every CTA's digit counts (a G x R matrix, CTA-major so the reads
// coalesce) and forming its own per-digit output positions; "scatter" ranks 4096 items per round
// (warp-level peer masks, cross-warp prefix per digit) and writes them through shared memory so
// global writes are contiguous per digit. Data another CTA wrote in an earlier phase is read with
// ld.global.cg (L2), never through the non-coherent path.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

constexpr int kT = 1024;                 // threads per CTA, one CTA per SM
constexpr int kW = kT / 32;
constexpr int kItems = 4;                // items per thread per ranking round
constexpr int kRound = kT * kItems;      // 4096
constexpr int kMaxBits = 9;
constexpr int kMaxR = 1 << kMaxBits;
constexpr int kDepthBits = 8;
constexpr int kExpPer = 4;               // pairs per thread per expansion round
constexpr int kExpRound = kT * kExpPer;  // 4096
constexpr unsigned kBallotMax = 1u << 22;  // passes up to this many items rank with ballots
constexpr unsigned kSpinLimit = 1u << 22;  // polls of a grid barrier before the frame is declared void

struct RankSmem {
    unsigned keys[kRound];
    unsigned vals[kRound];
    unsigned wh[kW * kMaxR];  // per-warp digit counts, then each warp's offset within its digit
    unsigned cnt[kMaxR];
    unsigned dstart[kMaxR];
    unsigned gbase[kMaxR];
};
struct ExpSmem {
    unsigned off[kExpRound + 2];
    unsigned idx[kExpRound + 1];
    unsigned org[kExpRound + 1];       // global tile of the rectangle's corner
    unsigned short w[kExpRound + 1];   // rectangle width in tiles
    unsigned short tx[kExpRound + 1];  // tiles per row of the entry's view
    unsigned hist[kMaxR];
    unsigned next;
};
struct ScanSmem {
    unsigned before[kT];
    unsigned total[kT];
};
struct KeepSmem {                      // lives across the phases
    unsigned run[kMaxR];               // next global output position of each digit (this CTA)
    unsigned tmp[kW + 1];
    unsigned long long tmp64[kW];
    int ok;
};
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kPhaseBytes = std::max(sizeof(RankSmem), std::max(sizeof(ExpSmem), sizeof(ScanSmem)));
constexpr size_t kKeepBytes = align256(sizeof(KeepSmem));
constexpr size_t kSmemBytes = kKeepBytes + kPhaseBytes;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier number `epoch` (1, 2, ...; the same sequence in every CTA). Returns false in every
// thread when the frame is void: this CTA's wait gave up, or another CTA's did.
__device__ bool grid_barrier(Ctrl* ctrl, unsigned epoch, KeepSmem& k) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&ctrl->sort_barrier, 1u);
        const unsigned target = epoch * gridDim.x;
        int ok = 1;
        for (unsigned spins = 0; ld_acquire(&ctrl->sort_barrier) < target; ++spins) {
            if ((spins & 63u) == 63u && (ld_acquire(&ctrl->flags) & kFlagWaitTimeout)) {
                ok = 0;
                break;
            }
            if (spins >= kSpinLimit) {
                atomicOr(&ctrl->flags, kFlagWaitTimeout | kFlagOverflow);
                ok = 0;
                break;
            }
            if (spins >= 32) __nanosleep(64);
        }
        __threadfence();
        k.ok = ok;
    }
    __syncthreads();
    return k.ok != 0;
}

__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) { return a < b ? a : b; }

// This CTA's items [lo, hi) of a pass over n items.
__device__ __forceinline__ void chunk_of(unsigned n, unsigned& lo, unsigned& hi) {
    const unsigned long long T = (static_cast<unsigned long long>(n) + kSortBlockItems - 1) / kSortBlockItems;
    const unsigned long long G = gridDim.x, c = blockIdx.x;
    lo = static_cast<unsigned>(umin64(n, T * c / G * kSortBlockItems));
    hi = static_cast<unsigned>(umin64(n, T * (c + 1) / G * kSortBlockItems));
}

__device__ __forceinline__ unsigned rect_area(unsigned long long r) {
    const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu, y1 = r >> 48;
    return (x1 - x0 + 1) * (y1 - y0 + 1);
}

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v, KeepSmem& k) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) k.tmp64[warp] = v;
    __syncthreads();
    unsigned long long s = 0;
#pragma unroll
    for (int w = 0; w < kW; ++w) s += k.tmp64[w];
    __syncthreads();
    return s;
}

// Counts this CTA's chunk of a pass: row[d] = items with digit d (culled keys skipped if masked).
template <int BITS, bool kMasked>
__device__ void count_phase(const unsigned* keys, unsigned n, int shift, unsigned* row, RankSmem& s) {
    constexpr int R = 1 << BITS, P = kT / R, WP = kW / P;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int i = tid; i < kW * R; i += kT) s.wh[i] = 0;
    __syncthreads();
    unsigned lo, hi;
    chunk_of(n, lo, hi);
    for (unsigned long long i0 = lo + tid; i0 < hi; i0 += 4ull * kT) {
        unsigned key[4];
        bool valid[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long i = i0 + static_cast<unsigned long long>(u) * kT;
            valid[u] = i < hi;
            key[u] = valid[u] ? __ldcg(keys + i) : 0u;
            if (kMasked) valid[u] = valid[u] && key[u] != kCulledKey;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (valid[u]) atomicAdd(&s.wh[warp * R + ((key[u] >> shift) & (R - 1))], 1u);
    }
    __syncthreads();
    const int d = tid / P, p = tid % P;
    unsigned sum = 0;
#pragma unroll
    for (int j = 0; j < WP; ++j) sum += s.wh[(p * WP + j) * R + d];
#pragma unroll
    for (int o = P / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    if (p == 0) row[d] = sum;
}

// Reads every CTA's row of the count matrix and sets k.run[d] = this CTA's first output position
// for digit d (all digits before d, then the CTAs before this one). Returns the pass's item total.
template <int BITS>
__device__ unsigned scan_phase(const unsigned* counts, ScanSmem& s, KeepSmem& k) {
    constexpr int R = 1 << BITS, Q = kT / R;
    const int tid = threadIdx.x, d = tid % R, q = tid / R;
    const unsigned G = gridDim.x, c = blockIdx.x;
    const unsigned c0 = G * q / Q, c1 = G * (q + 1) / Q;
    unsigned before = 0, total = 0;
    for (unsigned r0 = c0; r0 < c1; r0 += 8) {
        unsigned v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = r0 + u < c1 ? __ldcg(counts + static_cast<size_t>(r0 + u) * R + d) : 0u;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            total += v[u];
            if (r0 + u < c) before += v[u];
        }
    }
    s.before[tid] = before;
    s.total[tid] = total;
    __syncthreads();
    unsigned b = 0, t = 0;
    if (tid < R)
#pragma unroll
        for (int qq = 0; qq < Q; ++qq) {
            b += s.before[qq * R + tid];
            t += s.total[qq * R + tid];
        }
    unsigned all;
    const unsigned ex = block_excl_scan<kT>(tid < R ? t : 0u, k.tmp, all);
    if (tid < R) k.run[tid] = ex + b;
    __syncthreads();
    return all;
}

// Ranks and scatters this CTA's chunk, 4096 items per round, stably: within a round items keep
// their position order per digit (warp peer masks in (item, lane) order, warps in order), rounds
// in order, CTAs in order through k.run. masked: the input is the depth keys in entry order, culled
// ones dropped, the entry index as the value.
template <int BITS, bool kMasked, bool kKeysOut, bool kBallot>
__device__ void scatter_phase(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out,
                              unsigned* vals_out, unsigned n, int shift, RankSmem& s, KeepSmem& k) {
    constexpr int R = 1 << BITS, P = kT / R, WP = kW / P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    unsigned lo, hi;
    chunk_of(n, lo, hi);
    for (unsigned long long base = lo; base < hi; base += kRound) {
        for (int i = tid; i < kW * R; i += kT) s.wh[i] = 0;
        unsigned key[kItems], val[kItems], dg[kItems];
#pragma unroll
        for (int q = 0; q < kItems; ++q) {
            const unsigned long long idx = base + warp * (kItems * 32) + q * 32 + lane;
            bool valid = idx < hi;
            key[q] = valid ? __ldcg(keys_in + idx) : 0u;
            if (kMasked) {
                valid = valid && key[q] != kCulledKey;
                val[q] = static_cast<unsigned>(idx);
            } else {
                val[q] = valid ? __ldcg(vals_in + idx) : 0u;
            }
            dg[q] = valid ? ((key[q] >> shift) & (R - 1)) : static_cast<unsigned>(R);
        }
        __syncthreads();
        unsigned rank[kItems];
#pragma unroll
        for (int q = 0; q < kItems; ++q) {
            unsigned peers;
            if (kBallot) {
                peers = 0xFFFFFFFFu;
#pragma unroll
                for (int b = 0; b <= BITS; ++b) {
                    const bool bit = (dg[q] >> b) & 1u;
                    const unsigned vb = __ballot_sync(0xFFFFFFFFu, bit);
                    peers &= bit ? vb : ~vb;
                }
            } else {
                peers = __match_any_sync(0xFFFFFFFFu, dg[q]);
            }
            const unsigned cnt = dg[q] < R ? s.wh[warp * R + dg[q]] : 0u;
            rank[q] = cnt + __popc(peers & lt);
            __syncwarp();
            if (dg[q] < R && lane == 31 - __clz(peers)) s.wh[warp * R + dg[q]] = cnt + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        {  // per digit: each warp's offset within the round's run of the digit, and the run's length
            const int d = tid / P, p = tid % P;
            unsigned c[WP], sum = 0;
#pragma unroll
            for (int j = 0; j < WP; ++j) {
                c[j] = s.wh[(p * WP + j) * R + d];
                sum += c[j];
            }
            unsigned incl = sum;
#pragma unroll
            for (int o = 1; o < P; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o, P);
                if (p >= o) incl += y;
            }
            unsigned ex = incl - sum;
#pragma unroll
            for (int j = 0; j < WP; ++j) {
                s.wh[(p * WP + j) * R + d] = ex;
                ex += c[j];
            }
            if (p == P - 1) s.cnt[d] = incl;
        }
        __syncthreads();
        unsigned round_total;
        const unsigned v = tid < R ? s.cnt[tid] : 0u;
        const unsigned dstart = block_excl_scan<kT>(v, k.tmp, round_total);
        if (tid < R) {
            s.dstart[tid] = dstart;
            s.gbase[tid] = k.run[tid] - dstart;
            k.run[tid] += v;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kItems; ++q) {
            if (dg[q] < R) {
                const unsigned pos = s.dstart[dg[q]] + s.wh[warp * R + dg[q]] + rank[q];
                s.keys[pos] = key[q];
                s.vals[pos] = val[q];
            }
        }
        __syncthreads();
        for (unsigned p = tid; p < round_total; p += kT) {
            const unsigned kk = s.keys[p];
            const unsigned g = s.gbase[(kk >> shift) & (R - 1)] + p;
            if (kKeysOut) keys_out[g] = kk;
            vals_out[g] = s.vals[p];
        }
        __syncthreads();
    }
}

template <int BITS, bool kMasked, bool kKeysOut>
__device__ __forceinline__ void scatter_any(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out,
                                            unsigned* vals_out, unsigned n, int shift, RankSmem& s, KeepSmem& k) {
    if (n <= kBallotMax)
        scatter_phase<BITS, kMasked, kKeysOut, true>(keys_in, vals_in, keys_out, vals_out, n, shift, s, k);
    else
        scatter_phase<BITS, kMasked, kKeysOut, false>(keys_in, vals_in, keys_out, vals_out, n, shift, s, k);
}

// Gathers this CTA's share of the depth-sorted entries' rectangles into sorted order, records
// their sorted positions (rank, for the adjoint) and stores the share's pair total.
__device__ void pair_count_phase(const SortFrameArgs& a, const unsigned* sorted_idx, unsigned V, KeepSmem& k) {
    const int tid = threadIdx.x;
    unsigned lo, hi;
    chunk_of(V, lo, hi);
    unsigned long long sum = 0;
    for (unsigned long long j0 = lo + tid; j0 < hi; j0 += 4ull * kT) {
        unsigned e[4];
        unsigned long long r[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long j = j0 + static_cast<unsigned long long>(u) * kT;
            e[u] = j < hi ? __ldcg(sorted_idx + j) : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long j = j0 + static_cast<unsigned long long>(u) * kT;
            r[u] = j < hi ? a.rect16[e[u]] : 0ull;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long j = j0 + static_cast<unsigned long long>(u) * kT;
            if (j < hi) {
                if (a.rank) a.rank[e[u]] = static_cast<unsigned>(j);
                a.rect_sorted[j] = r[u];
                sum += rect_area(r[u]);
            }
        }
    }
    sum = block_sum_u64(sum, k);
    if (tid == 0) a.span_sum[blockIdx.x] = sum;
}

// Every CTA forms the pair total (the same value everywhere; CTA 0 publishes it and flags an
// overflow of the pair capacity -- then every CTA returns false). This CTA then writes the first
// pair of each of its sorted entries and, for each CTA's expansion chunk (blocks
// [Tp c' / G, Tp (c' + 1) / G) of the P pairs), the entry that holds the chunk's first pair.
__device__ bool pair_offsets_phase(const SortFrameArgs& a, unsigned V, unsigned& P_out, KeepSmem& k) {
    const int tid = threadIdx.x;
    const unsigned G = gridDim.x, c = blockIdx.x;
    unsigned long long before = 0, total = 0;
    for (unsigned i = tid; i < G; i += kT) {
        const unsigned long long v = __ldcg(a.span_sum + i);
        total += v;
        if (i < c) before += v;
    }
    before = block_sum_u64(before, k);
    total = block_sum_u64(total, k);
    if (c == 0 && tid == 0) {
        a.ctrl->pair_total = total;
        if (total > a.pair_cap) atomicOr(&a.ctrl->flags, kFlagOverflow);
    }
    if (total > a.pair_cap) return false;
    P_out = static_cast<unsigned>(total);
    const unsigned long long Tp = (total + kSortBlockItems - 1) / kSortBlockItems;
    unsigned lo, hi;
    chunk_of(V, lo, hi);
    unsigned long long run = before;
    for (unsigned long long j0 = lo; j0 < hi; j0 += kT) {
        const unsigned long long j = j0 + tid;
        const unsigned cnt = j < hi ? rect_area(__ldcg(a.rect_sorted + j)) : 0u;
        unsigned tot;
        const unsigned ex = block_excl_scan<kT>(cnt, k.tmp, tot);
        if (j < hi) {
            const unsigned long long o = run + ex;
            a.offs[j] = static_cast<unsigned>(o);
            // chunks whose start lies in [o, o + cnt): start(c') = floor(Tp c' / G) * block >= o
            // exactly from c' = ceil(ceil(o / block) * G / Tp)
            const unsigned long long blk = (o + kSortBlockItems - 1) / kSortBlockItems;
            for (unsigned long long cp = (blk * G + Tp - 1) / Tp; cp < G; ++cp) {
                if (Tp * cp / G * kSortBlockItems >= o + cnt) break;
                a.chunk_first[cp] = static_cast<unsigned>(j);
            }
        }
        run += tot;
    }
    return true;
}

// This CTA's chunk of the pairs, row-major over each rectangle (gpu_render.cu:155-160) in depth
// order, tile ids global over the batch; counts their first tile digit into row (the first tile
// pass's counts: the chunk is exactly that pass's chunk of this CTA).
template <int BITS0>
__device__ void expand_phase(const SortFrameArgs& a, const unsigned* sorted_idx, unsigned V, unsigned P,
                             unsigned* row, ExpSmem& s) {
    constexpr int R0 = 1 << BITS0;
    const int tid = threadIdx.x;
    for (int i = tid; i < R0; i += kT) s.hist[i] = 0;
    unsigned plo, phi;
    chunk_of(P, plo, phi);
    unsigned j_start = plo < phi ? __ldcg(a.chunk_first + blockIdx.x) : 0u;
    if (j_start >= V) j_start = V > 0 ? V - 1 : 0u;  // never taken (every chunk start is marked); keeps reads in bounds
    __syncthreads();
    unsigned* pk = a.pair_key[0];
    unsigned* pv = a.pair_val[0];
    for (unsigned long long q0 = plo; q0 < phi; q0 += kExpRound) {
        const unsigned q1 = static_cast<unsigned>(umin64(phi, q0 + kExpRound));
        const unsigned avail = min(static_cast<unsigned>(kExpRound + 1), V - j_start);
        for (unsigned kk = tid; kk < avail; kk += kT) {
            const unsigned j = j_start + kk;
            const unsigned long long r = __ldcg(a.rect_sorted + j);
            const unsigned e = __ldcg(sorted_idx + j);
            const unsigned v = find_segment(a.tables.entry_base, a.tables.n_views, e);
            const unsigned tx = a.tables.tiles_x[v];
            const unsigned x0 = r & 0xFFFFu, y0 = (r >> 16) & 0xFFFFu, x1 = (r >> 32) & 0xFFFFu;
            s.off[kk] = __ldcg(a.offs + j);
            s.idx[kk] = e;
            s.org[kk] = a.tables.tile_base[v] + y0 * tx + x0;
            s.w[kk] = static_cast<unsigned short>(x1 - x0 + 1);
            s.tx[kk] = static_cast<unsigned short>(tx);
        }
        if (tid == 0) s.off[avail] = j_start + avail < V ? __ldcg(a.offs + j_start + avail) : P;
        __syncthreads();
        const unsigned long long p0 = q0 + static_cast<unsigned long long>(tid) * kExpPer;
        if (p0 < q1) {
            const unsigned p = static_cast<unsigned>(p0);
            unsigned lo = 0, hi = avail - 1;  // last staged entry whose first pair is <= p
            while (lo < hi) {
                const unsigned mid = (lo + hi + 1) >> 1;
                if (s.off[mid] <= p) lo = mid;
                else hi = mid - 1;
            }
            unsigned w = s.w[lo], tx = s.tx[lo], org = s.org[lo], idx = s.idx[lo], next = s.off[lo + 1];
            const unsigned kk = p - s.off[lo];
            unsigned rw = kk / w, col = kk - rw * w;
            unsigned key[kExpPer], val[kExpPer];
#pragma unroll
            for (int i = 0; i < kExpPer; ++i) {
                key[i] = org + rw * tx + col;
                val[i] = idx;
                if (p + i + 1 == next && p + i + 1 < P) {  // the next pair starts the next entry
                    ++lo;
                    w = s.w[lo];
                    tx = s.tx[lo];
                    org = s.org[lo];
                    idx = s.idx[lo];
                    next = s.off[lo + 1];
                    rw = 0;
                    col = 0;
                } else if (++col == w) {
                    col = 0;
                    ++rw;
                }
            }
            if (p + kExpPer <= q1) {
                *reinterpret_cast<uint4*>(pk + p) = make_uint4(key[0], key[1], key[2], key[3]);
                *reinterpret_cast<uint4*>(pv + p) = make_uint4(val[0], val[1], val[2], val[3]);
            } else {
#pragma unroll
                for (int i = 0; i < kExpPer; ++i)
                    if (p + i < q1) {
                        pk[p + i] = key[i];
                        pv[p + i] = val[i];
                    }
            }
#pragma unroll
            for (int i = 0; i < kExpPer; ++i)
                if (p + i < q1) atomicAdd(&s.hist[key[i] & (R0 - 1)], 1u);
        }
        __syncthreads();
        if (tid == 0 && q1 < phi) {  // the entry holding pair q1 starts the next round
            unsigned lo = 0, hi = avail - 1;
            while (lo < hi) {
                const unsigned mid = (lo + hi + 1) >> 1;
                if (s.off[mid] <= q1) lo = mid;
                else hi = mid - 1;
            }
            s.next = j_start + lo;
        }
        __syncthreads();
        j_start = s.next;
        __syncthreads();
    }
    for (int i = tid; i < R0; i += kT) row[i] = s.hist[i];
}

// ranges[tile] = [first, last + 1) over the sorted tile keys (gpu_render.cu:164-177), this CTA's
// chunk of the positions.
__device__ void ranges_phase(const unsigned* keys, unsigned P, uint2* ranges) {
    unsigned lo, hi;
    chunk_of(P, lo, hi);
    for (unsigned long long i = lo + threadIdx.x; i < hi; i += kT) {
        const unsigned t = __ldcg(keys + i);
        if (i == 0) {
            ranges[t].x = 0;
        } else {
            const unsigned prev = __ldcg(keys + i - 1);
            if (prev != t) {
                ranges[prev].y = static_cast<unsigned>(i);
                ranges[t].x = static_cast<unsigned>(i);
            }
        }
        if (i == P - 1) ranges[t].y = P;
    }
}

template <int BITS>
__device__ bool tile_pass(const SortFrameArgs& a, int t, int shift, unsigned P, unsigned& epoch, RankSmem& rs,
                          ScanSmem& ss, KeepSmem& k) {
    constexpr int R = 1 << BITS;
    unsigned* counts = a.counts[t & 1];
    const int src = t & 1, dst = src ^ 1;
    if (t > 0) {
        count_phase<BITS, false>(a.pair_key[src], P, shift, counts + static_cast<size_t>(blockIdx.x) * R, rs);
        if (!grid_barrier(a.ctrl, ++epoch, k)) return false;
    }
    scan_phase<BITS>(counts, ss, k);
    scatter_any<BITS, false, true>(a.pair_key[src], a.pair_val[src], a.pair_key[dst], a.pair_val[dst], P, shift, rs,
                                   k);
    return grid_barrier(a.ctrl, ++epoch, k);
}

__global__ void __launch_bounds__(kT, 1) sort_frame_kernel(SortFrameArgs a) {
    chain_entry();
    extern __shared__ __align__(256) unsigned char smem[];
    KeepSmem& k = *reinterpret_cast<KeepSmem*>(smem);
    unsigned char* ph = smem + kKeepBytes;
    RankSmem& rs = *reinterpret_cast<RankSmem*>(ph);
    ExpSmem& es = *reinterpret_cast<ExpSmem*>(ph);
    ScanSmem& ss = *reinterpret_cast<ScanSmem*>(ph);
    constexpr int R8 = 1 << kDepthBits;
    const unsigned c = blockIdx.x;
    unsigned epoch = 0;

    // depth pass 0: all entries in entry order, culled ones dropped
    const unsigned E = a.entries;
    if (!a.first_counted) {
        count_phase<kDepthBits, true>(a.depth_key, E, 0, a.counts[0] + static_cast<size_t>(c) * R8, rs);
        if (!grid_barrier(a.ctrl, ++epoch, k)) return;
    }
    const unsigned V = scan_phase<kDepthBits>(a.counts[0], ss, k);
    if (c == 0 && threadIdx.x == 0) a.ctrl->vis_count = V;
    scatter_any<kDepthBits, true, true>(a.depth_key, nullptr, a.vis_key[0], a.vis_idx[0], E, 0, rs, k);
    if (!grid_barrier(a.ctrl, ++epoch, k)) return;
    // depth passes 1-3 over the V visible entries
    for (int p = 1; p < 4; ++p) {
        const int src = (p + 1) & 1, dst = p & 1;
        unsigned* counts = a.counts[p & 1];
        count_phase<kDepthBits, false>(a.vis_key[src], V, kDepthBits * p, counts + static_cast<size_t>(c) * R8, rs);
        if (!grid_barrier(a.ctrl, ++epoch, k)) return;
        scan_phase<kDepthBits>(counts, ss, k);
        if (p < 3)
            scatter_any<kDepthBits, false, true>(a.vis_key[src], a.vis_idx[src], a.vis_key[dst], a.vis_idx[dst], V,
                                                 kDepthBits * p, rs, k);
        else
            scatter_any<kDepthBits, false, false>(a.vis_key[src], a.vis_idx[src], nullptr, a.vis_idx[dst], V,
                                                  kDepthBits * p, rs, k);
        if (!grid_barrier(a.ctrl, ++epoch, k)) return;
    }
    const unsigned* sorted_idx = a.vis_idx[1];

    // pair count, pair offsets, expansion
    pair_count_phase(a, sorted_idx, V, k);
    if (!grid_barrier(a.ctrl, ++epoch, k)) return;
    unsigned P = 0;
    if (!pair_offsets_phase(a, V, P, k)) return;  // the same decision in every CTA
    if (!grid_barrier(a.ctrl, ++epoch, k)) return;
    const int b0 = a.tile_bits[0];
    if (b0 == 9) expand_phase<9>(a, sorted_idx, V, P, a.counts[0] + static_cast<size_t>(c) * 512, es);
    else expand_phase<8>(a, sorted_idx, V, P, a.counts[0] + static_cast<size_t>(c) * 256, es);
    if (!grid_barrier(a.ctrl, ++epoch, k)) return;

    // tile passes, ranges
    for (int t = 0, shift = 0; t < a.tile_passes; shift += a.tile_bits[t], ++t) {
        const bool ok = a.tile_bits[t] == 9 ? tile_pass<9>(a, t, shift, P, epoch, rs, ss, k)
                                            : tile_pass<8>(a, t, shift, P, epoch, rs, ss, k);
        if (!ok) return;
    }
    ranges_phase(a.pair_key[a.tile_passes & 1], P, a.ranges);
}

bool sort_env_persistent() {
    static const bool persistent = [] {
        const char* v = std::getenv("ANISO_B200_SORT");
        return v && std::strcmp(v, "persistent") == 0;
    }();
    return persistent;
}

constexpr int kMaxDevices = 64;
int g_ctas[kMaxDevices];  // 0: not yet probed; -1: not supported; else the CTA count

}  // namespace

unsigned persistent_sort_ctas() {
    if (!sort_env_persistent()) return 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return 0;
    }
    if (g_ctas[dev] == 0) {
        int coop = 0, sms = 0, occ = 0;
        bool ok = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess &&
                  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
                  cudaFuncSetAttribute(sort_frame_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kSmemBytes)) == cudaSuccess &&
                  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sort_frame_kernel, kT, kSmemBytes) ==
                      cudaSuccess;
        if (!ok) cudaGetLastError();
        g_ctas[dev] = (ok && coop && occ >= 1 && sms > 0 && sms <= kT) ? sms : -1;
    }
    return g_ctas[dev] > 0 ? static_cast<unsigned>(g_ctas[dev]) : 0u;
}

size_t persistent_sort_count_words(unsigned ctas) { return static_cast<size_t>(ctas) * kMaxR; }

cudaError_t launch_sort_frame(const SortFrameArgs& args, unsigned ctas, cudaStream_t stream) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(kT);
    cfg.dynamicSmemBytes = kSmemBytes;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    note_chained_launch();
    return cudaLaunchKernelEx(&cfg, sort_frame_kernel, args);
}

}  // namespace ab2
