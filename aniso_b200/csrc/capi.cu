// The C ABI (include/aniso_b200.h): scenes, batches, the differentiable path.
//
// Everything renders through one plan: V views of S scenes. A frame is a fixed, host-sync-free
// sequence of kernels on one stream (capturable in a CUDA graph), launched with programmatic
// stream serialisation: upload of the plan's view table, frame_begin (control block, first digit
// counts, tile ranges), preprocess, 4 depth LSD passes, pair scan, pair expansion, 1-4 tile LSD
// passes, tile ranges, blend. After a synchronous frame one more kernel hands the control block
// to the host. Data-dependent sizes (visible entries, pairs) stay on the
// device; grids are sized for capacity and surplus blocks exit at once. The reference instead reads
// the pair count back mid-frame (gpu_render.cu:329) to size its buffers; here a frame whose pairs
// exceed the capacity sets an overflow flag instead of writing them, and the host grows the
// buffers and renders it again.
#include "aniso_b200.h"
#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace {

using namespace ab2;

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();  // clear a non-sticky error so the context stays usable
    return fail(e == cudaErrorMemoryAllocation ? ANISO_B200_ERR_OUT_OF_MEMORY : ANISO_B200_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define AB_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
    } while (0)

#define AB_TRY(expr)              \
    do {                          \
        int rc_ = (expr);         \
        if (rc_ != 0) return rc_; \
    } while (0)

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), cap(o.cap) {
        o.p = nullptr;
        o.cap = 0;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    // Grows to at least n elements (contents are not kept); zero-fills new memory if asked.
    int reserve(size_t n, bool zero = false) {
        if (n <= cap && p) return 0;
        release();
        AB_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)));
        cap = std::max<size_t>(n, 1);
        if (zero) AB_CUDA(cudaMemset(p, 0, cap * sizeof(T)));
        return 0;
    }
};

unsigned chunks_of(uint64_t n, unsigned per) { return static_cast<unsigned>((n + per - 1) / per); }

int bits_for(uint32_t v) {  // bits needed to hold v
    int b = 0;
    while (b < 32 && (1ull << b) <= v) ++b;
    return b;
}

constexpr uint64_t kMaxEntries = 0xFFFFFFFFull;  // entry and tile indices are 32-bit
constexpr uint64_t kMaxPairs = 0x3FFFFFFFull;    // pair positions and the span arithmetic are 32-bit

// Work buffers of one frame at a time, sized for `n` entries and a pair capacity.
struct Arena {
    int64_t n = -1;
    unsigned pair_cap = 0;
    DevBuf<SplatRecord> rec;
    DevBuf<unsigned long long> rect16;
    DevBuf<unsigned> depth_key;
    DevBuf<unsigned> vis_key[2], vis_idx[2];
    DevBuf<unsigned> pair_key[2], pair_val[2];
    DevBuf<unsigned> offs, rank, chunk_start;
    DevBuf<unsigned long long> rect_sorted;
    DevBuf<uint2> ranges;
    DevBuf<Ctrl> ctrl;
    DevBuf<unsigned> sort_scratch;          // per-span digit counts of the pass in flight
    DevBuf<unsigned long long> span_sum;    // pairs per span of the pair-offset scan
    // The persistent sort (one CTA per SM, `ctas` of them; 0 = the multi-kernel sort runs): two
    // CTA-major count matrices and the entry holding each CTA's first expansion pair.
    unsigned ctas = 0;
    DevBuf<unsigned> pcounts;
    DevBuf<unsigned> chunk_first;
    // The one-pass tile binning (frames of at most bin_max_tiles() tiles): the (block, tile) count
    // matrix, sized for the pair capacity and the widest such frame seen (bin_tiles), and the
    // tiles' starts.
    unsigned bin_tiles = 0;
    DevBuf<unsigned> bin_counts;
    DevBuf<unsigned> tile_start;
    // Counts the (re)allocations of these buffers: a recorded graph is valid while it is unchanged.
    // Global so that a re-initialised arena never repeats an older arena's value.
    uint64_t gen = 0;
    static uint64_t next_gen() {
        static uint64_t g = 0;
        return ++g;
    }

    int init(int64_t count, unsigned cap) {
        n = count;
        gen = next_gen();
        const size_t nn = static_cast<size_t>(std::max<int64_t>(count, 1));
        AB_TRY(rec.reserve(nn));
        AB_TRY(rect16.reserve(nn));
        AB_TRY(depth_key.reserve(nn));
        for (int k = 0; k < 2; ++k) {
            AB_TRY(vis_key[k].reserve(nn));
            AB_TRY(vis_idx[k].reserve(nn));
        }
        AB_TRY(ctrl.reserve(1, true));
        AB_TRY(sort_scratch.reserve(2 * sort_scratch_words()));  // two count matrices and the totals
        ctas = persistent_sort_ctas();
        AB_TRY(span_sum.reserve(std::max<size_t>(sort_span_sums(), ctas)));
        if (ctas) {
            AB_TRY(pcounts.reserve(2 * persistent_sort_count_words(ctas)));
            AB_TRY(chunk_first.reserve(ctas + 1));
        }
        AB_TRY(offs.reserve(nn));
        AB_TRY(rank.reserve(nn));
        AB_TRY(rect_sorted.reserve(nn));
        return grow_pairs(cap);
    }

    // Makes room for at least `entries` entries (re-initialising when it grows).
    int ensure(int64_t entries) {
        if (n >= entries) return 0;
        const uint64_t cap = std::max<uint64_t>(
            std::max<uint64_t>(1u << 20, 2ull * static_cast<uint64_t>(entries)), pair_cap);
        this->~Arena();
        new (this) Arena();
        return init(entries, static_cast<unsigned>(std::min<uint64_t>(cap, kMaxPairs)));
    }

    // Tile ranges for `tiles` tiles, and the tile binning's buffers when it takes such frames.
    int reserve_ranges(size_t tiles) {
        if (tiles > ranges.cap || !ranges.p) gen = next_gen();
        AB_TRY(ranges.reserve(tiles));
        if (tiles > bin_tiles && tiles <= bin_max_tiles()) {
            bin_tiles = static_cast<unsigned>(tiles);
            return reserve_bins();
        }
        return 0;
    }

    int reserve_bins() {
        if (!bin_tiles || pair_cap > bin_max_pairs()) return 0;
        const size_t words = bin_count_words(pair_cap, bin_tiles);
        if (words > bin_counts.cap || !bin_counts.p || !tile_start.p) gen = next_gen();
        AB_TRY(bin_counts.reserve(words));
        return tile_start.reserve(bin_max_tiles());
    }

    // The tile binning can sort a frame of `tiles` tiles at the current pair capacity.
    bool bins_for(unsigned tiles) const {
        return tiles > 0 && tiles <= bin_tiles && pair_cap <= bin_max_pairs() && tile_start.p &&
               bin_counts.cap >= bin_count_words(pair_cap, tiles);
    }

    int grow_pairs(unsigned cap) {
        if (cap <= pair_cap && pair_key[0].p) return 0;
        gen = next_gen();
        for (int k = 0; k < 2; ++k) {
            AB_TRY(pair_key[k].reserve(cap));
            AB_TRY(pair_val[k].reserve(cap));
        }
        pair_cap = cap;
        AB_TRY(reserve_bins());
        return chunk_start.reserve(chunks_of(cap, expand_chunk_pairs()) + 2);
    }
};

// Largest pass (in items, host capacity) whose digits the kernels that write its keys count, in
// place of an upsweep launch. Below it a pass is latency-bound and one atomic add per key costs less
// than a counting kernel; above it the counting kernel's streaming read is the cheaper of the two.
constexpr uint64_t kProducerCountMax = 1ull << 22;

// Depth passes: four 8-bit digits over the 32-bit depth keys, or three 9-bit digits over the low
// 27 bits when every visible depth of the frame is known to be below 8192 (a "short" frame: its
// keys are below 2^27, common.cuh).
constexpr int kDepthPasses = 4;
constexpr int kDepthBits = 8;
constexpr int kShortDepthPasses = 3;
constexpr int kShortDepthBits = 9;
static_assert(kShortDepthPasses * kShortDepthBits == kShortDepthKeyBits, "the short passes cover the short keys");

// Digit widths of the tile passes: as few passes as digits of at most max_bits (8 or 9) allow, each
// pass 8 bits wide unless 9 are needed to stay within that count (17 tile bits: 9 + 8).
int tile_pass_widths(unsigned tiles, int max_bits, int widths[4]) {
    const int total = std::max(1, bits_for(tiles > 0 ? tiles - 1 : 0));
    const int n = (total + max_bits - 1) / max_bits;
    for (int k = 0, shift = 0; k < n; ++k) {
        widths[k] = total - shift > 8 * (n - k) ? 9 : 8;
        shift += widths[k];
    }
    return n;
}

unsigned* count_matrix(Arena& A, int q) { return A.sort_scratch.p + (q & 1) * sort_count_words(); }

// The digit counts of the first depth pass when the preprocess accumulates them (the frame is
// small enough), else {NULL}. *zero_words: the cells frame_begin must clear for it. The persistent
// sort chunks the pass over its CTAs and keeps the matrix CTA-major (its passes are always 8-bit);
// the multi-kernel sort over its spans, digit-major, with 9-bit digits in a short frame.
PassCounts first_pass_counts(Arena& A, unsigned entries, bool short_depth, unsigned* zero_words) {
    *zero_words = 0;
    if (entries == 0 || entries > kProducerCountMax) return PassCounts{};
    if (A.ctas) {
        *zero_words = A.ctas << kDepthBits;
        return PassCounts{A.pcounts.p, A.ctas, 0u, (1u << kDepthBits) - 1, 1u, 1u << kDepthBits};
    }
    const int bits = short_depth ? kShortDepthBits : kDepthBits;
    const unsigned spans = sort_spans(entries);
    *zero_words = spans << bits;
    return PassCounts{count_matrix(A, 0), spans, 0u, (1u << bits) - 1, spans, 1u};
}

// Steps 2-4 of a frame as one cooperative launch (sort_persistent.cu); *final_buf as enqueue_sort.
int enqueue_sort_persistent(Arena& A, unsigned entries, unsigned tiles, const BatchTables& tables, bool keep_rank,
                            int bits, bool first_counted, cudaStream_t st, int* final_buf) {
    SortFrameArgs a{};
    a.depth_key = A.depth_key.p;
    a.rect16 = A.rect16.p;
    for (int k = 0; k < 2; ++k) {
        a.vis_key[k] = A.vis_key[k].p;
        a.vis_idx[k] = A.vis_idx[k].p;
        a.pair_key[k] = A.pair_key[k].p;
        a.pair_val[k] = A.pair_val[k].p;
        a.counts[k] = A.pcounts.p + k * persistent_sort_count_words(A.ctas);
    }
    a.offs = A.offs.p;
    a.rank = keep_rank ? A.rank.p : nullptr;
    a.rect_sorted = A.rect_sorted.p;
    a.chunk_first = A.chunk_first.p;
    a.span_sum = A.span_sum.p;
    a.ranges = A.ranges.p;
    a.ctrl = A.ctrl.p;
    a.tables = tables;
    a.entries = entries;
    a.pair_cap = A.pair_cap;
    a.tile_passes = tile_pass_widths(tiles, bits, a.tile_bits);
    a.first_counted = first_counted ? 1 : 0;
    AB_CUDA(launch_sort_frame(a, A.ctas, st));
    *final_buf = a.tile_passes & 1;
    return 0;
}

// Depth passes over `entries` depth keys (the first compacts the visible ones), pair scan and
// expansion, tile passes over `tiles` global tiles, and ranges (cleared beforehand by
// frame_begin). *final_buf = the pair buffer that holds the sorted pairs. keep_rank: also record
// each visible entry's depth-sorted position (the adjoint reads it). first_counted: the depth
// keys' producer accumulated the first depth pass's digit counts (first_pass_counts). In a small
// frame the expansion likewise counts the first tile pass, the last depth pass's span scan clearing
// that count matrix first; every other pass has its own upsweep. (Counting in the downsweeps too
// was measured slower: keys written next to each other often share the next digit, the high depth
// digits taking few values, so one atomic per key contends -- 0.177 ms against 0.139 ms for the
// sort of the 740k / 1280x720 frame.) A frame of at most bin_max_tiles() tiles (A.bins_for) takes
// the one-pass tile binning after the expansion instead of the tile passes and the ranges.
// short_depth: every visible key is below 2^27 (Plan::bound_depth), so three 9-bit depth passes
// replace the four 8-bit ones (measured 0.119 -> 0.111 ms of sort for the 740k frame). Where the
// persistent sort is selected (A.ctas), it replaces this whole sequence with one launch and the
// same outputs.
int enqueue_sort(Arena& A, unsigned entries, unsigned tiles, const BatchTables& tables, bool keep_rank, int bits,
                 bool first_counted, bool short_depth, cudaStream_t st, int* final_buf) {
    if (A.ctas)
        return enqueue_sort_persistent(A, entries, tiles, tables, keep_rank, bits, first_counted, st, final_buf);
    const int depth_passes = short_depth ? kShortDepthPasses : kDepthPasses;
    const int depth_bits = short_depth ? kShortDepthBits : kDepthBits;
    Ctrl* ctrl = A.ctrl.p;
    const unsigned cap = static_cast<unsigned>(std::max<int64_t>(A.n, 0));
    unsigned* totals = A.sort_scratch.p + 2 * sort_count_words();
    int tile_bits[4];
    const int tile_passes = tile_pass_widths(tiles, bits, tile_bits);
    const bool bins = A.bins_for(tiles);
    const bool expand_counts = !bins && A.pair_cap <= kProducerCountMax;
    const unsigned tile_spans = sort_spans(A.pair_cap);
    const PassCounts first_tile =
        expand_counts
            ? PassCounts{count_matrix(A, depth_passes), tile_spans, 0u, (1u << tile_bits[0]) - 1, tile_spans, 1u}
            : PassCounts{};

    for (int p = 0; p < depth_passes; ++p) {
        const int src = (p + 1) & 1, dst = p & 1;  // pass 0 reads depth_key and writes buffer 0
        const unsigned* keys_in = p == 0 ? A.depth_key.p : A.vis_key[src].p;
        const SortCount count = p == 0 ? SortCount::kFixed : SortCount::kVisible;
        const unsigned capacity = p == 0 ? entries : cap;
        if (!(p == 0 && first_counted))
            launch_radix_count(keys_in, p == 0, count, entries, capacity, p * depth_bits, depth_bits,
                               count_matrix(A, p), ctrl, st);
        const bool last = p == depth_passes - 1;
        launch_radix_scatter(keys_in, p == 0 ? nullptr : A.vis_idx[src].p, last ? nullptr : A.vis_key[dst].p,
                             A.vis_idx[dst].p, p == 0, count, entries, capacity, p * depth_bits, depth_bits,
                             count_matrix(A, p), totals, last ? first_tile.counts : nullptr,
                             last && expand_counts ? tile_spans << tile_bits[0] : 0u, ctrl, st);
    }
    const int sorted = (depth_passes - 1) & 1;
    const DupBuffers dup{A.offs.p, keep_rank ? A.rank.p : nullptr, A.rect_sorted.p, A.chunk_start.p, A.span_sum.p};
    if (bins) {  // one stable counting pass over the tile id (and the ranges) instead of the tile passes
        launch_duplicate(A.vis_idx[sorted].p, A.rect16.p, ctrl, A.pair_cap, entries, tables, dup, A.pair_key[0].p,
                         A.pair_val[0].p, st, PassCounts{}, A.bin_counts.p, tiles);
        launch_tile_bins(A.pair_key[0].p, A.pair_val[0].p, A.pair_key[1].p, A.pair_val[1].p, A.bin_counts.p, tiles,
                         A.tile_start.p, A.ranges.p, ctrl, A.pair_cap, st);
        *final_buf = 1;
        return 0;
    }
    launch_duplicate(A.vis_idx[sorted].p, A.rect16.p, ctrl, A.pair_cap, entries, tables, dup, A.pair_key[0].p,
                     A.pair_val[0].p, st, first_tile);
    for (int t = 0, shift = 0; t < tile_passes; shift += tile_bits[t], ++t) {
        const int q = depth_passes + t;
        const int src = t & 1, dst = src ^ 1;
        if (!(t == 0 && expand_counts))
            launch_radix_count(A.pair_key[src].p, false, SortCount::kPairs, 0u, A.pair_cap, shift, tile_bits[t],
                               count_matrix(A, q), ctrl, st);
        launch_radix_scatter(A.pair_key[src].p, A.pair_val[src].p, A.pair_key[dst].p, A.pair_val[dst].p, false,
                             SortCount::kPairs, 0u, A.pair_cap, shift, tile_bits[t], count_matrix(A, q), totals,
                             nullptr, 0u, ctrl, st);
    }
    const int fin = tile_passes & 1;
    launch_ranges(A.pair_key[fin].p, ctrl, A.pair_cap, A.ranges.p, st);
    *final_buf = fin;
    return 0;
}

// The per-view constants, packed as gpu_render.cu:301-316 packs them (doubles cast to float; the
// eye is Camera::centre(), camera.cpp:19-23, computed in double); tiles in the plan's shape.
int pack_camera(int scene_degree, int rendered_degree, const aniso_b200_camera* c, float splat_scale, int tile_w,
                int tile_h, CamParams& cp) {
    if (!c) return fail(ANISO_B200_ERR_ARGUMENT, "camera is NULL");
    if (c->width <= 0 || c->height <= 0 || c->width > 32767 || c->height > 32767)
        return fail(ANISO_B200_ERR_ARGUMENT, "camera size must be in [1, 32767]");
    std::memset(&cp, 0, sizeof cp);
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) cp.R[r * 3 + k] = static_cast<float>(c->R[r * 3 + k]);
        cp.t[r] = static_cast<float>(c->t[r]);
    }
    const double* R = c->R;
    const double* t = c->t;
    cp.eye[0] = static_cast<float>(-(R[0] * t[0] + R[3] * t[1] + R[6] * t[2]));
    cp.eye[1] = static_cast<float>(-(R[1] * t[0] + R[4] * t[1] + R[7] * t[2]));
    cp.eye[2] = static_cast<float>(-(R[2] * t[0] + R[5] * t[1] + R[8] * t[2]));
    cp.fx = static_cast<float>(c->fx);
    cp.fy = static_cast<float>(c->fy);
    cp.cx = static_cast<float>(c->cx);
    cp.cy = static_cast<float>(c->cy);
    cp.width = c->width;
    cp.height = c->height;
    cp.tilesX = (c->width + tile_w - 1) / tile_w;
    cp.tilesY = (c->height + tile_h - 1) / tile_h;
    cp.shDegree = rendered_degree;
    cp.shCoeffs = (scene_degree + 1) * (scene_degree + 1);
    cp.splatScale = splat_scale;
    return 0;
}

// ---- plans ---------------------------------------------------------------------------------

// Launch shape of a plan. A single-view render uses 16x16 tiles (the reference's) and 128-splat
// blend rounds (measured 0.321 against 0.325 ms per 740k frame with 256); batches take theirs from
// their options (the autotuner's choice).
struct PlanShape {
    int tile_w = kTile, tile_h = kTile, blend_batch = 128, sh_degree = 3, radix_bits = kRadixBits;
    float splat_scale = 1.0f;
    bool use_graph = false;
};

int check_options(const aniso_b200_batch_options* o, PlanShape& shape) {
    if (!o) return 0;
    shape.sh_degree = o->sh_degree;
    shape.splat_scale = o->splat_scale;
    shape.tile_w = o->tile_w ? o->tile_w : kTile;
    shape.tile_h = o->tile_h ? o->tile_h : kTile;
    shape.blend_batch = o->blend_batch ? o->blend_batch : 256;
    shape.radix_bits = o->radix_bits ? o->radix_bits : kRadixBits;
    shape.use_graph = o->use_graph != 0;
    if (shape.sh_degree < 0) return fail(ANISO_B200_ERR_ARGUMENT, "sh_degree must be >= 0");
    if (!radix_bits_supported(shape.radix_bits)) return fail(ANISO_B200_ERR_ARGUMENT, "radix_bits must be 8 or 9");
    if (!blend_shape_supported(shape.tile_w, shape.tile_h))
        return fail(ANISO_B200_ERR_ARGUMENT, "tile shape must be 8x8, 16x16 or 16x32");
    return 0;
}

// The axis-aligned box of a scene's Gaussian positions, measured once when the scene is made;
// finite is false when the scene has a position that is not finite (or no box was measured).
struct PositionBox {
    bool finite = false;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// Whether every depth this camera can give a position in `box` is below the short keys' limit
// (8192): the largest camera-space z over the box's corners, plus a margin far above the rounding
// of the projection's fp32 z (R[6] x + R[7] y + R[8] z + t[2]), must stay below it.
bool depth_short(const PositionBox& box, const CamParams& cam) {
    if (!box.finite) return false;
    double z = cam.t[2], mag = std::fabs(cam.t[2]);
    for (int i = 0; i < 3; ++i) {
        const double r = cam.R[6 + i];
        z += std::max(r * box.lo[i], r * box.hi[i]);
        mag += std::fabs(r) * std::max(std::fabs(box.lo[i]), std::fabs(box.hi[i]));
    }
    // 2^27 keys above 0.125's bits span 2^(27 - 23) = 16 binades: depths below 0.125 * 2^16.
    const double limit = std::ldexp(0.125, 1 << (kShortDepthKeyBits - 23));
    return z + 1e-5 * mag + 1.0 < limit;  // false for a NaN
}

// V views of S scenes: host tables, uploaded as one blob to a slot before each frame.
template <class Src>
struct Plan {
    PlanShape shape;
    std::vector<ViewInfo> views;
    std::vector<BatchScene<Src>> scenes;
    std::vector<unsigned> entry_base, tile_base, tiles_x;
    std::vector<RawGrads> grads;  // the backward's gradient buffers, one per scene (empty otherwise)
    uint64_t entries = 0, tiles = 0;
    unsigned pre_blocks = 0;
    bool short_depth = false;  // three 9-bit depth passes (bound_depth)

    // srcs[s], stored degree deg[s]; view k of scene view_scene[k] (consecutive per scene).
    int build(const std::vector<Src>& srcs, const std::vector<int>& deg, const int32_t* view_scene, int n_views,
              const aniso_b200_camera* cameras, const PlanShape& sh) {
        shape = sh;
        const int S = static_cast<int>(srcs.size());
        if (S <= 0 || n_views <= 0 || !view_scene || !cameras)
            return fail(ANISO_B200_ERR_ARGUMENT, "a batch needs at least one scene and one view");
        // Each view is coloured up to min(option, its scene's degree, 3), as gpu_render.cu:314 does
        // per scene; the preprocess kernel is instantiated for the largest of them.
        const int wanted = std::min(sh.sh_degree, 3);
        views.assign(n_views, ViewInfo{});
        scenes.assign(S, BatchScene<Src>{});
        entry_base.assign(n_views, 0);
        tile_base.assign(n_views, 0);
        tiles_x.assign(n_views, 0);
        std::vector<int> first(S, -1), last(S, -1);
        entries = tiles = 0;
        for (int k = 0; k < n_views; ++k) {
            const int s = view_scene[k];
            if (s < 0 || s >= S) return fail(ANISO_B200_ERR_ARGUMENT, "view_scene out of range");
            if (first[s] < 0) first[s] = k;
            else if (last[s] != k - 1) return fail(ANISO_B200_ERR_ARGUMENT, "the views of a scene must be consecutive");
            last[s] = k;
            ViewInfo& v = views[k];
            AB_TRY(pack_camera(deg[s], std::min(wanted, deg[s]), &cameras[k], sh.splat_scale, sh.tile_w, sh.tile_h,
                               v.cam));
            v.scene = static_cast<unsigned>(s);
            v.n = static_cast<unsigned>(srcs[s].n);
            v.entry_base = static_cast<unsigned>(entries);
            v.tile_base = static_cast<unsigned>(tiles);
            entry_base[k] = v.entry_base;
            tile_base[k] = v.tile_base;
            tiles_x[k] = static_cast<unsigned>(v.cam.tilesX);
            entries += static_cast<uint64_t>(srcs[s].n);
            tiles += static_cast<uint64_t>(v.cam.tilesX) * v.cam.tilesY;
            if (entries > kMaxEntries || tiles > kMaxEntries)
                return fail(ANISO_B200_ERR_ARGUMENT, "more than 2^32 entries or tiles in one batch");
        }
        pre_blocks = 0;
        for (int s = 0; s < S; ++s) {
            scenes[s].src = srcs[s];
            scenes[s].view_begin = first[s] < 0 ? 0u : static_cast<unsigned>(first[s]);
            scenes[s].view_end = first[s] < 0 ? 0u : static_cast<unsigned>(last[s] + 1);
            scenes[s].block_base = pre_blocks;
            if (first[s] >= 0) pre_blocks += chunks_of(static_cast<uint64_t>(srcs[s].n), preprocess_gaussians_per_block());
        }
        return 0;
    }

    // Picks the short depth passes when every view's scene box (boxes[s], NULL: unknown) keeps its
    // depths below 8192 for the view's camera, and the frame has at most kProducerCountMax entries
    // (larger frames' 9-bit passes were measured slower: the 64-view 1M batch 8.69 -> 8.75 ms).
    // Without a call (the training path's positions change every step) the frame keeps 8-bit passes.
    void bound_depth(const std::vector<const PositionBox*>& boxes) {
        short_depth = entries > 0 && entries <= kProducerCountMax;
        for (const auto& v : views)
            if (v.scene >= boxes.size() || !boxes[v.scene] || !depth_short(*boxes[v.scene], v.cam)) short_depth = false;
    }

    // The largest degree any view is coloured with (the preprocess kernel's instantiation).
    int rendered_degree() const {
        int d = 0;
        for (const auto& v : views) d = std::max(d, v.cam.shDegree);
        return d;
    }
    // Blob layout: views, scenes, the three per-view tables, then (16-byte aligned) the gradients.
    size_t grads_offset() const {
        const size_t b = views.size() * sizeof(ViewInfo) + scenes.size() * sizeof(BatchScene<Src>) +
                         3 * views.size() * sizeof(unsigned);
        return (b + 15) / 16 * 16;
    }
    size_t blob_bytes() const { return grads_offset() + grads.size() * sizeof(RawGrads); }
    // Same launch geometry (the only thing a recorded graph fixes besides the slot).
    bool same_geometry(const Plan& o) const {
        if (views.size() != o.views.size() || scenes.size() != o.scenes.size() || entries != o.entries ||
            tiles != o.tiles || grads.size() != o.grads.size())
            return false;
        for (size_t s = 0; s < scenes.size(); ++s)
            if (scenes[s].src.n != o.scenes[s].src.n) return false;
        for (size_t k = 0; k < views.size(); ++k)
            if (views[k].cam.width != o.views[k].cam.width || views[k].cam.height != o.views[k].cam.height ||
                views[k].cam.shDegree != o.views[k].cam.shDegree)
                return false;
        return shape.tile_w == o.shape.tile_w && shape.tile_h == o.shape.tile_h &&
               shape.blend_batch == o.shape.blend_batch && shape.radix_bits == o.shape.radix_bits &&
               rendered_degree() == o.rendered_degree() && short_depth == o.short_depth;
    }
};

// The address at which the current device writes the host buffer p, when p is page-locked host
// memory mapped for this device (cudaHostAlloc, torch's pinned tensors, cudaHostRegister with
// mapping); else NULL (pageable memory, or pinned memory another device mapped).
uint8_t* mapped_host(void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? static_cast<uint8_t*>(a.devicePointer) : nullptr;
}

// Device copy of a plan's tables, filled from a pinned staging blob on the render stream (by the
// frame's first kernel through the blob's device mapping, else by a copy). A slot is restaged only
// after the frame that read it has run (its event). The blob's size depends only on the numbers of
// views and scenes, which a recorded graph's geometry fixes, so restaging a graph's slot never
// moves the blob the recorded upload reads.
struct Slot {
    DevBuf<unsigned char> dev;
    unsigned char* pinned = nullptr;
    const unsigned char* pinned_dev = nullptr;  // the device's address of `pinned`, NULL if unmapped
    size_t cap = 0;
    cudaEvent_t done = nullptr;
    bool pending = false;
    Slot() = default;
    Slot(const Slot&) = delete;
    Slot& operator=(const Slot&) = delete;
    ~Slot() {
        if (pinned) cudaFreeHost(pinned);
        if (done) cudaEventDestroy(done);
    }
    // Writes the blob (after the frame that last read this slot has run) without copying it.
    template <class Src>
    int stage(const Plan<Src>& P) {
        if (pending) {
            AB_CUDA(cudaEventSynchronize(done));
            pending = false;
        }
        const size_t bytes = P.blob_bytes();
        if (bytes > cap) {
            if (pinned) cudaFreeHost(pinned);
            pinned = nullptr;
            pinned_dev = nullptr;
            AB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&pinned), bytes));
            pinned_dev = mapped_host(pinned);
            AB_TRY(dev.reserve(bytes));
            cap = bytes;
        }
        if (!done) AB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        const size_t V = P.views.size(), S = P.scenes.size();
        unsigned char* h = pinned;
        std::memcpy(h, P.views.data(), V * sizeof(ViewInfo));
        std::memcpy(h + V * sizeof(ViewInfo), P.scenes.data(), S * sizeof(BatchScene<Src>));
        unsigned* t = reinterpret_cast<unsigned*>(h + V * sizeof(ViewInfo) + S * sizeof(BatchScene<Src>));
        std::memcpy(t, P.entry_base.data(), V * sizeof(unsigned));
        std::memcpy(t + V, P.tile_base.data(), V * sizeof(unsigned));
        std::memcpy(t + 2 * V, P.tiles_x.data(), V * sizeof(unsigned));
        if (!P.grads.empty()) std::memcpy(h + P.grads_offset(), P.grads.data(), P.grads.size() * sizeof(RawGrads));
        return 0;
    }
    // The device address of the blob's gradient table (after fill).
    template <class Src>
    const RawGrads* grads_dev(const Plan<Src>& P) const {
        return reinterpret_cast<const RawGrads*>(dev.p + P.grads_offset());
    }
    // Stages the blob and enqueues its upload on `st` (a chained kernel reading the mapped staging
    // buffer, else a copy); returns the device views, scenes, tables. With `begin`, the frame's
    // start (frame_begin's clears) is enqueued too, in the same kernel as the upload where that is
    // a kernel.
    struct FrameBegin {
        Ctrl* ctrl;
        unsigned* zero;
        unsigned zero_words;
        uint2* ranges;
        unsigned tiles;
    };
    template <class Src>
    int fill(const Plan<Src>& P, cudaStream_t st, const ViewInfo** views, const BatchScene<Src>** scenes,
             BatchTables& tables, const FrameBegin* begin = nullptr) {
        AB_TRY(stage(P));
        const size_t bytes = P.blob_bytes();
        if (pinned_dev && bytes % 4 == 0) {
            if (begin)
                launch_frame_start(reinterpret_cast<const unsigned*>(pinned_dev), reinterpret_cast<unsigned*>(dev.p),
                                   static_cast<unsigned>(bytes / 4), begin->ctrl, begin->zero, begin->zero_words,
                                   begin->ranges, begin->tiles, st);
            else
                launch_upload(reinterpret_cast<const unsigned*>(pinned_dev), reinterpret_cast<unsigned*>(dev.p),
                              static_cast<unsigned>(bytes / 4), st);
        } else {
            AB_CUDA(cudaMemcpyAsync(dev.p, pinned, bytes, cudaMemcpyHostToDevice, st));
            if (begin)
                launch_frame_begin(begin->ctrl, begin->zero, begin->zero_words, begin->ranges, begin->tiles, st);
        }
        const size_t V = P.views.size(), S = P.scenes.size();
        unsigned char* d = dev.p;
        *views = reinterpret_cast<const ViewInfo*>(d);
        *scenes = reinterpret_cast<const BatchScene<Src>*>(d + V * sizeof(ViewInfo));
        const unsigned* dt = reinterpret_cast<const unsigned*>(d + V * sizeof(ViewInfo) + S * sizeof(BatchScene<Src>));
        tables.entry_base = dt;
        tables.tile_base = dt + V;
        tables.tiles_x = dt + 2 * V;
        tables.n_views = static_cast<unsigned>(V);
        return 0;
    }
    int mark(cudaStream_t st) {
        AB_CUDA(cudaEventRecord(done, st));
        pending = true;
        return 0;
    }
};

void launch_preprocess_any(const BatchScene<SceneView>* sc, const Plan<SceneView>& P, const ViewInfo* views, Arena& A,
                           const DebugProjection* dbg, const PassCounts& counts, cudaStream_t st) {
    launch_preprocess(sc, static_cast<unsigned>(P.scenes.size()), P.pre_blocks, views, P.rendered_degree(),
                      P.shape.tile_w, P.shape.tile_h, A.rec.p, A.rect16.p, A.depth_key.p, dbg, counts,
                      static_cast<unsigned>(P.entries), st);
}
void launch_preprocess_any(const BatchScene<RawParams>* sc, const Plan<RawParams>& P, const ViewInfo* views,
                           Arena& A, const DebugProjection*, const PassCounts& counts, cudaStream_t st) {
    launch_preprocess_raw(sc, static_cast<unsigned>(P.scenes.size()), P.pre_blocks, views, P.rendered_degree(),
                          P.shape.tile_w, P.shape.tile_h, A.rec.p, A.rect16.p, A.depth_key.p, counts,
                          static_cast<unsigned>(P.entries), st);
}

// Enqueues one frame of a plan. ev (4 events, may be NULL) brackets the stages.
template <class Src>
int enqueue_plan(Arena& A, Slot& slot, const Plan<Src>& P, cudaStream_t st, cudaEvent_t* ev,
                 const DebugProjection* dbg, bool stop_after_sort, bool train, int* final_buf, bool mark_slot = true) {
    const ViewInfo* views = nullptr;
    const BatchScene<Src>* scenes = nullptr;
    BatchTables tables;
    AB_TRY(A.reserve_ranges(static_cast<size_t>(P.tiles)));
    unsigned zero_words = 0;
    const PassCounts first = first_pass_counts(A, static_cast<unsigned>(P.entries), P.short_depth, &zero_words);
    if (ev) AB_CUDA(cudaEventRecord(ev[0], st));
    const Slot::FrameBegin begin{A.ctrl.p, first.counts, zero_words, A.ranges.p, static_cast<unsigned>(P.tiles)};
    AB_TRY(slot.fill(P, st, &views, &scenes, tables, &begin));
    launch_preprocess_any(scenes, P, views, A, dbg, first, st);
    if (ev) AB_CUDA(cudaEventRecord(ev[1], st));
    int fin = 0;
    AB_TRY(enqueue_sort(A, static_cast<unsigned>(P.entries), static_cast<unsigned>(P.tiles), tables, train,
                        P.shape.radix_bits, first.counts != nullptr, P.short_depth, st, &fin));
    if (ev) AB_CUDA(cudaEventRecord(ev[2], st));
    if (!stop_after_sort)
        launch_blend(static_cast<unsigned>(P.tiles), A.ranges.p, A.pair_val[fin].p, A.rec.p, A.ctrl.p, views, tables,
                     P.shape.tile_w, P.shape.tile_h, P.shape.blend_batch, train, st);
    if (ev) AB_CUDA(cudaEventRecord(ev[3], st));
    AB_CUDA(cudaGetLastError());
    if (mark_slot) AB_TRY(slot.mark(st));
    if (final_buf) *final_buf = fin;
    return 0;
}

// Reads the control block of the last frame on `st` (waits for it) into `host` (page-locked). The
// frame's flags are then consumed: they are cleared on the device, so that the next frame_begin
// does not fold them into the sticky flags as if no one had seen them. Where the device maps
// `host`, one chained kernel does both; else a copy and a memset.
int read_ctrl(const Arena& A, Ctrl* host, cudaStream_t st) {
    if (Ctrl* mapped = reinterpret_cast<Ctrl*>(mapped_host(host))) {
        launch_publish_ctrl(A.ctrl.p, mapped, st);
        AB_CUDA(cudaGetLastError());
    } else {
        AB_CUDA(cudaMemcpyAsync(host, A.ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        AB_CUDA(cudaMemsetAsync(&A.ctrl.p->flags, 0, sizeof(unsigned), st));
    }
    AB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

// After a synchronised frame: grows the pair buffers on overflow (*again = 1: render it again).
// With all_frames, also looks at the frames before the last one (the sticky fields). The caller
// has waited for every frame that used the buffers (read_ctrl after the owner's last frame), so
// they are released without waiting for the rest of the device.
int settle(Arena& A, const Ctrl& h, int* again, bool all_frames) {
    *again = 0;
    const unsigned flags = h.flags | (all_frames ? h.sticky_flags : 0u);
    const uint64_t pairs = all_frames ? std::max(h.pair_total, h.max_pair_total) : h.pair_total;
    if (flags & kFlagWaitTimeout)  // the persistent sort's bounded grid-barrier wait gave up
        return fail(ANISO_B200_ERR_DEVICE_WAIT, "a sort grid barrier wait gave up: the frame was not rendered");
    if (flags & kFlagOverflow) {
        const uint64_t need = pairs + pairs / 4 + 1024;
        if (need > kMaxPairs) return fail(ANISO_B200_ERR_ARGUMENT, "more than 2^30 splat-tile pairs");
        AB_TRY(A.grow_pairs(static_cast<unsigned>(need)));
        *again = 1;
    }
    return 0;
}

int clear_sticky(Arena& A, cudaStream_t st) {
    AB_CUDA(cudaMemsetAsync(&A.ctrl.p->sticky_flags, 0, sizeof(unsigned), st));
    AB_CUDA(cudaMemsetAsync(&A.ctrl.p->max_pair_total, 0, sizeof(unsigned long long), st));
    AB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

constexpr int kSlots = 8;

// The order of one object's frames (a scene's, a batch's or a trainer's, which share its work
// buffers) over the caller streams they are enqueued on, and the wait for them. Frames on one
// stream are ordered by the stream; when the caller switches streams, the new stream first waits
// (an event) for the last frame on the old one, so the object's frames form one chain. Waiting for
// the object then means waiting for the end of that chain -- never for the rest of the device, so
// objects rendering on different streams do not serialise each other's syncs.
struct StreamChain {
    cudaStream_t last = nullptr;
    bool any = false;
    cudaEvent_t ev = nullptr;
    StreamChain() = default;
    StreamChain(const StreamChain&) = delete;
    StreamChain& operator=(const StreamChain&) = delete;
    ~StreamChain() {
        if (ev) cudaEventDestroy(ev);
    }
    // Makes `st` wait for the chain's last frame if that went to another stream.
    int join(cudaStream_t st) {
        if (!any || st == last) return 0;
        if (!ev) AB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        AB_CUDA(cudaEventRecord(ev, last));
        AB_CUDA(cudaStreamWaitEvent(st, ev, 0));
        return 0;
    }
    // A frame was enqueued on `st` (after join(st)).
    void extend(cudaStream_t st) {
        last = st;
        any = true;
    }
    // Blocks the host until the chain's last frame has run (for destructors; errors ignored).
    void wait_host() {
        if (!any) return;
        if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        if (cudaEventRecord(ev, last) == cudaSuccess) cudaEventSynchronize(ev);
        cudaGetLastError();
        // The chain stays as it is: work enqueued after this wait still goes to `last`, and the
        // next join must order behind it.
    }
};

}  // namespace

namespace ab2 {
// For entry points defined in other files: sets the aniso_b200_last_error message, returns code.
int report_error(int code, const char* msg) { return fail(code, msg); }

static thread_local uint64_t t_chained_launches = 0;
uint64_t chained_launches() { return t_chained_launches; }
void note_chained_launch() { ++t_chained_launches; }

bool chain_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("ANISO_B200_CHAIN");
        return !(v && v[0] == '0');
    }();
    return on;
}
}  // namespace ab2

// ---- scenes ------------------------------------------------------------------------------------

struct aniso_b200_scene {
    int64_t n = 0;
    int degree = 0;
    int planes = 0;
    DevBuf<float4> pos_op, scale, rot, sh;
    PositionBox box;  // of pos_op's positions, measured when the scene is made
    Arena arena;  // work buffers of the scene's own renders
    Slot slots[kSlots];
    int next_slot = 0;
    DevBuf<uint8_t> image;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    Ctrl* host_ctrl = nullptr;  // pinned
    // Stage events of profiled render_device frames: 4 per frame, reused after each read.
    bool profiling = false;
    std::vector<cudaEvent_t> prof_ev;
    size_t prof_frames = 0;
    int32_t frame_kernels = 0;  // kernels the last frame launched
    StreamChain chain;          // the streams the scene's frames went to

    SceneView view() const {
        SceneView v;
        v.pos_op = pos_op.p;
        v.scale = scale.p;
        v.rot = rot.p;
        v.sh = sh.p;
        v.n = n;
        v.sh_planes = planes;
        return v;
    }
    Slot& slot() { return slots[next_slot++ % kSlots]; }
    ~aniso_b200_scene() {
        chain.wait_host();
        if (stream) cudaStreamSynchronize(stream);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : prof_ev) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        if (host_ctrl) cudaFreeHost(host_ctrl);
    }
};

namespace {

__global__ void ingest_kernel(const float* __restrict__ gauss, const float* __restrict__ shin, int64_t n, int k3,
                              int planes, float4* __restrict__ pos_op, float4* __restrict__ scale,
                              float4* __restrict__ rot, float4* __restrict__ sh) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* g = gauss + i * 11;
    pos_op[i] = make_float4(g[0], g[1], g[2], g[10]);
    scale[i] = make_float4(g[3], g[4], g[5], 0.f);
    rot[i] = make_float4(g[6], g[7], g[8], g[9]);
    const float* s = shin + i * k3;
    for (int p = 0; p < planes; ++p) {
        float4 f;
        f.x = 4 * p + 0 < k3 ? s[4 * p + 0] : 0.f;
        f.y = 4 * p + 1 < k3 ? s[4 * p + 1] : 0.f;
        f.z = 4 * p + 2 < k3 ? s[4 * p + 2] : 0.f;
        f.w = 4 * p + 3 < k3 ? s[4 * p + 3] : 0.f;
        sh[i * planes + p] = f;
    }
}

// ply_loader.cpp:124-138 on the device: exp(scale), sigmoid(opacity), normalised quaternion,
// f_rest reordered from channel-major to [coefficient][channel].
__global__ void ingest_raw_kernel(const float* __restrict__ xyz, const float* __restrict__ f_dc,
                                  const float* __restrict__ f_rest, const float* __restrict__ opacity,
                                  const float* __restrict__ log_scale, const float* __restrict__ rotin, int64_t n,
                                  int coeffs, int planes, float4* __restrict__ pos_op, float4* __restrict__ scale,
                                  float4* __restrict__ rot, float4* __restrict__ sh) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pos_op[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 1.0f / (1.0f + expf(-opacity[i])));
    scale[i] = make_float4(expf(log_scale[3 * i]), expf(log_scale[3 * i + 1]), expf(log_scale[3 * i + 2]), 0.f);
    const float qw = rotin[4 * i], qx = rotin[4 * i + 1], qy = rotin[4 * i + 2], qz = rotin[4 * i + 3];
    const float nrm = sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    rot[i] = nrm > 0 ? make_float4(qw / nrm, qx / nrm, qy / nrm, qz / nrm) : make_float4(1.f, 0.f, 0.f, 0.f);
    const int k3 = coeffs * 3, rest = coeffs - 1;
    for (int p = 0; p < planes; ++p) {
        float v[4];
        for (int e = 0; e < 4; ++e) {
            const int f = 4 * p + e;  // float index in [coefficient][channel] order
            if (f >= k3) {
                v[e] = 0.f;
                continue;
            }
            const int k = f / 3, c = f % 3;
            v[e] = k == 0 ? f_dc[3 * i + c] : f_rest[i * 3 * rest + c * rest + (k - 1)];
        }
        sh[i * planes + p] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// Where each needed value sits in a PLY vertex row (float columns, in file order).
struct PlyColumns {
    int stride;                  // floats per row
    int x, y, z, opacity;
    int scale[3], rot[4], dc[3];
    int rest[72];                // f_rest_0.. (channel-major), 3((d+1)^2 - 1) of them, d <= 4
};

// ply_loader.cpp:113-134 on the device, straight from the file's vertex block (one row of `stride`
// floats per Gaussian): position, exp(scale), sigmoid(opacity), the normalised quaternion, and
// f_dc / f_rest reordered to [coefficient][channel]; packed into the 16-byte SoA words.
__global__ void ingest_ply_kernel(const float* __restrict__ body, int64_t n, PlyColumns col, int coeffs, int planes,
                                  float4* __restrict__ pos_op, float4* __restrict__ scale, float4* __restrict__ rot,
                                  float4* __restrict__ sh) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* v = body + i * col.stride;
    pos_op[i] = make_float4(v[col.x], v[col.y], v[col.z], 1.0f / (1.0f + expf(-v[col.opacity])));
    scale[i] = make_float4(expf(v[col.scale[0]]), expf(v[col.scale[1]]), expf(v[col.scale[2]]), 0.f);
    const float qw = v[col.rot[0]], qx = v[col.rot[1]], qy = v[col.rot[2]], qz = v[col.rot[3]];
    const float nrm = sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    rot[i] = nrm > 0 ? make_float4(qw / nrm, qx / nrm, qy / nrm, qz / nrm) : make_float4(1.f, 0.f, 0.f, 0.f);
    const int k3 = coeffs * 3, rest = coeffs - 1;
    for (int p = 0; p < planes; ++p) {
        float w[4];
        for (int e = 0; e < 4; ++e) {
            const int f = 4 * p + e;  // float index in [coefficient][channel] order
            if (f >= k3) {
                w[e] = 0.f;
                continue;
            }
            const int k = f / 3, c = f % 3;
            w[e] = k == 0 ? v[col.dc[c]] : v[col.rest[c * rest + (k - 1)]];
        }
        sh[i * planes + p] = make_float4(w[0], w[1], w[2], w[3]);
    }
}

// The header rules and messages of ply_loader.cpp:20-65 and 77-104: binary little-endian, one
// vertex element of float properties (others must be empty), the named columns present, the
// f_rest count matching a degree 0..4.
int parse_ply_header(FILE* f, const std::string& name, int64_t* count, PlyColumns* col, int* degree, long* body) {
    char line[512];
    if (!std::fgets(line, sizeof line, f) || std::strncmp(line, "ply", 3) != 0)
        return fail(ANISO_B200_ERR_ARGUMENT, name + ": not a PLY file");
    bool in_vertex = false, saw_format = false;
    int64_t n = 0;
    std::vector<std::string> props;
    while (std::fgets(line, sizeof line, f)) {
        std::string l(line);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
        char w0[64] = {0}, w1[128] = {0}, w2[128] = {0};
        const int got = std::sscanf(l.c_str(), "%63s %127s %127s", w0, w1, w2);
        if (got < 1) continue;
        const std::string word = w0;
        if (word == "format") {
            if (std::string(w1) != "binary_little_endian")
                return fail(ANISO_B200_ERR_ARGUMENT,
                            name + ": only binary_little_endian PLY is supported, got " + std::string(w1));
            saw_format = true;
        } else if (word == "element") {
            const long long c = got >= 3 ? std::atoll(w2) : 0;
            in_vertex = std::string(w1) == "vertex";
            if (in_vertex) n = c;
            else if (c != 0) return fail(ANISO_B200_ERR_ARGUMENT, name + ": unexpected element '" + std::string(w1) + "'");
        } else if (word == "property") {
            if (!in_vertex) continue;
            const std::string type = w1;
            if (type != "float" && type != "float32")
                return fail(ANISO_B200_ERR_ARGUMENT,
                            name + ": property '" + std::string(w2) + "' has type " + type + ", expected float");
            props.push_back(w2);
        } else if (word == "end_header") {
            if (!saw_format) return fail(ANISO_B200_ERR_ARGUMENT, name + ": missing format line");
            *body = std::ftell(f);
            const auto find = [&](const std::string& p, int* out) {
                for (size_t k = 0; k < props.size(); ++k)
                    if (props[k] == p) {
                        *out = static_cast<int>(k);
                        return 0;
                    }
                return fail(ANISO_B200_ERR_ARGUMENT, name + ": missing property '" + p + "'");
            };
            col->stride = static_cast<int>(props.size());
            AB_TRY(find("x", &col->x));
            AB_TRY(find("y", &col->y));
            AB_TRY(find("z", &col->z));
            AB_TRY(find("opacity", &col->opacity));
            for (int k = 0; k < 3; ++k) AB_TRY(find("scale_" + std::to_string(k), &col->scale[k]));
            for (int k = 0; k < 4; ++k) AB_TRY(find("rot_" + std::to_string(k), &col->rot[k]));
            for (int k = 0; k < 3; ++k) AB_TRY(find("f_dc_" + std::to_string(k), &col->dc[k]));
            int rest = 0;
            while (rest < 72) {
                int c = -1;
                const std::string p = "f_rest_" + std::to_string(rest);
                bool found = false;
                for (size_t k = 0; k < props.size(); ++k)
                    if (props[k] == p) {
                        c = static_cast<int>(k);
                        found = true;
                        break;
                    }
                if (!found) break;
                col->rest[rest++] = c;
            }
            *degree = -1;
            for (int d = 0; d <= 4; ++d)
                if (rest == 3 * ((d + 1) * (d + 1) - 1)) *degree = d;
            if (*degree < 0)
                return fail(ANISO_B200_ERR_ARGUMENT,
                            name + ": " + std::to_string(rest) + " f_rest properties do not match any SH degree");
            *count = n;
            return 0;
        }
    }
    return fail(ANISO_B200_ERR_ARGUMENT, name + ": header has no end_header");
}

// Scenes may store up to degree 4 (the degrees the reference loader accepts, ply_loader.cpp:67-73);
// colour is evaluated up to degree 3, as both reference renderers do.
int validate_degree(int d) {
    if (d < 0 || d > 4) return fail(ANISO_B200_ERR_ARGUMENT, "scene sh_degree must be 0..4");
    return 0;
}

int device_present() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(ANISO_B200_ERR_NO_DEVICE, "no CUDA device");
    }
    return 0;
}

constexpr int kBoxBlocks = 296;  // 2 CTAs per SM, 256 threads each, grid-strided

// Per CTA, 7 floats: the smallest and largest x, y, z over the finite coordinates of the positions
// (x, y, z of pos[i]) this CTA visits, and 1 when one of its coordinates was not finite, else 0.
__global__ void __launch_bounds__(256) position_box_kernel(const float4* __restrict__ pos, int64_t n,
                                                           float* __restrict__ out) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float bad = 0.f;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float4 p = pos[i];
        const float c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (!isfinite(c[k])) {
                bad = 1.f;
                continue;
            }
            lo[k] = fminf(lo[k], c[k]);
            hi[k] = fmaxf(hi[k], c[k]);
        }
    }
    __shared__ float s[8][7];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], o));
        }
        bad = fmaxf(bad, __shfl_xor_sync(0xFFFFFFFFu, bad, o));
    }
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) {
            s[warp][k] = lo[k];
            s[warp][3 + k] = hi[k];
        }
        s[warp][6] = bad;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        float v = s[0][threadIdx.x];
        for (int w = 1; w < 8; ++w)
            v = threadIdx.x < 3 ? fminf(v, s[w][threadIdx.x]) : fmaxf(v, s[w][threadIdx.x]);
        out[blockIdx.x * 7 + threadIdx.x] = v;
    }
}

// Measures the scene's position box (after the positions were written on s->stream; waits).
int measure_box(aniso_b200_scene* s) {
    s->box = PositionBox{};
    if (s->n <= 0) return 0;
    DevBuf<float> d;
    AB_TRY(d.reserve(kBoxBlocks * 7));
    position_box_kernel<<<kBoxBlocks, 256, 0, s->stream>>>(s->pos_op.p, s->n, d.p);
    AB_CUDA(cudaGetLastError());
    std::vector<float> h(kBoxBlocks * 7);
    AB_CUDA(cudaMemcpyAsync(h.data(), d.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    AB_CUDA(cudaStreamSynchronize(s->stream));
    PositionBox b;
    b.finite = true;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = INFINITY;
        b.hi[k] = -INFINITY;
    }
    for (int c = 0; c < kBoxBlocks; ++c) {
        const float* r = &h[c * 7];
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = std::min(b.lo[k], static_cast<double>(r[k]));
            b.hi[k] = std::max(b.hi[k], static_cast<double>(r[3 + k]));
        }
        if (r[6] != 0.f) b.finite = false;
    }
    for (int k = 0; k < 3; ++k)
        if (!(b.lo[k] <= b.hi[k])) b.finite = false;  // no finite coordinate on an axis
    s->box = b;
    return 0;
}

int new_scene(int64_t n, int degree, aniso_b200_scene** out, aniso_b200_scene** made) {
    if (!out) return fail(ANISO_B200_ERR_ARGUMENT, "out is NULL");
    if (n < 0 || n >= (int64_t(1) << 31)) return fail(ANISO_B200_ERR_ARGUMENT, "n must be in [0, 2^31)");
    AB_TRY(validate_degree(degree));
    AB_TRY(device_present());
    aniso_b200_scene* s = new (std::nothrow) aniso_b200_scene();
    if (!s) return fail(ANISO_B200_ERR_OUT_OF_MEMORY, "host allocation failed");
    *made = s;
    s->n = n;
    s->degree = degree;
    const int coeffs = (degree + 1) * (degree + 1);
    s->planes = (coeffs * 3 + 3) / 4;
    const size_t nn = static_cast<size_t>(std::max<int64_t>(n, 1));
    AB_TRY(s->pos_op.reserve(nn));
    AB_TRY(s->scale.reserve(nn));
    AB_TRY(s->rot.reserve(nn));
    AB_TRY(s->sh.reserve(nn * s->planes));
    AB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    for (auto& e : s->ev) AB_CUDA(cudaEventCreate(&e));
    AB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s->host_ctrl), sizeof(Ctrl)));
    std::memset(s->host_ctrl, 0, sizeof(Ctrl));
    return s->arena.ensure(std::max<int64_t>(n, 1));
}

PlanShape scene_shape(const aniso_b200_options* o) {
    PlanShape shape;
    shape.sh_degree = o ? o->sh_degree : 3;
    shape.splat_scale = o ? o->splat_scale : 1.0f;
    return shape;
}

// A plan of one view of one scene.
int single_plan(aniso_b200_scene* s, const aniso_b200_camera* camera, const aniso_b200_options* options,
                Plan<SceneView>& P) {
    if (options && options->sh_degree < 0) return fail(ANISO_B200_ERR_ARGUMENT, "sh_degree must be >= 0");
    const int32_t vs = 0;
    AB_TRY(P.build({s->view()}, {s->degree}, &vs, 1, camera, scene_shape(options)));
    P.bound_depth({&s->box});
    return 0;
}

}  // namespace

extern "C" {

size_t aniso_b200_last_error(char* buf, size_t len) {
    if (buf && len) {
        const size_t k = std::min(len - 1, g_err.size());
        std::memcpy(buf, g_err.data(), k);
        buf[k] = '\0';
    }
    return g_err.size();
}

int aniso_b200_available(int32_t* available) {
    if (!available) return fail(ANISO_B200_ERR_ARGUMENT, "available is NULL");
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) cudaGetLastError();
    *available = (e == cudaSuccess && count > 0) ? 1 : 0;
    return ANISO_B200_OK;
}

int aniso_b200_scene_create(const float* gaussians, const float* sh, int64_t n, int32_t sh_degree,
                            aniso_b200_scene** out) {
    if (n > 0 && (!gaussians || !sh)) return fail(ANISO_B200_ERR_ARGUMENT, "gaussians/sh is NULL");
    aniso_b200_scene* s = nullptr;
    int rc = new_scene(n, sh_degree, out, &s);
    if (rc == 0 && n > 0) {
        const int k3 = (sh_degree + 1) * (sh_degree + 1) * 3;
        float *dg = nullptr, *ds = nullptr;
        cudaError_t e = cudaMalloc(&dg, static_cast<size_t>(n) * 11 * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&ds, static_cast<size_t>(n) * k3 * sizeof(float));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dg, gaussians, static_cast<size_t>(n) * 11 * sizeof(float), cudaMemcpyHostToDevice,
                                s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ds, sh, static_cast<size_t>(n) * k3 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) {
            ingest_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s->stream>>>(
                dg, ds, n, k3, s->planes, s->pos_op.p, s->scale.p, s->rot.p, s->sh.p);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (dg) cudaFree(dg);
        if (ds) cudaFree(ds);
        if (e != cudaSuccess) rc = cuda_fail(e, "scene upload");
        else rc = measure_box(s);
    }
    if (rc != 0) {
        delete s;
        if (out) *out = nullptr;
        return rc;
    }
    *out = s;
    return ANISO_B200_OK;
}

int aniso_b200_scene_create_raw(const float* xyz, const float* f_dc, const float* f_rest, const float* opacity,
                                const float* log_scale, const float* rot, int64_t n, int32_t sh_degree,
                                aniso_b200_scene** out) {
    const int coeffs = (sh_degree + 1) * (sh_degree + 1);
    if (n > 0 && (!xyz || !f_dc || !opacity || !log_scale || !rot || (coeffs > 1 && !f_rest)))
        return fail(ANISO_B200_ERR_ARGUMENT, "an input array is NULL");
    aniso_b200_scene* s = nullptr;
    int rc = new_scene(n, sh_degree, out, &s);
    if (rc == 0 && n > 0) {
        const size_t nn = static_cast<size_t>(n);
        const size_t rest = static_cast<size_t>(coeffs - 1) * 3;
        const size_t floats = nn * (3 + 3 + rest + 1 + 3 + 4);
        float* d = nullptr;
        cudaError_t e = cudaMalloc(&d, floats * sizeof(float));
        float* dx = d;
        float* ddc = dx + nn * 3;
        float* drest = ddc + nn * 3;
        float* dop = drest + nn * rest;
        float* dsc = dop + nn;
        float* drot = dsc + nn * 3;
        struct {
            float* dst;
            const float* src;
            size_t count;
        } copies[] = {{dx, xyz, nn * 3}, {ddc, f_dc, nn * 3}, {drest, f_rest, nn * rest},
                      {dop, opacity, nn}, {dsc, log_scale, nn * 3}, {drot, rot, nn * 4}};
        for (auto& c : copies)
            if (e == cudaSuccess && c.count)
                e = cudaMemcpyAsync(c.dst, c.src, c.count * sizeof(float), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) {
            ingest_raw_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s->stream>>>(
                dx, ddc, drest, dop, dsc, drot, n, coeffs, s->planes, s->pos_op.p, s->scale.p, s->rot.p, s->sh.p);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (d) cudaFree(d);
        if (e != cudaSuccess) rc = cuda_fail(e, "scene upload");
        else rc = measure_box(s);
    }
    if (rc != 0) {
        delete s;
        if (out) *out = nullptr;
        return rc;
    }
    *out = s;
    return ANISO_B200_OK;
}

int aniso_b200_scene_load_ply(const char* path, aniso_b200_scene** out) {
    if (!path || !out) return fail(ANISO_B200_ERR_ARGUMENT, "path/out is NULL");
    const std::string name = path;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ANISO_B200_ERR_ARGUMENT, name + ": cannot open");
    int64_t n = 0;
    int degree = 0;
    long body_at = 0;
    PlyColumns col{};
    int rc = parse_ply_header(f, name, &n, &col, &degree, &body_at);
    std::vector<float> body;
    if (rc == 0) {
        body.resize(static_cast<size_t>(n) * col.stride);
        std::fseek(f, body_at, SEEK_SET);
        const size_t got = body.empty() ? 0 : std::fread(body.data(), sizeof(float), body.size(), f);
        if (got != body.size())
            rc = fail(ANISO_B200_ERR_ARGUMENT, name + ": file is shorter than the header promises (" +
                                                   std::to_string(n) + " Gaussians)");
    }
    std::fclose(f);
    if (rc != 0) return rc;
    aniso_b200_scene* s = nullptr;
    rc = new_scene(n, degree, out, &s);
    if (rc == 0 && n > 0) {
        float* d = nullptr;
        cudaError_t e = cudaMalloc(&d, body.size() * sizeof(float));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d, body.data(), body.size() * sizeof(float), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) {
            ingest_ply_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s->stream>>>(
                d, n, col, (degree + 1) * (degree + 1), s->planes, s->pos_op.p, s->scale.p, s->rot.p, s->sh.p);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (d) cudaFree(d);
        if (e != cudaSuccess) rc = cuda_fail(e, "scene upload");
        else rc = measure_box(s);
    }
    if (rc != 0) {
        delete s;
        *out = nullptr;
        return rc;
    }
    *out = s;
    return ANISO_B200_OK;
}

int aniso_b200_scene_destroy(aniso_b200_scene* scene) {
    delete scene;
    return ANISO_B200_OK;
}

int aniso_b200_render(aniso_b200_scene* s, const aniso_b200_camera* camera, const aniso_b200_options* options,
                      uint8_t* rgb_host, aniso_b200_stats* stats) {
    if (!s || !rgb_host) return fail(ANISO_B200_ERR_ARGUMENT, "scene/rgb_host is NULL");
    Plan<SceneView> P;
    AB_TRY(single_plan(s, camera, options, P));
    const size_t bytes = static_cast<size_t>(camera->width) * camera->height * 3;
    // Pinned host memory that this device can address is written by the blend itself, across the
    // bus while the frame is blended, instead of by a copy after it; other memory gets the copy.
    uint8_t* direct = mapped_host(rgb_host);
    if (!direct) {
        AB_TRY(s->image.reserve(bytes));
        P.views[0].rgb8 = s->image.p;
    } else {
        P.views[0].rgb8 = direct;
    }
    AB_TRY(s->chain.join(s->stream));  // after any frame the caller enqueued on another stream
    s->chain.extend(s->stream);
    for (int attempt = 0; attempt < 3; ++attempt) {
        const uint64_t k0 = chained_launches();
        AB_TRY(enqueue_plan(s->arena, s->slot(), P, s->stream, stats ? s->ev : nullptr, nullptr, false, false,
                            nullptr));
        s->frame_kernels = static_cast<int32_t>(chained_launches() - k0);
        if (!direct) AB_CUDA(cudaMemcpyAsync(rgb_host, s->image.p, bytes, cudaMemcpyDeviceToHost, s->stream));
        AB_TRY(read_ctrl(s->arena, s->host_ctrl, s->stream));
        int again = 0;
        AB_TRY(settle(s->arena, *s->host_ctrl, &again, false));
        if (again) continue;
        if (stats) {
            float a = 0, b = 0, c = 0;
            cudaEventElapsedTime(&a, s->ev[0], s->ev[1]);
            cudaEventElapsedTime(&b, s->ev[1], s->ev[2]);
            cudaEventElapsedTime(&c, s->ev[2], s->ev[3]);
            stats->visible = s->host_ctrl->vis_count;
            stats->tile_pairs = s->host_ctrl->pair_total;
            stats->project_ms = a;
            stats->sort_ms = b;
            stats->blend_ms = c;
        }
        return ANISO_B200_OK;
    }
    return fail(ANISO_B200_ERR_ARGUMENT, "pair capacity kept overflowing");
}

int aniso_b200_render_device(aniso_b200_scene* s, const aniso_b200_camera* camera, const aniso_b200_options* options,
                             uint8_t* rgb_device, void* stream) {
    if (!s || !rgb_device) return fail(ANISO_B200_ERR_ARGUMENT, "scene/rgb_device is NULL");
    Plan<SceneView> P;
    AB_TRY(single_plan(s, camera, options, P));
    P.views[0].rgb8 = rgb_device;
    cudaEvent_t* ev = nullptr;
    if (s->profiling) {
        while (s->prof_ev.size() < 4 * (s->prof_frames + 1)) {
            cudaEvent_t e;
            AB_CUDA(cudaEventCreate(&e));
            s->prof_ev.push_back(e);
        }
        ev = &s->prof_ev[4 * s->prof_frames++];
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    AB_TRY(s->chain.join(st));
    const uint64_t k0 = chained_launches();
    const int rc = enqueue_plan(s->arena, s->slot(), P, st, ev, nullptr, false, false, nullptr);
    s->frame_kernels = static_cast<int32_t>(chained_launches() - k0);
    s->chain.extend(st);
    return rc;
}

int aniso_b200_frame_kernels(aniso_b200_scene* s, int32_t* kernels) {
    if (!s || !kernels) return fail(ANISO_B200_ERR_ARGUMENT, "scene/kernels is NULL");
    *kernels = s->frame_kernels;
    return ANISO_B200_OK;
}

int aniso_b200_profile(aniso_b200_scene* s, int32_t enable) {
    if (!s) return fail(ANISO_B200_ERR_ARGUMENT, "scene is NULL");
    s->profiling = enable != 0;
    if (s->profiling) s->prof_frames = 0;
    return ANISO_B200_OK;
}

int aniso_b200_profile_read(aniso_b200_scene* s, double* project_ms, double* sort_ms, double* blend_ms,
                            int64_t* frames) {
    if (!s) return fail(ANISO_B200_ERR_ARGUMENT, "scene is NULL");
    double t[3] = {0, 0, 0};
    for (size_t f = 0; f < s->prof_frames; ++f) {
        const cudaEvent_t* e = &s->prof_ev[4 * f];
        AB_CUDA(cudaEventSynchronize(e[3]));
        for (int k = 0; k < 3; ++k) {
            float ms = 0;
            AB_CUDA(cudaEventElapsedTime(&ms, e[k], e[k + 1]));
            t[k] += ms;
        }
    }
    if (project_ms) *project_ms = t[0];
    if (sort_ms) *sort_ms = t[1];
    if (blend_ms) *blend_ms = t[2];
    if (frames) *frames = static_cast<int64_t>(s->prof_frames);
    return ANISO_B200_OK;
}

int aniso_b200_sync(aniso_b200_scene* s, aniso_b200_stats* stats) {
    if (!s) return fail(ANISO_B200_ERR_ARGUMENT, "scene is NULL");
    // The control-block read goes on the scene's own stream after its last frame, and waits for it.
    AB_TRY(s->chain.join(s->stream));
    s->chain.extend(s->stream);
    AB_TRY(read_ctrl(s->arena, s->host_ctrl, s->stream));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->visible = s->host_ctrl->vis_count;
        stats->tile_pairs = s->host_ctrl->pair_total;
    }
    AB_TRY(clear_sticky(s->arena, s->stream));
    int again = 0;
    AB_TRY(settle(s->arena, *s->host_ctrl, &again, true));
    if (again) return fail(ANISO_B200_ERR_ARGUMENT, "pair capacity exceeded");
    return ANISO_B200_OK;
}

int aniso_b200_debug_projection(aniso_b200_scene* s, const aniso_b200_camera* camera,
                                const aniso_b200_options* options, float* uv, float* conic_opacity, float* depth,
                                float* rgb, uint32_t* rect, uint32_t* tiles_touched) {
    if (!s) return fail(ANISO_B200_ERR_ARGUMENT, "scene is NULL");
    Plan<SceneView> P;
    AB_TRY(single_plan(s, camera, options, P));
    const size_t nn = static_cast<size_t>(std::max<int64_t>(s->n, 1));
    DevBuf<float2> duv;
    DevBuf<float4> dco;
    DevBuf<float> ddepth, drgb;
    DevBuf<uint4> drect;
    DevBuf<unsigned> dtt;
    AB_TRY(duv.reserve(nn, true));
    AB_TRY(dco.reserve(nn, true));
    AB_TRY(ddepth.reserve(nn, true));
    AB_TRY(drgb.reserve(nn * 3, true));
    AB_TRY(drect.reserve(nn, true));
    AB_TRY(dtt.reserve(nn, true));
    DebugProjection dbg;
    dbg.uv = duv.p;
    dbg.conic_opacity = dco.p;
    dbg.depth = ddepth.p;
    dbg.rgb = drgb.p;
    dbg.rect = drect.p;
    dbg.tiles_touched = dtt.p;
    Arena& A = s->arena;
    const ViewInfo* views = nullptr;
    const BatchScene<SceneView>* scenes = nullptr;
    BatchTables tables;
    Slot& slot = s->slot();
    AB_TRY(s->chain.join(s->stream));
    s->chain.extend(s->stream);
    AB_TRY(slot.fill(P, s->stream, &views, &scenes, tables));
    launch_frame_begin(A.ctrl.p, s->stream);
    launch_preprocess_any(scenes, P, views, A, &dbg, PassCounts{}, s->stream);
    AB_TRY(slot.mark(s->stream));
    AB_CUDA(cudaGetLastError());
    AB_CUDA(cudaStreamSynchronize(s->stream));
    const size_t n = static_cast<size_t>(s->n);
    if (uv) AB_CUDA(cudaMemcpy(uv, duv.p, n * sizeof(float2), cudaMemcpyDeviceToHost));
    if (conic_opacity) AB_CUDA(cudaMemcpy(conic_opacity, dco.p, n * sizeof(float4), cudaMemcpyDeviceToHost));
    if (depth) AB_CUDA(cudaMemcpy(depth, ddepth.p, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (rgb) AB_CUDA(cudaMemcpy(rgb, drgb.p, n * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    if (rect) AB_CUDA(cudaMemcpy(rect, drect.p, n * sizeof(uint4), cudaMemcpyDeviceToHost));
    if (tiles_touched) AB_CUDA(cudaMemcpy(tiles_touched, dtt.p, n * sizeof(unsigned), cudaMemcpyDeviceToHost));
    return ANISO_B200_OK;
}

int aniso_b200_debug_sorted(aniso_b200_scene* s, const aniso_b200_camera* camera, const aniso_b200_options* options,
                            uint32_t* tiles, uint32_t* values, uint64_t capacity, uint32_t* ranges, uint64_t* pairs) {
    if (!s || !pairs) return fail(ANISO_B200_ERR_ARGUMENT, "scene/pairs is NULL");
    Plan<SceneView> P;
    AB_TRY(single_plan(s, camera, options, P));
    int fin = 0;
    AB_TRY(s->chain.join(s->stream));
    s->chain.extend(s->stream);
    for (int attempt = 0; attempt < 3; ++attempt) {
        AB_TRY(enqueue_plan(s->arena, s->slot(), P, s->stream, nullptr, nullptr, true, false, &fin));
        AB_TRY(read_ctrl(s->arena, s->host_ctrl, s->stream));
        int again = 0;
        AB_TRY(settle(s->arena, *s->host_ctrl, &again, false));
        if (!again) break;
    }
    const uint64_t Pn = s->host_ctrl->pair_total;
    *pairs = Pn;
    if (Pn > capacity) return fail(ANISO_B200_ERR_ARGUMENT, "capacity too small");
    const Arena& A = s->arena;
    if (tiles && Pn) AB_CUDA(cudaMemcpy(tiles, A.pair_key[fin].p, Pn * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (values && Pn) AB_CUDA(cudaMemcpy(values, A.pair_val[fin].p, Pn * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (ranges)
        AB_CUDA(cudaMemcpy(ranges, A.ranges.p, static_cast<size_t>(P.tiles) * sizeof(uint2), cudaMemcpyDeviceToHost));
    return ANISO_B200_OK;
}

int aniso_b200_sort_projection(int64_t n, const uint32_t* tiles_touched, const uint32_t* rect, const float* depth,
                               int32_t tiles_x, int32_t tiles_y, uint32_t* tiles, uint32_t* values,
                               uint64_t capacity, uint32_t* ranges, uint64_t* pairs) {
    if (n < 0 || n >= (int64_t(1) << 31) || tiles_x <= 0 || tiles_y <= 0 || !pairs)
        return fail(ANISO_B200_ERR_ARGUMENT, "bad size or NULL pairs");
    if (n > 0 && (!tiles_touched || !rect || !depth)) return fail(ANISO_B200_ERR_ARGUMENT, "input is NULL");
    uint64_t Pn = 0;
    bool short_depth = true;  // every listed depth in [0.125, 8192): offset keys, three 9-bit passes
    for (int64_t i = 0; i < n; ++i) {
        Pn += tiles_touched[i];
        if (tiles_touched[i] && !(depth[i] >= 0.125f && depth[i] < 8192.0f)) short_depth = false;
    }
    *pairs = Pn;
    if (Pn > capacity) return fail(ANISO_B200_ERR_ARGUMENT, "capacity too small");
    if (Pn > kMaxPairs) return fail(ANISO_B200_ERR_ARGUMENT, "more than 2^30 pairs");
    AB_TRY(device_present());
    Arena A;
    AB_TRY(A.init(std::max<int64_t>(n, 1), static_cast<unsigned>(std::max<uint64_t>(Pn, 1))));
    const size_t nn = static_cast<size_t>(std::max<int64_t>(n, 1));
    DevBuf<unsigned> dtt, dtab;
    DevBuf<uint4> drect;
    DevBuf<float> ddepth;
    AB_TRY(dtt.reserve(nn));
    AB_TRY(drect.reserve(nn));
    AB_TRY(ddepth.reserve(nn));
    AB_TRY(dtab.reserve(3));
    const unsigned tab[3] = {0u, 0u, static_cast<unsigned>(tiles_x)};  // one view: entry base, tile base, tiles_x
    AB_CUDA(cudaMemcpy(dtab.p, tab, sizeof tab, cudaMemcpyHostToDevice));
    const size_t un = static_cast<size_t>(n);
    if (n > 0) {
        AB_CUDA(cudaMemcpy(dtt.p, tiles_touched, un * sizeof(unsigned), cudaMemcpyHostToDevice));
        AB_CUDA(cudaMemcpy(drect.p, rect, un * sizeof(uint4), cudaMemcpyHostToDevice));
        AB_CUDA(cudaMemcpy(ddepth.p, depth, un * sizeof(float), cudaMemcpyHostToDevice));
    }
    cudaStream_t st = nullptr;
    const BatchTables tables{dtab.p, dtab.p + 1, dtab.p + 2, 1u};
    const unsigned T = static_cast<unsigned>(tiles_x) * static_cast<unsigned>(tiles_y);
    AB_TRY(A.reserve_ranges(T));
    launch_frame_begin(A.ctrl.p, nullptr, 0u, A.ranges.p, T, st);
    launch_projection_keys(n, dtt.p, ddepth.p, drect.p, A.depth_key.p, A.rect16.p, st,
                           short_depth ? kDepthKeyBase : 0u);
    int fin = 0;
    AB_TRY(enqueue_sort(A, static_cast<unsigned>(n), T, tables, false, kRadixBits, false, short_depth, st, &fin));
    AB_CUDA(cudaGetLastError());
    AB_CUDA(cudaStreamSynchronize(st));
    Ctrl h;
    AB_CUDA(cudaMemcpy(&h, A.ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    if (h.pair_total != Pn) return fail(ANISO_B200_ERR_CUDA, "device pair count disagrees with the host");
    if (tiles && Pn) AB_CUDA(cudaMemcpy(tiles, A.pair_key[fin].p, Pn * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (values && Pn) AB_CUDA(cudaMemcpy(values, A.pair_val[fin].p, Pn * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (ranges) AB_CUDA(cudaMemcpy(ranges, A.ranges.p, static_cast<size_t>(T) * sizeof(uint2), cudaMemcpyDeviceToHost));
    return ANISO_B200_OK;
}

}  // extern "C"

// ---- batches -------------------------------------------------------------------------------

struct aniso_b200_batch {
    std::vector<aniso_b200_scene*> scenes;
    std::vector<int32_t> view_scene;
    PlanShape shape;
    bool use_graph = false;
    Arena arena;
    Slot slots[kSlots];
    int next_slot = 0;
    Slot graph_slot;
    Plan<SceneView> graph_plan;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t capture_stream = nullptr;
    Ctrl* host_ctrl = nullptr;
    StreamChain chain;  // the streams the batch's frames went to
    ~aniso_b200_batch() {
        chain.wait_host();
        if (capture_stream) cudaStreamSynchronize(capture_stream);
        if (graph) cudaGraphExecDestroy(graph);
        if (capture_stream) cudaStreamDestroy(capture_stream);
        if (host_ctrl) cudaFreeHost(host_ctrl);
    }
};

extern "C" {

int aniso_b200_batch_create(aniso_b200_scene* const* scenes, int32_t n_scenes, const int32_t* view_scene,
                            int32_t n_views, const aniso_b200_batch_options* options, aniso_b200_batch** out) {
    if (!out || !scenes || !view_scene || n_scenes <= 0 || n_views <= 0)
        return fail(ANISO_B200_ERR_ARGUMENT, "a batch needs scenes, views and out");
    for (int s = 0; s < n_scenes; ++s)
        if (!scenes[s]) return fail(ANISO_B200_ERR_ARGUMENT, "a scene is NULL");
    PlanShape shape;
    AB_TRY(check_options(options, shape));
    aniso_b200_batch* b = new (std::nothrow) aniso_b200_batch();
    if (!b) return fail(ANISO_B200_ERR_OUT_OF_MEMORY, "host allocation failed");
    b->scenes.assign(scenes, scenes + n_scenes);
    b->view_scene.assign(view_scene, view_scene + n_views);
    b->shape = shape;
    b->use_graph = options && options->use_graph;
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&b->host_ctrl), sizeof(Ctrl));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "batch create");
    }
    std::memset(b->host_ctrl, 0, sizeof(Ctrl));
    *out = b;
    return ANISO_B200_OK;
}

int aniso_b200_batch_destroy(aniso_b200_batch* batch) {
    delete batch;
    return ANISO_B200_OK;
}

int aniso_b200_batch_render(aniso_b200_batch* b, const aniso_b200_camera* cameras, uint8_t* const* rgb_device,
                            void* stream) {
    if (!b || !cameras || !rgb_device) return fail(ANISO_B200_ERR_ARGUMENT, "batch/cameras/rgb_device is NULL");
    std::vector<SceneView> srcs;
    std::vector<int> degs;
    for (auto* s : b->scenes) {
        srcs.push_back(s->view());
        degs.push_back(s->degree);
    }
    Plan<SceneView> P;
    AB_TRY(P.build(srcs, degs, b->view_scene.data(), static_cast<int>(b->view_scene.size()), cameras, b->shape));
    std::vector<const PositionBox*> boxes;
    for (auto* s : b->scenes) boxes.push_back(&s->box);
    P.bound_depth(boxes);
    for (size_t k = 0; k < P.views.size(); ++k) {
        if (!rgb_device[k]) return fail(ANISO_B200_ERR_ARGUMENT, "an output buffer is NULL");
        P.views[k].rgb8 = rgb_device[k];
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (b->arena.n < static_cast<int64_t>(P.entries)) {
        b->chain.wait_host();  // the buffers are about to move: the batch's frames must be done
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);  // record again
            b->graph = nullptr;
        }
    }
    AB_TRY(b->arena.ensure(static_cast<int64_t>(std::max<uint64_t>(P.entries, 1))));
    AB_TRY(b->chain.join(st));
    b->chain.extend(st);
    if (!b->use_graph)
        return enqueue_plan(b->arena, b->slots[b->next_slot++ % kSlots], P, st, nullptr, nullptr, false, false,
                            nullptr);
    if (b->graph && !P.same_geometry(b->graph_plan)) {
        b->chain.wait_host();
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (!b->graph) {
        // Record the sequence on a private stream. The recorded upload reads the graph slot's
        // pinned blob at every replay, and each replay refreshes that blob first.
        // Every allocation the sequence needs happens first: none may happen while capturing.
        AB_TRY(b->graph_slot.stage(P));
        AB_TRY(b->arena.reserve_ranges(static_cast<size_t>(P.tiles)));
        cudaGraph_t g = nullptr;
        AB_CUDA(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_plan(b->arena, b->graph_slot, P, b->capture_stream, nullptr, nullptr, false, false,
                                    nullptr, false);
        const cudaError_t ce = cudaStreamEndCapture(b->capture_stream, &g);
        if (rc != 0) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
        b->graph_plan = P;
    } else {
        AB_TRY(b->graph_slot.stage(P));  // waits for the previous replay to have read it
    }
    AB_CUDA(cudaGraphLaunch(b->graph, st));
    return b->graph_slot.mark(st);
}

int aniso_b200_batch_sync(aniso_b200_batch* b, aniso_b200_stats* stats) {
    if (!b) return fail(ANISO_B200_ERR_ARGUMENT, "batch is NULL");
    AB_TRY(b->chain.join(b->capture_stream));  // the control-block read follows the batch's last frame
    b->chain.extend(b->capture_stream);
    AB_TRY(read_ctrl(b->arena, b->host_ctrl, b->capture_stream));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->visible = b->host_ctrl->vis_count;
        stats->tile_pairs = b->host_ctrl->pair_total;
    }
    AB_TRY(clear_sticky(b->arena, b->capture_stream));
    int again = 0;
    AB_TRY(settle(b->arena, *b->host_ctrl, &again, true));
    if (again) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);  // buffers moved: record again
            b->graph = nullptr;
        }
        return fail(ANISO_B200_ERR_ARGUMENT, "pair capacity exceeded");
    }
    return ANISO_B200_OK;
}

}  // extern "C"

// ---- the differentiable path ---------------------------------------------------------------

struct aniso_b200_trainer {
    Arena arena;
    Slot slots[kSlots];
    int next_slot = 0;
    Ctrl* host_ctrl = nullptr;  // pinned
    std::vector<DevBuf<float>> t_final;
    std::vector<DevBuf<unsigned>> n_contrib;
    DevBuf<float> grad_pair;
    DevBuf<unsigned> vis_list;    // one view's visible Gaussians (the backward's work list)
    DevBuf<unsigned> vis_counts;  // their count, one word per view
    // The state of the last forward, for its backward.
    bool has_forward = false;
    Plan<RawParams> plan;
    int fin = 0;
    StreamChain chain;  // the streams the trainer's forwards and backwards went to
    // CUDA graphs of a batch (batch options with use_graph): the forward's and the backward's
    // launch sequences, each recorded once per launch geometry and replayed after restaging its
    // slot's tables (cameras, parameter, image and gradient pointers all travel in the tables).
    cudaStream_t capture_stream = nullptr;
    Slot graph_slot_f, graph_slot_b;
    cudaGraphExec_t fwd_graph = nullptr, bwd_graph = nullptr;
    Plan<RawParams> fwd_plan, bwd_plan;
    uint64_t fwd_gen = 0, bwd_gen = 0;     // the work buffers' generation each was recorded against
    int fwd_fin = 0;                       // the pair buffer the recorded forward leaves sorted
    int bwd_fin = -1;                      // the pair buffer the recorded backward reads
    std::vector<int> bwd_fresh;            // per view: the fresh flag the backward was recorded with
    const void* bwd_buffers[3] = {nullptr, nullptr, nullptr};
    Slot& slot() { return slots[next_slot++ % kSlots]; }
    void drop_graphs() {
        if (fwd_graph) cudaGraphExecDestroy(fwd_graph);
        if (bwd_graph) cudaGraphExecDestroy(bwd_graph);
        fwd_graph = bwd_graph = nullptr;
    }
    ~aniso_b200_trainer() {
        chain.wait_host();
        drop_graphs();
        if (capture_stream) cudaStreamDestroy(capture_stream);
        if (host_ctrl) cudaFreeHost(host_ctrl);
    }
};

namespace {

int raw_of(const aniso_b200_raw_params& P, RawParams& raw) {
    if (P.n < 0 || P.n >= (int64_t(1) << 31)) return fail(ANISO_B200_ERR_ARGUMENT, "n must be in [0, 2^31)");
    if (P.sh_degree != 1 && P.sh_degree != 3)
        return fail(ANISO_B200_ERR_ARGUMENT, "stored SH degree must be 1 or 3 (whole 16-byte words per Gaussian)");
    if (P.n > 0 && (!P.means || !P.log_scales || !P.quats || !P.opacity_logits || !P.sh))
        return fail(ANISO_B200_ERR_ARGUMENT, "a parameter pointer is NULL");
    if ((reinterpret_cast<uintptr_t>(P.quats) | reinterpret_cast<uintptr_t>(P.sh)) & 15)
        return fail(ANISO_B200_ERR_ARGUMENT, "quats and sh must be 16-byte aligned");
    raw.means = P.means;
    raw.log_scales = P.log_scales;
    raw.quats = reinterpret_cast<const float4*>(P.quats);
    raw.logits = P.opacity_logits;
    raw.sh = reinterpret_cast<const float4*>(P.sh);
    raw.n = P.n;
    raw.sh_planes = (P.sh_degree + 1) * (P.sh_degree + 1) * 3 / 4;
    return 0;
}

// Records `enqueue` on the trainer's private stream as a CUDA graph and instantiates it in *exec.
template <typename F>
int record_graph(aniso_b200_trainer* t, cudaGraphExec_t* exec, F&& enqueue) {
    if (!t->capture_stream) AB_CUDA(cudaStreamCreateWithFlags(&t->capture_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    AB_CUDA(cudaStreamBeginCapture(t->capture_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue(t->capture_stream);
    const cudaError_t ce = cudaStreamEndCapture(t->capture_stream, &g);
    if (rc != 0) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        *exec = nullptr;
        return cuda_fail(ie, "cudaGraphInstantiate");
    }
    return 0;
}

// The forward of a batch from its recorded graph: recorded (after every allocation it needs) when
// the launch geometry or the work buffers changed, else replayed after restaging the graph's slot.
int train_forward_graph(aniso_b200_trainer* t, const Plan<RawParams>& P, cudaStream_t st, int* fin) {
    Arena& A = t->arena;
    AB_TRY(A.reserve_ranges(static_cast<size_t>(P.tiles)));
    AB_TRY(t->graph_slot_f.stage(P));
    if (!t->fwd_graph || t->fwd_gen != A.gen || !P.same_geometry(t->fwd_plan)) {
        if (t->fwd_graph) {
            t->chain.wait_host();  // no replay of the old graph may still be in flight
            cudaGraphExecDestroy(t->fwd_graph);
            t->fwd_graph = nullptr;
        }
        int rec_fin = 0;
        AB_TRY(record_graph(t, &t->fwd_graph, [&](cudaStream_t cs) {
            return enqueue_plan(A, t->graph_slot_f, P, cs, nullptr, nullptr, false, true, &rec_fin, false);
        }));
        t->fwd_plan = P;
        t->fwd_gen = A.gen;
        t->fwd_fin = rec_fin;
    }
    *fin = t->fwd_fin;
    AB_CUDA(cudaGraphLaunch(t->fwd_graph, st));
    return t->graph_slot_f.mark(st);
}

int train_forward(aniso_b200_trainer* t, const aniso_b200_raw_params* params, int32_t n_scenes,
                  const int32_t* view_scene, const aniso_b200_camera* cameras, int32_t n_views, const PlanShape& shape,
                  float* const* images, cudaStream_t st) {
    if (!t || !params || !images) return fail(ANISO_B200_ERR_ARGUMENT, "trainer/params/images is NULL");
    t->has_forward = false;
    std::vector<RawParams> srcs(n_scenes);
    std::vector<int> degs(n_scenes);
    for (int s = 0; s < n_scenes; ++s) {
        AB_TRY(raw_of(params[s], srcs[s]));
        degs[s] = params[s].sh_degree;
    }
    Plan<RawParams>& P = t->plan;
    AB_TRY(P.build(srcs, degs, view_scene, n_views, cameras, shape));
    if (t->t_final.size() < static_cast<size_t>(n_views)) {
        t->t_final.resize(n_views);
        t->n_contrib.resize(n_views);
    }
    for (int k = 0; k < n_views; ++k) {
        if (!images[k]) return fail(ANISO_B200_ERR_ARGUMENT, "an image buffer is NULL");
        const size_t px = static_cast<size_t>(P.views[k].cam.width) * P.views[k].cam.height;
        AB_TRY(t->t_final[k].reserve(px));
        AB_TRY(t->n_contrib[k].reserve(px));
        P.views[k].rgbf = images[k];
        P.views[k].t_final = t->t_final[k].p;
        P.views[k].n_contrib = t->n_contrib[k].p;
    }
    Arena& A = t->arena;
    AB_TRY(A.ensure(static_cast<int64_t>(std::max<uint64_t>(P.entries, 1))));
    AB_TRY(t->chain.join(st));  // after the trainer's last backward, wherever it went
    t->chain.extend(st);
    for (int attempt = 0; attempt < 3; ++attempt) {
        int fin = 0;
        if (shape.use_graph) {
            AB_TRY(train_forward_graph(t, P, st, &fin));
        } else {
            AB_TRY(enqueue_plan(A, t->slot(), P, st, nullptr, nullptr, false, true, &fin));
        }
        AB_TRY(read_ctrl(A, t->host_ctrl, st));
        int again = 0;
        AB_TRY(settle(A, *t->host_ctrl, &again, false));
        if (again) continue;
        t->fin = fin;
        t->has_forward = true;
        return ANISO_B200_OK;
    }
    return fail(ANISO_B200_ERR_ARGUMENT, "pair capacity kept overflowing");
}

int train_backward(aniso_b200_trainer* t, const float* const* grad_images, const aniso_b200_raw_grads* grads,
                   cudaStream_t st) {
    if (!t || !grad_images || !grads) return fail(ANISO_B200_ERR_ARGUMENT, "trainer/grad_images/grads is NULL");
    if (!t->has_forward) return fail(ANISO_B200_ERR_ARGUMENT, "no forward to differentiate");
    Plan<RawParams>& P = t->plan;
    for (size_t k = 0; k < P.views.size(); ++k) {
        if (!grad_images[k]) return fail(ANISO_B200_ERR_ARGUMENT, "a gradient image is NULL");
        P.views[k].grad_img = grad_images[k];
    }
    for (size_t s = 0; s < P.scenes.size(); ++s)
        if (P.scenes[s].src.n > 0 && (!grads[s].means || !grads[s].log_scales || !grads[s].quats ||
                                      !grads[s].opacity_logits || !grads[s].sh))
            return fail(ANISO_B200_ERR_ARGUMENT, "a gradient pointer is NULL");
    for (size_t s = 0; s < P.scenes.size(); ++s) {
        if (grads[s].grad2d && !grads[s].visible)
            return fail(ANISO_B200_ERR_ARGUMENT, "grad2d needs its visible counts");
        if ((reinterpret_cast<uintptr_t>(grads[s].quats) | reinterpret_cast<uintptr_t>(grads[s].sh)) & 15)
            return fail(ANISO_B200_ERR_ARGUMENT, "the quats and sh gradients must be 16-byte aligned");
    }
    Arena& A = t->arena;
    const Ctrl& h = *t->host_ctrl;
    const bool graph = P.shape.use_graph;
    // The pairs' gradient slots; sized for the pair capacity when a recorded graph replays (the
    // graph fixes the buffer, whatever the frame's own pair count).
    AB_TRY(t->grad_pair.reserve(std::max<uint64_t>(graph ? A.pair_cap : h.pair_total, 1) * 9));
    int64_t max_n = 1;
    for (const auto& sc : P.scenes) max_n = std::max<int64_t>(max_n, sc.src.n);
    AB_TRY(t->vis_list.reserve(static_cast<size_t>(max_n)));
    AB_TRY(t->vis_counts.reserve(P.views.size()));
    // The scenes' gradient buffers travel in the frame's tables; the scene's first view of a fresh
    // gradient stores without reading the zeros (a separate kernel instantiation).
    P.grads.assign(P.scenes.size(), RawGrads{});
    for (size_t s = 0; s < P.scenes.size(); ++s) {
        const aniso_b200_raw_grads& g = grads[s];
        P.grads[s] = RawGrads{g.means, g.log_scales, g.quats, g.opacity_logits, g.sh, g.grad2d,
                              g.grad2d ? g.visible : nullptr, g.fresh != 0 ? 1u : 0u, 0u};
    }
    std::vector<int> fresh(P.views.size());
    for (size_t k = 0; k < P.views.size(); ++k) {
        const unsigned s = P.views[k].scene;
        fresh[k] = grads[s].fresh != 0 && k == P.scenes[s].view_begin;
    }
    const auto enqueue = [&](Slot& slot, cudaStream_t cs) -> int {
        const ViewInfo* views = nullptr;
        const BatchScene<RawParams>* scenes = nullptr;
        BackwardIn in;
        AB_TRY(slot.fill(P, cs, &views, &scenes, in.tables));
        in.ranges = A.ranges.p;
        in.vals = A.pair_val[t->fin].p;
        in.rec = A.rec.p;
        in.ctrl = A.ctrl.p;
        in.views = views;
        in.rank = A.rank.p;
        in.offs = A.offs.p;
        in.rect_sorted = A.rect_sorted.p;
        AB_CUDA(cudaMemsetAsync(t->vis_counts.p, 0, P.views.size() * sizeof(unsigned), cs));
        launch_blend_backward(in, static_cast<unsigned>(P.tiles), P.shape.tile_w, P.shape.tile_h, t->grad_pair.p, cs);
        for (size_t k = 0; k < P.views.size(); ++k) {
            const unsigned s = P.views[k].scene;
            const GaussBackwardArgs ga{scenes, s, views, static_cast<unsigned>(k), slot.grads_dev(P),
                                       P.scenes[s].src.n, P.views[k].entry_base, P.views[k].cam.shDegree,
                                       fresh[k] != 0};
            launch_gauss_backward(ga, A.ctrl.p, A.depth_key.p, A.rank.p, A.offs.p, A.rect_sorted.p, t->grad_pair.p,
                                  t->vis_list.p, t->vis_counts.p + k, cs);
        }
        AB_CUDA(cudaGetLastError());
        return 0;
    };
    AB_TRY(t->chain.join(st));
    t->chain.extend(st);
    if (!graph) {
        Slot& slot = t->slot();
        AB_TRY(enqueue(slot, st));
        return slot.mark(st);
    }
    AB_TRY(t->graph_slot_b.stage(P));
    const void* bufs[3] = {t->grad_pair.p, t->vis_list.p, t->vis_counts.p};
    const bool valid = t->bwd_graph && t->bwd_gen == A.gen && P.same_geometry(t->bwd_plan) && t->bwd_fresh == fresh &&
                       std::equal(bufs, bufs + 3, t->bwd_buffers) && t->bwd_fin == t->fin;
    if (!valid) {
        if (t->bwd_graph) {
            t->chain.wait_host();  // no replay of the old graph may still be in flight
            cudaGraphExecDestroy(t->bwd_graph);
            t->bwd_graph = nullptr;
        }
        AB_TRY(record_graph(t, &t->bwd_graph, [&](cudaStream_t cs) { return enqueue(t->graph_slot_b, cs); }));
        t->bwd_plan = P;
        t->bwd_gen = A.gen;
        t->bwd_fresh = fresh;
        t->bwd_fin = t->fin;
        std::copy(bufs, bufs + 3, t->bwd_buffers);
    }
    AB_CUDA(cudaGraphLaunch(t->bwd_graph, st));
    return t->graph_slot_b.mark(st);
}

}  // namespace

extern "C" {

int aniso_b200_trainer_create(aniso_b200_trainer** out) {
    if (!out) return fail(ANISO_B200_ERR_ARGUMENT, "out is NULL");
    AB_TRY(device_present());
    aniso_b200_trainer* t = new (std::nothrow) aniso_b200_trainer();
    if (!t) return fail(ANISO_B200_ERR_OUT_OF_MEMORY, "host allocation failed");
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&t->host_ctrl), sizeof(Ctrl));
    if (e != cudaSuccess) {
        delete t;
        return cuda_fail(e, "cudaMallocHost");
    }
    std::memset(t->host_ctrl, 0, sizeof(Ctrl));
    *out = t;
    return ANISO_B200_OK;
}

int aniso_b200_trainer_destroy(aniso_b200_trainer* t) {
    delete t;
    return ANISO_B200_OK;
}

int aniso_b200_train_forward(aniso_b200_trainer* t, const aniso_b200_raw_params* params, const aniso_b200_camera* camera,
                             const aniso_b200_options* options, float* image_device, void* stream) {
    if (!image_device) return fail(ANISO_B200_ERR_ARGUMENT, "image is NULL");
    if (options && options->sh_degree < 0) return fail(ANISO_B200_ERR_ARGUMENT, "sh_degree must be >= 0");
    const int32_t vs = 0;
    float* images[1] = {image_device};
    return train_forward(t, params, 1, &vs, camera, 1, scene_shape(options), images, static_cast<cudaStream_t>(stream));
}

int aniso_b200_train_backward(aniso_b200_trainer* t, const float* grad_image_device, const aniso_b200_raw_grads* grads,
                              void* stream) {
    if (!grad_image_device) return fail(ANISO_B200_ERR_ARGUMENT, "grad_image is NULL");
    const float* g[1] = {grad_image_device};
    return train_backward(t, g, grads, static_cast<cudaStream_t>(stream));
}

int aniso_b200_train_batch_forward(aniso_b200_trainer* t, const aniso_b200_raw_params* params, int32_t n_scenes,
                                   const int32_t* view_scene, const aniso_b200_camera* cameras, int32_t n_views,
                                   const aniso_b200_batch_options* options, float* const* images_device,
                                   void* stream) {
    PlanShape shape;
    AB_TRY(check_options(options, shape));
    if (n_scenes <= 0) return fail(ANISO_B200_ERR_ARGUMENT, "n_scenes must be > 0");
    return train_forward(t, params, n_scenes, view_scene, cameras, n_views, shape, images_device,
                         static_cast<cudaStream_t>(stream));
}

int aniso_b200_train_batch_backward(aniso_b200_trainer* t, const float* const* grad_images_device,
                                    const aniso_b200_raw_grads* grads, void* stream) {
    return train_backward(t, grad_images_device, grads, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
