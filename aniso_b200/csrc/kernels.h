// Host-side launchers of the rasterizer kernels (internal to the library).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace ab2 {

// Optional per-Gaussian outputs in the reference kernel's own layout (gpu_render.cu:86-88), for
// the parity tests: uv float2, conicOpacity float4, depth float, rgb float3, rect uint4,
// tilesTouched uint32 (0 for culled Gaussians).
struct DebugProjection {
    float2* uv = nullptr;
    float4* conic_opacity = nullptr;
    float* depth = nullptr;
    float* rgb = nullptr;
    uint4* rect = nullptr;
    unsigned* tiles_touched = nullptr;
};

// Clears the frame's control block (counts and flags; the flags are folded into the sticky ones),
// `zero_words` words at `zero` (the first LSD pass's digit counts, which the preprocess adds to)
// and the first `tiles` tile ranges (to [0, 0), which a tile without pairs keeps).
void launch_frame_begin(Ctrl* ctrl, cudaStream_t stream);
// Copies `words` 32-bit words from `src_mapped` (the device's address of page-locked host memory)
// to `dst` in device memory.
void launch_upload(const unsigned* src_mapped, unsigned* dst, unsigned words, cudaStream_t stream);
// Writes the control block to `host_mapped` (the device's address of page-locked host memory) and
// clears the block's flags.
void launch_publish_ctrl(Ctrl* ctrl, Ctrl* host_mapped, cudaStream_t stream);
void launch_frame_begin(Ctrl* ctrl, unsigned* zero, unsigned zero_words, uint2* ranges, unsigned tiles,
                        cudaStream_t stream);
// launch_upload and then launch_frame_begin, as one kernel.
void launch_frame_start(const unsigned* src_mapped, unsigned* dst, unsigned words, Ctrl* ctrl, unsigned* zero,
                        unsigned zero_words, uint2* ranges, unsigned tiles, cudaStream_t stream);

// Projection of every (view, Gaussian) entry of a batch; `blocks` = sum over scenes of
// ceil(n / preprocess_gaussians_per_block()) (scene s starts at block scenes[s].block_base). counts.counts set: each visible
// entry's depth key is also added to the digit counts of the first depth pass, whose items are the
// `entries` depth keys in entry order.
unsigned preprocess_gaussians_per_block();
void launch_preprocess(const BatchScene<SceneView>* scenes, unsigned n_scenes, unsigned blocks, const ViewInfo* views,
                       int sh_degree, int tile_w, int tile_h, SplatRecord* rec, unsigned long long* rect16,
                       unsigned* depth_key, const DebugProjection* dbg, const PassCounts& counts, unsigned entries,
                       cudaStream_t stream);
// The same projection of the optimizer's raw tensors (activated in the kernel).
void launch_preprocess_raw(const BatchScene<RawParams>* scenes, unsigned n_scenes, unsigned blocks,
                           const ViewInfo* views, int sh_degree, int tile_w, int tile_h, SplatRecord* rec,
                           unsigned long long* rect16, unsigned* depth_key, const PassCounts& counts,
                           unsigned entries, cudaStream_t stream);

// Where a sort pass finds its item count: a host value, the visible count the first depth pass
// publishes, or the frame's pair total.
enum class SortCount : int { kFixed = 0, kVisible = 1, kPairs = 2 };

// One stable LSD radix pass over (key, value) u32 pairs, a `bits`-bit digit (8 or 9) at `shift`
// (three launches: upsweep, per-digit span scan, downsweep). masked: the input is the N depth keys in entry order,
// culled ones dropped, the entry index as value (the first depth pass; it publishes the visible
// count); keys_out may be NULL on the last pass. Grids are sized for `capacity` (`fixed` for
// kFixed) items. scratch holds sort_scratch_words() words.
size_t sort_scratch_words();
bool radix_bits_supported(int bits);
void launch_radix_pass(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                       bool masked, SortCount src, unsigned fixed, unsigned capacity, int shift, int bits,
                       unsigned* scratch, Ctrl* ctrl, cudaStream_t stream);
// The same pass in two parts, for passes whose digit counts the key producer accumulates
// (PassCounts, common.cuh): launch_radix_count is the upsweep alone (writes every (digit, span)
// cell of `counts`); launch_radix_scatter the span scan and the downsweep over counts that are
// complete. The span scan also clears `zero_words` words at `zero` (a later pass's counts, which
// a producer accumulates). One count matrix is sort_count_words() words; the pass's span count is
// sort_spans(capacity or fixed).
size_t sort_count_words();
unsigned sort_spans(uint64_t max_items);
void launch_radix_count(const unsigned* keys_in, bool masked, SortCount src, unsigned fixed, unsigned capacity,
                        int shift, int bits, unsigned* counts, Ctrl* ctrl, cudaStream_t stream);
void launch_radix_scatter(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                          bool masked, SortCount src, unsigned fixed, unsigned capacity, int shift, int bits,
                          unsigned* counts, unsigned* totals, unsigned* zero, unsigned zero_words, Ctrl* ctrl,
                          cudaStream_t stream);

// Expands the depth-sorted visible list into (tile, entry) pairs in depth order; sets kFlagOverflow
// (and writes no pairs) if they exceed capacity. Three kernels: per-span pair counts, pair offsets,
// and an expansion with a fixed number of pairs per CTA, which with first.counts set also adds the
// pairs' tile keys to the first tile pass's digit counts (cleared beforehand).
struct DupBuffers {
    unsigned* offs;                   // [N] exclusive pair offset of each depth-sorted entry
    unsigned* rank;                   // [N] depth-sorted position of each visible entry (or NULL)
    unsigned long long* rect_sorted;  // [N] its tile rectangle, in sorted order
    unsigned* chunk_start;            // [capacity / expand_chunk_pairs() + 2] first entry per chunk
    unsigned long long* span_sum;     // [sort_span_sums()] pairs per span
};
size_t sort_span_sums();
unsigned expand_chunk_pairs();
// bin_counts (with bin_tiles = the frame's global tiles): the expansion also writes each block's
// per-tile pair counts there, for the one-pass tile binning (launch_tile_bins).
void launch_duplicate(const unsigned* sorted_idx, const unsigned long long* rect16, Ctrl* ctrl, unsigned capacity,
                      unsigned max_visible, const BatchTables& tables, const DupBuffers& buf, unsigned* pair_key,
                      unsigned* pair_val, cudaStream_t stream, const PassCounts& first = PassCounts{},
                      unsigned* bin_counts = nullptr, unsigned bin_tiles = 0);

// The tile order in one stable counting pass over the tile id, for frames of at most
// bin_max_tiles() global tiles and at most bin_max_pairs() pair capacity: keys_in / vals_in are
// the expansion's depth-ordered pairs, counts its (block, tile) matrix (bin_count_words words;
// made into offsets in place); writes the tile-ordered pairs, the tiles' starts (tile_start, one
// word per tile) and every tile's range. Two kernels; same outputs as the LSD tile passes and
// launch_ranges.
unsigned bin_max_tiles();
unsigned bin_max_pairs();
size_t bin_count_words(unsigned capacity, unsigned tiles);
void launch_tile_bins(const unsigned* keys_in, const unsigned* vals_in, unsigned* keys_out, unsigned* vals_out,
                      unsigned* counts, unsigned tiles, unsigned* tile_start, uint2* ranges, Ctrl* ctrl,
                      unsigned capacity, cudaStream_t stream);

// ranges[tile] = [start, end) over the sorted tile keys (gpu_render.cu:164-177); ranges must be
// zeroed before.
void launch_ranges(const unsigned* sorted_keys, const Ctrl* ctrl, unsigned capacity, uint2* ranges,
                   cudaStream_t stream);

// Depth keys and rectangles of a projection computed elsewhere (tiles_touched, rect, depth in the
// reference kernel's layout); a visible entry's key is its depth's bits less key_base (the
// preprocess kernel's keys with kDepthKeyBase, the raw bits with 0).
void launch_projection_keys(int64_t n, const unsigned* tiles_touched, const float* depth, const uint4* rect,
                            unsigned* depth_key, unsigned long long* rect16, cudaStream_t stream,
                            unsigned key_base = 0);

// ---- the persistent sort: steps 2-4 of a frame (depth passes, pair scan and expansion, tile
// passes, tile ranges) as ONE cooperative launch of one 1024-thread CTA per SM, its phases
// separated by grid barriers whose waits are bounded (sort_persistent.cu). Same outputs as the
// multi-kernel sequence above, bit for bit.
struct SortFrameArgs {
    const unsigned* depth_key;            // [entries] depth bits, kCulledKey when culled
    const unsigned long long* rect16;     // [entries] tile rectangles of visible entries
    unsigned* vis_key[2];                 // [entries] ping-pong depth passes
    unsigned* vis_idx[2];
    unsigned* pair_key[2];                // [pair_cap] ping-pong tile passes
    unsigned* pair_val[2];
    unsigned* offs;                       // [entries] pair offset of each depth-sorted entry
    unsigned* rank;                       // [entries] depth-sorted position of each entry, or NULL
    unsigned long long* rect_sorted;      // [entries]
    unsigned* chunk_first;                // [ctas + 1] entry holding each expansion chunk's first pair
    unsigned long long* span_sum;         // [ctas] pairs of each CTA's share of the sorted entries
    unsigned* counts[2];                  // two count matrices of ctas x 512 words (CTA-major)
    uint2* ranges;                        // [tiles], cleared beforehand
    Ctrl* ctrl;
    BatchTables tables;
    unsigned entries;
    unsigned pair_cap;
    int tile_passes;
    int tile_bits[4];
    int first_counted;                    // counts[0] holds depth pass 0's digit counts already
};
// CTAs of the persistent sort on the current device (one per SM) when ANISO_B200_SORT=persistent
// is set in the environment, else 0 (the multi-kernel sequence runs: measured faster, 0.125 against
// 0.169 ms per 740k frame); also 0 where it cannot run (no cooperative launch, or not one CTA per
// SM resident).
unsigned persistent_sort_ctas();
size_t persistent_sort_count_words(unsigned ctas);  // words of one count matrix
cudaError_t launch_sort_frame(const SortFrameArgs& args, unsigned ctas, cudaStream_t stream);

// Blends every tile of a batch (blockIdx = global tile); outputs go to each view's ViewInfo.
// train: also the float colour, final transmittance and last contributor per pixel.
bool blend_shape_supported(int tile_w, int tile_h);
void launch_blend(unsigned tiles, const uint2* ranges, const unsigned* sorted_vals, const SplatRecord* rec,
                  const Ctrl* ctrl, const ViewInfo* views, const BatchTables& tables, int tile_w, int tile_h,
                  int batch, bool train, cudaStream_t stream);

// ---- the adjoint ----------------------------------------------------------------------------
struct BackwardIn {
    const uint2* ranges;
    const unsigned* vals;                // sorted pair values (entries)
    const SplatRecord* rec;
    const Ctrl* ctrl;
    const ViewInfo* views;               // t_final, n_contrib, grad_img per view
    BatchTables tables;
    const unsigned* rank;                // depth-sorted position of each visible entry
    const unsigned* offs;                // pair offset of each depth-sorted entry
    const unsigned long long* rect_sorted;
};
// Gradients of the raw parameters of one scene (device, the layout of RawParams). Added to.
struct RawGrads {
    float* means;
    float* log_scales;
    float* quats;
    float* logits;
    float* sh;
    float* grad2d;   // optional (NULL): per Gaussian, |dL/d(screen position)| in NDC units, added over views
    float* visible;  // with grad2d: per Gaussian, the number of views it was visible in, added
    unsigned fresh;  // 1: the buffers hold zeros (the scene's first view of a fresh gradient): store, do not read
    unsigned pad;
};
// grad_pair: 9 floats per pair, at the pair's depth-ordered slot.
void launch_blend_backward(const BackwardIn& in, unsigned tiles, int tile_w, int tile_h, float* grad_pair,
                           cudaStream_t stream);
// One view of one scene, everything the kernel reads about them in the frame's device tables: the
// scene's raw tensors (scenes[scene].src), the view's camera and entry base (views[view]), the
// scene's gradient buffers (grads[scene]). n, entry_base and sh_degree (the view's rendered degree)
// size and choose the launch; fresh: the scene's first view of a fresh gradient (store, do not read).
struct GaussBackwardArgs {
    const BatchScene<RawParams>* scenes;
    unsigned scene;
    const ViewInfo* views;
    unsigned view;
    const RawGrads* grads;
    int64_t n;
    unsigned entry_base;
    int sh_degree;
    bool fresh;
};
// The view's visible Gaussians add their gradients to the scene's buffers. list (the scene's n
// words) and *list_count (zero on entry) are work space for the compacted visible list.
void launch_gauss_backward(const GaussBackwardArgs& args, const Ctrl* ctrl, const unsigned* depth_key,
                           const unsigned* rank, const unsigned* offs, const unsigned long long* rect_sorted,
                           const float* grad_pair, unsigned* list, unsigned* list_count, cudaStream_t stream);

}  // namespace ab2
