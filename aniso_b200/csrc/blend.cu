// Step 5 of the rasterizer: front-to-back blending, one block per tile of a batch (any view),
// for tile shapes TW x TH of 8x8, 16x16 (the reference's) and 16x32 pixels.
//
// Per pixel this is the blend of render.cpp:195-220 / gpu_render.cu:180-233:
//   power = -(A dx^2 + C dy^2)/2 - B dx dy; skip if power > 0
//   alpha = min(0.99, opacity * exp(power)); skip if alpha < 1/255
//   stop (without applying) once T (1 - alpha) < 1e-4; else C += rgb alpha T, T *= 1 - alpha
// evaluated in base 2 on the pre-scaled conic of the SplatRecord (one MUFU ex2 per evaluation).
//
// B200 mapping (the kernel is FP32-issue bound, so the layout minimises instructions per pixel):
//   * each warp owns one 8x8 pixel block -- exactly one tile of the CPU renderer -- with two
//     horizontally adjacent pixels per lane; the row terms of the exponent (with log2(opacity)
//     folded in) are shared, and the two pixels' offsets and FMAs are packed FP32x2 instructions
//     (three for both pixels' exponents);
//   * the block stages kBatch splat records per round in shared memory and, per splat, a mask of
//     the warp blocks it can touch (staged_block_mask): its pixel bounds (the CPU 8x8-tile
//     rectangle cut by the bounding box of the ellipse where alpha can reach 1/255, with a margin)
//     against each 8x8 block -- which gives every pixel exactly the splat list of the CPU renderer
//     whatever the tile shape (so the image does not depend on it) -- and, in training, the
//     record's block bits (the blocks where the ellipse itself reaches the cut, set once per splat
//     by the training preprocess), which only drop splats that cannot pass the alpha test anywhere
//     in the block, so they change no result. The plain forward leaves them out: their cost in the
//     preprocess (+14 us per 740k frame) is more than the blend steps they save (-9 us), where the
//     training step, whose adjoint replays every step at about four times the cost, gains (forward
//     and adjoint at 2.2M: 1.84 -> 1.73 ms; the 8-scene training batch 29.0 -> 27.0 ms a step).
//     Testing every block against the ellipse in each tile's staging instead cost more than it
//     saved: 0.161 -> 0.186 ms of blend;
//   * each warp walks only its splats (listed once per round from the masks by ballot and
//     popcount); a finished pixel holds T = 0 (T >= 1e-4 while it is not finished), so no
//     separate flag is carried; the warp leaves once all 64 pixels are finished and the block
//     stops loading once all its warps have (__syncthreads_or).
#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

// Both of a lane's pixels' step for one splat. p is each pixel's base-2 exponent including
// log2(opacity) L, so alpha = min(0.99, 2^p) and the reference's "power > 0" skip is p > L. The
// new transmittance is T - alpha T (one instruction fewer than T (1 - alpha); it differs only in
// rounding); once it would fall below 1e-4 the pixel is finished: T = 0 and the splat is not
// applied (T = 0 keeps a finished pixel finished). The weights, new transmittances and colour sums
// are packed FP32x2 instructions (per component the rounding of the scalar ones; T + (-1) w in one
// rounding is T - w) and the conditions selects: a pixel that does not take the splat adds 0 x
// colour, which leaves its sum as it was for the finite colours the blend stages (measured 0.153
// -> 0.139 ms of blend per 740k frame against a scalar step with branches). In training mode tfin
// keeps the transmittance after the last applied splat and last the list position one past it.
template <bool kTrain>
__device__ __forceinline__ void blend_px2(float2 p, float L, float r, float g, float b, float2& T, float2& cr,
                                          float2& cg, float2& cb, float2& tfin, unsigned& last0, unsigned& last1,
                                          unsigned pos) {
    bool v0, v1;
    const float a0 = splat_alpha(p.x, L, v0), a1 = splat_alpha(p.y, L, v1);
    const float2 w = __fmul2_rn(make_float2(a0, a1), T);
    const float2 nt = __ffma2_rn(make_float2(-1.f, -1.f), w, T);
    const bool k0 = v0 && !(nt.x < 1e-4f), k1 = v1 && !(nt.y < 1e-4f);
    T.x = v0 ? (k0 ? nt.x : 0.f) : T.x;  // taken, finished, or skipped
    T.y = v1 ? (k1 ? nt.y : 0.f) : T.y;
    const float2 wk = make_float2(k0 ? w.x : 0.f, k1 ? w.y : 0.f);
    cr = __ffma2_rn(make_float2(r, r), wk, cr);
    cg = __ffma2_rn(make_float2(g, g), wk, cg);
    cb = __ffma2_rn(make_float2(b, b), wk, cb);
    if (kTrain) {
        tfin.x = k0 ? nt.x : tfin.x;
        tfin.y = k1 ? nt.y : tfin.y;
        last0 = k0 ? pos : last0;
        last1 = k1 ? pos : last1;
    }
}

// The training outputs of one pixel: float colour, final transmittance, one past the last splat.
__device__ __forceinline__ void store_train_px(const ViewInfo& vi, int x, int y, float tfin, float cr, float cg,
                                               float cb, unsigned last) {
    const int width = vi.cam.width;
    if (x >= width || y >= vi.cam.height) return;
    const size_t p = static_cast<size_t>(y) * width + x;
    vi.rgbf[p * 3 + 0] = cr;
    vi.rgbf[p * 3 + 1] = cg;
    vi.rgbf[p * 3 + 2] = cb;
    vi.t_final[p] = tfin;
    vi.n_contrib[p] = last;
}

// One 8-bit channel as render.cpp quantises it: clamp to [0, 1], scale by 255, round half up.
__device__ __forceinline__ unsigned quantise(float c) {
    return static_cast<unsigned>(static_cast<uint8_t>(fminf(fmaxf(c, 0.f), 1.f) * 255.f + 0.5f));
}

// Copies the tile's RGB8 pixels, staged in s_px (TH rows of TW * 3 bytes, 16-byte aligned), to
// the image as whole row segments: 16-byte stores where the image rows and the segment allow,
// else 4-byte ones, else single bytes. Wide contiguous stores matter most when `out` is pinned
// host memory written across PCIe during the blend (each store instruction becomes a few bus
// writes, where per-pixel bytes would become many partial ones); in device memory they cost no
// more than per-pixel stores.
template <int TW, int TH, int kThreads>
__device__ __forceinline__ void write_tile_rgb8(const unsigned char* s_px, uint8_t* out, int width, int height,
                                                int ox, int oy) {
    constexpr int kRow = TW * 3;
    const int rows = min(TH, height - oy), seg = min(TW, width - ox) * 3;  // both >= 1: the tile starts inside
    const size_t pitch = static_cast<size_t>(width) * 3;
    uint8_t* dst = out + static_cast<size_t>(oy) * pitch + static_cast<size_t>(ox) * 3;
    const uintptr_t a = reinterpret_cast<uintptr_t>(dst) | pitch | static_cast<unsigned>(seg) | kRow;
    if ((a & 15) == 0) {
        const int per = seg >> 4;
        for (int i = threadIdx.x; i < rows * per; i += kThreads) {
            const int r = i / per, c = i - r * per;
            *reinterpret_cast<uint4*>(dst + r * pitch + c * 16) =
                *reinterpret_cast<const uint4*>(s_px + r * kRow + c * 16);
        }
    } else if ((a & 3) == 0) {
        const int per = seg >> 2;
        for (int i = threadIdx.x; i < rows * per; i += kThreads) {
            const int r = i / per, c = i - r * per;
            *reinterpret_cast<unsigned*>(dst + r * pitch + c * 4) =
                *reinterpret_cast<const unsigned*>(s_px + r * kRow + c * 4);
        }
    } else {
        for (int i = threadIdx.x; i < rows * seg; i += kThreads) {
            const int r = i / seg, c = i - r * seg;
            dst[r * pitch + c] = s_px[r * kRow + c];
        }
    }
}

template <int TW, int TH, int kBatch, bool kTrain>
__global__ void __launch_bounds__(TW * TH / 2) blend_kernel(const uint2* __restrict__ ranges,
                                                            const unsigned* __restrict__ vals,
                                                            const SplatRecord* __restrict__ rec, const Ctrl* ctrl,
                                                            const ViewInfo* __restrict__ views, BatchTables tables) {
    chain_entry();
    constexpr int kThreads = TW * TH / 2;  // two pixels per lane
    constexpr int kWarpsX = TW / 8;
    __shared__ float4 s_r0[kBatch];
    __shared__ float4 s_r1[kBatch];
    __shared__ float s_b[kBatch];
    __shared__ unsigned char s_mask[kBatch];
    __shared__ unsigned short s_list[kThreads / 32][kBatch];  // each warp's splats of the round
    __shared__ __align__(16) unsigned char s_px[TH * TW * 3];  // the tile's RGB8, staged for row stores

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned gtile = blockIdx.x;
    const unsigned v = find_segment(tables.tile_base, tables.n_views, gtile);
    const ViewInfo& vi = views[v];
    const int tiles_x = vi.cam.tilesX;
    const unsigned local = gtile - vi.tile_base;
    const int ox = static_cast<int>(local % tiles_x) * TW, oy = static_cast<int>(local / tiles_x) * TH;
    const int x0 = ox + (warp % kWarpsX) * 8 + 2 * (lane & 3), y = oy + (warp / kWarpsX) * 8 + (lane >> 2);
    const int width = vi.cam.width, height = vi.cam.height;
    const float px0 = x0 + 0.5f, py = y + 0.5f;
    const uint2 range = (ctrl->flags & kFlagOverflow) ? make_uint2(0, 0) : ranges[gtile];
    const unsigned lt = lanemask_lt();

    // Pixels outside the image start finished.
    float2 T = make_float2((x0 < width && y < height) ? 1.0f : 0.f, (x0 + 1 < width && y < height) ? 1.0f : 0.f);
    float2 cr = make_float2(0.f, 0.f), cg = cr, cb = cr;
    unsigned last0 = range.x, last1 = range.x;
    float2 tf = make_float2(1.0f, 1.0f);

    for (unsigned base = range.x; base < range.y; base += kBatch) {
        if (!__syncthreads_or(T.x + T.y > 0.f)) break;
#pragma unroll
        for (int h = 0; h < kBatch / kThreads; ++h) {
            const int slot = tid + h * kThreads;
            const unsigned j = base + slot;
            unsigned m = 0;
            if (j < range.y) {
                const SplatRecord r = rec[vals[j]];
                constexpr float kMax = 3.40282347e38f;  // an infinite colour quantises as the largest finite one
                s_r0[slot] = r.r0;
                s_r1[slot] = make_float4(r.r1.x, r.r1.y, fminf(r.r1.z, kMax), fminf(r.r1.w, kMax));
                s_b[slot] = fminf(r.r2.x, kMax);
                m = staged_block_mask<TW, TH, kTrain>(r, ox, oy);
            }
            s_mask[slot] = static_cast<unsigned char>(m);
        }
        __syncthreads();
        const unsigned cnt = min(static_cast<unsigned>(kBatch), range.y - base);
        if (!__any_sync(0xFFFFFFFFu, T.x + T.y > 0.f)) continue;  // the warp is finished
        // The warp's splats of the round in list order, compacted once (a ballot per 32 staged)
        // rather than found bit by bit in each step (0.1395 -> 0.1376 ms per 740k frame).
        unsigned n = 0;
        for (unsigned c = 0; c * 32 < cnt; ++c) {
            const unsigned idx = c * 32 + lane;
            const bool mine = idx < cnt && ((s_mask[idx] >> warp) & 1u);
            const unsigned bits = __ballot_sync(0xFFFFFFFFu, mine);
            if (mine) s_list[warp][n + __popc(bits & lt)] = static_cast<unsigned short>(idx);
            n += __popc(bits);
        }
        __syncwarp();
        for (unsigned i = 0; i < n; i += 4) {
            // Up to four splats per vote on whether the warp is finished (a vote per splat, or per
            // two, costs more than the steps a finished warp walks in vain: 0.161 -> 0.154 ms per
            // 740k frame from two to four).
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (i + u >= n) break;
                const unsigned jj = s_list[warp][i + u];
                const float4 a = s_r0[jj];
                const float4 k = s_r1[jj];
                const float bb = s_b[jj];
                float2 dx;
                const float2 pp = splat_exponents2(a, k, make_float2(px0, px0 + 1.0f), __fsub_rn(py, a.y), dx);
                blend_px2<kTrain>(pp, k.y, k.z, k.w, bb, T, cr, cg, cb, tf, last0, last1, base + jj + 1);
            }
            if (!__any_sync(0xFFFFFFFFu, T.x + T.y > 0.f)) break;
        }
    }
    if (kTrain) {
        store_train_px(vi, x0, y, tf.x, cr.x, cg.x, cb.x, last0);
        store_train_px(vi, x0 + 1, y, tf.y, cr.y, cg.y, cb.y, last1);
    }
    if (vi.rgb8) {  // the same for the whole block: one view per tile
        // The lane's two pixels are 6 bytes at an even pixel column: three 2-byte words.
        unsigned short* q = reinterpret_cast<unsigned short*>(s_px + ((y - oy) * TW + (x0 - ox)) * 3);
        q[0] = static_cast<unsigned short>(quantise(cr.x) | quantise(cg.x) << 8);
        q[1] = static_cast<unsigned short>(quantise(cb.x) | quantise(cr.y) << 8);
        q[2] = static_cast<unsigned short>(quantise(cg.y) | quantise(cb.y) << 8);
        __syncthreads();
        write_tile_rgb8<TW, TH, kThreads>(s_px, vi.rgb8, width, height, ox, oy);
    }
}

template <int TW, int TH, int kBatch>
void launch_shape(unsigned tiles, const uint2* ranges, const unsigned* vals, const SplatRecord* rec, const Ctrl* ctrl,
                  const ViewInfo* views, const BatchTables& tables, bool train, cudaStream_t stream) {
    if (train)
        launch_chained(blend_kernel<TW, TH, kBatch, true>, dim3(tiles), dim3(TW * TH / 2), stream, ranges, vals, rec,
                       ctrl, views, tables);
    else
        launch_chained(blend_kernel<TW, TH, kBatch, false>, dim3(tiles), dim3(TW * TH / 2), stream, ranges, vals, rec,
                       ctrl, views, tables);
}

}  // namespace

bool blend_shape_supported(int tile_w, int tile_h) {
    return (tile_w == 8 && tile_h == 8) || (tile_w == 16 && tile_h == 16) || (tile_w == 16 && tile_h == 32);
}

void launch_blend(unsigned tiles, const uint2* ranges, const unsigned* sorted_vals, const SplatRecord* rec,
                  const Ctrl* ctrl, const ViewInfo* views, const BatchTables& tables, int tile_w, int tile_h,
                  int batch, bool train, cudaStream_t stream) {
    if (tiles == 0) return;
    const bool big = batch >= 256;
    if (tile_w == 8) {
        if (big) launch_shape<8, 8, 256>(tiles, ranges, sorted_vals, rec, ctrl, views, tables, train, stream);
        else launch_shape<8, 8, 128>(tiles, ranges, sorted_vals, rec, ctrl, views, tables, train, stream);
    } else if (tile_h == 32) {
        if (big) launch_shape<16, 32, 512>(tiles, ranges, sorted_vals, rec, ctrl, views, tables, train, stream);
        else launch_shape<16, 32, 256>(tiles, ranges, sorted_vals, rec, ctrl, views, tables, train, stream);
    } else {
        if (big) launch_shape<16, 16, 256>(tiles, ranges, sorted_vals, rec, ctrl, views, tables, train, stream);
        else launch_shape<16, 16, 128>(tiles, ranges, sorted_vals, rec, ctrl, views, tables, train, stream);
    }
}

}  // namespace ab2
