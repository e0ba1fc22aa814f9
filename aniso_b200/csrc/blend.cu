// Step 5 of the rasterizer: front-to-back blending, one 256-thread block per 16x16 tile.
//
// Per pixel this is the blend of render.cpp:195-220 / gpu_render.cu:180-233:
//   power = -(A dx^2 + C dy^2)/2 - B dx dy; skip if power > 0
//   alpha = min(0.99, opacity * exp(power)); skip if alpha < 1/255
//   stop (without applying) once T (1 - alpha) < 1e-4; else C += rgb alpha T, T *= 1 - alpha
// evaluated in base 2 on the pre-scaled conic of the SplatRecord (one MUFU ex2 per evaluation).
//
// B200 mapping:
//   * each warp owns an 8x4 pixel block (lane -> pixel), so a tile is 2 x 4 warp blocks and every
//     warp block lies inside one 8x8 tile of the CPU renderer;
//   * the block stages 256 splat records per round in shared memory and, per splat, builds an
//     8-bit mask of the warp blocks it can touch: its pixel bounds (the CPU 8x8-tile rectangle cut
//     by the ellipse where alpha can reach 1/255) against each warp block. The 8x8 part makes every
//     pixel see exactly the splat list the CPU renderer gives it; the ellipse part only drops splats
//     that cannot pass the alpha test anywhere in the warp block, so it changes no result;
//   * each warp walks only its set bits (ballot + ffs), exits as soon as all 32 pixels are opaque,
//     and the block stops loading once all 256 pixels are done (__syncthreads_count).
#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

__device__ __forceinline__ bool overlaps(int lo, int hi, int a, int b) { return lo <= b && hi >= a; }

template <bool kTrain>
__global__ void __launch_bounds__(256) blend_kernel(const uint2* __restrict__ ranges,
                                                    const unsigned* __restrict__ vals,
                                                    const SplatRecord* __restrict__ rec, const Ctrl* ctrl, int width,
                                                    int height, int tiles_x, BlendOut out) {
    __shared__ float4 s_r0[256];
    __shared__ float4 s_r1[256];
    __shared__ float s_b[256];
    __shared__ unsigned char s_mask[256];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tile = blockIdx.x;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    const int ox = tx * kTile, oy = ty * kTile;
    const int pxi = ox + (warp & 1) * 8 + (lane & 7), pyi = oy + (warp >> 1) * 4 + (lane >> 3);
    const bool inside = pxi < width && pyi < height;
    const float px = pxi + 0.5f, py = pyi + 0.5f;
    const uint2 range = (ctrl->flags & kFlagOverflow) ? make_uint2(0, 0) : ranges[tile];

    float T = 1.0f, cr = 0.f, cg = 0.f, cb = 0.f;
    bool done = !inside;
    unsigned last = range.x;

    for (unsigned b0 = range.x; b0 < range.y; b0 += 256) {
        if (__syncthreads_count(done) == 256) break;
        const unsigned j = b0 + tid;
        unsigned m = 0;
        if (j < range.y) {
            const SplatRecord r = rec[vals[j]];
            s_r0[tid] = r.r0;
            s_r1[tid] = r.r1;
            s_b[tid] = r.r2.x;
            const unsigned bx = __float_as_uint(r.r2.y), by = __float_as_uint(r.r2.z);
            const int xlo = unpack_lo(bx), xhi = unpack_hi(bx), ylo = unpack_lo(by), yhi = unpack_hi(by);
            const unsigned cols = (overlaps(xlo, xhi, ox, ox + 7) ? 1u : 0u) | (overlaps(xlo, xhi, ox + 8, ox + 15) ? 2u : 0u);
#pragma unroll
            for (int row = 0; row < 4; ++row)
                if (overlaps(ylo, yhi, oy + 4 * row, oy + 4 * row + 3)) m |= cols << (2 * row);
        }
        s_mask[tid] = static_cast<unsigned char>(m);
        __syncthreads();
        const unsigned cnt = min(256u, range.y - b0);
        bool warp_done = __all_sync(0xFFFFFFFFu, done);
        for (unsigned c = 0; c * 32 < cnt && !warp_done; ++c) {
            const unsigned idx = c * 32 + lane;
            unsigned bits = __ballot_sync(0xFFFFFFFFu, idx < cnt && ((s_mask[idx] >> warp) & 1u));
            while (bits) {
                const unsigned jj = c * 32 + (__ffs(bits) - 1);
                bits &= bits - 1;
                const float4 a = s_r0[jj];
                const float4 q1 = s_r1[jj];
                const float dx = px - a.x, dy = py - a.y;
                const float q = fmaf(dx, fmaf(a.z, dx, a.w * dy), q1.x * dy * dy);
                const float alpha = fminf(0.99f, ex2_approx(q + q1.y));
                if (!done && !(q > 0.f) && alpha >= 1.0f / 255.0f) {
                    const float nt = T * (1.0f - alpha);
                    if (nt < 1e-4f) {
                        done = true;
                    } else {
                        const float w = alpha * T;
                        cr = fmaf(q1.z, w, cr);
                        cg = fmaf(q1.w, w, cg);
                        cb = fmaf(s_b[jj], w, cb);
                        T = nt;
                        if (kTrain) last = b0 + jj + 1;
                    }
                }
                if (__all_sync(0xFFFFFFFFu, done)) {
                    warp_done = true;
                    break;
                }
            }
        }
    }
    if (inside) {
        const size_t p = static_cast<size_t>(pyi) * width + pxi;
        if (out.rgb8) {
            uint8_t* o = out.rgb8 + p * 3;
            o[0] = static_cast<uint8_t>(fminf(fmaxf(cr, 0.f), 1.f) * 255.f + 0.5f);
            o[1] = static_cast<uint8_t>(fminf(fmaxf(cg, 0.f), 1.f) * 255.f + 0.5f);
            o[2] = static_cast<uint8_t>(fminf(fmaxf(cb, 0.f), 1.f) * 255.f + 0.5f);
        }
        if (kTrain) {
            out.rgbf[p * 3 + 0] = cr;
            out.rgbf[p * 3 + 1] = cg;
            out.rgbf[p * 3 + 2] = cb;
            out.t_final[p] = T;
            out.n_contrib[p] = last;
        }
    }
}

}  // namespace

void launch_blend(const uint2* ranges, const unsigned* sorted_vals, const SplatRecord* rec, const Ctrl* ctrl,
                  int width, int height, int tiles_x, int tiles_y, const BlendOut& out, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>(tiles_x) * static_cast<unsigned>(tiles_y);
    if (blocks == 0) return;
    if (out.rgbf)
        blend_kernel<true><<<blocks, 256, 0, stream>>>(ranges, sorted_vals, rec, ctrl, width, height, tiles_x, out);
    else
        blend_kernel<false><<<blocks, 256, 0, stream>>>(ranges, sorted_vals, rec, ctrl, width, height, tiles_x, out);
}

}  // namespace ab2
