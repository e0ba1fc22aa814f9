// Shared device-side definitions of the B200 Gaussian-splat rasterizer.
//
// Layout in HBM (one scene, N Gaussians, all 16-byte aligned so every load is a 128-bit load):
//   pos_op  float4[N]   x, y, z, opacity (activated)
//   scale   float4[N]   sx, sy, sz, 0     (activated, i.e. exp of the PLY's log-scale)
//   rot     float4[N]   w, x, y, z        (normalised)
//   sh      float4[N][P]  P = ceil(3K/4): the Gaussian's 3K SH floats in [coefficient][channel]
//                         order (gaussian.h:33-35), padded to 16 bytes. Per Gaussian, not planar:
//                         only visible Gaussians read their SH, and a planar layout would pull the
//                         sectors of culled neighbours from DRAM too.
// Per view:
//   rec     float4[3][N]  blend record of each visible Gaussian (see SplatRecord)
//   rect    uint64[N]     16x16-tile rectangle x0 | y0 << 16 | x1 << 32 | y1 << 48
//   depth_key uint32[N]   float bits of each Gaussian's depth less kDepthKeyBase, kCulledKey when culled
//   vis_key / vis_idx     the visible list being depth-sorted: depth bits and Gaussian index
//   pair_key / pair_val   one (tile, Gaussian) pair per tile a splat touches
//   ranges  uint2[tiles]  [start, end) of each tile's run in the sorted pair list
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ab2 {

constexpr int kTile = 16;     // key / blend tile edge in pixels (gpu_render.cu:15)
constexpr int kCpuTile = 8;   // the CPU renderer's binning tile (render.cpp:16)
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxPasses = 4;

// Per-view constants, packed on the host exactly as gpu_render.cu:301-316 packs CameraParams.
struct CamParams {
    float R[9];  // world to camera, row major
    float t[3];
    float eye[3];
    float fx, fy, cx, cy;
    int width, height, tilesX, tilesY;
    int shDegree;   // rendered degree: min(option, scene)
    int shCoeffs;   // coefficients per channel stored in the scene
    float splatScale;
};

struct SceneView {
    const float4* pos_op;
    const float4* scale;
    const float4* rot;
    const float4* sh;   // [n][sh_planes]
    int64_t n;
    int sh_planes;

    // Activated position + opacity, scale and rotation of Gaussian i.
    __device__ __forceinline__ void load(int64_t i, float4& pg, float4& sg, float4& q) const {
        pg = pos_op[i];
        sg = scale[i];
        q = rot[i];
    }
};

// The optimizer's raw per-Gaussian tensors (device memory, row-major): means n x 3, log-scales
// n x 3, quaternions n x 4 (w first, any norm), opacity logits n, SH n x K x 3 with 3K a multiple
// of 4 (sh_planes = 3K / 4). Activated on the fly as the reference loader activates a PLY
// (ply_loader.cpp:124-131): exp, sigmoid, normalise.
struct RawParams {
    const float* means;
    const float* log_scales;
    const float4* quats;
    const float* logits;
    const float4* sh;
    int64_t n;
    int sh_planes;

    __device__ __forceinline__ void load(int64_t i, float4& pg, float4& sg, float4& q) const {
        pg = make_float4(means[3 * i], means[3 * i + 1], means[3 * i + 2], 1.0f / (1.0f + expf(-logits[i])));
        sg = make_float4(expf(log_scales[3 * i]), expf(log_scales[3 * i + 1]), expf(log_scales[3 * i + 2]), 0.f);
        const float4 r = quats[i];
        const float nrm = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
        q = nrm > 0 ? make_float4(r.x / nrm, r.y / nrm, r.z / nrm, r.w / nrm) : make_float4(1.f, 0.f, 0.f, 0.f);
    }
};

// ---- batches: V views of S scenes rendered by one launch sequence ----------------------------
// Each (view, Gaussian of its scene) is an entry with a global index entry_base + i; each
// (view, tile) a global tile tile_base + local tile. Entries of one view, and tiles of one view,
// are contiguous; views of one scene are contiguous.
struct ViewInfo {
    CamParams cam;          // tilesX / tilesY in units of the batch's tile shape
    unsigned scene;
    unsigned entry_base;
    unsigned tile_base;
    unsigned n;             // Gaussians of its scene
    uint8_t* rgb8;          // outputs, any may be null: RGB8 image, float colour, and for the
    float* rgbf;            // backward the final transmittance and last contributor per pixel
    float* t_final;
    unsigned* n_contrib;
    const float* grad_img;  // dL/d(colour) of the view, for the backward
};

template <class Src>
struct BatchScene {
    Src src;
    unsigned view_begin, view_end;  // its views
    unsigned block_base;            // its first preprocess block
};

// Compact per-view tables of a batch (device arrays of n_views entries) for the kernels that map
// an entry or a global tile back to its view.
struct BatchTables {
    const unsigned* entry_base;
    const unsigned* tile_base;
    const unsigned* tiles_x;
    unsigned n_views;
};

// Largest k in [0, count) with bases[k] <= x (bases ascending, bases[0] <= x).
__device__ __forceinline__ unsigned find_segment(const unsigned* bases, unsigned count, unsigned x) {
    unsigned lo = 0, hi = count - 1;
    while (lo < hi) {
        const unsigned mid = (lo + hi + 1) >> 1;
        if (bases[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Control block of one frame. Cleared (the flags folded into the sticky ones) by frame_begin.
struct Ctrl {
    unsigned long long pair_total;      // sum of tiles touched over visible entries
    unsigned int vis_count;             // visible entries
    unsigned int flags;                 // kFlag* bits, read back by the host after the frame
    unsigned int sticky_flags;          // OR of the flags of earlier frames since the host last read it
    unsigned int sort_barrier;          // arrivals at the persistent sort's grid barriers, or CTAs done
                                        // with the tile-bin scan (cleared per frame)
    unsigned long long max_pair_total;  // largest pair_total of earlier frames since then
};

// Depth key of a culled Gaussian. A visible entry's key is its depth's float bits less
// kDepthKeyBase; visible depths are >= 0.2, so the keys never have the sign bit set.
constexpr unsigned kCulledKey = 0xFFFFFFFFu;

// The float bits of 0.125. Every visible depth is >= 0.2 > 0.125, so subtracting them keeps the
// keys' order (positive floats order as their bits), and a depth below 8192 = 0.125 * 2^16 leaves
// a key below 2^27: three 9-bit LSD passes then order the keys as four 8-bit passes over the
// 32-bit depth bits do.
constexpr unsigned kDepthKeyBase = 0x3E000000u;
constexpr unsigned kShortDepthKeyBits = 27;

enum : unsigned {
    kFlagOverflow = 1u,     // pairs exceeded the pair capacity: nothing after duplication ran
    kFlagWaitTimeout = 2u,  // a bounded grid-barrier wait gave up (never expected): the frame is void
};

// ---- digit counts of an LSD pass, accumulated by the kernel that writes the pass's keys ---------
// An LSD pass splits its items into blocks of kSortBlockItems and the blocks into `spans` runs (one
// CTA each; span b holds blocks [T b / spans, T (b + 1) / spans) of the T = ceil(items / block)).
// It needs, per (digit, span), the number of items. Instead of a counting kernel that re-reads
// the keys, the kernel that writes them adds each key to its cell as it goes:
//   counts[digit(key) * digit_stride + span(position) * span_stride] += 1,
// with span(position) = ((position / kSortBlockItems + 1) * spans - 1) / T (the span whose block
// range holds the position). The multi-kernel sort keeps the matrix digit-major (digit_stride =
// spans, span_stride = 1), the persistent sort span-major (1, radix). The cells must be zero
// beforehand; integer adds make the totals independent of their order.
constexpr unsigned kSortBlockItems = 2048;

struct PassCounts {
    unsigned* counts;  // NULL: nothing is counted
    unsigned spans;
    unsigned shift;
    unsigned mask;     // radix - 1
    unsigned digit_stride;
    unsigned span_stride;
};

__device__ __forceinline__ unsigned span_of(unsigned position, unsigned spans, unsigned blocks) {
    return ((position / kSortBlockItems + 1) * spans - 1) / blocks;  // < 2^31: blocks <= 2^21, spans <= 592
}

__device__ __forceinline__ void count_key(const PassCounts& pc, unsigned blocks, unsigned position, unsigned key) {
    atomicAdd(&pc.counts[((key >> pc.shift) & pc.mask) * pc.digit_stride +
                         span_of(position, pc.spans, blocks) * pc.span_stride],
              1u);
}

// ---- programmatic dependent launch --------------------------------------------------------------
// The frame is a chain of ~25 dependent kernels, most of them a few microseconds long, so the gap
// between one kernel's end and the next kernel's start (grid completion, memory flush, launch,
// CTA dispatch) is a visible share of the frame. Kernels of the chain are launched with
// programmatic stream serialisation (launch_chained), which lets the next launch be prepared while
// the previous kernel runs; every chained kernel calls chain_entry() as its first statement, in
// every CTA, which waits until every earlier kernel of the stream has completed and its writes are
// visible. Because the wait is at the top and unconditional, a chained kernel never completes
// before its predecessor, so the ordering stays transitive along the chain, and nothing in the
// kernel touches memory before the wait (no read of an older kernel's output, no write over data
// an older kernel still reads). The wait is the hardware's own grid dependency, not a spin on
// memory; launched without the attribute (or with chaining switched off) it is a no-op.
// No kernel triggers its dependants early (griddepcontrol.launch_dependents): the trigger then
// comes when its CTAs exit. An early trigger lets the CTAs of several later kernels sit resident
// and waiting, holding registers and shared memory that the running kernel's successors need;
// measured on the 740k / 1280x720 frame it gave 0.382 ms against 0.352 ms without it (0.402 ms
// unchained).
__device__ __forceinline__ void chain_entry() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Chaining on unless the environment sets ANISO_B200_CHAIN=0 (read once per process).
bool chain_enabled();
// Kernels launched through launch_chained by the calling host thread so far.
uint64_t chained_launches();
void note_chained_launch();

// kernel<<<grid, block, smem, stream>>>(args...) with programmatic stream serialisation.
template <typename... P, typename... A>
inline void launch_chained_smem(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                A&&... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = chain_enabled() ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    note_chained_launch();
    cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...);
}

// kernel<<<grid, block, 0, stream>>>(args...) with programmatic stream serialisation.
template <typename... P, typename... A>
inline void launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, cudaStream_t stream, A&&... args) {
    launch_chained_smem(kernel, grid, block, 0, stream, static_cast<A&&>(args)...);
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan.
__device__ __forceinline__ unsigned warp_incl_scan(unsigned v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// Exclusive scan over a block of NT threads (NT a multiple of 32, at most 1024); s_tmp holds
// NT/32 words. Returns the thread's exclusive prefix and the block total.
template <int NT>
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned* s_tmp, unsigned& total) {
    constexpr int W = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned incl = warp_incl_scan(v);
    if (lane == 31) s_tmp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned x = lane < W ? s_tmp[lane] : 0u;
        x = warp_incl_scan(x);
        if (lane < W) s_tmp[lane] = x;
    }
    __syncthreads();
    total = s_tmp[W - 1];
    const unsigned before = warp > 0 ? s_tmp[warp - 1] : 0u;
    __syncthreads();
    return before + incl - v;
}

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Blend record: three float4 per visible Gaussian.
//   r0 = (u, v, A2, B2)     r1 = (C2, L, r, g)     r2 = (b, bx, by, block bits)
// where the exponent of the Gaussian in base 2 is A2 dx^2 + B2 dx dy + C2 dy^2 (the conic scaled
// by -log2(e)/2, -log2(e), -log2(e)/2), L = log2(opacity), and bx / by hold two int16 pixel bounds
// (lo | hi << 16): the pixels that lie both in the splat's 8x8-tile rectangle (render.cpp:166-171)
// and inside the ellipse where alpha can reach 1/255 (with a safety margin); the block bits
// (record_block_bits) mark the 8x8 pixel blocks of those bounds where the splat can pass the
// alpha test.
struct SplatRecord {
    float4 r0, r1, r2;
};

// The base-2 exponents of a splat at a lane's two horizontally adjacent pixel centres
// px = (x + 0.5, x + 1.5) of one row (dy = py - v already formed): A2 dx^2 + B2 dx dy + C2 dy^2 + L
// from the record (r0 = u, v, A2, B2; r1 = C2, L, ..), dx = px - u returned too. The row terms are
// shared; the per-pixel operations go as packed FP32x2 instructions (sm_100: one instruction for
// both pixels, per component the rounding of the scalar __fsub_rn / __fmaf_rn). Written with
// explicit roundings so the forward and backward blends compute the same bits (the backward
// replays the forward's alpha tests). Measured: 0.344 -> 0.335 ms per 740k frame, the 64-view
// batch 9.5 -> 9.0 ms.
__device__ __forceinline__ float2 splat_exponents2(const float4& r0, const float4& r1, float2 px, float dy,
                                                   float2& dx) {
    dx = __fadd2_rn(px, make_float2(-r0.x, -r0.x));
    const float t1 = __fmul_rn(r0.w, dy);
    const float t3 = __fmaf_rn(__fmul_rn(r1.x, dy), dy, r1.y);
    const float2 in = __ffma2_rn(make_float2(r0.z, r0.z), dx, make_float2(t1, t1));
    return __ffma2_rn(dx, in, make_float2(t3, t3));
}

// alpha of a splat from its exponent; valid = the reference's tests pass (power <= 0 is p <= L,
// alpha >= 1/255).
__device__ __forceinline__ float splat_alpha(float p, float L, bool& valid) {
    const float alpha = fminf(0.99f, ex2_approx(p));
    valid = !(p > L) && alpha >= 1.0f / 255.0f;
    return alpha;
}

__device__ __forceinline__ unsigned pack_i16x2(int lo, int hi) {
    return (static_cast<unsigned>(lo) & 0xFFFFu) | (static_cast<unsigned>(hi) << 16);
}
__device__ __forceinline__ int unpack_lo(unsigned v) { return static_cast<int>(static_cast<short>(v & 0xFFFFu)); }
__device__ __forceinline__ int unpack_hi(unsigned v) { return static_cast<int>(static_cast<short>(v >> 16)); }

__device__ __forceinline__ float sqrt_mufu(float x) {  // MUFU square root, relative error ~2^-22
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The x-offset interval [xl, xr] (from the splat centre) over which A x^2 + B x y + C y^2 >= D for
// some y in [Y0, Y1]; false when there is none. The form is concave (A, C < 0, 4AC > B^2), so the
// region is an ellipse: its right boundary is concave in y, largest (the half-width W) at
// y = yr = -B W / 2C, so over the band it is largest at the band's point nearest yr (there the
// larger root of the quadratic in x); the left boundary likewise, mirrored (y = -yr). inv2a =
// 1 / 2A. MUFU square roots: the caller widens the interval far beyond their error.
__device__ __forceinline__ bool band_extent(float A, float B, float C, float D, float inv2a, float W, float yr,
                                            float Y0, float Y1, float& xl, float& xr) {
    const auto root = [&](float Y, float sign, float& x) {  // sign -1: the larger root, +1: the smaller
        const float by = B * Y, disc = by * by - 4.f * A * (C * Y * Y - D);
        if (!(disc >= 0.f)) return false;
        x = (sign * sqrt_mufu(disc) - by) * inv2a;
        return true;
    };
    if (yr >= Y0 && yr <= Y1) xr = W;
    else if (!root(yr > Y1 ? Y1 : Y0, -1.f, xr)) return false;
    const float yl = -yr;
    if (yl >= Y0 && yl <= Y1) xl = -W;
    else if (!root(yl > Y1 ? Y1 : Y0, 1.f, xl)) return false;
    return xl <= xr;
}

// The block bits of a blend record (its r2.w), made once per visible entry by the training
// preprocess (the plain one leaves every bit set): over the 8x8 pixel blocks (absolute: block x
// covers pixels [8x, 8x + 7]) that the splat's pixel bounds (r2.y, r2.z: its 8x8-tile rectangle of
// the CPU renderer cut by the bounding box of the ellipse where alpha can reach 1/255) overlap,
// x0b = xlo >> 3 .. and wb blocks wide, bit j * wb + i is set unless the splat's exponent stays
// below log2(1/255) at every pixel centre of block (x0b + i, y0b + j): per block row, the x-extent
// of the ellipse over the row band's centre offsets (band_extent, a continuous superset of the
// centres), widened, against the blocks' centre offsets. The cut is lowered by 0.02 plus a term
// relative to the size of the form's terms over the bounds (in log2 units), and the extent widened
// by 1e-3 of the half-width plus 0.01 pixel, which covers the rounding of this test and of the
// blend's own evaluation. Bounds of more than 32 blocks, or a degenerate form (a coefficient that
// is 0 or not finite, or not concave), set every bit. A blend skips a splat on a block whose bit is
// clear: no pixel there could take anything from it, so the image does not change (and does not
// depend on the tile shape: the blocks are the image's, not the tile's); only warp steps that could
// apply nothing are saved.
__device__ __forceinline__ unsigned record_block_bits(const SplatRecord& r) {
    constexpr float kCut = -7.99435343685885793f;  // log2(1/255)
    const unsigned bx = __float_as_uint(r.r2.y), by = __float_as_uint(r.r2.z);
    const int xlo = unpack_lo(bx), xhi = unpack_hi(bx), ylo = unpack_lo(by), yhi = unpack_hi(by);
    if (xhi < xlo || yhi < ylo) return 0u;
    const int x0b = xlo >> 3, y0b = ylo >> 3, wb = (xhi >> 3) - x0b + 1, hb = (yhi >> 3) - y0b + 1;
    const float u = r.r0.x, v = r.r0.y, A = r.r0.z, B = r.r0.w, C = r.r1.x, L = r.r1.y;
    const float det4 = 4.f * A * C - B * B;
    if (wb * hb > 32 || !(A < 0.f && C < 0.f && det4 > 0.f && isfinite(A + B + C + L + det4))) return 0xFFFFFFFFu;
    const float mx = fmaxf(fabsf(xlo + 0.5f - u), fabsf(xhi + 0.5f - u));
    const float my = fmaxf(fabsf(ylo + 0.5f - v), fabsf(yhi + 0.5f - v));
    const float size = fabsf(A) * mx * mx + fabsf(B) * mx * my + fabsf(C) * my * my;
    const float D = kCut - 0.02f - 1e-5f * size - L;  // the form must reach D somewhere
    if (D > 0.f) return 0u;                             // it cannot: its largest value is 0
    const float W = sqrt_mufu(D * (4.f * C) * __frcp_rn(det4));  // half-width: D / (A - B^2 / 4C)
    const float yr = -B * W * __frcp_rn(2.f * C);
    const float inv2a = __frcp_rn(2.f * A);
    const float eps = 1e-3f * W + 0.01f;
    unsigned bits = 0;
    for (int j = 0; j < hb; ++j) {
        const int y0 = max(ylo, 8 * (y0b + j)), y1 = min(yhi, 8 * (y0b + j) + 7);
        float xl, xr;
        if (!band_extent(A, B, C, D, inv2a, W, yr, y0 + 0.5f - v, y1 + 0.5f - v, xl, xr)) continue;
        // blocks whose centre offsets [8 b + 0.5 - u, 8 b + 7.5 - u] meet [xl - eps, xr + eps]
        const int lo = max(0, static_cast<int>(ceilf((u + xl - eps - 7.5f) * 0.125f)) - x0b);
        const int hi = min(wb - 1, static_cast<int>(floorf((u + xr + eps - 0.5f) * 0.125f)) - x0b);
        if (lo <= hi) bits |= ((2u << hi) - (1u << lo)) << (j * wb);  // bits lo..hi (2u << 31 wraps to 0)
    }
    return bits;
}

// The 8x8 pixel blocks of a TW x TH tile at pixel (ox, oy, multiples of 8) that a staged splat
// record may touch, bit rr * (TW / 8) + c for block (c, rr): the blocks its pixel bounds overlap,
// and with kBits only those whose bit in the record's block bits is set. The training forward and
// the adjoint stage the same masks.
template <int TW, int TH, bool kBits>
__device__ __forceinline__ unsigned staged_block_mask(const SplatRecord& r, int ox, int oy) {
    constexpr int kWX = TW / 8, kWY = TH / 8;
    const unsigned bx = __float_as_uint(r.r2.y), by = __float_as_uint(r.r2.z);
    const int xlo = unpack_lo(bx), xhi = unpack_hi(bx), ylo = unpack_lo(by), yhi = unpack_hi(by);
    unsigned m = 0;
    if (!kBits) {
        unsigned cols = 0;
#pragma unroll
        for (int c = 0; c < kWX; ++c)
            if (xlo <= ox + 8 * c + 7 && xhi >= ox + 8 * c) cols |= 1u << c;
#pragma unroll
        for (int rr = 0; rr < kWY; ++rr)
            if (ylo <= oy + 8 * rr + 7 && yhi >= oy + 8 * rr) m |= cols << (kWX * rr);
        return m;
    }
    const unsigned bits = __float_as_uint(r.r2.w);
    const int x0b = xlo >> 3, y0b = ylo >> 3, wb = (xhi >> 3) - x0b + 1;
#pragma unroll
    for (int rr = 0; rr < kWY; ++rr) {
        const int py = oy + 8 * rr;
        if (ylo > py + 7 || yhi < py) continue;
#pragma unroll
        for (int c = 0; c < kWX; ++c) {
            const int px = ox + 8 * c;
            if (xlo > px + 7 || xhi < px) continue;
            const int idx = ((py >> 3) - y0b) * wb + ((px >> 3) - x0b);
            if (idx >= 32 || ((bits >> idx) & 1u)) m |= 1u << (rr * kWX + c);
        }
    }
    return m;
}

}  // namespace ab2
