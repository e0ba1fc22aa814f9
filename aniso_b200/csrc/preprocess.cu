// Step 1 of the rasterizer: every (view, Gaussian) entry of a batch, each Gaussian read once for
// all the views of its scene (early test per lane, exact projection by warp-wide work queue).
//
// Projects each Gaussian the way gpu_render.cu:86-145 does (the same fp32 expressions in the same
// order, compiled without fast-math, so depth, rectangle and conic come out bit-identical to the
// reference kernel built without --use_fast_math), then, fused into the same kernel:
//   * writes the blend record (SplatRecord) and the tile rectangle of visible Gaussians;
//   * writes every entry's depth key (the float bits of its depth; a sentinel if culled) -- the
//     first LSD pass of the depth sort compacts the visible ones as it ranks them.
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

constexpr float kShC1 = 0.4886025119029199f;
constexpr float kShC2_0 = 1.0925484305920792f, kShC2_1 = -1.0925484305920792f, kShC2_2 = 0.31539156525252005f,
                kShC2_3 = -1.0925484305920792f, kShC2_4 = 0.5462742152960396f;
constexpr float kShC3_0 = -0.5900435899266435f, kShC3_1 = 2.890611442640554f, kShC3_2 = -0.4570457994644658f,
                kShC3_3 = 0.3731763325901154f, kShC3_4 = -0.4570457994644658f, kShC3_5 = 1.445305721320277f,
                kShC3_6 = -0.5900435899266435f;

// MUFU approximations (relative error ~2^-22) for quantities that carry their own margins (the
// early screen test, the pixel bounds, log2 of the opacity), never the reference's bit-exact
// geometry (depth, conic, radius, rectangle) or colour.
__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// SH colour of degree D along (x, y, z): the basis of sh.cpp:18-58 / gpu_render.cu:56-83, then
// +0.5 and clamped at 0. The coefficients are streamed straight from the Gaussian's 16-byte words
// ([coefficient][channel] order), so nothing stays live across views; each channel still sums its
// terms in ascending coefficient order, as the reference does.
template <int D>
__device__ __forceinline__ float3 sh_color(const float4* __restrict__ shp, float x, float y, float z) {
    float b[16];
    b[0] = 0.28209479177387814f;
    if (D >= 1) {
        b[1] = -kShC1 * y; b[2] = kShC1 * z; b[3] = -kShC1 * x;
    }
    if (D >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        b[4] = kShC2_0 * x * y; b[5] = kShC2_1 * y * z; b[6] = kShC2_2 * (2 * zz - xx - yy);
        b[7] = kShC2_3 * x * z; b[8] = kShC2_4 * (xx - yy);
        if (D >= 3) {
            b[9] = kShC3_0 * y * (3 * xx - yy); b[10] = kShC3_1 * x * y * z; b[11] = kShC3_2 * y * (4 * zz - xx - yy);
            b[12] = kShC3_3 * z * (2 * zz - 3 * xx - 3 * yy); b[13] = kShC3_4 * x * (4 * zz - xx - yy);
            b[14] = kShC3_5 * z * (xx - yy); b[15] = kShC3_6 * x * (xx - 3 * yy);
        }
    }
    constexpr int kFloats = (D + 1) * (D + 1) * 3;
    constexpr int kPlanes = (kFloats + 3) / 4;
    float c[3] = {0.5f, 0.5f, 0.5f};
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) {
        const float4 f = shp[k];
        const float v[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int idx = 4 * k + e;
            if (idx < kFloats) c[idx % 3] += b[idx / 3] * v[e];
        }
    }
    return make_float3(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f), fmaxf(c[2], 0.f));
}

// The colour at the view's own degree (<= D, and <= the scene's stored degree, so the words read
// are the Gaussian's own): views of scenes with different degrees share one launch.
template <int D>
__device__ __forceinline__ float3 sh_color_upto(int degree, const float4* __restrict__ shp, float x, float y, float z) {
    if (D >= 3 && degree >= 3) return sh_color<3>(shp, x, y, z);
    if (D >= 2 && degree == 2) return sh_color<(D >= 2 ? 2 : 0)>(shp, x, y, z);
    if (D >= 1 && degree == 1) return sh_color<(D >= 1 ? 1 : 0)>(shp, x, y, z);
    return sh_color<0>(shp, x, y, z);
}

struct Projected {
    float u, v, depth;
    float a, b, c, det;       // 2D covariance (with the 0.3 low-pass) and its determinant
    float conicA, conicB, conicC;
    int radius;
    int x0, y0, x1, y1;       // 16x16-tile rectangle
};

// The view-independent part of gpu_render.cu:101-111, evaluated once per Gaussian for all its
// views with the same expressions in the same order: the 3D covariance S = M M^T with
// M = R(q) diag(s * splat_scale), and tr(S) for the early screen test. S is kept as its upper
// triangle: S[c][r] and S[r][c] are the same products summed in the same order, so equal bits.
struct Cov3 {
    float s00, s01, s02, s11, s12, s22;
    float trace;
    __device__ __forceinline__ float at(int r, int c) const {
        const int lo = r < c ? r : c, hi = r < c ? c : r;
        return lo == 0 ? (hi == 0 ? s00 : hi == 1 ? s01 : s02) : lo == 1 ? (hi == 1 ? s11 : s12) : s22;
    }
};

__device__ __forceinline__ void covariance(const float4 sg, const float4 q, float splat_scale, Cov3& o) {
    const float w = q.x, x = q.y, y = q.z, z = q.w;
    const float Rq[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                            {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                            {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
    const float s[3] = {sg.x * splat_scale, sg.y * splat_scale, sg.z * splat_scale};
    float M[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) M[r][c] = Rq[r][c] * s[c];
    const auto dot = [&](int r, int c) { return M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2]; };
    o.s00 = dot(0, 0);
    o.s01 = dot(0, 1);
    o.s02 = dot(0, 2);
    o.s11 = dot(1, 1);
    o.s12 = dot(1, 2);
    o.s22 = dot(2, 2);
    o.trace = o.s00 + o.s11 + o.s22;
}

// The conservative early screen test (see project()) of a camera-space centre with pz >= 0.2.
__device__ __forceinline__ bool early_screen(float px, float py, float pz, float limX, float limY, const Cov3& cov,
                                             const CamParams& cam) {
    const float iz = __frcp_rn(pz);
    const float ex = fminf(limX, fmaxf(-limX, px * iz)) * pz, ey = fminf(limY, fmaxf(-limY, py * iz)) * pz;
    const float j00 = cam.fx * iz, j02 = -cam.fx * ex * iz * iz, j11 = cam.fy * iz, j12 = -cam.fy * ey * iz * iz;
    float tn = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float t0 = j00 * cam.R[c] + j02 * cam.R[6 + c];
        const float t1 = j11 * cam.R[3 + c] + j12 * cam.R[6 + c];
        tn += t0 * t0 + t1 * t1;
    }
    const float rb = 3.0f * sqrt_approx((tn * cov.trace + 0.92f) * 1.001f) + 1.0f;
    const float uu = cam.fx * px * iz + cam.cx, vv = cam.fy * py * iz + cam.cy;
    const float du = 1e-5f * (fabsf(uu) + fabsf(cam.cx)) + 0.01f + rb;
    const float dv = 1e-5f * (fabsf(vv) + fabsf(cam.cy)) + 0.01f + rb;
    return !(uu + du < 0.f || vv + dv < 0.f || uu - du >= cam.width || vv - dv >= cam.height);
}

// The culling and projection of gpu_render.cu:93-135 (the rectangle in units of tile_w x tile_h
// pixels; 16 x 16 is the reference's), on the precomputed covariance. Returns false when the
// Gaussian is culled.
//
// Before the exact screen test (which needs the 2D covariance, its eigenvalue and eight IEEE
// divisions), a conservative one: lambda <= a + c + sqrt(0.1) <= ||T||_F^2 tr(S) + 0.6 + 0.317,
// because tr(T S T^T) <= lambda_max(S) ||T||_F^2 <= tr(S) ||T||_F^2, evaluated with a rounded
// reciprocal and widened (x1.001 under the root, +1 pixel for the ceiling, a relative margin on
// the centre) so that it only culls what the exact test culls. NaN or infinite inputs never pass
// it and fall through to the exact test.
// The near-plane cut and the conservative early screen test alone (true: the exact test may pass).
__device__ __forceinline__ bool early_visible(const float4 pg, const Cov3& cov, const CamParams& cam) {
    const float gx = pg.x, gy = pg.y, gz = pg.z;
    const float px = cam.R[0] * gx + cam.R[1] * gy + cam.R[2] * gz + cam.t[0];
    const float py = cam.R[3] * gx + cam.R[4] * gy + cam.R[5] * gz + cam.t[1];
    const float pz = cam.R[6] * gx + cam.R[7] * gy + cam.R[8] * gz + cam.t[2];
    if (pz < 0.2f) return false;
    const float limX = 1.3f * 0.5f * cam.width / cam.fx, limY = 1.3f * 0.5f * cam.height / cam.fy;
    return early_screen(px, py, pz, limX, limY, cov, cam);
}

__device__ __forceinline__ bool project(const float4 pg, const Cov3& cov, const CamParams& cam, int tile_w, int tile_h,
                                        Projected& o) {
    const float gx = pg.x, gy = pg.y, gz = pg.z;
    const float px = cam.R[0] * gx + cam.R[1] * gy + cam.R[2] * gz + cam.t[0];
    const float py = cam.R[3] * gx + cam.R[4] * gy + cam.R[5] * gz + cam.t[1];
    const float pz = cam.R[6] * gx + cam.R[7] * gy + cam.R[8] * gz + cam.t[2];
    if (pz < 0.2f) return false;

    const float limX = 1.3f * 0.5f * cam.width / cam.fx, limY = 1.3f * 0.5f * cam.height / cam.fy;
    if (!early_screen(px, py, pz, limX, limY, cov, cam)) return false;

    const float tx = fminf(limX, fmaxf(-limX, px / pz)) * pz;
    const float ty = fminf(limY, fmaxf(-limY, py / pz)) * pz;
    const float J[2][3] = {{cam.fx / pz, 0, -cam.fx * tx / (pz * pz)}, {0, cam.fy / pz, -cam.fy * ty / (pz * pz)}};
    float T[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) T[r][c] = J[r][0] * cam.R[c] + J[r][1] * cam.R[3 + c] + J[r][2] * cam.R[6 + c];
    float TS[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) TS[r][c] = T[r][0] * cov.at(0, c) + T[r][1] * cov.at(1, c) + T[r][2] * cov.at(2, c);
    const float a = TS[0][0] * T[0][0] + TS[0][1] * T[0][1] + TS[0][2] * T[0][2] + 0.3f;
    const float b = TS[0][0] * T[1][0] + TS[0][1] * T[1][1] + TS[0][2] * T[1][2];
    const float c = TS[1][0] * T[1][0] + TS[1][1] * T[1][1] + TS[1][2] * T[1][2] + 0.3f;
    const float det = a * c - b * b;
    if (det <= 0) return false;
    // A projection that is not finite (a NaN or infinite position, scale or rotation, or an
    // overflow on the way) or a radius of a billion pixels or more is culled. The reference leaves
    // these cases to undefined float-to-int conversions (render.cpp:84-89, gpu_render.cu:126-132),
    // which on x86-64 leave such a splat with no tile; culling them gives that image everywhere.
    // Finite, representable projections are unaffected (bit for bit).
    if (!(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(det))) return false;

    const float mid = 0.5f * (a + c);
    const float lambda = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
    const float r3 = 3.0f * sqrtf(lambda);
    if (!(r3 < 1.0e9f)) return false;
    const int radius = (int)ceilf(r3);
    const float u = cam.fx * px / pz + cam.cx, v = cam.fy * py / pz + cam.cy;
    if (!(isfinite(u) && isfinite(v))) return false;
    if (u + radius < 0 || v + radius < 0 || u - radius >= cam.width || v - radius >= cam.height) return false;

    const int x0 = max(0, (int)(u - radius) / tile_w), y0 = max(0, (int)(v - radius) / tile_h);
    const int x1 = min(cam.tilesX - 1, (int)(u + radius) / tile_w), y1 = min(cam.tilesY - 1, (int)(v + radius) / tile_h);
    if (x1 < x0 || y1 < y0) return false;

    o.u = u; o.v = v; o.depth = pz;
    o.a = a; o.b = b; o.c = c; o.det = det;
    o.conicA = c / det; o.conicB = -b / det; o.conicC = a / det;
    o.radius = radius;
    o.x0 = x0; o.y0 = y0; o.x1 = x1; o.y1 = y1;
    return true;
}

// Pixel bounds [lo, hi] on one axis that a splat can reach with alpha >= 1/255, cut to the pixels
// of its 8x8-tile rectangle (render.cpp:166-171) and to the image.
__device__ __forceinline__ unsigned axis_bounds(float centre, float cov, float tau, int radius, int size) {
    const int tiles8 = (size + kCpuTile - 1) / kCpuTile;
    const int t0 = max(0, (int)(centre - radius) / kCpuTile);
    const int t1 = min(tiles8 - 1, (int)(centre + radius) / kCpuTile);
    int lo = t0 * kCpuTile, hi = min(t1 * kCpuTile + kCpuTile - 1, size - 1);
    if (tau >= 0.f) {
        const float h = sqrt_approx(2.0f * tau * cov) * 1.001f + 0.05f;
        const float flo = fminf(fmaxf(ceilf(centre - h - 0.5f), -1.0f), (float)size);
        const float fhi = fminf(fmaxf(floorf(centre + h - 0.5f), -1.0f), (float)size);
        lo = max(lo, (int)flo);
        hi = min(hi, (int)fhi);
    } else {
        lo = 1;
        hi = 0;
    }
    if (lo > hi) {
        lo = 1;
        hi = 0;
    }
    return pack_i16x2(lo, hi);
}

constexpr int kMaxStagedViews = 64;  // cameras of a scene's views kept in shared memory
constexpr int kPreThreads = 256;
constexpr int kPreWarps = kPreThreads / 32;
constexpr int kPreGroups = 1;  // groups of 32 Gaussians each warp tests (2 and 4 measured slower)
constexpr int kPreGaussians = kPreThreads * kPreGroups;  // Gaussians per CTA

// The projection of one entry that passed the early test, by any lane of the warp (the Gaussian's
// activated position / opacity and covariance come from its owner lane through shared memory):
// the exact test, then colour, blend record, rectangle and depth key, all indexed by entry.
template <int D, bool kDebug, class Src>
__device__ __forceinline__ void project_entry(const Src& src, int64_t i, const float4 pg, const Cov3& cov,
                                              const CamParams& cam, unsigned e, int tile_w,
                                              int tile_h, SplatRecord* __restrict__ rec,
                                              unsigned long long* __restrict__ rect16, unsigned* __restrict__ depth_key,
                                              const DebugProjection& dbg, const PassCounts& counts,
                                              unsigned count_blocks) {
    Projected p;
    if (!project(pg, cov, cam, tile_w, tile_h, p)) {
        depth_key[e] = kCulledKey;
        if (kDebug) dbg.tiles_touched[e] = 0;
        return;
    }
    // log2(opacity) for the record. alpha = min(0.99, opacity * exp(power)) >= 1/255 needs
    // power >= -ln(255 opacity) = -ln2 (log2(opacity) + log2(255)): a margin of 1% + 0.02 on that
    // bound keeps the cut conservative under rounding. A NaN opacity gives alpha 0.99 everywhere
    // (as fminf does in the reference), so no cut then.
    const float log2_opacity = lg2_approx(pg.w);
    float tau = (log2_opacity + 7.99435343685885793f) * (0.69314718055994530942f * 1.01f) + 0.02f;
    if (isnan(tau)) tau = 3.0e38f;
    // Colour along the unit direction from the camera centre, normalised with an IEEE square root
    // and three IEEE divisions as gpu_render.cu:137-139 does, so the colour is bit-identical to the
    // reference kernel's too (a few instructions per visible entry).
    float3 d = make_float3(pg.x - cam.eye[0], pg.y - cam.eye[1], pg.z - cam.eye[2]);
    const float len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
    const float3 rgb = sh_color_upto<D>(cam.shDegree, src.sh + i * src.sh_planes, d.x / len, d.y / len, d.z / len);

    const unsigned bx = axis_bounds(p.u, p.a, tau, p.radius, cam.width);
    const unsigned by = axis_bounds(p.v, p.c, tau, p.radius, cam.height);
    constexpr float kHalfLog2e = -0.72134752044448170368f;  // -log2(e) / 2
    constexpr float kLog2e = -1.44269504088896340736f;      // -log2(e)
    SplatRecord r;
    r.r0 = make_float4(p.u, p.v, kHalfLog2e * p.conicA, kLog2e * p.conicB);
    r.r1 = make_float4(kHalfLog2e * p.conicC, log2_opacity, rgb.x, rgb.y);
    r.r2 = make_float4(rgb.z, __uint_as_float(bx), __uint_as_float(by), __uint_as_float(0xFFFFFFFFu));
    if (std::is_same<Src, RawParams>::value) r.r2.w = __uint_as_float(record_block_bits(r));  // training
    rec[e] = r;
    rect16[e] = static_cast<unsigned long long>(p.x0) | (static_cast<unsigned long long>(p.y0) << 16) |
                (static_cast<unsigned long long>(p.x1) << 32) | (static_cast<unsigned long long>(p.y1) << 48);
    // The depth key (the depth's bits less kDepthKeyBase: visible depths are >= 0.2, so the sign
    // bit of kCulledKey never collides). The first depth pass compacts the visible entries.
    const unsigned key = __float_as_uint(p.depth) - kDepthKeyBase;
    depth_key[e] = key;
    if (counts.counts) count_key(counts, count_blocks, e, key);
    if (kDebug) {
        dbg.uv[e] = make_float2(p.u, p.v);
        dbg.conic_opacity[e] = make_float4(p.conicA, p.conicB, p.conicC, pg.w);
        dbg.depth[e] = p.depth;
        dbg.rgb[3 * e + 0] = rgb.x;
        dbg.rgb[3 * e + 1] = rgb.y;
        dbg.rgb[3 * e + 2] = rgb.z;
        dbg.rect[e] = make_uint4(p.x0, p.y0, p.x1, p.y1);
        dbg.tiles_touched[e] = static_cast<unsigned>((p.x1 - p.x0 + 1) * (p.y1 - p.y0 + 1));
    }
}

// Every (view, Gaussian) entry of a scene's views. Each warp owns kPreGroups x 32 Gaussians. For
// each group it reads the 32 Gaussians once (one per lane) and runs the early screen test of
// project() for every view of the scene; entries that fail it are written culled at once, the
// others are queued in shared memory as (Gaussian, view) items. Whenever 32 items are queued the
// whole warp projects them, one per lane (project_entry), so the expensive part -- the exact
// test, the SH colour, the record -- runs without idle lanes however the visible entries are
// spread over the Gaussians and views (a quarter of the entries of a 64-view batch are visible,
// scattered over every warp). Outputs are indexed by entry, so the queue order does not matter.
// The kernel is latency-bound, so it is held to 64 registers for four CTAs per SM. Measured: the
// 64-view batch 10.2 -> 9.5 ms per batch, the 740k view 0.350 -> 0.344 ms per frame.
template <int D, bool kDebug, class Src>
__global__ void __launch_bounds__(kPreThreads, 4) preprocess_kernel(const BatchScene<Src>* __restrict__ scenes,
                                                                    unsigned n_scenes, const ViewInfo* __restrict__ views,
                                                                    int tile_w, int tile_h, SplatRecord* __restrict__ rec,
                                                                    unsigned long long* __restrict__ rect16,
                                                                    unsigned* __restrict__ depth_key, DebugProjection dbg,
                                                                    PassCounts counts, unsigned entries) {
    chain_entry();
    __shared__ CamParams s_cam[kMaxStagedViews];
    __shared__ unsigned s_ebase[kMaxStagedViews];
    __shared__ unsigned s_queue[kPreWarps][64];
    __shared__ float4 s_pos[kPreWarps][32 * kPreGroups];     // activated position + opacity
    __shared__ float4 s_cova[kPreWarps][32 * kPreGroups];    // s00, s01, s02, s11
    __shared__ float4 s_covb[kPreWarps][32 * kPreGroups];    // s12, s22, trace, splat scale
    __shared__ unsigned s_scene;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        unsigned sidx = 0;
        for (unsigned k = 1; k < n_scenes; ++k)
            if (scenes[k].block_base <= blockIdx.x) sidx = k;
        s_scene = sidx;
    }
    __syncthreads();
    const BatchScene<Src> sc = scenes[s_scene];
    const unsigned nv = sc.view_end - sc.view_begin;
    const unsigned staged = min(nv, static_cast<unsigned>(kMaxStagedViews));
    for (unsigned k = tid; k < staged * (sizeof(CamParams) / 4); k += kPreThreads)
        reinterpret_cast<unsigned*>(s_cam)[k] =
            reinterpret_cast<const unsigned*>(&views[sc.view_begin + k / (sizeof(CamParams) / 4)].cam)[k % (sizeof(CamParams) / 4)];
    for (unsigned k = tid; k < staged; k += kPreThreads) s_ebase[k] = views[sc.view_begin + k].entry_base;
    __syncthreads();
    const unsigned count_blocks = (entries + kSortBlockItems - 1) / kSortBlockItems;
    const int64_t warp_base =
        static_cast<int64_t>(blockIdx.x - sc.block_base) * kPreGaussians + static_cast<int64_t>(warp) * 32 * kPreGroups;
    unsigned* queue = s_queue[warp];
    const unsigned lt = lanemask_lt();
    unsigned queued = 0;  // items in the warp's queue (warp-uniform)

    for (int g = 0; g < kPreGroups; ++g) {
        const int64_t i = warp_base + g * 32 + lane;
        const bool have = i < sc.src.n;
        float4 pg = make_float4(0.f, 0.f, 0.f, 0.f);
        Cov3 cov{};
        float cov_scale = 0.f;
        bool prefetched = false;
        if (have) {
            float4 sg, q;
            sc.src.load(i, pg, sg, q);
            cov_scale = nv > 0 ? s_cam[0].splatScale : 1.0f;
            covariance(sg, q, cov_scale, cov);
        }
        s_pos[warp][g * 32 + lane] = pg;
        s_cova[warp][g * 32 + lane] = make_float4(cov.s00, cov.s01, cov.s02, cov.s11);
        s_covb[warp][g * 32 + lane] = make_float4(cov.s12, cov.s22, cov.trace, cov_scale);
        for (unsigned vk = 0; vk < nv;) {
            // Test views until the queue holds a warp's worth of items (or the views run out).
            for (; vk < nv && queued < 32; ++vk) {
                const CamParams& cam = vk < kMaxStagedViews ? s_cam[vk] : views[sc.view_begin + vk].cam;
                bool pass = false;
                if (have) {
                    if (cam.splatScale != cov_scale) {
                        float4 pg2, sg, q;
                        sc.src.load(i, pg2, sg, q);
                        cov_scale = cam.splatScale;
                        covariance(sg, q, cov_scale, cov);
                    }
                    pass = early_visible(pg, cov, cam);
                    if (!pass) {
                        const unsigned e = (vk < kMaxStagedViews ? s_ebase[vk] : views[sc.view_begin + vk].entry_base) +
                                           static_cast<unsigned>(i);
                        depth_key[e] = kCulledKey;
                        if (kDebug) dbg.tiles_touched[e] = 0;
                    } else if (!prefetched) {
                        // Its SH words start towards L2 now; the warp projects it later.
                        const char* shp = reinterpret_cast<const char*>(sc.src.sh + i * sc.src.sh_planes);
                        for (int off = 0; off < sc.src.sh_planes * 16; off += 128)
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(shp + off));
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(shp + sc.src.sh_planes * 16 - 1));
                        prefetched = true;
                    }
                }
                const unsigned m = __ballot_sync(0xFFFFFFFFu, pass);
                if (pass) queue[queued + __popc(m & lt)] = static_cast<unsigned>(g * 32 + lane) | (vk << 8);
                queued += __popc(m);
            }
            __syncwarp();
            // A full warp of items (or, after the last group, what is left) is projected.
            const bool last = g == kPreGroups - 1 && vk == nv;
            while (queued >= 32 || (last && queued > 0)) {
                const unsigned take = min(queued, 32u);
                if (static_cast<unsigned>(lane) < take) {
                    const unsigned item = queue[queued - take + lane];
                    const unsigned ivk = item >> 8;
                    const int64_t gi = warp_base + (item & 0xFFu);
                    const CamParams& cam = ivk < kMaxStagedViews ? s_cam[ivk] : views[sc.view_begin + ivk].cam;
                    const unsigned e = (ivk < kMaxStagedViews ? s_ebase[ivk] : views[sc.view_begin + ivk].entry_base) +
                                       static_cast<unsigned>(gi);
                    const float4 ip = s_pos[warp][item & 0xFFu];
                    const float4 ca = s_cova[warp][item & 0xFFu], cb = s_covb[warp][item & 0xFFu];
                    Cov3 icov{ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z};
                    if (cam.splatScale != cb.w) {  // a view with another splat scale than the first
                        float4 pg2, sg, q;
                        sc.src.load(gi, pg2, sg, q);
                        covariance(sg, q, cam.splatScale, icov);
                    }
                    project_entry<D, kDebug>(sc.src, gi, ip, icov, cam, e, tile_w, tile_h, rec, rect16, depth_key, dbg,
                                             counts, count_blocks);
                }
                queued -= take;
                __syncwarp();
            }
        }
    }
}

}  // namespace

unsigned preprocess_gaussians_per_block() { return kPreGaussians; }

namespace {

template <bool kDebug, class Src>
void launch_preprocess_t(const BatchScene<Src>* scenes, unsigned n_scenes, unsigned blocks, const ViewInfo* views,
                         int sh_degree, int tile_w, int tile_h, SplatRecord* rec,
                         unsigned long long* rect16, unsigned* depth_key, const DebugProjection& dbg,
                         const PassCounts& counts, unsigned entries, cudaStream_t stream) {
    if (blocks == 0) return;
    const dim3 grid(blocks), block(kPreThreads);
    switch (sh_degree) {
        case 0: launch_chained(preprocess_kernel<0, kDebug, Src>, grid, block, stream, scenes, n_scenes, views, tile_w,
                               tile_h, rec, rect16, depth_key, dbg, counts, entries); break;
        case 1: launch_chained(preprocess_kernel<1, kDebug, Src>, grid, block, stream, scenes, n_scenes, views, tile_w,
                               tile_h, rec, rect16, depth_key, dbg, counts, entries); break;
        case 2: launch_chained(preprocess_kernel<2, kDebug, Src>, grid, block, stream, scenes, n_scenes, views, tile_w,
                               tile_h, rec, rect16, depth_key, dbg, counts, entries); break;
        default: launch_chained(preprocess_kernel<3, kDebug, Src>, grid, block, stream, scenes, n_scenes, views, tile_w,
                                tile_h, rec, rect16, depth_key, dbg, counts, entries); break;
    }
}

}  // namespace

void launch_preprocess(const BatchScene<SceneView>* scenes, unsigned n_scenes, unsigned blocks, const ViewInfo* views,
                       int sh_degree, int tile_w, int tile_h, SplatRecord* rec, unsigned long long* rect16,
                       unsigned* depth_key, const DebugProjection* dbg, const PassCounts& counts, unsigned entries,
                       cudaStream_t stream) {
    if (dbg)
        launch_preprocess_t<true>(scenes, n_scenes, blocks, views, sh_degree, tile_w, tile_h, rec, rect16,
                                  depth_key, *dbg, counts, entries, stream);
    else
        launch_preprocess_t<false>(scenes, n_scenes, blocks, views, sh_degree, tile_w, tile_h, rec, rect16,
                                   depth_key, DebugProjection{}, counts, entries, stream);
}

void launch_preprocess_raw(const BatchScene<RawParams>* scenes, unsigned n_scenes, unsigned blocks,
                           const ViewInfo* views, int sh_degree, int tile_w, int tile_h, SplatRecord* rec,
                           unsigned long long* rect16, unsigned* depth_key, const PassCounts& counts,
                           unsigned entries, cudaStream_t stream) {
    launch_preprocess_t<false>(scenes, n_scenes, blocks, views, sh_degree, tile_w, tile_h, rec, rect16,
                               depth_key, DebugProjection{}, counts, entries, stream);
}

}  // namespace ab2
