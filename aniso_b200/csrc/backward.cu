// The adjoint of the rasterizer (no counterpart in the reference, which has no backward pass; the
// forward it differentiates is render.cpp:39-104 / 195-220 on the GPU path's lists).
//
// blend_backward: one block per tile of a batch, the forward's pixel layout (8x8 per warp, two
//   pixels per lane). Each pixel walks its tile list back to front from its last applied
//   splat, replaying the forward's alpha tests bit for bit (same record, same exponent code) and
//   recovering the transmittance in front of each splat (T_j = T_{j+1} / (1 - a_j));
//   nothing per pixel is stored but the final T and the last contributor. Per splat, the gradient
//   with respect to its nine record parameters (u, v, A2, B2, C2, L, r, g, b) is reduced over the
//   warp (12 shuffles for the 9 values; skipped when no pixel of the warp took the splat), summed
//   over the warps in a fixed order, and written
//   to the pair's slot in the depth-ordered pair list -- no atomics, so the result does not depend
//   on scheduling.
// gauss_backward: one launch per view over the Gaussians visible in it (compacted first, so no lane
//   idles on a culled one); each sums its pairs' slots (contiguous, in a fixed order), applies the
//   chain rule through the record
//   (conic, log2 opacity, SH colour), the EWA projection (2D covariance, clamped Jacobian, camera
//   transform), the 3D covariance M M^T with M = R(q) diag(s), and the activations (exp, sigmoid,
//   quaternion normalisation) to the 59 raw parameters, and adds them to the scene's gradients.
//   Views are launched one after another, so the sum over views also runs in a fixed order.
#include "common.cuh"
#include "kernels.h"

namespace ab2 {
namespace {

constexpr int kBatch = 128;
constexpr int kG = 9;
constexpr float kLn2 = 0.69314718055994530942f;
constexpr float kHalfLog2e = -0.72134752044448170368f;  // A2 = kHalfLog2e * A, C2 likewise
constexpr float kNegLog2e = -1.44269504088896340736f;   // B2 = kNegLog2e * B

// Sums v[0..8] over the warp; afterwards the even lanes hold one sum each: value index *k (-1 for
// none). 12 shuffles: each step hands half of the values to the partner lane.
__device__ __forceinline__ float warp_reduce9(const float v[kG], int lane, int& k) {
    const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4, b2 = lane & 2;
    float a[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const float lo = v[i], hi = i + 5 < kG ? v[i + 5] : 0.f;
        a[i] = (b16 ? hi : lo) + __shfl_xor_sync(0xFFFFFFFFu, b16 ? lo : hi, 16);
    }
    float b[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float lo = a[i], hi = i + 3 < 5 ? a[i + 3] : 0.f;
        b[i] = (b8 ? hi : lo) + __shfl_xor_sync(0xFFFFFFFFu, b8 ? lo : hi, 8);
    }
    float c[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float lo = b[i], hi = i + 2 < 3 ? b[i + 2] : 0.f;
        c[i] = (b4 ? hi : lo) + __shfl_xor_sync(0xFFFFFFFFu, b4 ? lo : hi, 4);
    }
    const float d = (b2 ? c[1] : c[0]) + __shfl_xor_sync(0xFFFFFFFFu, b2 ? c[0] : c[1], 2);
    const float e = d + __shfl_xor_sync(0xFFFFFFFFu, d, 1);
    const int ci = b2 ? 1 : 0;
    const int bi = ci + (b4 ? 2 : 0);
    const int ai = bi + (b8 ? 3 : 0);
    const int vi = ai + (b16 ? 5 : 0);
    k = ((lane & 1) == 0 && bi < 3 && ai < 5 && vi < kG) ? vi : -1;
    return e;
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The backward state of a lane's two pixels, as pairs (x: the left pixel, y: the right one).
struct PixelState2 {
    float2 T;                 // transmittance behind the splat being visited (starts at the final T)
    float2 ar, ag, ab;        // colour accumulated from the splats behind it
    float2 gr, gg, gb;        // dL/dC of the pixel
    unsigned last0, last1;    // list position one past each pixel's last applied splat
};

// One adjoint step for splat j (list position pos) at both pixels of the lane, each pair of
// operations one packed FP32x2 instruction (sm_100; per component the rounding of the scalar
// form). A pixel the splat does not apply to in the forward (behind its last applied splat, or
// failing the alpha tests, replayed with the forward's exponent bits) takes alpha = 0, which
// leaves its state unchanged (1/(1 - 0) = 1, w = 0) and adds zeros. G[k] receives the two pixels'
// gradients of the nine record parameters (u, v, A2, B2, C2, L, r, g, b); the caller adds the
// halves. Returns whether the splat applied to either pixel. 1/(1 - alpha) is the approximate
// reciprocal (relative error below 2^-22): the recovered transmittance drifts by that much per
// splat, far inside the gradients' tolerance. Packing the two pixels took the fwd+bwd of the
// 2.2M-Gaussian view from 1.95 to 1.86 ms.

__device__ __forceinline__ bool pixel_step2(PixelState2& s, unsigned pos, float2 p, float2 dx, float dy,
                                            const float4& r0, const float4& r1, float rb, float2 G[kG]) {
    const float e0 = ex2_approx(p.x), e1 = ex2_approx(p.y);
    const float a0 = fminf(0.99f, e0), a1 = fminf(0.99f, e1);
    const bool v0 = pos < s.last0 && !(p.x > r1.y) && a0 >= 1.0f / 255.0f;
    const bool v1 = pos < s.last1 && !(p.y > r1.y) && a1 >= 1.0f / 255.0f;
    if (!(v0 || v1)) return false;
    const float2 alpha = make_float2(v0 ? a0 : 0.f, v1 ? a1 : 0.f);
    const float2 om = __fadd2_rn(make_float2(1.0f, 1.0f), make_float2(-alpha.x, -alpha.y));
    const float2 inv_om = make_float2(rcp_approx(om.x), rcp_approx(om.y));
    const float2 Tb = __fmul2_rn(s.T, inv_om);  // transmittance in front of the splat
    const float2 w = __fmul2_rn(alpha, Tb);
    G[6] = __fmul2_rn(s.gr, w);
    G[7] = __fmul2_rn(s.gg, w);
    G[8] = __fmul2_rn(s.gb, w);
    const float2 tr = __ffma2_rn(make_float2(r1.z, r1.z), Tb, __fmul2_rn(make_float2(-s.ar.x, -s.ar.y), inv_om));
    const float2 tg = __ffma2_rn(make_float2(r1.w, r1.w), Tb, __fmul2_rn(make_float2(-s.ag.x, -s.ag.y), inv_om));
    const float2 tb = __ffma2_rn(make_float2(rb, rb), Tb, __fmul2_rn(make_float2(-s.ab.x, -s.ab.y), inv_om));
    const float2 dalpha = __ffma2_rn(s.gb, tb, __ffma2_rn(s.gg, tg, __fmul2_rn(s.gr, tr)));
    s.ar = __ffma2_rn(make_float2(r1.z, r1.z), w, s.ar);
    s.ag = __ffma2_rn(make_float2(r1.w, r1.w), w, s.ag);
    s.ab = __ffma2_rn(make_float2(rb, rb), w, s.ab);
    s.T = Tb;
    // d alpha / d p = alpha ln 2 unless clamped (alpha = 0 for a pixel that takes no part)
    float2 dp = __fmul2_rn(__fmul2_rn(dalpha, alpha), make_float2(kLn2, kLn2));
    if (e0 > 0.99f) dp.x = 0.f;
    if (e1 > 0.99f) dp.y = 0.f;
    const float2 ndp = make_float2(-dp.x, -dp.y);
    const float bdy = r0.w * dy, cdy2 = 2.0f * r1.x * dy;
    G[0] = __fmul2_rn(ndp, __ffma2_rn(make_float2(2.0f * r0.z, 2.0f * r0.z), dx, make_float2(bdy, bdy)));
    G[1] = __fmul2_rn(ndp, __ffma2_rn(make_float2(r0.w, r0.w), dx, make_float2(cdy2, cdy2)));
    const float2 dpdx = __fmul2_rn(dp, dx);
    G[2] = __fmul2_rn(dpdx, dx);
    G[3] = __fmul2_rn(dpdx, make_float2(dy, dy));
    G[4] = __fmul2_rn(dp, make_float2(dy * dy, dy * dy));
    G[5] = dp;
    return true;
}

template <int TW, int TH>
__global__ void __launch_bounds__(TW * TH / 2) blend_backward_kernel(BackwardIn in, float* __restrict__ grad_pair) {
    chain_entry();
    constexpr int kThreads = TW * TH / 2;
    constexpr int kWarps = kThreads / 32;
    constexpr int kWarpsX = TW / 8;
    __shared__ float4 s_r0[kBatch];
    __shared__ float4 s_r1[kBatch];
    __shared__ float s_b[kBatch];
    __shared__ unsigned s_pos[kBatch];
    __shared__ unsigned char s_mask[kBatch];
    __shared__ unsigned s_hit[kBatch];
    __shared__ float s_grad[kWarps][kBatch][kG];
    __shared__ unsigned s_maxlast;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned gtile = blockIdx.x;
    const unsigned v = find_segment(in.tables.tile_base, in.tables.n_views, gtile);
    const ViewInfo& vi = in.views[v];
    const unsigned local = gtile - vi.tile_base;
    const int tx = static_cast<int>(local % vi.cam.tilesX), ty = static_cast<int>(local / vi.cam.tilesX);
    const int ox = tx * TW, oy = ty * TH;
    const int x0 = ox + (warp % kWarpsX) * 8 + 2 * (lane & 3), y = oy + (warp / kWarpsX) * 8 + (lane >> 2);
    const int width = vi.cam.width, height = vi.cam.height;
    const float px0 = x0 + 0.5f, py = y + 0.5f;
    const uint2 range = (in.ctrl->flags & kFlagOverflow) ? make_uint2(0, 0) : in.ranges[gtile];

    PixelState2 st;
    st.T = make_float2(1.f, 1.f);
    st.ar = st.ag = st.ab = st.gr = st.gg = st.gb = make_float2(0.f, 0.f);
    st.last0 = st.last1 = range.x;
    if (x0 < width && y < height) {
        const size_t p = static_cast<size_t>(y) * width + x0;
        st.T.x = vi.t_final[p];
        st.last0 = vi.n_contrib[p];
        st.gr.x = vi.grad_img[3 * p];
        st.gg.x = vi.grad_img[3 * p + 1];
        st.gb.x = vi.grad_img[3 * p + 2];
    }
    if (x0 + 1 < width && y < height) {
        const size_t p = static_cast<size_t>(y) * width + x0 + 1;
        st.T.y = vi.t_final[p];
        st.last1 = vi.n_contrib[p];
        st.gr.y = vi.grad_img[3 * p];
        st.gg.y = vi.grad_img[3 * p + 1];
        st.gb.y = vi.grad_img[3 * p + 2];
    }
    if (tid == 0) s_maxlast = range.x;
    __syncthreads();
    const unsigned mylast = max(st.last0, st.last1);
    const unsigned wlast = __reduce_max_sync(0xFFFFFFFFu, mylast);
    if (lane == 0) atomicMax(&s_maxlast, wlast);
    __syncthreads();
    const unsigned end = s_maxlast;

    // Pairs behind every pixel's last applied splat get zero gradient.
    for (unsigned q = end + tid; q < range.y; q += kThreads) {
        const unsigned g = in.vals[q];
        const unsigned j = in.rank[g];
        const unsigned long long rc = in.rect_sorted[j];
        const unsigned rx0 = rc & 0xFFFFu, ry0 = (rc >> 16) & 0xFFFFu, rx1 = (rc >> 32) & 0xFFFFu;
        float* out = grad_pair +
                     static_cast<size_t>(in.offs[j] + (static_cast<unsigned>(ty) - ry0) * (rx1 - rx0 + 1) +
                                         (static_cast<unsigned>(tx) - rx0)) * kG;
#pragma unroll
        for (int k = 0; k < kG; ++k) out[k] = 0.f;
    }

    for (unsigned top = end; top > range.x;) {
        const unsigned start = top > range.x + kBatch ? top - kBatch : range.x;
        const unsigned cnt = top - start;
        // Stage the batch [start, top): records, warp masks and each pair's slot in the
        // depth-ordered pair list (the slot of (Gaussian g, tile t) is offs[rank[g]] plus t's
        // row-major index in g's rectangle).
        for (unsigned slot = tid; slot < cnt; slot += kThreads) {
            const unsigned g = in.vals[start + slot];
            const SplatRecord r = in.rec[g];
            s_r0[slot] = r.r0;
            s_r1[slot] = r.r1;
            s_b[slot] = r.r2.x;
            // The forward's masks (the same function), so the adjoint walks exactly its splats.
            s_mask[slot] = static_cast<unsigned char>(staged_block_mask<TW, TH, true>(r, ox, oy));
            s_hit[slot] = 0;
            const unsigned j = in.rank[g];
            const unsigned long long rc = in.rect_sorted[j];
            const unsigned rx0 = rc & 0xFFFFu, ry0 = (rc >> 16) & 0xFFFFu, rx1 = (rc >> 32) & 0xFFFFu;
            s_pos[slot] = in.offs[j] + (static_cast<unsigned>(ty) - ry0) * (rx1 - rx0 + 1) + (static_cast<unsigned>(tx) - rx0);
        }
        __syncthreads();
        if (start < wlast) {  // some pixel of the warp applied a splat of this batch
            for (int c = static_cast<int>((cnt - 1) / 32); c >= 0; --c) {
                const unsigned idx = c * 32 + lane;
                unsigned bits = __ballot_sync(0xFFFFFFFFu, idx < cnt && ((s_mask[idx] >> warp) & 1u));
                while (bits) {
                    const int b = 31 - __clz(bits);
                    bits &= ~(1u << b);
                    const unsigned jj = c * 32 + b;
                    const unsigned pos = start + jj;
                    if (pos >= wlast) continue;  // behind every pixel's last applied splat
                    const float4 r0 = s_r0[jj];
                    const float4 r1 = s_r1[jj];
                    const float rb = s_b[jj];
                    const float dy = __fsub_rn(py, r0.y);
                    float2 dx;
                    const float2 pp = splat_exponents2(r0, r1, make_float2(px0, px0 + 1.0f), dy, dx);
                    float2 G[kG];
                    const bool any = pixel_step2(st, pos, pp, dx, dy, r0, r1, rb, G);
                    // No pixel of the warp took the splat: its share is zero, leave it out of the sum.
                    if (!__any_sync(0xFFFFFFFFu, any)) continue;
                    float g[kG];
#pragma unroll
                    for (int q = 0; q < kG; ++q) g[q] = any ? G[q].x + G[q].y : 0.f;
                    int k;
                    const float sum = warp_reduce9(g, lane, k);
                    if (k >= 0) s_grad[warp][jj][k] = sum;
                    if (lane == 0) atomicOr(&s_hit[jj], 1u << warp);
                }
            }
        }
        __syncthreads();
        // Fixed-order sum over the warps; every staged pair's slot is written.
        for (unsigned slot = tid; slot < cnt; slot += kThreads) {
            const unsigned hit = s_hit[slot];
            float acc[kG];
#pragma unroll
            for (int k = 0; k < kG; ++k) acc[k] = 0.f;
#pragma unroll
            for (int w = 0; w < kWarps; ++w)
                if (hit & (1u << w))
#pragma unroll
                    for (int k = 0; k < kG; ++k) acc[k] += s_grad[w][slot][k];
            float* out = grad_pair + static_cast<size_t>(s_pos[slot]) * kG;
#pragma unroll
            for (int k = 0; k < kG; ++k) out[k] = acc[k];
        }
        __syncthreads();
        top = start;
    }
}

// SH basis (sh.cpp:18-58 order) and its derivatives along x, y, z, for degree D.
// Adds one view's gradient to the caller's buffer. The add is rounded on its own (never fused with
// the product that formed v), so accumulating views here equals summing per-view gradients.
__device__ __forceinline__ void accumulate(float* p, float v) { *p = __fadd_rn(*p, v); }
// The same where the old value is known to be zero (the first view of a fresh gradient) and is not
// read: 0 + v rounds as the add would.
template <bool kFresh>
__device__ __forceinline__ void add_grad(float* p, float v) {
    *p = __fadd_rn(kFresh ? 0.f : *p, v);
}

template <int D>
__device__ __forceinline__ void sh_basis(float x, float y, float z, float b[16], float bx[16], float by[16],
                                         float bz[16]) {
    const float C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
    const float C20 = 1.0925484305920792f, C21 = -1.0925484305920792f, C22 = 0.31539156525252005f,
                C23 = -1.0925484305920792f, C24 = 0.5462742152960396f;
    const float C30 = -0.5900435899266435f, C31 = 2.890611442640554f, C32 = -0.4570457994644658f,
                C33 = 0.3731763325901154f, C34 = -0.4570457994644658f, C35 = 1.445305721320277f,
                C36 = -0.5900435899266435f;
#pragma unroll
    for (int k = 0; k < 16; ++k) b[k] = bx[k] = by[k] = bz[k] = 0.f;
    b[0] = C0;
    if (D >= 1) {
        b[1] = -C1 * y; by[1] = -C1;
        b[2] = C1 * z; bz[2] = C1;
        b[3] = -C1 * x; bx[3] = -C1;
    }
    if (D >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        b[4] = C20 * x * y; bx[4] = C20 * y; by[4] = C20 * x;
        b[5] = C21 * y * z; by[5] = C21 * z; bz[5] = C21 * y;
        b[6] = C22 * (2 * zz - xx - yy); bx[6] = -2 * C22 * x; by[6] = -2 * C22 * y; bz[6] = 4 * C22 * z;
        b[7] = C23 * x * z; bx[7] = C23 * z; bz[7] = C23 * x;
        b[8] = C24 * (xx - yy); bx[8] = 2 * C24 * x; by[8] = -2 * C24 * y;
        if (D >= 3) {
            b[9] = C30 * y * (3 * xx - yy); bx[9] = C30 * 6 * x * y; by[9] = C30 * (3 * xx - 3 * yy);
            b[10] = C31 * x * y * z; bx[10] = C31 * y * z; by[10] = C31 * x * z; bz[10] = C31 * x * y;
            b[11] = C32 * y * (4 * zz - xx - yy); bx[11] = -2 * C32 * x * y; by[11] = C32 * (4 * zz - xx - 3 * yy);
            bz[11] = 8 * C32 * y * z;
            b[12] = C33 * z * (2 * zz - 3 * xx - 3 * yy); bx[12] = -6 * C33 * x * z; by[12] = -6 * C33 * y * z;
            bz[12] = C33 * (6 * zz - 3 * xx - 3 * yy);
            b[13] = C34 * x * (4 * zz - xx - yy); bx[13] = C34 * (4 * zz - 3 * xx - yy); by[13] = -2 * C34 * x * y;
            bz[13] = 8 * C34 * x * z;
            b[14] = C35 * z * (xx - yy); bx[14] = 2 * C35 * x * z; by[14] = -2 * C35 * y * z; bz[14] = C35 * (xx - yy);
            b[15] = C36 * x * (xx - 3 * yy); bx[15] = C36 * (3 * xx - 3 * yy); by[15] = -6 * C36 * x * y;
        }
    }
}

constexpr int kListItems = 4;  // entries per thread of the visible-list compaction

// The Gaussians of one view that are visible in it, appended in any order: the adjoint of each is
// independent of where it sits in the list, so the order does not change any result.
__global__ void __launch_bounds__(256) visible_list_kernel(int64_t n, unsigned entry_base,
                                                           const unsigned* __restrict__ depth_key,
                                                           unsigned* __restrict__ list, unsigned* counter) {
    chain_entry();
    __shared__ unsigned s_tmp[8];
    __shared__ unsigned s_base;
    const int64_t i0 = static_cast<int64_t>(blockIdx.x) * (256 * kListItems) + threadIdx.x;
    bool vis[kListItems];
    unsigned mine = 0;
#pragma unroll
    for (int k = 0; k < kListItems; ++k) {
        const int64_t i = i0 + k * 256;
        vis[k] = i < n && depth_key[entry_base + static_cast<unsigned>(i)] != kCulledKey;
        mine += vis[k];
    }
    // One atomic per CTA on the shared counter (one per warp contended on it for ~50 us at 2.2M).
    unsigned total;
    unsigned at = block_excl_scan<256>(mine, s_tmp, total);
    if (threadIdx.x == 0) s_base = total ? atomicAdd(counter, total) : 0u;
    __syncthreads();
    at += s_base;
#pragma unroll
    for (int k = 0; k < kListItems; ++k)
        if (vis[k]) list[at++] = static_cast<unsigned>(i0 + k * 256);
}

// The view's camera, its scene's raw tensors and gradient buffers come from the frame's device
// tables (copied into shared memory by each CTA), not from kernel arguments, so a recorded CUDA graph
// of the backward stays valid when the parameters, gradients or cameras move between replays.
template <typename T>
__device__ __forceinline__ void copy_words(T& dst, const T& src) {
    static_assert(sizeof(T) % 4 == 0, "copied as 32-bit words");
    if (threadIdx.x < sizeof(T) / 4)
        reinterpret_cast<unsigned*>(&dst)[threadIdx.x] = reinterpret_cast<const unsigned*>(&src)[threadIdx.x];
}

// Held to 128 registers (four CTAs per SM): the kernel waits on memory, and the extra warps
// measured faster where it runs many times per step (the 8-scene training batch: 27.0 -> 25.2 ms a
// step; 102 registers spilled and was no faster; the adjoint blend held to 64 was slower).
template <int D, bool kFresh>
__global__ void __launch_bounds__(128, 4) gauss_backward_kernel(const BatchScene<RawParams>* __restrict__ scenes,
                                                             unsigned scene, const ViewInfo* __restrict__ views,
                                                             unsigned view, const RawGrads* __restrict__ grads_table,
                                                             const Ctrl* ctrl, const unsigned* __restrict__ list,
                                                             const unsigned* __restrict__ list_count,
                                                             const unsigned* __restrict__ rank,
                                                             const unsigned* __restrict__ offs,
                                                             const unsigned long long* __restrict__ rect_sorted,
                                                             const float* __restrict__ grad_pair) {
    chain_entry();
    __shared__ CamParams s_cam;
    __shared__ RawParams s_raw;
    __shared__ RawGrads s_out;
    __shared__ unsigned s_entry_base;
    copy_words(s_cam, views[view].cam);
    copy_words(s_raw, scenes[scene].src);
    copy_words(s_out, grads_table[scene]);
    if (threadIdx.x == 0) s_entry_base = views[view].entry_base;
    __syncthreads();
    const CamParams& cam = s_cam;
    const RawParams raw = s_raw;
    const RawGrads out = s_out;
    const unsigned entry_base = s_entry_base;
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (ctrl->flags & kFlagOverflow) return;
    // The view's visible entries in entry order (the compacted list), so that a warp's reads of the
    // raw parameters and its gradient writes fall on neighbouring rows. (Walking the depth-sorted
    // list instead makes the pair-slot reads contiguous but every parameter row a random gather:
    // measured 0.22 -> 0.30 ms at 2.2M Gaussians.)
    const unsigned count = *list_count;
    if (blockIdx.x * blockDim.x >= count) return;
    const int lane = threadIdx.x & 31;
    // Past the end of the list: no Gaussian, but the lane still helps its warp.
    const bool active = t < count;
    const unsigned e = active ? entry_base + list[t] : entry_base;
    const int64_t i = e - entry_base;
    unsigned cnt = 0, off = 0;
    if (active) {
        const unsigned j = rank[e];
        const unsigned long long rc = rect_sorted[j];
        cnt = ((rc >> 32 & 0xFFFFu) - (rc & 0xFFFFu) + 1) * ((rc >> 48) - (rc >> 16 & 0xFFFFu) + 1);
        off = offs[j];
    }
    // The sum of the Gaussian's per-pair gradients, in a fixed order: a short list by its own lane,
    // slot after slot; a long one (the nearest splats own thousands of tiles) by the whole warp,
    // lane l taking slots l, l + 32, ..., then a fixed shuffle tree -- so one huge splat does not
    // hold its warp for thousands of serial loads.
    constexpr unsigned kSolo = 16;
    float g9[kG] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (cnt <= kSolo) {
        const float* gp = grad_pair + static_cast<size_t>(off) * kG;
        for (unsigned k = 0; k < cnt; ++k)
#pragma unroll
            for (int c = 0; c < kG; ++c) g9[c] += gp[k * kG + c];
    }
    for (unsigned big = __ballot_sync(0xFFFFFFFFu, cnt > kSolo); big; big &= big - 1) {
        const int src = __ffs(big) - 1;
        const unsigned bc = __shfl_sync(0xFFFFFFFFu, cnt, src), bo = __shfl_sync(0xFFFFFFFFu, off, src);
        const float* gp = grad_pair + static_cast<size_t>(bo) * kG;
        float part[kG] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (unsigned k = lane; k < bc; k += 32)
#pragma unroll
            for (int c = 0; c < kG; ++c) part[c] += gp[k * kG + c];
#pragma unroll
        for (int c = 0; c < kG; ++c) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part[c] += __shfl_down_sync(0xFFFFFFFFu, part[c], o);
            part[c] = __shfl_sync(0xFFFFFFFFu, part[c], 0);
            if (lane == src) g9[c] = part[c];
        }
    }
    if (!active) return;

    // ---- forward quantities (the preprocess kernel's, in the same order) ----
    float4 pg, sg, qn;
    raw.load(i, pg, sg, qn);
    const float4 qraw = raw.quats[i];
    const float qlen = sqrtf(qraw.x * qraw.x + qraw.y * qraw.y + qraw.z * qraw.z + qraw.w * qraw.w);
    const float gx = pg.x, gy = pg.y, gz = pg.z, o = pg.w;
    const float* W = cam.R;
    const float px = W[0] * gx + W[1] * gy + W[2] * gz + cam.t[0];
    const float py = W[3] * gx + W[4] * gy + W[5] * gz + cam.t[1];
    const float pz = W[6] * gx + W[7] * gy + W[8] * gz + cam.t[2];
    const float qw = qn.x, qx = qn.y, qy = qn.z, qz = qn.w;
    const float Rq[3][3] = {{1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)},
                            {2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx)},
                            {2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)}};
    const float s[3] = {sg.x * cam.splatScale, sg.y * cam.splatScale, sg.z * cam.splatScale};
    float M[3][3], S[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) M[r][c] = Rq[r][c] * s[c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) S[r][c] = M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2];
    const float limX = 1.3f * 0.5f * cam.width / cam.fx, limY = 1.3f * 0.5f * cam.height / cam.fy;
    const float rx = px / pz, ry = py / pz;
    const bool clx = rx < -limX || rx > limX, cly = ry < -limY || ry > limY;
    const float tx = fminf(limX, fmaxf(-limX, rx)) * pz;
    const float ty = fminf(limY, fmaxf(-limY, ry)) * pz;
    const float iz = 1.0f / pz, iz2 = iz * iz;
    const float J[2][3] = {{cam.fx * iz, 0.f, -cam.fx * tx * iz2}, {0.f, cam.fy * iz, -cam.fy * ty * iz2}};
    float T[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) T[r][c] = J[r][0] * W[c] + J[r][1] * W[3 + c] + J[r][2] * W[6 + c];
    float ST[2][3];  // S T_r^T for r = 0, 1 (S symmetric)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) ST[r][c] = S[c][0] * T[r][0] + S[c][1] * T[r][1] + S[c][2] * T[r][2];
    const float a = T[0][0] * ST[0][0] + T[0][1] * ST[0][1] + T[0][2] * ST[0][2] + 0.3f;
    const float b = T[1][0] * ST[0][0] + T[1][1] * ST[0][1] + T[1][2] * ST[0][2];
    const float c = T[1][0] * ST[1][0] + T[1][1] * ST[1][1] + T[1][2] * ST[1][2] + 0.3f;
    const float det = a * c - b * b;

    // ---- record parameters -> conic, opacity, colour ----
    const float gu = g9[0], gv = g9[1];
    // What densification reads (gsplat's DefaultStrategy): the screen-space gradient in NDC units
    // (x width/2, x height/2), its norm added over views, and the number of views that saw it.
    if (out.grad2d) {
        const float nu = gu * (0.5f * cam.width), nv = gv * (0.5f * cam.height);
        accumulate(&out.grad2d[i], sqrtf(nu * nu + nv * nv));
        accumulate(&out.visible[i], 1.0f);
    }
    const float gA = g9[2] * kHalfLog2e, gB = g9[3] * kNegLog2e, gC = g9[4] * kHalfLog2e;
    const float go = g9[5] / (o * kLn2);  // L = log2(o)
    float* gsh = out.sh + static_cast<size_t>(i) * raw.sh_planes * 4;
    float gm[3] = {0.f, 0.f, 0.f};
    {
        float3 d = make_float3(gx - cam.eye[0], gy - cam.eye[1], gz - cam.eye[2]);
        const float len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        const float ux = d.x / len, uy = d.y / len, uz = d.z / len;
        float bs[16], bxs[16], bys[16], bzs[16];
        sh_basis<D>(ux, uy, uz, bs, bxs, bys, bzs);
        constexpr int count = (D + 1) * (D + 1);
        const float4* shp = raw.sh + static_cast<size_t>(i) * raw.sh_planes;
        float shv[48];
#pragma unroll
        for (int k = 0; k < (count * 3 + 3) / 4; ++k) {
            const float4 f = shp[k];
            shv[4 * k] = f.x;
            if (4 * k + 1 < 48) shv[4 * k + 1] = f.y;
            if (4 * k + 2 < 48) shv[4 * k + 2] = f.z;
            if (4 * k + 3 < 48) shv[4 * k + 3] = f.w;
        }
        float gdir[3] = {0.f, 0.f, 0.f};
        const float grgb[3] = {g9[6], g9[7], g9[8]};
        float gc3[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            float pre = 0.5f;
#pragma unroll
            for (int k = 0; k < count; ++k) pre += bs[k] * shv[k * 3 + ch];
            const float gc = pre > 0.f ? grgb[ch] : 0.f;  // rgb = max(0, pre)
            gc3[ch] = gc;
#pragma unroll
            for (int k = 0; k < count; ++k) {
                gdir[0] += shv[k * 3 + ch] * bxs[k] * gc;
                gdir[1] += shv[k * 3 + ch] * bys[k] * gc;
                gdir[2] += shv[k * 3 + ch] * bzs[k] * gc;
            }
        }
        // d rgb / d sh = basis (x) gc, added 16 bytes at a time: float f of the row is coefficient f/3,
        // channel f%3 (each element still gets its own rounded add).
        constexpr int kFloats = count * 3;
        float4* gsh4 = reinterpret_cast<float4*>(gsh);
#pragma unroll
        for (int pl = 0; pl < (kFloats + 3) / 4; ++pl) {
            const float4 o = kFresh ? make_float4(0.f, 0.f, 0.f, 0.f) : gsh4[pl];
            float w[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int f = 4 * pl + e;
                if (f < kFloats) w[e] = __fadd_rn(w[e], bs[f / 3] * gc3[f % 3]);
            }
            gsh4[pl] = make_float4(w[0], w[1], w[2], w[3]);
        }
        const float dd = ux * gdir[0] + uy * gdir[1] + uz * gdir[2];
        gm[0] += (gdir[0] - ux * dd) / len;
        gm[1] += (gdir[1] - uy * dd) / len;
        gm[2] += (gdir[2] - uz * dd) / len;
    }
    add_grad<kFresh>(&out.logits[i], go * o * (1.0f - o));

    // ---- conic (A, B, C) = (c, -b, a) / det -> 2D covariance (a, b, c) ----
    const float id2 = 1.0f / (det * det);
    const float ga = (-c * c * gA + b * c * gB - b * b * gC) * id2;
    const float gb = (2.0f * b * c * gA - (det + 2.0f * b * b) * gB + 2.0f * a * b * gC) * id2;
    const float gc2 = (-b * b * gA + a * b * gB - a * a * gC) * id2;

    // ---- covariance = T S T^T + 0.3 I -> S, T ----
    float gS[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            gS[r][q] = ga * T[0][r] * T[0][q] + gb * T[0][r] * T[1][q] + gc2 * T[1][r] * T[1][q];
    float gT[2][3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        gT[0][q] = 2.0f * ga * ST[0][q] + gb * ST[1][q];
        gT[1][q] = gb * ST[0][q] + 2.0f * gc2 * ST[1][q];
    }
    // ---- T = J W -> J -> camera-space position ----
    float gJ[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) gJ[r][k] = gT[r][0] * W[3 * k] + gT[r][1] * W[3 * k + 1] + gT[r][2] * W[3 * k + 2];
    float gpx = gu * cam.fx * iz, gpy = gv * cam.fy * iz;
    float gpz = -(gu * cam.fx * px + gv * cam.fy * py) * iz2;
    gpz += -(gJ[0][0] * cam.fx + gJ[1][1] * cam.fy) * iz2;
    const float iz3 = iz2 * iz;
    if (!clx) {
        gpx += gJ[0][2] * (-cam.fx * iz2);
        gpz += gJ[0][2] * (2.0f * cam.fx * tx * iz3);
    } else {
        gpz += gJ[0][2] * (cam.fx * (tx * iz) * iz2);  // tx = lim pz: J02 = -fx lim / pz
    }
    if (!cly) {
        gpy += gJ[1][2] * (-cam.fy * iz2);
        gpz += gJ[1][2] * (2.0f * cam.fy * ty * iz3);
    } else {
        gpz += gJ[1][2] * (cam.fy * (ty * iz) * iz2);
    }
    // camera transform p_cam = W p + t
    gm[0] += W[0] * gpx + W[3] * gpy + W[6] * gpz;
    gm[1] += W[1] * gpx + W[4] * gpy + W[7] * gpz;
    gm[2] += W[2] * gpx + W[5] * gpy + W[8] * gpz;
    add_grad<kFresh>(&out.means[3 * i], gm[0]);
    add_grad<kFresh>(&out.means[3 * i + 1], gm[1]);
    add_grad<kFresh>(&out.means[3 * i + 2], gm[2]);

    // ---- S = M M^T -> M = R(q) diag(s) -> s, R(q) ----
    float gM[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            gM[r][k] = (gS[r][0] + gS[0][r]) * M[0][k] + (gS[r][1] + gS[1][r]) * M[1][k] + (gS[r][2] + gS[2][r]) * M[2][k];
    float gR[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float gs = 0.f;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            gR[r][k] = gM[r][k] * s[k];
            gs += gM[r][k] * Rq[r][k];
        }
        add_grad<kFresh>(&out.log_scales[3 * i + k], gs * s[k]);  // s = exp(log s) * splat_scale
    }
    const float gqw = 2.0f * (-qz * gR[0][1] + qy * gR[0][2] + qz * gR[1][0] - qx * gR[1][2] - qy * gR[2][0] + qx * gR[2][1]);
    const float gqx = 2.0f * (qy * gR[0][1] + qz * gR[0][2] + qy * gR[1][0] - 2.0f * qx * gR[1][1] - qw * gR[1][2] +
                              qz * gR[2][0] + qw * gR[2][1] - 2.0f * qx * gR[2][2]);
    const float gqy = 2.0f * (-2.0f * qy * gR[0][0] + qx * gR[0][1] + qw * gR[0][2] + qx * gR[1][0] + qz * gR[1][2] -
                              qw * gR[2][0] + qz * gR[2][1] - 2.0f * qy * gR[2][2]);
    const float gqz = 2.0f * (-2.0f * qz * gR[0][0] - qw * gR[0][1] + qx * gR[0][2] + qw * gR[1][0] -
                              2.0f * qz * gR[1][1] + qy * gR[1][2] + qx * gR[2][0] + qy * gR[2][1]);
    // q_n = q / |q|
    const float dq = qw * gqw + qx * gqx + qy * gqy + qz * gqz;
    const float il = qlen > 0 ? 1.0f / qlen : 0.f;
    float4* gq4 = reinterpret_cast<float4*>(out.quats) + i;
    const float4 oq = kFresh ? make_float4(0.f, 0.f, 0.f, 0.f) : *gq4;
    *gq4 = make_float4(__fadd_rn(oq.x, (gqw - qw * dq) * il), __fadd_rn(oq.y, (gqx - qx * dq) * il),
                       __fadd_rn(oq.z, (gqy - qy * dq) * il), __fadd_rn(oq.w, (gqz - qz * dq) * il));
}

}  // namespace

void launch_blend_backward(const BackwardIn& in, unsigned tiles, int tile_w, int tile_h, float* grad_pair,
                           cudaStream_t stream) {
    if (tiles == 0) return;
    if (tile_w == 8) launch_chained(blend_backward_kernel<8, 8>, dim3(tiles), dim3(32), stream, in, grad_pair);
    else if (tile_h == 32)
        launch_chained(blend_backward_kernel<16, 32>, dim3(tiles), dim3(256), stream, in, grad_pair);
    else launch_chained(blend_backward_kernel<16, 16>, dim3(tiles), dim3(128), stream, in, grad_pair);
}

namespace {
// The fresh and the accumulating gradient passes are separate instantiations: a run-time flag
// inside the kernel made the accumulating one (a batch's later views) slower.
template <bool kFresh>
void launch_gauss_backward_t(const GaussBackwardArgs& a, const Ctrl* ctrl, const unsigned* list,
                             const unsigned* list_count, const unsigned* rank, const unsigned* offs,
                             const unsigned long long* rect_sorted, const float* grad_pair, dim3 grid, dim3 block,
                             cudaStream_t stream) {
    switch (a.sh_degree) {
        case 0: launch_chained(gauss_backward_kernel<0, kFresh>, grid, block, stream, a.scenes, a.scene, a.views,
                               a.view, a.grads, ctrl, list, list_count, rank, offs, rect_sorted, grad_pair); break;
        case 1: launch_chained(gauss_backward_kernel<1, kFresh>, grid, block, stream, a.scenes, a.scene, a.views,
                               a.view, a.grads, ctrl, list, list_count, rank, offs, rect_sorted, grad_pair); break;
        case 2: launch_chained(gauss_backward_kernel<2, kFresh>, grid, block, stream, a.scenes, a.scene, a.views,
                               a.view, a.grads, ctrl, list, list_count, rank, offs, rect_sorted, grad_pair); break;
        default: launch_chained(gauss_backward_kernel<3, kFresh>, grid, block, stream, a.scenes, a.scene, a.views,
                                a.view, a.grads, ctrl, list, list_count, rank, offs, rect_sorted, grad_pair); break;
    }
}
}  // namespace

void launch_gauss_backward(const GaussBackwardArgs& a, const Ctrl* ctrl, const unsigned* depth_key,
                           const unsigned* rank, const unsigned* offs, const unsigned long long* rect_sorted,
                           const float* grad_pair, unsigned* list, unsigned* list_count, cudaStream_t stream) {
    const unsigned lblocks = static_cast<unsigned>((a.n + 256 * kListItems - 1) / (256 * kListItems));
    if (lblocks == 0) return;
    launch_chained(visible_list_kernel, dim3(lblocks), dim3(256), stream, a.n, a.entry_base, depth_key, list,
                   list_count);
    const dim3 grid(static_cast<unsigned>((a.n + 127) / 128)), block(128);
    if (a.fresh)
        launch_gauss_backward_t<true>(a, ctrl, list, list_count, rank, offs, rect_sorted, grad_pair, grid, block,
                                      stream);
    else
        launch_gauss_backward_t<false>(a, ctrl, list, list_count, rank, offs, rect_sorted, grad_pair, grid, block,
                                       stream);
}

}  // namespace ab2
