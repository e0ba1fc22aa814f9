// The C ABI (include/aniso_b200.h): scene upload, per-frame work buffers, the frame pipeline.
//
// A frame is a fixed, host-sync-free sequence of launches on one stream (capturable in a CUDA
// graph): frame_begin, preprocess (+compaction), 4 depth onesweep passes, pair scan, pair
// expansion, 1-4 tile onesweep passes, tile ranges, blend. Data-dependent sizes (visible count V, pair count P) stay
// on the device; grids are sized for capacity and surplus blocks exit at once. The reference
// instead reads P back mid-frame (gpu_render.cu:329) to size its buffers; here a frame whose P
// exceeds the pair capacity sets an overflow flag instead of writing, and the host grows the
// buffers and renders it again.
#include "aniso_b200.h"
#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
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

// Work buffers of one frame at a time, sized for N Gaussians and a pair capacity.
struct Arena {
    int64_t n = -1;
    unsigned pair_cap = 0;
    uint64_t frames = 0;
    DevBuf<SplatRecord> rec;
    DevBuf<unsigned long long> rect16;
    DevBuf<unsigned> depth_key;
    DevBuf<unsigned> vis_key[2], vis_idx[2];
    DevBuf<unsigned> pair_key[2], pair_val[2];
    DevBuf<unsigned> offs, rank, chunk_start;
    DevBuf<unsigned long long> rect_sorted;
    DevBuf<uint2> ranges;
    DevBuf<Ctrl> ctrl;
    DevBuf<unsigned long long> st_depth, st_dup, st_tile;
    DevBuf<uint8_t> image;

    unsigned depth_chunks() const { return chunks_of(static_cast<uint64_t>(std::max<int64_t>(n, 1)), onesweep_chunk_items()); }
    unsigned tile_chunks() const { return chunks_of(std::max(pair_cap, 1u), onesweep_chunk_items()); }
    // The vis_idx buffer that holds the depth-sorted visible list after the depth passes.
    static int sorted_buf() { return (kMaxPasses - 1) & 1; }

    int init(int64_t count, unsigned cap) {
        n = count;
        const size_t nn = static_cast<size_t>(std::max<int64_t>(count, 1));
        AB_TRY(rec.reserve(nn));
        AB_TRY(rect16.reserve(nn));
        AB_TRY(depth_key.reserve(nn));
        for (int k = 0; k < 2; ++k) {
            AB_TRY(vis_key[k].reserve(nn));
            AB_TRY(vis_idx[k].reserve(nn));
        }
        AB_TRY(ctrl.reserve(1, true));
        AB_TRY(st_depth.reserve(static_cast<size_t>(kMaxPasses) * depth_chunks() * kRadix, true));
        AB_TRY(st_dup.reserve(chunks_of(nn, pair_scan_chunk_items()), true));
        AB_TRY(offs.reserve(nn));
        AB_TRY(rank.reserve(nn));
        AB_TRY(rect_sorted.reserve(nn));
        return grow_pairs(cap);
    }

    int grow_pairs(unsigned cap) {
        if (cap <= pair_cap && pair_key[0].p) return 0;
        for (int k = 0; k < 2; ++k) {
            AB_TRY(pair_key[k].reserve(cap));
            AB_TRY(pair_val[k].reserve(cap));
        }
        pair_cap = cap;
        AB_TRY(chunk_start.reserve(chunks_of(cap, expand_chunk_pairs()) + 2));
        st_tile.release();
        return st_tile.reserve(static_cast<size_t>(kMaxPasses) * tile_chunks() * kRadix, true);
    }

    // Status words carry a 30-bit frame epoch; clear them long before it could wrap.
    int tick(cudaStream_t st) {
        if (++frames % (1ull << 29) == 0) {
            AB_CUDA(cudaMemsetAsync(st_depth.p, 0, st_depth.cap * sizeof(unsigned long long), st));
            AB_CUDA(cudaMemsetAsync(st_dup.p, 0, st_dup.cap * sizeof(unsigned long long), st));
            AB_CUDA(cudaMemsetAsync(st_tile.p, 0, st_tile.cap * sizeof(unsigned long long), st));
        }
        return 0;
    }
};

// Depth passes (the first one compacts the visible Gaussians out of depth_key), pair scan and
// expansion, tile passes and ranges. Returns the buffer index holding the final sorted pairs.
int enqueue_sort(Arena& A, int tiles_x, int tiles_y, cudaStream_t st, int* final_buf) {
    Ctrl* ctrl = A.ctrl.p;
    const unsigned nmax = static_cast<unsigned>(std::max<int64_t>(A.n, 0));
    for (int p = 0; p < kMaxPasses; ++p) {
        const int src = (p + 1) & 1, dst = p & 1;  // pass 0 reads depth_key and writes buffer 0
        launch_onesweep(p == 0 ? A.depth_key.p : A.vis_key[src].p, p == 0 ? nullptr : A.vis_idx[src].p,
                        p == kMaxPasses - 1 ? nullptr : A.vis_key[dst].p, A.vis_idx[dst].p, p == 0 ? nmax : 0u, nmax,
                        p * kRadixBits, &ctrl->depth_hist[p * kRadix],
                        A.st_depth.p + static_cast<size_t>(p) * A.depth_chunks() * kRadix,
                        &ctrl->chunk_ctr[kCtrDepth0 + p], ctrl, st);
    }
    const int sorted = A.sorted_buf();
    const unsigned tiles = static_cast<unsigned>(tiles_x) * static_cast<unsigned>(tiles_y);
    const int tile_passes = std::max(1, (bits_for(tiles - 1) + kRadixBits - 1) / kRadixBits);
    const DupBuffers dup{A.offs.p, A.rank.p, A.rect_sorted.p, A.chunk_start.p};
    launch_duplicate(A.vis_idx[sorted].p, A.rect16.p, ctrl, A.pair_cap, nmax, tiles_x, tile_passes, dup,
                     A.pair_key[0].p, A.pair_val[0].p, A.st_dup.p, st);
    for (int p = 0; p < tile_passes; ++p) {
        const int src = p & 1, dst = src ^ 1;
        launch_onesweep(A.pair_key[src].p, A.pair_val[src].p, A.pair_key[dst].p, A.pair_val[dst].p, 0u, A.pair_cap,
                        p * kRadixBits, &ctrl->tile_hist[p * kRadix],
                        A.st_tile.p + static_cast<size_t>(p) * A.tile_chunks() * kRadix,
                        &ctrl->chunk_ctr[kCtrTile0 + p], ctrl, st);
    }
    const int fin = tile_passes & 1;
    AB_TRY(A.ranges.reserve(tiles));
    AB_CUDA(cudaMemsetAsync(A.ranges.p, 0, static_cast<size_t>(tiles) * sizeof(uint2), st));
    launch_ranges(A.pair_key[fin].p, ctrl, A.pair_cap, A.ranges.p, st);
    *final_buf = fin;
    return 0;
}

}  // namespace

struct aniso_b200_scene {
    int64_t n = 0;
    int degree = 0;
    int planes = 0;
    DevBuf<float4> pos_op, scale, rot, sh;
    Arena arena;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    Ctrl* host_ctrl = nullptr;  // pinned
    // Stage events of profiled render_device frames: 4 per frame, reused after each read.
    bool profiling = false;
    std::vector<cudaEvent_t> prof_ev;
    size_t prof_frames = 0;

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
    ~aniso_b200_scene() {
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

// Scenes may store up to degree 4 (the degrees the reference loader accepts, ply_loader.cpp:67-73);
// colour is evaluated up to degree 3, as both reference renderers do.
int validate_degree(int d) {
    if (d < 0 || d > 4) return fail(ANISO_B200_ERR_ARGUMENT, "scene sh_degree must be 0..4");
    return 0;
}

int new_scene(int64_t n, int degree, aniso_b200_scene** out, aniso_b200_scene** made) {
    if (!out) return fail(ANISO_B200_ERR_ARGUMENT, "out is NULL");
    if (n < 0 || n >= (int64_t(1) << 31)) return fail(ANISO_B200_ERR_ARGUMENT, "n must be in [0, 2^31)");
    AB_TRY(validate_degree(degree));
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(ANISO_B200_ERR_NO_DEVICE, "no CUDA device");
    }
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
    const uint64_t cap = std::max<uint64_t>(1u << 20, 4ull * static_cast<uint64_t>(n));
    AB_TRY(s->arena.init(n, static_cast<unsigned>(std::min<uint64_t>(cap, 0x3FFFFFFFull))));
    return 0;
}

// The per-view constants, packed as gpu_render.cu:301-316 packs them (doubles cast to float; the
// eye is Camera::centre(), camera.cpp:19-23, computed in double).
int pack_camera_deg(int scene_degree, const aniso_b200_camera* c, const aniso_b200_options* o, CamParams& cp) {
    if (!c) return fail(ANISO_B200_ERR_ARGUMENT, "camera is NULL");
    if (c->width <= 0 || c->height <= 0 || c->width > 32767 || c->height > 32767)
        return fail(ANISO_B200_ERR_ARGUMENT, "camera size must be in [1, 32767]");
    const int opt_degree = o ? o->sh_degree : 3;
    if (opt_degree < 0) return fail(ANISO_B200_ERR_ARGUMENT, "sh_degree must be >= 0");
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
    cp.tilesX = (c->width + kTile - 1) / kTile;
    cp.tilesY = (c->height + kTile - 1) / kTile;
    cp.shDegree = std::min(std::min(opt_degree, scene_degree), 3);
    cp.shCoeffs = (scene_degree + 1) * (scene_degree + 1);
    cp.splatScale = o ? o->splat_scale : 1.0f;
    return 0;
}

int pack_camera(const aniso_b200_scene* s, const aniso_b200_camera* c, const aniso_b200_options* o, CamParams& cp) {
    return pack_camera_deg(s->degree, c, o, cp);
}

// Enqueues one frame; ev (4 events, may be NULL) brackets the stages. With stop_after_sort, the
// blend is skipped (introspection).
int enqueue_frame(aniso_b200_scene* s, const CamParams& cam, const BlendOut& out, cudaStream_t st, cudaEvent_t* ev,
                  const DebugProjection* dbg, bool stop_after_sort, int* final_buf) {
    Arena& A = s->arena;
    AB_TRY(A.tick(st));
    if (ev) AB_CUDA(cudaEventRecord(ev[0], st));
    launch_frame_begin(A.ctrl.p, st);
    launch_preprocess(s->view(), cam, A.ctrl.p, A.rec.p, A.rect16.p, A.depth_key.p, dbg, st);
    if (ev) AB_CUDA(cudaEventRecord(ev[1], st));
    int fin = 0;
    AB_TRY(enqueue_sort(A, cam.tilesX, cam.tilesY, st, &fin));
    if (ev) AB_CUDA(cudaEventRecord(ev[2], st));
    if (!stop_after_sort)
        launch_blend(A.ranges.p, A.pair_val[fin].p, A.rec.p, A.ctrl.p, cam.width, cam.height, cam.tilesX, cam.tilesY,
                     out, st);
    if (ev) AB_CUDA(cudaEventRecord(ev[3], st));
    AB_CUDA(cudaGetLastError());
    if (final_buf) *final_buf = fin;
    return 0;
}

// After a synchronised frame: grows the pair buffers on overflow (returns 1 = render again).
// With all_frames, also looks at the frames before the last one (the sticky fields).
int settle(aniso_b200_scene* s, int* again, bool all_frames = false) {
    *again = 0;
    const Ctrl& h = *s->host_ctrl;
    const unsigned flags = h.flags | (all_frames ? h.sticky_flags : 0u);
    const uint64_t pairs = all_frames ? std::max(h.pair_total, h.max_pair_total) : h.pair_total;
    if (flags & kFlagTimeout) return fail(ANISO_B200_ERR_DEVICE_WAIT, "a device-side look-back wait gave up");
    if (flags & kFlagOverflow) {
        const uint64_t need = pairs + pairs / 4 + 1024;
        if (need > 0x3FFFFFFFull) return fail(ANISO_B200_ERR_ARGUMENT, "more than 2^30 splat-tile pairs");
        AB_CUDA(cudaStreamSynchronize(s->stream));
        AB_TRY(s->arena.grow_pairs(static_cast<unsigned>(need)));
        *again = 1;
    }
    return 0;
}

int read_ctrl(aniso_b200_scene* s, cudaStream_t st) {
    AB_CUDA(cudaMemcpyAsync(s->host_ctrl, s->arena.ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    AB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace

struct aniso_b200_trainer {
    Arena arena;
    Ctrl* host_ctrl = nullptr;  // pinned
    DevBuf<float> t_final, grad_pair;
    DevBuf<unsigned> n_contrib;
    // The state of the last forward, for its backward.
    bool has_forward = false;
    RawParams raw{};
    CamParams cam{};
    int fin = 0;
    ~aniso_b200_trainer() {
        if (host_ctrl) cudaFreeHost(host_ctrl);
    }
};

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
    }
    if (rc != 0) {
        delete s;
        if (out) *out = nullptr;
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
    CamParams cam;
    AB_TRY(pack_camera(s, camera, options, cam));
    const size_t bytes = static_cast<size_t>(cam.width) * cam.height * 3;
    AB_TRY(s->arena.image.reserve(bytes));
    BlendOut out;
    out.rgb8 = s->arena.image.p;
    for (int attempt = 0; attempt < 3; ++attempt) {
        AB_TRY(enqueue_frame(s, cam, out, s->stream, stats ? s->ev : nullptr, nullptr, false, nullptr));
        AB_CUDA(cudaMemcpyAsync(rgb_host, out.rgb8, bytes, cudaMemcpyDeviceToHost, s->stream));
        AB_TRY(read_ctrl(s, s->stream));
        int again = 0;
        AB_TRY(settle(s, &again));
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
    CamParams cam;
    AB_TRY(pack_camera(s, camera, options, cam));
    BlendOut out;
    out.rgb8 = rgb_device;
    cudaEvent_t* ev = nullptr;
    if (s->profiling) {
        while (s->prof_ev.size() < 4 * (s->prof_frames + 1)) {
            cudaEvent_t e;
            AB_CUDA(cudaEventCreate(&e));
            s->prof_ev.push_back(e);
        }
        ev = &s->prof_ev[4 * s->prof_frames++];
    }
    return enqueue_frame(s, cam, out, static_cast<cudaStream_t>(stream), ev, nullptr, false, nullptr);
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
    AB_CUDA(cudaDeviceSynchronize());
    AB_TRY(read_ctrl(s, s->stream));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->visible = s->host_ctrl->vis_count;
        stats->tile_pairs = s->host_ctrl->pair_total;
    }
    // Clear the sticky record of earlier frames once read.
    AB_CUDA(cudaMemsetAsync(&s->arena.ctrl.p->sticky_flags, 0, sizeof(unsigned), s->stream));
    AB_CUDA(cudaMemsetAsync(&s->arena.ctrl.p->max_pair_total, 0, sizeof(unsigned long long), s->stream));
    AB_CUDA(cudaStreamSynchronize(s->stream));
    int again = 0;
    AB_TRY(settle(s, &again, true));
    if (again) return fail(ANISO_B200_ERR_ARGUMENT, "pair capacity exceeded");
    return ANISO_B200_OK;
}

int aniso_b200_debug_projection(aniso_b200_scene* s, const aniso_b200_camera* camera,
                                const aniso_b200_options* options, float* uv, float* conic_opacity, float* depth,
                                float* rgb, uint32_t* rect, uint32_t* tiles_touched) {
    if (!s) return fail(ANISO_B200_ERR_ARGUMENT, "scene is NULL");
    CamParams cam;
    AB_TRY(pack_camera(s, camera, options, cam));
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
    AB_TRY(A.tick(s->stream));
    launch_frame_begin(A.ctrl.p, s->stream);
    launch_preprocess(s->view(), cam, A.ctrl.p, A.rec.p, A.rect16.p, A.depth_key.p, &dbg, s->stream);
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
    CamParams cam;
    AB_TRY(pack_camera(s, camera, options, cam));
    int fin = 0;
    for (int attempt = 0; attempt < 3; ++attempt) {
        AB_TRY(enqueue_frame(s, cam, BlendOut{}, s->stream, nullptr, nullptr, true, &fin));
        AB_TRY(read_ctrl(s, s->stream));
        int again = 0;
        AB_TRY(settle(s, &again));
        if (!again) break;
    }
    const uint64_t P = s->host_ctrl->pair_total;
    *pairs = P;
    if (P > capacity) return fail(ANISO_B200_ERR_ARGUMENT, "capacity too small");
    const Arena& A = s->arena;
    if (tiles && P) AB_CUDA(cudaMemcpy(tiles, A.pair_key[fin].p, P * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (values && P) AB_CUDA(cudaMemcpy(values, A.pair_val[fin].p, P * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (ranges)
        AB_CUDA(cudaMemcpy(ranges, A.ranges.p, static_cast<size_t>(cam.tilesX) * cam.tilesY * sizeof(uint2),
                           cudaMemcpyDeviceToHost));
    return ANISO_B200_OK;
}

int aniso_b200_sort_projection(int64_t n, const uint32_t* tiles_touched, const uint32_t* rect, const float* depth,
                               int32_t tiles_x, int32_t tiles_y, uint32_t* tiles, uint32_t* values,
                               uint64_t capacity, uint32_t* ranges, uint64_t* pairs) {
    if (n < 0 || n >= (int64_t(1) << 31) || tiles_x <= 0 || tiles_y <= 0 || !pairs)
        return fail(ANISO_B200_ERR_ARGUMENT, "bad size or NULL pairs");
    if (n > 0 && (!tiles_touched || !rect || !depth)) return fail(ANISO_B200_ERR_ARGUMENT, "input is NULL");
    uint64_t P = 0;
    for (int64_t i = 0; i < n; ++i) P += tiles_touched[i];
    *pairs = P;
    if (P > capacity) return fail(ANISO_B200_ERR_ARGUMENT, "capacity too small");
    if (P > 0x3FFFFFFFull) return fail(ANISO_B200_ERR_ARGUMENT, "more than 2^30 pairs");
    Arena A;
    AB_TRY(A.init(n, static_cast<unsigned>(std::max<uint64_t>(P, 1))));
    const size_t nn = static_cast<size_t>(std::max<int64_t>(n, 1));
    DevBuf<unsigned> dtt;
    DevBuf<uint4> drect;
    DevBuf<float> ddepth;
    AB_TRY(dtt.reserve(nn));
    AB_TRY(drect.reserve(nn));
    AB_TRY(ddepth.reserve(nn));
    const size_t un = static_cast<size_t>(n);
    if (n > 0) {
        AB_CUDA(cudaMemcpy(dtt.p, tiles_touched, un * sizeof(unsigned), cudaMemcpyHostToDevice));
        AB_CUDA(cudaMemcpy(drect.p, rect, un * sizeof(uint4), cudaMemcpyHostToDevice));
        AB_CUDA(cudaMemcpy(ddepth.p, depth, un * sizeof(float), cudaMemcpyHostToDevice));
    }
    cudaStream_t st = nullptr;
    AB_TRY(A.tick(st));
    launch_frame_begin(A.ctrl.p, st);
    launch_projection_keys(n, dtt.p, ddepth.p, drect.p, A.ctrl.p, A.depth_key.p, A.rect16.p, st);
    int fin = 0;
    AB_TRY(enqueue_sort(A, tiles_x, tiles_y, st, &fin));
    AB_CUDA(cudaGetLastError());
    AB_CUDA(cudaDeviceSynchronize());
    Ctrl h;
    AB_CUDA(cudaMemcpy(&h, A.ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    if (h.flags & kFlagTimeout) return fail(ANISO_B200_ERR_DEVICE_WAIT, "a device-side look-back wait gave up");
    if (h.pair_total != P) return fail(ANISO_B200_ERR_CUDA, "device pair count disagrees with the host");
    if (tiles && P) AB_CUDA(cudaMemcpy(tiles, A.pair_key[fin].p, P * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (values && P) AB_CUDA(cudaMemcpy(values, A.pair_val[fin].p, P * sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (ranges)
        AB_CUDA(cudaMemcpy(ranges, A.ranges.p, static_cast<size_t>(tiles_x) * tiles_y * sizeof(uint2),
                           cudaMemcpyDeviceToHost));
    return ANISO_B200_OK;
}

int aniso_b200_trainer_create(aniso_b200_trainer** out) {
    if (!out) return fail(ANISO_B200_ERR_ARGUMENT, "out is NULL");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(ANISO_B200_ERR_NO_DEVICE, "no CUDA device");
    }
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
    if (t) cudaDeviceSynchronize();
    delete t;
    return ANISO_B200_OK;
}

int aniso_b200_train_forward(aniso_b200_trainer* t, const aniso_b200_raw_params* params, const aniso_b200_camera* camera,
                             const aniso_b200_options* options, float* image_device, void* stream) {
    if (!t || !params || !image_device) return fail(ANISO_B200_ERR_ARGUMENT, "trainer/params/image is NULL");
    const aniso_b200_raw_params& P = *params;
    if (P.n < 0 || P.n >= (int64_t(1) << 31)) return fail(ANISO_B200_ERR_ARGUMENT, "n must be in [0, 2^31)");
    if (P.sh_degree != 1 && P.sh_degree != 3)
        return fail(ANISO_B200_ERR_ARGUMENT, "stored SH degree must be 1 or 3 (whole 16-byte words per Gaussian)");
    if (P.n > 0 && (!P.means || !P.log_scales || !P.quats || !P.opacity_logits || !P.sh))
        return fail(ANISO_B200_ERR_ARGUMENT, "a parameter pointer is NULL");
    if ((reinterpret_cast<uintptr_t>(P.quats) | reinterpret_cast<uintptr_t>(P.sh)) & 15)
        return fail(ANISO_B200_ERR_ARGUMENT, "quats and sh must be 16-byte aligned");
    CamParams cam;
    AB_TRY(pack_camera_deg(P.sh_degree, camera, options, cam));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Arena& A = t->arena;
    if (A.n < P.n) {
        const uint64_t cap = std::max<uint64_t>(1u << 20, 4ull * static_cast<uint64_t>(P.n));
        A.~Arena();
        new (&A) Arena();
        AB_TRY(A.init(P.n, static_cast<unsigned>(std::min<uint64_t>(cap, 0x3FFFFFFFull))));
    }
    const size_t pixels = static_cast<size_t>(cam.width) * cam.height;
    AB_TRY(t->t_final.reserve(pixels));
    AB_TRY(t->n_contrib.reserve(pixels));
    RawParams raw;
    raw.means = P.means;
    raw.log_scales = P.log_scales;
    raw.quats = reinterpret_cast<const float4*>(P.quats);
    raw.logits = P.opacity_logits;
    raw.sh = reinterpret_cast<const float4*>(P.sh);
    raw.n = P.n;
    raw.sh_planes = (P.sh_degree + 1) * (P.sh_degree + 1) * 3 / 4;
    BlendOut out;
    out.rgbf = image_device;
    out.t_final = t->t_final.p;
    out.n_contrib = t->n_contrib.p;
    const int64_t saved_n = A.n;
    A.n = P.n;  // grids follow this frame's Gaussian count
    int rc = ANISO_B200_OK;
    for (int attempt = 0; attempt < 3; ++attempt) {
        rc = A.tick(st);
        if (rc) break;
        launch_frame_begin(A.ctrl.p, st);
        launch_preprocess_raw(raw, cam, A.ctrl.p, A.rec.p, A.rect16.p, A.depth_key.p, st);
        int fin = 0;
        rc = enqueue_sort(A, cam.tilesX, cam.tilesY, st, &fin);
        if (rc) break;
        launch_blend(A.ranges.p, A.pair_val[fin].p, A.rec.p, A.ctrl.p, cam.width, cam.height, cam.tilesX, cam.tilesY,
                     out, st);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(t->host_ctrl, A.ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "train forward");
            break;
        }
        const Ctrl& h = *t->host_ctrl;
        if (h.flags & kFlagTimeout) {
            rc = fail(ANISO_B200_ERR_DEVICE_WAIT, "a device-side look-back wait gave up");
            break;
        }
        if (h.flags & kFlagOverflow) {
            const uint64_t need = h.pair_total + h.pair_total / 4 + 1024;
            if (need > 0x3FFFFFFFull) {
                rc = fail(ANISO_B200_ERR_ARGUMENT, "more than 2^30 splat-tile pairs");
                break;
            }
            rc = A.grow_pairs(static_cast<unsigned>(need));
            if (rc) break;
            rc = fail(ANISO_B200_ERR_ARGUMENT, "pair capacity kept overflowing");
            continue;
        }
        t->has_forward = true;
        t->raw = raw;
        t->cam = cam;
        t->fin = fin;
        rc = ANISO_B200_OK;
        break;
    }
    A.n = std::max(A.n, saved_n);
    if (rc != ANISO_B200_OK) t->has_forward = false;
    return rc;
}

int aniso_b200_train_backward(aniso_b200_trainer* t, const float* grad_image_device, const aniso_b200_raw_grads* grads,
                              void* stream) {
    if (!t || !grad_image_device || !grads) return fail(ANISO_B200_ERR_ARGUMENT, "trainer/grad_image/grads is NULL");
    if (!t->has_forward) return fail(ANISO_B200_ERR_ARGUMENT, "no forward to differentiate");
    if (t->raw.n > 0 && (!grads->means || !grads->log_scales || !grads->quats || !grads->opacity_logits || !grads->sh))
        return fail(ANISO_B200_ERR_ARGUMENT, "a gradient pointer is NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Arena& A = t->arena;
    const Ctrl& h = *t->host_ctrl;
    AB_TRY(t->grad_pair.reserve(std::max<uint64_t>(h.pair_total, 1) * 9));
    BackwardIn in;
    in.ranges = A.ranges.p;
    in.vals = A.pair_val[t->fin].p;
    in.rec = A.rec.p;
    in.ctrl = A.ctrl.p;
    in.t_final = t->t_final.p;
    in.n_contrib = t->n_contrib.p;
    in.grad_img = grad_image_device;
    in.rank = A.rank.p;
    in.offs = A.offs.p;
    in.rect_sorted = A.rect_sorted.p;
    in.width = t->cam.width;
    in.height = t->cam.height;
    in.tiles_x = t->cam.tilesX;
    launch_blend_backward(in, t->cam.tilesY, t->grad_pair.p, st);
    RawGrads g{grads->means, grads->log_scales, grads->quats, grads->opacity_logits, grads->sh};
    launch_gauss_backward(t->raw, t->cam, A.ctrl.p, A.vis_idx[A.sorted_buf()].p, A.offs.p, A.rect_sorted.p,
                          t->grad_pair.p, h.vis_count, g, st);
    AB_CUDA(cudaGetLastError());
    return ANISO_B200_OK;
}

}  // extern "C"
