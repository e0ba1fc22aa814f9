// Test infrastructure, not product code: the "key oracle". A C-ABI that drives the reference's own
// CUDA kernels (gpu_render.cu), compiled from the reference source where it lies (oracle/Makefile
// defines REF_GPU_RENDER_CU) for sm_100a, once without --use_fast_math (the bit-exact parity build)
// and once with it (the reference as shipped, for timing). Only tests/ and the profiling recipes
// under oracle/ load the libraries this file builds.
//
// Each stage is exposed separately so a test can feed the reference's sort exactly the projection
// the product computed ("given the same fp32 projection"), and compare keys, values and tile ranges
// bit for bit.
#include REF_GPU_RENDER_CU

#include <cstdint>
#include <cstring>
#include <string>

namespace {

thread_local std::string g_err;

#define RG_CHECK(call)                                         \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) {                               \
            g_err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return 1;                                          \
        }                                                      \
    } while (0)

aniso::Camera makeCamera(const double* cam, int w, int h) {
    aniso::Camera c;
    c.width = w;
    c.height = h;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) c.R[r][k] = cam[r * 3 + k];
    for (int k = 0; k < 3; ++k) c.t[k] = cam[9 + k];
    c.fx = cam[12];
    c.fy = cam[13];
    c.cx = cam[14];
    c.cy = cam[15];
    return c;
}

// The same packing as GpuRenderer::render (gpu_render.cu:301-316).
aniso::CameraParams pack(const aniso::Camera& camera, int optDegree, int sceneDegree, float splatScale) {
    aniso::CameraParams cp{};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) cp.R[r * 3 + c] = static_cast<float>(camera.R[r][c]);
        cp.t[r] = static_cast<float>(camera.t[r]);
    }
    const aniso::Vec3 eye = camera.centre();
    cp.eye[0] = eye.x; cp.eye[1] = eye.y; cp.eye[2] = eye.z;
    cp.fx = static_cast<float>(camera.fx); cp.fy = static_cast<float>(camera.fy);
    cp.cx = static_cast<float>(camera.cx); cp.cy = static_cast<float>(camera.cy);
    cp.width = camera.width; cp.height = camera.height;
    cp.tilesX = (camera.width + aniso::kTile - 1) / aniso::kTile;
    cp.tilesY = (camera.height + aniso::kTile - 1) / aniso::kTile;
    cp.shDegree = std::min(optDegree, sceneDegree);
    cp.shCoeffs = (sceneDegree + 1) * (sceneDegree + 1);
    cp.splatScale = splatScale;
    return cp;
}

}  // namespace

extern "C" {

const char* refgpu_last_error() { return g_err.c_str(); }

// preprocess (gpu_render.cu:86-145) on device SoA arrays laid out as GpuRenderer::Impl holds them:
// pos float3[n], scale float3[n], rot float4[n] (w,x,y,z), opacity float[n], sh float[n*coeffs*3].
// Outputs: uv float2[n], conicOpacity float4[n], depth float[n], rgb float3[n], rect uint4[n],
// tilesTouched uint32[n].
int refgpu_preprocess(int n, uint64_t pos, uint64_t scale, uint64_t rot, uint64_t opacity, uint64_t sh,
                      int scene_degree, const double* cam, int w, int h, int sh_degree, float splat_scale,
                      uint64_t uv, uint64_t conic_opacity, uint64_t depth, uint64_t rgb, uint64_t rect,
                      uint64_t tiles_touched) {
    const aniso::CameraParams cp = pack(makeCamera(cam, w, h), sh_degree, scene_degree, splat_scale);
    const int threads = 256, blocks = (n + threads - 1) / threads;
    if (n > 0)
        aniso::preprocess<<<blocks, threads>>>(
            n, reinterpret_cast<const float3*>(pos), reinterpret_cast<const float3*>(scale),
            reinterpret_cast<const float4*>(rot), reinterpret_cast<const float*>(opacity),
            reinterpret_cast<const float*>(sh), cp, reinterpret_cast<float2*>(uv),
            reinterpret_cast<float4*>(conic_opacity), reinterpret_cast<float*>(depth),
            reinterpret_cast<float3*>(rgb), reinterpret_cast<uint4*>(rect), reinterpret_cast<uint32_t*>(tiles_touched));
    RG_CHECK(cudaGetLastError());
    RG_CHECK(cudaDeviceSynchronize());
    return 0;
}

// Steps 2-4 of GpuRenderer::render (gpu_render.cu:324-345): inclusive scan of tilesTouched,
// duplicate, CUB SortPairs over bits [0, 32 + bitsFor(tileCount)), tileRanges. Writes the sorted
// keys/values (capacity entries at most) and tiles_x*tiles_y ranges; *total receives the pair count.
// Returns 2 if capacity is too small (total is still set).
int refgpu_sort(int n, uint64_t tiles_touched, uint64_t rect, uint64_t depth, int tiles_x, int tiles_y,
                uint64_t keys_out, uint64_t values_out, uint64_t capacity, uint64_t ranges_out, uint64_t* total) {
    const int tileCount = tiles_x * tiles_y;
    uint32_t* offsets = nullptr;
    void* temp = nullptr;
    std::size_t tempBytes = 0;
    RG_CHECK(cudaMalloc(&offsets, std::max(n, 1) * sizeof(uint32_t)));
    cub::DeviceScan::InclusiveSum(nullptr, tempBytes, reinterpret_cast<const uint32_t*>(tiles_touched), offsets, n);
    RG_CHECK(cudaMalloc(&temp, std::max<std::size_t>(tempBytes, 1)));
    cub::DeviceScan::InclusiveSum(temp, tempBytes, reinterpret_cast<const uint32_t*>(tiles_touched), offsets, n);
    uint32_t t = 0;
    if (n > 0) RG_CHECK(cudaMemcpy(&t, offsets + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    cudaFree(temp);
    *total = t;
    RG_CHECK(cudaMemset(reinterpret_cast<void*>(ranges_out), 0, tileCount * sizeof(uint2)));
    if (t > capacity) {
        cudaFree(offsets);
        g_err = "capacity too small";
        return 2;
    }
    if (t > 0) {
        uint64_t *keys = nullptr, *keysAlt = nullptr;
        uint32_t *values = nullptr, *valuesAlt = nullptr;
        RG_CHECK(cudaMalloc(&keys, t * sizeof(uint64_t)));
        RG_CHECK(cudaMalloc(&keysAlt, t * sizeof(uint64_t)));
        RG_CHECK(cudaMalloc(&values, t * sizeof(uint32_t)));
        RG_CHECK(cudaMalloc(&valuesAlt, t * sizeof(uint32_t)));
        const int threads = 256, blocks = (n + threads - 1) / threads;
        aniso::duplicate<<<blocks, threads>>>(n, offsets, reinterpret_cast<const uint32_t*>(tiles_touched),
                                              reinterpret_cast<const uint4*>(rect),
                                              reinterpret_cast<const float*>(depth), tiles_x, keys, values);
        RG_CHECK(cudaGetLastError());
        cub::DoubleBuffer<uint64_t> k(keys, keysAlt);
        cub::DoubleBuffer<uint32_t> v(values, valuesAlt);
        const int endBit = 32 + aniso::bitsFor(static_cast<uint32_t>(tileCount));
        tempBytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, k, v, t, 0, endBit);
        RG_CHECK(cudaMalloc(&temp, std::max<std::size_t>(tempBytes, 1)));
        cub::DeviceRadixSort::SortPairs(temp, tempBytes, k, v, t, 0, endBit);
        aniso::tileRanges<<<(t + threads - 1) / threads, threads>>>(static_cast<int>(t), k.Current(),
                                                                     reinterpret_cast<uint2*>(ranges_out));
        RG_CHECK(cudaGetLastError());
        RG_CHECK(cudaMemcpy(reinterpret_cast<void*>(keys_out), k.Current(), t * sizeof(uint64_t),
                            cudaMemcpyDeviceToDevice));
        RG_CHECK(cudaMemcpy(reinterpret_cast<void*>(values_out), v.Current(), t * sizeof(uint32_t),
                            cudaMemcpyDeviceToDevice));
        RG_CHECK(cudaDeviceSynchronize());
        cudaFree(temp);
        cudaFree(keys);
        cudaFree(keysAlt);
        cudaFree(values);
        cudaFree(valuesAlt);
    }
    cudaFree(offsets);
    RG_CHECK(cudaDeviceSynchronize());
    return 0;
}

// blend (gpu_render.cu:180-233) into a device RGB8 image.
int refgpu_blend(uint64_t ranges, uint64_t values, uint64_t uv, uint64_t conic_opacity, uint64_t rgb, int w, int h,
                 uint64_t out) {
    const int tx = (w + aniso::kTile - 1) / aniso::kTile, ty = (h + aniso::kTile - 1) / aniso::kTile;
    aniso::blend<<<dim3(tx, ty), dim3(aniso::kTile, aniso::kTile)>>>(
        reinterpret_cast<const uint2*>(ranges), reinterpret_cast<const uint32_t*>(values),
        reinterpret_cast<const float2*>(uv), reinterpret_cast<const float4*>(conic_opacity),
        reinterpret_cast<const float3*>(rgb), w, h, tx, reinterpret_cast<uint8_t*>(out));
    RG_CHECK(cudaGetLastError());
    RG_CHECK(cudaDeviceSynchronize());
    return 0;
}

// The whole GpuRenderer as shipped: constructed from a host scene (n x 11 activated floats:
// pos, scale, rot w-first, opacity; plus SH), rendered with a host camera into a host image.
void* refgpu_renderer_create(const float* gauss, const float* sh, int64_t n, int degree) {
    try {
        aniso::Scene s;
        s.shDegree = degree;
        s.gaussians.resize(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            const float* g = gauss + i * 11;
            aniso::Gaussian& o = s.gaussians[static_cast<std::size_t>(i)];
            o.position = {g[0], g[1], g[2]};
            o.scale = {g[3], g[4], g[5]};
            o.rotation = {g[6], g[7], g[8], g[9]};
            o.opacity = g[10];
        }
        s.sh.assign(sh, sh + static_cast<std::size_t>(n) * s.shCoeffsPerChannel() * 3);
        return new aniso::GpuRenderer(s);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// stats: visible, tilePairs, projectMs, sortMs, blendMs (RenderStats).
int refgpu_renderer_render(void* r, const double* cam, int w, int h, int sh_degree, float splat_scale,
                           uint8_t* out_rgb, double* stats) {
    try {
        aniso::RenderOptions o;
        o.shDegree = sh_degree;
        o.splatScale = splat_scale;
        aniso::RenderStats st;
        const aniso::Image img = static_cast<aniso::GpuRenderer*>(r)->render(makeCamera(cam, w, h), &st, o);
        std::memcpy(out_rgb, img.rgb.data(), img.rgb.size());
        if (stats) {
            stats[0] = static_cast<double>(st.visible);
            stats[1] = static_cast<double>(st.tilePairs);
            stats[2] = st.projectMs;
            stats[3] = st.sortMs;
            stats[4] = st.blendMs;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

void refgpu_renderer_destroy(void* r) { delete static_cast<aniso::GpuRenderer*>(r); }

}  // extern "C"
