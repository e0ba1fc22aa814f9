// Test infrastructure, not product code. A C-ABI around the reference's own CPU renderer, compiled
// from the reference sources where they lie (see oracle/Makefile). Only tests/, the smoke check and
// bench.py's CPU-baseline / reference arms load the library this file builds.
//
// render.cpp is included (not linked) so that its anonymous-namespace makeSplat() can be called
// directly to dump the per-Gaussian projection that feeds the blend (render.cpp:39-104).
// The Makefile defines REF_RENDER_CPP as the quoted path of the reference's src/render.cpp.
#include REF_RENDER_CPP

#include "aniso/camera.h"
#include "aniso/gaussian.h"
#include "aniso/image.h"
#include "aniso/ply_loader.h"
#include "aniso/render.h"
#include "aniso/sh.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

namespace {

thread_local std::string g_err;

aniso::Scene makeScene(const float* gauss, const float* sh, int64_t n, int degree) {
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
    const std::size_t k = static_cast<std::size_t>(s.shCoeffsPerChannel()) * 3;
    s.sh.assign(sh, sh + static_cast<std::size_t>(n) * k);
    return s;
}

// cam: R[9] row-major, t[3], fx, fy, cx, cy (16 doubles); size (w, h).
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

}  // namespace

extern "C" {

const char* ref_cpu_last_error() { return g_err.c_str(); }

// aniso::render (render.cpp:140-223). stats: visible, tilePairs, projectMs, sortMs, blendMs.
int ref_cpu_render(const float* gauss, const float* sh, int64_t n, int scene_degree, const double* cam, int w, int h,
                   int sh_degree, float splat_scale, uint8_t* out_rgb, double* stats) {
    try {
        const aniso::Scene s = makeScene(gauss, sh, n, scene_degree);
        const aniso::Camera c = makeCamera(cam, w, h);
        aniso::RenderOptions o;
        o.shDegree = sh_degree;
        o.splatScale = splat_scale;
        aniso::RenderStats st;
        const aniso::Image img = aniso::render(s, c, &st, o);
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

// A scene built once, as the reference CLI builds it (main.cpp loads the PLY once and renders each
// view from the same Scene), so that a timed loop of ref_cpu_scene_render calls measures
// aniso::render alone (render.cpp:140-223), not the Scene construction.
void* ref_cpu_scene_create(const float* gauss, const float* sh, int64_t n, int scene_degree) {
    try {
        return new aniso::Scene(makeScene(gauss, sh, n, scene_degree));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_cpu_scene_destroy(void* scene) { delete static_cast<aniso::Scene*>(scene); }

// aniso::render of a scene made by ref_cpu_scene_create; stats as ref_cpu_render.
int ref_cpu_scene_render(const void* scene, const double* cam, int w, int h, int sh_degree, float splat_scale,
                         uint8_t* out_rgb, double* stats) {
    try {
        const aniso::Scene& s = *static_cast<const aniso::Scene*>(scene);
        const aniso::Camera c = makeCamera(cam, w, h);
        aniso::RenderOptions o;
        o.shDegree = sh_degree;
        o.splatScale = splat_scale;
        aniso::RenderStats st;
        const aniso::Image img = aniso::render(s, c, &st, o);
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

// makeSplat (render.cpp:39-104) for every Gaussian. out: n x 10 floats
// (u, v, conicA, conicB, conicC, opacity, depth, r, g, b); radius: n ints; alive: n bytes.
int ref_cpu_make_splats(const float* gauss, const float* sh, int64_t n, int scene_degree, const double* cam, int w,
                        int h, int sh_degree, float splat_scale, float* out, int32_t* radius, uint8_t* alive) {
    try {
        const aniso::Scene s = makeScene(gauss, sh, n, scene_degree);
        const aniso::Camera c = makeCamera(cam, w, h);
        const aniso::Vec3 eye = c.centre();
        for (int64_t i = 0; i < n; ++i) {
            aniso::Splat sp;
            const bool ok = aniso::makeSplat(s, static_cast<std::size_t>(i), c, eye, sh_degree, splat_scale, sp);
            float* o = out + i * 10;
            o[0] = sp.u; o[1] = sp.v; o[2] = sp.conicA; o[3] = sp.conicB; o[4] = sp.conicC;
            o[5] = sp.opacity; o[6] = sp.depth; o[7] = sp.rgb[0]; o[8] = sp.rgb[1]; o[9] = sp.rgb[2];
            radius[i] = sp.radius;
            alive[i] = ok ? 1 : 0;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// shColor (sh.cpp:18-58) for one Gaussian's coefficients.
int ref_cpu_sh_color(const float* sh, int scene_degree, float x, float y, float z, int degree, float* out3) {
    aniso::Scene s;
    s.shDegree = scene_degree;
    s.gaussians.resize(1);
    s.sh.assign(sh, sh + s.shCoeffsPerChannel() * 3);
    const auto c = aniso::shColor(s, 0, aniso::Vec3{x, y, z}, degree);
    out3[0] = c[0]; out3[1] = c[1]; out3[2] = c[2];
    return 0;
}

// loadPly (ply_loader.cpp:77-141), two calls: with gauss == nullptr only n and degree are returned.
int ref_cpu_load_ply(const char* path, int64_t* n, int* degree, float* gauss, float* sh) {
    try {
        const aniso::Scene s = aniso::loadPly(path);
        *n = static_cast<int64_t>(s.size());
        *degree = s.shDegree;
        if (gauss) {
            for (std::size_t i = 0; i < s.size(); ++i) {
                const aniso::Gaussian& g = s.gaussians[i];
                float* o = gauss + i * 11;
                o[0] = g.position.x; o[1] = g.position.y; o[2] = g.position.z;
                o[3] = g.scale.x; o[4] = g.scale.y; o[5] = g.scale.z;
                o[6] = g.rotation.w; o[7] = g.rotation.x; o[8] = g.rotation.y; o[9] = g.rotation.z;
                o[10] = g.opacity;
            }
            std::memcpy(sh, s.sh.data(), s.sh.size() * sizeof(float));
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// loadColmapCameras (camera.cpp:105-140), two calls: with out == nullptr only the count is returned.
// out per camera: w, h, fx, fy, cx, cy, R[9], t[3] (20 doubles).
int ref_cpu_load_colmap(const char* dir, int* count, double* out) {
    try {
        const auto cams = aniso::loadColmapCameras(dir);
        *count = static_cast<int>(cams.size());
        if (out) {
            for (std::size_t i = 0; i < cams.size(); ++i) {
                const aniso::Camera& c = cams[i];
                double* o = out + i * 20;
                o[0] = c.width; o[1] = c.height; o[2] = c.fx; o[3] = c.fy; o[4] = c.cx; o[5] = c.cy;
                for (int r = 0; r < 3; ++r)
                    for (int k = 0; k < 3; ++k) o[6 + r * 3 + k] = c.R[r][k];
                for (int k = 0; k < 3; ++k) o[15 + k] = c.t[k];
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Camera::centre (camera.cpp:19-23), as floats.
void ref_cpu_camera_centre(const double* cam, float* out3) {
    const aniso::Camera c = makeCamera(cam, 1, 1);
    const aniso::Vec3 e = c.centre();
    out3[0] = e.x; out3[1] = e.y; out3[2] = e.z;
}

}  // extern "C"
