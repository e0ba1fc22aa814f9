// aniso::GpuRenderer (include/aniso/gpu_render.h:22-37) re-implemented on the C ABI of
// libaniso_b200.so, so the reference's callers -- the CLI (main.cpp:158-165, 227-243), the viewer
// (viewer.cpp:102-103, 133, 244) and tests/test_gpu_render.cpp -- compile unchanged and link this
// file plus -laniso_b200 in place of src/gpu_render.cu.
//
// Same contract as the reference: the scene is uploaded once in the constructor and not retained;
// render() returns an owning host RGB8 Image and fills RenderStats with GPU stage times; any
// failure throws std::runtime_error("CUDA <what>: <message>") (gpu_render.cu:18-21). Unlike the
// reference, stats->visible is the real visible count (the reference reports 0, gpu_render.cu:372).
#include "aniso/gpu_render.h"
#include "aniso_b200.h"

#include <stdexcept>
#include <string>

namespace aniso {

static_assert(sizeof(Gaussian) == 11 * sizeof(float), "aniso::Gaussian must be 11 packed floats");

namespace {

void check(int rc, const char* what) {
    if (rc == ANISO_B200_OK) return;
    char buf[512];
    aniso_b200_last_error(buf, sizeof buf);
    throw std::runtime_error(std::string("CUDA ") + what + ": " + buf);
}

}  // namespace

struct GpuRenderer::Impl {
    aniso_b200_scene* scene = nullptr;
};

bool GpuRenderer::available() {
    int32_t a = 0;
    return aniso_b200_available(&a) == ANISO_B200_OK && a != 0;
}

GpuRenderer::GpuRenderer(const Scene& scene) : impl_(std::make_unique<Impl>()) {
    check(aniso_b200_scene_create(reinterpret_cast<const float*>(scene.gaussians.data()), scene.sh.data(),
                                  static_cast<int64_t>(scene.size()), scene.shDegree, &impl_->scene),
          "scene upload");
}

GpuRenderer::~GpuRenderer() {
    if (impl_) aniso_b200_scene_destroy(impl_->scene);
}

Image GpuRenderer::render(const Camera& camera, RenderStats* stats, const RenderOptions& options) {
    aniso_b200_camera c{};
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) c.R[r * 3 + k] = camera.R[r][k];
        c.t[r] = camera.t[r];
    }
    c.fx = camera.fx;
    c.fy = camera.fy;
    c.cx = camera.cx;
    c.cy = camera.cy;
    c.width = camera.width;
    c.height = camera.height;
    const aniso_b200_options o{options.shDegree, options.splatScale};
    Image img(camera.width, camera.height);
    aniso_b200_stats st{};
    check(aniso_b200_render(impl_->scene, &c, &o, img.rgb.data(), stats ? &st : nullptr), "render");
    if (stats) {
        stats->visible = st.visible;
        stats->tilePairs = st.tile_pairs;
        stats->projectMs = st.project_ms;
        stats->sortMs = st.sort_ms;
        stats->blendMs = st.blend_ms;
    }
    return img;
}

}  // namespace aniso
