// aniso::loadColmapCameras (include/aniso/camera.h:51, src/camera.cpp:105-140) re-implemented on
// aniso_b200_colmap_load, for the drop-in CLI: the same cameras, order and PlyError messages for
// the binary model the reference reads, and COLMAP's text model (cameras.txt + images.txt) where
// there is no cameras.bin -- the form the workload descriptions are written in. The drop-in build
// links this file and compiles the reference's camera.cpp with its own loadColmapCameras renamed
// out of the way (oracle/Makefile, `dropin`), so main.cpp compiles unchanged.
#include "aniso/camera.h"
#include "aniso/ply_loader.h"
#include "aniso_b200.h"

#include <string>
#include <vector>

namespace aniso {

std::vector<Camera> loadColmapCameras(const std::filesystem::path& sparseDir) {
    const std::string dir = sparseDir.string();
    const auto fail = [] {
        char buf[1024];
        aniso_b200_last_error(buf, sizeof buf);
        throw PlyError(buf);
    };
    int32_t n = 0;
    if (aniso_b200_colmap_load(dir.c_str(), nullptr, 0, &n) != ANISO_B200_OK) fail();
    std::vector<aniso_b200_colmap_camera> raw(static_cast<size_t>(n));
    if (n > 0 && aniso_b200_colmap_load(dir.c_str(), raw.data(), n, &n) != ANISO_B200_OK) fail();
    std::vector<Camera> out;
    out.reserve(raw.size());
    for (const aniso_b200_colmap_camera& r : raw) {
        Camera c;
        c.imageName = r.image_name;
        c.width = r.camera.width;
        c.height = r.camera.height;
        c.fx = r.camera.fx;
        c.fy = r.camera.fy;
        c.cx = r.camera.cx;
        c.cy = r.camera.cy;
        for (int i = 0; i < 3; ++i) {
            for (int k = 0; k < 3; ++k) c.R[i][k] = r.camera.R[i * 3 + k];
            c.t[i] = r.camera.t[i];
        }
        out.push_back(std::move(c));
    }
    return out;
}

}  // namespace aniso
