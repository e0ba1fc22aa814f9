// aniso_b200_colmap_load: the cameras of a COLMAP sparse model, binary or text, for C callers and
// for the GpuRenderer drop-in's CLI (host code only).
//
// Binary (cameras.bin + images.bin): the format and rules of aniso::loadColmapCameras
// (camera.cpp:61-140) -- little-endian records, camera model ids with COLMAP's parameter counts,
// PINHOLE (1) and SIMPLE_PINHOLE (0) only, each image's 2D points skipped, the quaternion normalised
// in double into R, cameras sorted by image name -- with the same error messages. Text
// (cameras.txt + images.txt, read when cameras.bin is absent): COLMAP's text model, '#' comments,
// "CAMERA_ID MODEL WIDTH HEIGHT PARAMS..." and two lines per image ("IMAGE_ID QW QX QY QZ TX TY TZ
// CAMERA_ID NAME", then its 2D points), the same models, conversion and order.
#include "aniso_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace ab2 {
int report_error(int code, const char* msg);  // capi.cu: status code + aniso_b200_last_error text
}

namespace {

struct Intrinsics {
    int width = 0, height = 0;
    double fx = 0, fy = 0, cx = 0, cy = 0;
};

struct Failure {
    std::string what;
};

// COLMAP's camera models (models.h) by id: name and parameter count.
const char* const kModelNames[] = {"SIMPLE_PINHOLE", "PINHOLE", "SIMPLE_RADIAL", "RADIAL", "OPENCV", "OPENCV_FISHEYE",
                                   "FULL_OPENCV", "FOV", "SIMPLE_RADIAL_FISHEYE", "RADIAL_FISHEYE", "THIN_PRISM_FISHEYE"};
const int kModelParams[] = {3, 4, 4, 5, 8, 8, 12, 5, 4, 5, 12};

Intrinsics pinhole(int model, const std::vector<double>& p, int width, int height, const std::string& where,
                   const std::string& model_name) {
    Intrinsics c;
    c.width = width;
    c.height = height;
    if (model == 0) {  // SIMPLE_PINHOLE: f, cx, cy
        c.fx = c.fy = p[0];
        c.cx = p[1];
        c.cy = p[2];
    } else if (model == 1) {  // PINHOLE: fx, fy, cx, cy
        c.fx = p[0];
        c.fy = p[1];
        c.cx = p[2];
        c.cy = p[3];
    } else {
        throw Failure{where + ": camera model " + model_name + " has lens distortion; undistort the images first"};
    }
    return c;
}

// The rotation of the normalised quaternion (w, x, y, z), in double (camera.cpp:95-101).
void quat_to_matrix(double w, double x, double y, double z, double* R) {
    const double n = std::sqrt(w * w + x * x + y * y + z * z);
    w /= n;
    x /= n;
    y /= n;
    z /= n;
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z);     R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);     R[7] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}

struct Image {
    std::string name;
    double q[4], t[3];
    uint32_t camera;
};

template <typename T>
T read_pod(std::ifstream& in, const std::string& file) {
    T v{};
    in.read(reinterpret_cast<char*>(&v), sizeof(T));
    if (!in) throw Failure{file + ": unexpected end of file"};
    return v;
}

void read_binary(const std::string& dir, std::map<uint32_t, Intrinsics>& cams, std::vector<Image>& images) {
    {
        const std::string file = dir + "/cameras.bin";
        std::ifstream in(file, std::ios::binary);
        if (!in) throw Failure{file + ": cannot open"};
        const auto count = read_pod<uint64_t>(in, file);
        for (uint64_t i = 0; i < count; ++i) {
            const auto id = read_pod<uint32_t>(in, file);
            const auto model = read_pod<int32_t>(in, file);
            const int width = static_cast<int>(read_pod<uint64_t>(in, file));
            const int height = static_cast<int>(read_pod<uint64_t>(in, file));
            if (model < 0 || model >= 11) throw Failure{file + ": unknown camera model " + std::to_string(model)};
            std::vector<double> p(kModelParams[model]);
            for (double& v : p) v = read_pod<double>(in, file);
            cams[id] = pinhole(model, p, width, height, file, std::to_string(model));
        }
    }
    const std::string file = dir + "/images.bin";
    std::ifstream in(file, std::ios::binary);
    if (!in) throw Failure{file + ": cannot open"};
    const auto count = read_pod<uint64_t>(in, file);
    for (uint64_t i = 0; i < count; ++i) {
        Image im;
        read_pod<uint32_t>(in, file);  // image id, unused
        for (double& v : im.q) v = read_pod<double>(in, file);
        for (double& v : im.t) v = read_pod<double>(in, file);
        im.camera = read_pod<uint32_t>(in, file);
        for (char ch; (ch = read_pod<char>(in, file)) != '\0';) im.name.push_back(ch);
        const auto points = read_pod<uint64_t>(in, file);
        in.seekg(static_cast<std::streamoff>(points * 24), std::ios::cur);  // x, y, point3D id
        images.push_back(std::move(im));
    }
}

// Data lines of a text model file (comments and blank lines dropped unless keep_blank).
std::vector<std::string> text_lines(const std::string& file, bool keep_blank) {
    std::ifstream in(file);
    if (!in) throw Failure{file + ": cannot open"};
    std::vector<std::string> out;
    for (std::string line; std::getline(in, line);) {
        while (!line.empty() && (line.back() == '\r' || line.back() == '\n')) line.pop_back();
        if (!line.empty() && line[0] == '#') continue;
        if (line.find_first_not_of(" \t") == std::string::npos && !keep_blank) continue;
        out.push_back(line);
    }
    return out;
}

void read_text(const std::string& dir, std::map<uint32_t, Intrinsics>& cams, std::vector<Image>& images) {
    {
        const std::string file = dir + "/cameras.txt";
        for (const std::string& line : text_lines(file, false)) {
            std::istringstream s(line);
            long long id = 0, width = 0, height = 0;
            std::string name;
            if (!(s >> id >> name >> width >> height)) throw Failure{file + ": malformed camera line '" + line + "'"};
            int model = -1;
            for (int m = 0; m < 11; ++m)
                if (name == kModelNames[m]) model = m;
            if (model < 0) throw Failure{file + ": unknown camera model " + name};
            std::vector<double> p(kModelParams[model]);
            for (double& v : p)
                if (!(s >> v)) throw Failure{file + ": camera " + std::to_string(id) + " has too few parameters"};
            cams[static_cast<uint32_t>(id)] = pinhole(model, p, static_cast<int>(width), static_cast<int>(height), file,
                                                      name);
        }
    }
    const std::string file = dir + "/images.txt";
    const std::vector<std::string> lines = text_lines(file, true);
    // Two lines per image: the pose line, then its 2D points (possibly an empty line).
    for (size_t i = 0; i < lines.size(); ++i) {
        if (lines[i].find_first_not_of(" \t") == std::string::npos) continue;
        std::istringstream s(lines[i]);
        Image im;
        long long id = 0, cam = 0;
        if (!(s >> id >> im.q[0] >> im.q[1] >> im.q[2] >> im.q[3] >> im.t[0] >> im.t[1] >> im.t[2] >> cam >> im.name))
            throw Failure{file + ": malformed image line '" + lines[i] + "'"};
        im.camera = static_cast<uint32_t>(cam);
        images.push_back(std::move(im));
        ++i;  // skip the points line
    }
}

}  // namespace

extern "C" int aniso_b200_colmap_load(const char* folder, aniso_b200_colmap_camera* out, int32_t capacity,
                                      int32_t* count) {
    if (!folder || !count) return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "folder/count is NULL");
    if (out && capacity < 0) return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "capacity must be >= 0");
    const std::string dir = folder;
    std::map<uint32_t, Intrinsics> cams;
    std::vector<Image> images;
    std::vector<aniso_b200_colmap_camera> result;
    try {
        std::ifstream probe(dir + "/cameras.bin", std::ios::binary);
        const bool binary = static_cast<bool>(probe);
        probe.close();
        if (binary) read_binary(dir, cams, images);
        else read_text(dir, cams, images);
        const std::string file = dir + (binary ? "/images.bin" : "/images.txt");
        for (const Image& im : images) {
            const auto it = cams.find(im.camera);
            if (it == cams.end()) throw Failure{file + ": image " + im.name + " refers to a missing camera"};
            if (im.name.size() >= sizeof(aniso_b200_colmap_camera::image_name))
                throw Failure{file + ": image name " + im.name + " is longer than 255 bytes"};
            aniso_b200_colmap_camera c{};
            std::memcpy(c.image_name, im.name.data(), im.name.size());
            c.camera.width = it->second.width;
            c.camera.height = it->second.height;
            c.camera.fx = it->second.fx;
            c.camera.fy = it->second.fy;
            c.camera.cx = it->second.cx;
            c.camera.cy = it->second.cy;
            quat_to_matrix(im.q[0], im.q[1], im.q[2], im.q[3], c.camera.R);
            for (int k = 0; k < 3; ++k) c.camera.t[k] = im.t[k];
            result.push_back(c);
        }
    } catch (const Failure& f) {
        return ab2::report_error(ANISO_B200_ERR_ARGUMENT, f.what.c_str());
    } catch (const std::exception& e) {
        return ab2::report_error(ANISO_B200_ERR_ARGUMENT, e.what());
    }
    std::stable_sort(result.begin(), result.end(), [](const aniso_b200_colmap_camera& a,
                                                      const aniso_b200_colmap_camera& b) {
        return std::strcmp(a.image_name, b.image_name) < 0;
    });
    if (result.size() > 0x7FFFFFFFu) return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "too many images");
    *count = static_cast<int32_t>(result.size());
    if (!out) return ANISO_B200_OK;
    if (capacity < *count) return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "capacity too small");
    std::copy(result.begin(), result.end(), out);
    return ANISO_B200_OK;
}
