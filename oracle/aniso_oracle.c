/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's CPU rasterizer path, used only by tests/, the smoke
 * check and bench.py's CPU-baseline leg, as the checker. The product never links it.
 *
 * Every function cites the reference file:line it restates. Arithmetic mirrors the reference's
 * types and evaluation order exactly (float vs double promotions, left-to-right sums, std::exp ->
 * expf, std::sqrt -> sqrtf), and it is compiled with the same gcc and without -mfma, so its
 * outputs equal the reference build's bit for bit; tests/test_oracle.py checks that against the
 * reference library compiled from its own sources and against the committed golden fixtures.
 *
 * Contents
 *   orc_activate        ply_loader.cpp:124-138  raw PLY values -> activated Gaussians
 *   orc_sh_color        sh.cpp:18-58            SH colour up to degree 3
 *   orc_camera_centre   camera.cpp:19-23        -R^T t in double, cast to float
 *   orc_make_splats     render.cpp:39-104       per-Gaussian projection (CPU path, double camera)
 *   orc_render          render.cpp:140-223      the whole CPU render (8x8 tiles), single thread
 *   orc_sort_keys       gpu_render.cu:148-177, 324-345
 *                                               scan, duplicate, stable sort of (tile|depth, index),
 *                                               tile ranges -- the GPU path's integer work
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_TILE_CPU 8

/* ---- ply_loader.cpp:124-138 ------------------------------------------------------------------ */
/* gauss out: n x 11 (x y z sx sy sz qw qx qy qz opacity); sh out: n x K x 3, [coeff][channel]. */
void orc_activate(int64_t n, const float* xyz, const float* f_dc, const float* f_rest, const float* opacity,
                  const float* scale, const float* rot, int degree, float* gauss, float* sh) {
    const int64_t coeffs = (int64_t)(degree + 1) * (degree + 1);
    const int64_t rest_per_channel = coeffs - 1;
    for (int64_t i = 0; i < n; ++i) {
        float* g = gauss + i * 11;
        g[0] = xyz[i * 3 + 0];
        g[1] = xyz[i * 3 + 1];
        g[2] = xyz[i * 3 + 2];
        g[3] = expf(scale[i * 3 + 0]);
        g[4] = expf(scale[i * 3 + 1]);
        g[5] = expf(scale[i * 3 + 2]);
        g[10] = 1.0f / (1.0f + expf(-opacity[i]));
        const float qw = rot[i * 4 + 0], qx = rot[i * 4 + 1], qy = rot[i * 4 + 2], qz = rot[i * 4 + 3];
        const float nrm = sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
        if (nrm > 0) {
            g[6] = qw / nrm; g[7] = qx / nrm; g[8] = qy / nrm; g[9] = qz / nrm;
        } else {
            g[6] = 1; g[7] = 0; g[8] = 0; g[9] = 0;
        }
        float* s = sh + i * coeffs * 3;
        for (int c = 0; c < 3; ++c) s[c] = f_dc[i * 3 + c];
        for (int c = 0; c < 3; ++c)
            for (int64_t k = 0; k < rest_per_channel; ++k)
                s[(k + 1) * 3 + c] = f_rest[i * 3 * rest_per_channel + c * rest_per_channel + k];
    }
}

/* ---- sh.cpp:10-14, 18-58 --------------------------------------------------------------------- */
static const float SH_C0 = 0.28209479177387814f;
static const float SH_C1 = 0.4886025119029199f;
static const float SH_C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                               -1.0925484305920792f, 0.5462742152960396f};
static const float SH_C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                               0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                               -0.5900435899266435f};

void orc_sh_color(const float* sh, int scene_degree, float x, float y, float z, int degree, float* out) {
    if (degree > scene_degree) degree = scene_degree;
    float basis[16];
    int count = 1;
    basis[0] = SH_C0;
    if (degree >= 1) {
        basis[1] = -SH_C1 * y;
        basis[2] = SH_C1 * z;
        basis[3] = -SH_C1 * x;
        count = 4;
    }
    if (degree >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        basis[4] = SH_C2[0] * x * y;
        basis[5] = SH_C2[1] * y * z;
        basis[6] = SH_C2[2] * (2 * zz - xx - yy);
        basis[7] = SH_C2[3] * x * z;
        basis[8] = SH_C2[4] * (xx - yy);
        count = 9;
        if (degree >= 3) {
            basis[9] = SH_C3[0] * y * (3 * xx - yy);
            basis[10] = SH_C3[1] * x * y * z;
            basis[11] = SH_C3[2] * y * (4 * zz - xx - yy);
            basis[12] = SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy);
            basis[13] = SH_C3[4] * x * (4 * zz - xx - yy);
            basis[14] = SH_C3[5] * z * (xx - yy);
            basis[15] = SH_C3[6] * x * (xx - 3 * yy);
            count = 16;
        }
    }
    float rgb[3] = {0.5f, 0.5f, 0.5f};
    for (int k = 0; k < count; ++k)
        for (int c = 0; c < 3; ++c) rgb[c] += basis[k] * sh[k * 3 + c];
    for (int c = 0; c < 3; ++c) out[c] = rgb[c] < 0.0f ? 0.0f : rgb[c]; /* std::max(0.0f, v) */
}

/* ---- camera.h:16-26, camera.cpp:12-23 -------------------------------------------------------- */
/* cam: R[9] row-major, t[3], fx, fy, cx, cy (16 doubles). */
void orc_camera_centre(const double* cam, float* out) {
    const double* R = cam;
    const double* t = cam + 9;
    out[0] = (float)(-(R[0] * t[0] + R[3] * t[1] + R[6] * t[2]));
    out[1] = (float)(-(R[1] * t[0] + R[4] * t[1] + R[7] * t[2]));
    out[2] = (float)(-(R[2] * t[0] + R[5] * t[1] + R[8] * t[2]));
}

static void to_camera(const double* cam, const float* p, float* out) {
    const double* R = cam;
    const double* t = cam + 9;
    const double x = p[0], y = p[1], z = p[2];
    out[0] = (float)(R[0] * x + R[1] * y + R[2] * z + t[0]);
    out[1] = (float)(R[3] * x + R[4] * y + R[5] * z + t[1]);
    out[2] = (float)(R[6] * x + R[7] * y + R[8] * z + t[2]);
}

/* ---- render.cpp:18-25, 31-104 ---------------------------------------------------------------- */
typedef struct {
    float u, v, A, B, C, opacity, depth, rgb[3];
    int radius;
} orc_splat;

static float clampf_(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); } /* std::clamp */

static int make_splat(const float* g, const float* sh, int scene_degree, const double* cam, int width, int height,
                      const float* eye, int sh_degree, float splat_scale, orc_splat* s) {
    float p[3];
    to_camera(cam, g, p);
    if (p[2] < 0.2f) return 0;

    const float w = g[6], x = g[7], y = g[8], z = g[9];
    float R[3][3];
    R[0][0] = 1 - 2 * (y * y + z * z); R[0][1] = 2 * (x * y - w * z);     R[0][2] = 2 * (x * z + w * y);
    R[1][0] = 2 * (x * y + w * z);     R[1][1] = 1 - 2 * (x * x + z * z); R[1][2] = 2 * (y * z - w * x);
    R[2][0] = 2 * (x * z - w * y);     R[2][1] = 2 * (y * z + w * x);     R[2][2] = 1 - 2 * (x * x + y * y);
    const float sc[3] = {g[3] * splat_scale, g[4] * splat_scale, g[5] * splat_scale};
    float M[3][3], Sigma[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) M[r][c] = R[r][c] * sc[c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Sigma[r][c] = M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2];

    const double cfx = cam[12], cfy = cam[13], ccx = cam[14], ccy = cam[15];
    const float limX = 1.3f * (float)(0.5 * width / cfx);
    const float limY = 1.3f * (float)(0.5 * height / cfy);
    const float tx = clampf_(p[0] / p[2], -limX, limX) * p[2];
    const float ty = clampf_(p[1] / p[2], -limY, limY) * p[2];
    const float fx = (float)cfx, fy = (float)cfy;
    const float J[2][3] = {{fx / p[2], 0, -fx * tx / (p[2] * p[2])}, {0, fy / p[2], -fy * ty / (p[2] * p[2])}};
    float T[2][3];
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c)
            T[r][c] = J[r][0] * (float)cam[0 * 3 + c] + J[r][1] * (float)cam[1 * 3 + c] + J[r][2] * (float)cam[2 * 3 + c];
    float TS[2][3];
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c) TS[r][c] = T[r][0] * Sigma[0][c] + T[r][1] * Sigma[1][c] + T[r][2] * Sigma[2][c];
    const float a = TS[0][0] * T[0][0] + TS[0][1] * T[0][1] + TS[0][2] * T[0][2] + 0.3f;
    const float b = TS[0][0] * T[1][0] + TS[0][1] * T[1][1] + TS[0][2] * T[1][2];
    const float c = TS[1][0] * T[1][0] + TS[1][1] * T[1][1] + TS[1][2] * T[1][2] + 0.3f;

    const float det = a * c - b * b;
    if (det <= 0) return 0;
    s->A = c / det;
    s->B = -b / det;
    s->C = a / det;

    const float mid = 0.5f * (a + c);
    const float m2 = mid * mid - det;
    const float lambda = mid + sqrtf(0.1f < m2 ? m2 : 0.1f); /* std::max(0.1f, ...) */
    s->radius = (int)ceilf(3.0f * sqrtf(lambda));

    s->u = fx * p[0] / p[2] + (float)ccx;
    s->v = fy * p[1] / p[2] + (float)ccy;
    if (s->u + s->radius < 0 || s->v + s->radius < 0 || s->u - s->radius >= width || s->v - s->radius >= height)
        return 0;

    s->depth = p[2];
    s->opacity = g[10];
    float d[3] = {g[0] - eye[0], g[1] - eye[1], g[2] - eye[2]};
    const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    d[0] = d[0] / len; d[1] = d[1] / len; d[2] = d[2] / len;
    orc_sh_color(sh, scene_degree, d[0], d[1], d[2], sh_degree, s->rgb);
    return 1;
}

/* out: n x 10 floats (u, v, A, B, C, opacity, depth, r, g, b); radius n ints; alive n bytes. */
void orc_make_splats(int64_t n, const float* gauss, const float* sh, int scene_degree, const double* cam, int width,
                     int height, int sh_degree, float splat_scale, float* out, int32_t* radius, uint8_t* alive) {
    float eye[3];
    orc_camera_centre(cam, eye);
    const int64_t stride = (int64_t)(scene_degree + 1) * (scene_degree + 1) * 3;
    for (int64_t i = 0; i < n; ++i) {
        orc_splat s;
        memset(&s, 0, sizeof s);
        const int ok = make_splat(gauss + i * 11, sh + i * stride, scene_degree, cam, width, height, eye, sh_degree,
                                  splat_scale, &s);
        float* o = out + i * 10;
        o[0] = s.u; o[1] = s.v; o[2] = s.A; o[3] = s.B; o[4] = s.C;
        o[5] = s.opacity; o[6] = s.depth; o[7] = s.rgb[0]; o[8] = s.rgb[1]; o[9] = s.rgb[2];
        radius[i] = s.radius;
        alive[i] = (uint8_t)ok;
    }
}

/* ---- render.cpp:119-136: stable LSD sort of indices by depth bits, 11 bits per pass ----------- */
static void radix_sort_by_depth(uint32_t* order, size_t n, const orc_splat* splats) {
    uint32_t* keys = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t* keys_tmp = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t* idx_tmp = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    for (size_t i = 0; i < n; ++i) memcpy(&keys[i], &splats[order[i]].depth, sizeof(float));
    for (int shift = 0; shift < 32; shift += 11) {
        uint32_t count[2049];
        memset(count, 0, sizeof count);
        for (size_t i = 0; i < n; ++i) ++count[((keys[i] >> shift) & 2047) + 1];
        for (int b = 0; b < 2048; ++b) count[b + 1] += count[b];
        for (size_t i = 0; i < n; ++i) {
            const uint32_t dst = count[(keys[i] >> shift) & 2047]++;
            keys_tmp[dst] = keys[i];
            idx_tmp[dst] = order[i];
        }
        uint32_t* t = keys; keys = keys_tmp; keys_tmp = t;
        memcpy(order, idx_tmp, n * sizeof(uint32_t));
    }
    free(keys); free(keys_tmp); free(idx_tmp);
}

static void tile_range8(const orc_splat* s, int tiles_x, int tiles_y, int* x0, int* y0, int* x1, int* y1) {
    int a;
    a = (int)(s->u - s->radius) / ORC_TILE_CPU; *x0 = a > 0 ? a : 0;
    a = (int)(s->v - s->radius) / ORC_TILE_CPU; *y0 = a > 0 ? a : 0;
    a = (int)(s->u + s->radius) / ORC_TILE_CPU; *x1 = a < tiles_x - 1 ? a : tiles_x - 1;
    a = (int)(s->v + s->radius) / ORC_TILE_CPU; *y1 = a < tiles_y - 1 ? a : tiles_y - 1;
}

/* ---- render.cpp:140-223: the CPU render. stats: visible, tilePairs (8x8). ------------------- */
int orc_render(int64_t n, const float* gauss, const float* sh, int scene_degree, const double* cam, int width,
               int height, int sh_degree, float splat_scale, uint8_t* out_rgb, int64_t* stats) {
    float eye[3];
    orc_camera_centre(cam, eye);
    const int64_t stride = (int64_t)(scene_degree + 1) * (scene_degree + 1) * 3;
    orc_splat* splats = (orc_splat*)calloc(n ? (size_t)n : 1, sizeof(orc_splat));
    uint32_t* order = (uint32_t*)malloc((n ? (size_t)n : 1) * sizeof(uint32_t));
    if (!splats || !order) return 1;
    size_t visible = 0;
    for (int64_t i = 0; i < n; ++i)
        if (make_splat(gauss + i * 11, sh + i * stride, scene_degree, cam, width, height, eye, sh_degree, splat_scale,
                       &splats[i]))
            order[visible++] = (uint32_t)i;
    radix_sort_by_depth(order, visible, splats);

    const int tiles_x = (width + ORC_TILE_CPU - 1) / ORC_TILE_CPU, tiles_y = (height + ORC_TILE_CPU - 1) / ORC_TILE_CPU;
    const size_t tile_count = (size_t)tiles_x * tiles_y;
    uint32_t* start = (uint32_t*)calloc(tile_count + 1, sizeof(uint32_t));
    for (size_t k = 0; k < visible; ++k) {
        int x0, y0, x1, y1;
        tile_range8(&splats[order[k]], tiles_x, tiles_y, &x0, &y0, &x1, &y1);
        for (int ty = y0; ty <= y1; ++ty)
            for (int tx = x0; tx <= x1; ++tx) ++start[(size_t)ty * tiles_x + tx + 1];
    }
    for (size_t t = 0; t < tile_count; ++t) start[t + 1] += start[t];
    const size_t pairs = start[tile_count];
    uint32_t* binned = (uint32_t*)malloc((pairs ? pairs : 1) * sizeof(uint32_t));
    uint32_t* fill = (uint32_t*)malloc((tile_count ? tile_count : 1) * sizeof(uint32_t));
    memcpy(fill, start, tile_count * sizeof(uint32_t));
    for (size_t k = 0; k < visible; ++k) {
        int x0, y0, x1, y1;
        tile_range8(&splats[order[k]], tiles_x, tiles_y, &x0, &y0, &x1, &y1);
        for (int ty = y0; ty <= y1; ++ty)
            for (int tx = x0; tx <= x1; ++tx) binned[fill[(size_t)ty * tiles_x + tx]++] = order[k];
    }

    memset(out_rgb, 0, (size_t)width * height * 3);
    for (size_t t = 0; t < tile_count; ++t) {
        const int tx = (int)(t % tiles_x), ty = (int)(t / tiles_x);
        const uint32_t* first = binned + start[t];
        const uint32_t* last = binned + start[t + 1];
        const int ye = (ty + 1) * ORC_TILE_CPU < height ? (ty + 1) * ORC_TILE_CPU : height;
        const int xe = (tx + 1) * ORC_TILE_CPU < width ? (tx + 1) * ORC_TILE_CPU : width;
        for (int y = ty * ORC_TILE_CPU; y < ye; ++y) {
            for (int x = tx * ORC_TILE_CPU; x < xe; ++x) {
                const float px = x + 0.5f, py = y + 0.5f;
                float T = 1.0f, C[3] = {0, 0, 0};
                for (const uint32_t* it = first; it != last; ++it) {
                    const orc_splat* s = &splats[*it];
                    const float dx = px - s->u, dy = py - s->v;
                    const float power = -0.5f * (s->A * dx * dx + s->C * dy * dy) - s->B * dx * dy;
                    if (power > 0) continue;
                    const float e = s->opacity * expf(power);
                    const float alpha = 0.99f < e ? 0.99f : e; /* std::min(0.99f, e) */
                    if (alpha < 1.0f / 255.0f) continue;
                    const float next_t = T * (1 - alpha);
                    if (next_t < 1e-4f) break;
                    for (int k = 0; k < 3; ++k) C[k] += s->rgb[k] * alpha * T;
                    T = next_t;
                }
                uint8_t* o = out_rgb + ((size_t)y * width + x) * 3;
                for (int k = 0; k < 3; ++k) o[k] = (uint8_t)(clampf_(C[k], 0.0f, 1.0f) * 255.0f + 0.5f);
            }
        }
    }
    if (stats) {
        stats[0] = (int64_t)visible;
        stats[1] = (int64_t)pairs;
    }
    free(splats); free(order); free(start); free(binned); free(fill);
    return 0;
}

/* ---- gpu_render.cu:148-177 and 324-345: the GPU path's integer work --------------------------- */
/* Given one projection (per Gaussian: tiles_touched, rect x0 y0 x1 y1, depth), produce what the
 * reference produces: keys (tile << 32 | depth bits) and values (Gaussian index) in the order of a
 * stable radix sort of the index-ordered duplicated list, and ranges[tile] = [start, end) with
 * empty tiles {0, 0}. Returns the pair count, or -1 if it exceeds capacity. */
int64_t orc_sort_keys(int64_t n, const uint32_t* tiles_touched, const uint32_t* rect, const float* depth, int tiles_x,
                      int tiles_y, uint64_t* keys, uint32_t* values, int64_t capacity, uint32_t* ranges) {
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) total += tiles_touched[i];
    const int64_t tile_count = (int64_t)tiles_x * tiles_y;
    memset(ranges, 0, (size_t)tile_count * 2 * sizeof(uint32_t));
    if (total > capacity) return -1;
    uint64_t* k0 = keys;
    uint32_t* v0 = values;
    int64_t out = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (tiles_touched[i] == 0) continue;
        uint32_t bits;
        memcpy(&bits, &depth[i], 4);
        const uint32_t* r = rect + i * 4;
        for (uint32_t ty = r[1]; ty <= r[3]; ++ty)
            for (uint32_t tx = r[0]; tx <= r[2]; ++tx) {
                k0[out] = ((uint64_t)(ty * (uint32_t)tiles_x + tx) << 32) | bits;
                v0[out] = (uint32_t)i;
                ++out;
            }
    }
    /* Stable LSD radix over bits [0, 32 + bitsFor(tileCount)), 16-bit digits. */
    int tile_bits = 0;
    while (tile_bits < 32 && (1u << tile_bits) <= (uint32_t)tile_count) ++tile_bits;
    const int end_bit = 32 + tile_bits;
    uint64_t* k1 = (uint64_t*)malloc((total ? total : 1) * sizeof(uint64_t));
    uint32_t* v1 = (uint32_t*)malloc((total ? total : 1) * sizeof(uint32_t));
    uint32_t* count = (uint32_t*)malloc((65536 + 1) * sizeof(uint32_t));
    uint64_t* ks = k0; uint32_t* vs = v0; uint64_t* kd = k1; uint32_t* vd = v1;
    for (int shift = 0; shift < end_bit; shift += 16) {
        const int bits = end_bit - shift < 16 ? end_bit - shift : 16;
        const uint64_t mask = (1ull << bits) - 1;
        memset(count, 0, (65536 + 1) * sizeof(uint32_t));
        for (int64_t i = 0; i < total; ++i) ++count[((ks[i] >> shift) & mask) + 1];
        for (int b = 0; b < 65536; ++b) count[b + 1] += count[b];
        for (int64_t i = 0; i < total; ++i) {
            const uint32_t dst = count[(ks[i] >> shift) & mask]++;
            kd[dst] = ks[i];
            vd[dst] = vs[i];
        }
        uint64_t* tk = ks; ks = kd; kd = tk;
        uint32_t* tv = vs; vs = vd; vd = tv;
    }
    if (ks != keys) {
        memcpy(keys, ks, (size_t)total * sizeof(uint64_t));
        memcpy(values, vs, (size_t)total * sizeof(uint32_t));
    }
    free(k1); free(v1); free(count);
    for (int64_t i = 0; i < total; ++i) {
        const uint32_t tile = (uint32_t)(keys[i] >> 32);
        if (i == 0) ranges[tile * 2 + 0] = 0;
        else {
            const uint32_t prev = (uint32_t)(keys[i - 1] >> 32);
            if (prev != tile) {
                ranges[prev * 2 + 1] = (uint32_t)i;
                ranges[tile * 2 + 0] = (uint32_t)i;
            }
        }
        if (i == total - 1) ranges[tile * 2 + 1] = (uint32_t)total;
    }
    return total;
}

/* ==== FP64 forward and adjoint of the training render (the gradient oracle) ====================
 *
 * The same algorithm as the CPU renderer (render.cpp:39-104 projection, 8x8-tile lists from the
 * 3-sigma rectangles render.cpp:166-171, depth order with index ties, render.cpp:195-220 blending
 * and thresholds), evaluated in double from the optimizer's raw parameters (exp scale, sigmoid
 * opacity, normalised quaternion), producing the unclamped colour. The adjoint is derived by hand
 * from the same equations. Camera values are rounded to float first, as the GPU path packs them
 * (gpu_render.cu:301-316), so both evaluate the same function.
 * params: means n x 3, log_scales n x 3, quats n x 4 (w first), logits n, sh n x K x 3. */

typedef struct {
    double R[9], t[3], eye[3], fx, fy, cx, cy;
    int w, h;
} orc_cam64;

static orc_cam64 cam64(const double* cam, int w, int h) {
    orc_cam64 c;
    for (int k = 0; k < 9; ++k) c.R[k] = (float)cam[k];
    for (int k = 0; k < 3; ++k) c.t[k] = (float)cam[9 + k];
    float e[3];
    orc_camera_centre(cam, e);
    for (int k = 0; k < 3; ++k) c.eye[k] = e[k];
    c.fx = (float)cam[12]; c.fy = (float)cam[13]; c.cx = (float)cam[14]; c.cy = (float)cam[15];
    c.w = w; c.h = h;
    return c;
}

typedef struct {
    int alive, x0, y0, x1, y1;      /* 8x8-tile rectangle */
    float depth32;                   /* ordering key */
    double u, v, A, B, C, o, rgb[3], pre[3];
    /* intermediates for the adjoint */
    double p[3], pc[3], qn[4], qlen, s[3], Rq[9], M[9], S[9], T[6], a, b, c, det, dir[3], len;
    int clx, cly;
} orc_sp64;

static void sh_basis64(double x, double y, double z, int D, double* b, double* bx, double* by, double* bz) {
    const double C0 = 0.28209479177387814, C1 = 0.4886025119029199;
    const double C20 = 1.0925484305920792, C21 = -1.0925484305920792, C22 = 0.31539156525252005,
                 C23 = -1.0925484305920792, C24 = 0.5462742152960396;
    const double C30 = -0.5900435899266435, C31 = 2.890611442640554, C32 = -0.4570457994644658,
                 C33 = 0.3731763325901154, C34 = -0.4570457994644658, C35 = 1.445305721320277,
                 C36 = -0.5900435899266435;
    for (int k = 0; k < 16; ++k) b[k] = bx[k] = by[k] = bz[k] = 0;
    b[0] = C0;
    if (D >= 1) { b[1] = -C1 * y; by[1] = -C1; b[2] = C1 * z; bz[2] = C1; b[3] = -C1 * x; bx[3] = -C1; }
    if (D >= 2) {
        const double xx = x * x, yy = y * y, zz = z * z;
        b[4] = C20 * x * y; bx[4] = C20 * y; by[4] = C20 * x;
        b[5] = C21 * y * z; by[5] = C21 * z; bz[5] = C21 * y;
        b[6] = C22 * (2 * zz - xx - yy); bx[6] = -2 * C22 * x; by[6] = -2 * C22 * y; bz[6] = 4 * C22 * z;
        b[7] = C23 * x * z; bx[7] = C23 * z; bz[7] = C23 * x;
        b[8] = C24 * (xx - yy); bx[8] = 2 * C24 * x; by[8] = -2 * C24 * y;
        if (D >= 3) {
            b[9] = C30 * y * (3 * xx - yy); bx[9] = 6 * C30 * x * y; by[9] = C30 * (3 * xx - 3 * yy);
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

static void splat64(const orc_cam64* cam, const double* means, const double* log_scales, const double* quats,
                    const double* logits, const double* sh, int K, int D, double splat_scale, int64_t i,
                    orc_sp64* s) {
    memset(s, 0, sizeof *s);
    const double* R = cam->R;
    for (int k = 0; k < 3; ++k) s->p[k] = means[3 * i + k];
    for (int r = 0; r < 3; ++r)
        s->pc[r] = R[3 * r] * s->p[0] + R[3 * r + 1] * s->p[1] + R[3 * r + 2] * s->p[2] + cam->t[r];
    const double px = s->pc[0], py = s->pc[1], pz = s->pc[2];
    if (pz < 0.2) return;
    const double* q = quats + 4 * i;
    s->qlen = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int k = 0; k < 4; ++k) s->qn[k] = s->qlen > 0 ? q[k] / s->qlen : (k == 0);
    const double w = s->qn[0], x = s->qn[1], y = s->qn[2], z = s->qn[3];
    double* Rq = s->Rq;
    Rq[0] = 1 - 2 * (y * y + z * z); Rq[1] = 2 * (x * y - w * z); Rq[2] = 2 * (x * z + w * y);
    Rq[3] = 2 * (x * y + w * z); Rq[4] = 1 - 2 * (x * x + z * z); Rq[5] = 2 * (y * z - w * x);
    Rq[6] = 2 * (x * z - w * y); Rq[7] = 2 * (y * z + w * x); Rq[8] = 1 - 2 * (x * x + y * y);
    for (int k = 0; k < 3; ++k) s->s[k] = exp(log_scales[3 * i + k]) * splat_scale;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) s->M[3 * r + c] = Rq[3 * r + c] * s->s[c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            s->S[3 * r + c] = s->M[3 * r] * s->M[3 * c] + s->M[3 * r + 1] * s->M[3 * c + 1] + s->M[3 * r + 2] * s->M[3 * c + 2];
    const double limX = 1.3 * 0.5 * cam->w / cam->fx, limY = 1.3 * 0.5 * cam->h / cam->fy;
    double rx = px / pz, ry = py / pz;
    s->clx = rx < -limX || rx > limX;
    s->cly = ry < -limY || ry > limY;
    rx = rx < -limX ? -limX : (rx > limX ? limX : rx);
    ry = ry < -limY ? -limY : (ry > limY ? limY : ry);
    const double tx = rx * pz, ty = ry * pz;
    const double J[6] = {cam->fx / pz, 0, -cam->fx * tx / (pz * pz), 0, cam->fy / pz, -cam->fy * ty / (pz * pz)};
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c) s->T[3 * r + c] = J[3 * r] * R[c] + J[3 * r + 1] * R[3 + c] + J[3 * r + 2] * R[6 + c];
    double ST[6];
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c)
            ST[3 * r + c] = s->S[3 * c] * s->T[3 * r] + s->S[3 * c + 1] * s->T[3 * r + 1] + s->S[3 * c + 2] * s->T[3 * r + 2];
    s->a = s->T[0] * ST[0] + s->T[1] * ST[1] + s->T[2] * ST[2] + 0.3;
    s->b = s->T[3] * ST[0] + s->T[4] * ST[1] + s->T[5] * ST[2];
    s->c = s->T[3] * ST[3] + s->T[4] * ST[4] + s->T[5] * ST[5] + 0.3;
    s->det = s->a * s->c - s->b * s->b;
    if (s->det <= 0) return;
    s->A = s->c / s->det; s->B = -s->b / s->det; s->C = s->a / s->det;
    const double mid = 0.5 * (s->a + s->c);
    const double m2 = mid * mid - s->det;
    const int radius = (int)ceil(3.0 * sqrt(mid + sqrt(m2 > 0.1 ? m2 : 0.1)));
    s->u = cam->fx * px / pz + cam->cx;
    s->v = cam->fy * py / pz + cam->cy;
    if (s->u + radius < 0 || s->v + radius < 0 || s->u - radius >= cam->w || s->v - radius >= cam->h) return;
    const int tx8 = (cam->w + 7) / 8, ty8 = (cam->h + 7) / 8;
    int a;
    a = (int)(s->u - radius) / 8; s->x0 = a > 0 ? a : 0;
    a = (int)(s->v - radius) / 8; s->y0 = a > 0 ? a : 0;
    a = (int)(s->u + radius) / 8; s->x1 = a < tx8 - 1 ? a : tx8 - 1;
    a = (int)(s->v + radius) / 8; s->y1 = a < ty8 - 1 ? a : ty8 - 1;
    s->depth32 = (float)pz;
    s->o = 1.0 / (1.0 + exp(-logits[i]));
    double d[3] = {s->p[0] - cam->eye[0], s->p[1] - cam->eye[1], s->p[2] - cam->eye[2]};
    s->len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int k = 0; k < 3; ++k) s->dir[k] = d[k] / s->len;
    double b[16], bx[16], by[16], bz[16];
    sh_basis64(s->dir[0], s->dir[1], s->dir[2], D, b, bx, by, bz);
    const int count = (D + 1) * (D + 1);
    for (int ch = 0; ch < 3; ++ch) {
        double v = 0.5;
        for (int k = 0; k < count; ++k) v += b[k] * sh[(i * K + k) * 3 + ch];
        s->pre[ch] = v;
        s->rgb[ch] = v > 0 ? v : 0;
    }
    s->alive = 1;
}

static const orc_sp64* g_sort_sp;
static int cmp_depth_index(const void* a, const void* b) {
    const uint32_t i = *(const uint32_t*)a, j = *(const uint32_t*)b;
    const float di = g_sort_sp[i].depth32, dj = g_sort_sp[j].depth32;
    if (di < dj) return -1;
    if (di > dj) return 1;
    return i < j ? -1 : (i > j);
}

/* Shared by forward and adjoint: splats, depth order, per-8x8-tile lists. */
typedef struct {
    orc_sp64* sp;
    uint32_t* order;
    size_t visible;
} orc_frame64;

static int frame64(const orc_cam64* cam, int64_t n, const double* means, const double* log_scales, const double* quats,
                   const double* logits, const double* sh, int K, int D, double splat_scale, orc_frame64* f) {
    f->sp = (orc_sp64*)calloc(n ? (size_t)n : 1, sizeof(orc_sp64));
    f->order = (uint32_t*)malloc((n ? (size_t)n : 1) * sizeof(uint32_t));
    if (!f->sp || !f->order) return 1;
    f->visible = 0;
    for (int64_t i = 0; i < n; ++i) {
        splat64(cam, means, log_scales, quats, logits, sh, K, D, splat_scale, i, &f->sp[i]);
        if (f->sp[i].alive) f->order[f->visible++] = (uint32_t)i;
    }
    g_sort_sp = f->sp;
    qsort(f->order, f->visible, sizeof(uint32_t), cmp_depth_index);
    return 0;
}

/* Applied contributors of one pixel, front to back: (index, alpha, T before, e^power, clamped). */
typedef struct { uint32_t idx; double alpha, T, ep, dx, dy; int clamped; } orc_contrib;

static size_t pixel64(const orc_frame64* f, int x, int y, orc_contrib* out, double* col) {
    const double px = x + 0.5, py = y + 0.5;
    const int sx = x / 8, sy = y / 8;
    double T = 1.0;
    size_t n = 0;
    col[0] = col[1] = col[2] = 0;
    for (size_t k = 0; k < f->visible; ++k) {
        const orc_sp64* s = &f->sp[f->order[k]];
        if (sx < s->x0 || sx > s->x1 || sy < s->y0 || sy > s->y1) continue;
        const double dx = px - s->u, dy = py - s->v;
        const double power = -0.5 * (s->A * dx * dx + s->C * dy * dy) - s->B * dx * dy;
        if (power > 0) continue;
        const double ep = exp(power);
        const double e = s->o * ep;
        const double alpha = e < 0.99 ? e : 0.99;
        if (alpha < 1.0 / 255.0) continue;
        const double nt = T * (1 - alpha);
        if (nt < 1e-4) break;
        for (int c = 0; c < 3; ++c) col[c] += s->rgb[c] * alpha * T;
        if (out) {
            out[n].idx = f->order[k]; out[n].alpha = alpha; out[n].T = T; out[n].ep = ep;
            out[n].dx = dx; out[n].dy = dy; out[n].clamped = !(e < 0.99);
        }
        ++n;
        T = nt;
    }
    return n;
}

int orc_train_forward_f64(int64_t n, const double* means, const double* log_scales, const double* quats,
                          const double* logits, const double* sh, int K, const double* camd, int w, int h,
                          int sh_degree, double splat_scale, double* out_img) {
    const orc_cam64 cam = cam64(camd, w, h);
    int D = sh_degree;
    if (D > 3) D = 3;
    if ((D + 1) * (D + 1) > K) return 2;
    orc_frame64 f;
    if (frame64(&cam, n, means, log_scales, quats, logits, sh, K, D, splat_scale, &f)) return 1;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) pixel64(&f, x, y, NULL, out_img + ((size_t)y * w + x) * 3);
    free(f.sp);
    free(f.order);
    return 0;
}

/* The adjoint of one Gaussian's projection and colour (splat64) given the gradients of its
 * splat g[9] = d/d(u, v, A, B, C, o, r, g, b): writes its 59 raw-parameter gradients. */
static void gauss_adjoint64(const orc_cam64* cam_, const orc_sp64* s, int64_t i, const double* g,
                            const double* sh, int K, int D, double* g_means, double* g_log_scales,
                            double* g_quats, double* g_logits, double* g_sh) {
    const orc_cam64 cam = *cam_;
    const int count = (D + 1) * (D + 1);
    /* colour and SH */
    double b[16], bx[16], by[16], bz[16];
    sh_basis64(s->dir[0], s->dir[1], s->dir[2], D, b, bx, by, bz);
    double gdir[3] = {0, 0, 0};
    for (int ch = 0; ch < 3; ++ch) {
        const double gcol = s->pre[ch] > 0 ? g[6 + ch] : 0;
        for (int q = 0; q < count; ++q) {
            const double shv = sh[((size_t)i * K + q) * 3 + ch];
            g_sh[((size_t)i * K + q) * 3 + ch] = b[q] * gcol;
            gdir[0] += shv * bx[q] * gcol;
            gdir[1] += shv * by[q] * gcol;
            gdir[2] += shv * bz[q] * gcol;
        }
    }
    const double dd = s->dir[0] * gdir[0] + s->dir[1] * gdir[1] + s->dir[2] * gdir[2];
    double gm[3];
    for (int q = 0; q < 3; ++q) gm[q] = (gdir[q] - s->dir[q] * dd) / s->len;
    g_logits[i] = g[5] * s->o * (1 - s->o);
    /* conic -> 2D covariance */
    const double a = s->a, bb = s->b, c = s->c, det = s->det, id2 = 1.0 / (det * det);
    const double gA = g[2], gB = g[3], gC = g[4];
    const double ga = (-c * c * gA + bb * c * gB - bb * bb * gC) * id2;
    const double gb = (2 * bb * c * gA - (det + 2 * bb * bb) * gB + 2 * a * bb * gC) * id2;
    const double gc2 = (-bb * bb * gA + a * bb * gB - a * a * gC) * id2;
    const double* T = s->T;
    const double* S = s->S;
    double ST[6];
    for (int r = 0; r < 2; ++r)
        for (int q = 0; q < 3; ++q) ST[3 * r + q] = S[3 * q] * T[3 * r] + S[3 * q + 1] * T[3 * r + 1] + S[3 * q + 2] * T[3 * r + 2];
    double gS[9], gT[6], gJ[6];
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q)
            gS[3 * r + q] = ga * T[r] * T[q] + gb * T[r] * T[3 + q] + gc2 * T[3 + r] * T[3 + q];
    for (int q = 0; q < 3; ++q) {
        gT[q] = 2 * ga * ST[q] + gb * ST[3 + q];
        gT[3 + q] = gb * ST[q] + 2 * gc2 * ST[3 + q];
    }
    const double* W = cam.R;
    for (int r = 0; r < 2; ++r)
        for (int kk = 0; kk < 3; ++kk) gJ[3 * r + kk] = gT[3 * r] * W[3 * kk] + gT[3 * r + 1] * W[3 * kk + 1] + gT[3 * r + 2] * W[3 * kk + 2];
    const double px = s->pc[0], py = s->pc[1], pz = s->pc[2], iz = 1 / pz, iz2 = iz * iz, iz3 = iz2 * iz;
    const double limX = 1.3 * 0.5 * cam.w / cam.fx, limY = 1.3 * 0.5 * cam.h / cam.fy;
    double rx = px / pz, ry = py / pz;
    rx = rx < -limX ? -limX : (rx > limX ? limX : rx);
    ry = ry < -limY ? -limY : (ry > limY ? limY : ry);
    const double tx = rx * pz, ty = ry * pz;
    double gpx = g[0] * cam.fx * iz, gpy = g[1] * cam.fy * iz;
    double gpz = -(g[0] * cam.fx * px + g[1] * cam.fy * py) * iz2 - (gJ[0] * cam.fx + gJ[4] * cam.fy) * iz2;
    if (!s->clx) { gpx += gJ[2] * (-cam.fx * iz2); gpz += gJ[2] * (2 * cam.fx * tx * iz3); }
    else gpz += gJ[2] * (cam.fx * rx * iz2);
    if (!s->cly) { gpy += gJ[5] * (-cam.fy * iz2); gpz += gJ[5] * (2 * cam.fy * ty * iz3); }
    else gpz += gJ[5] * (cam.fy * ry * iz2);
    for (int q = 0; q < 3; ++q) gm[q] += W[q] * gpx + W[3 + q] * gpy + W[6 + q] * gpz;
    for (int q = 0; q < 3; ++q) g_means[3 * i + q] = gm[q];
    /* S = M M^T, M = R(q) diag(s) */
    const double* M = s->M;
    const double* Rq = s->Rq;
    double gM[9], gR[9];
    for (int r = 0; r < 3; ++r)
        for (int kk = 0; kk < 3; ++kk) {
            double v = 0;
            for (int q = 0; q < 3; ++q) v += (gS[3 * r + q] + gS[3 * q + r]) * M[3 * q + kk];
            gM[3 * r + kk] = v;
        }
    for (int kk = 0; kk < 3; ++kk) {
        double gsv = 0;
        for (int r = 0; r < 3; ++r) {
            gR[3 * r + kk] = gM[3 * r + kk] * s->s[kk];
            gsv += gM[3 * r + kk] * Rq[3 * r + kk];
        }
        g_log_scales[3 * i + kk] = gsv * s->s[kk];
    }
    const double qw = s->qn[0], qx = s->qn[1], qy = s->qn[2], qz = s->qn[3];
    const double gqw = 2 * (-qz * gR[1] + qy * gR[2] + qz * gR[3] - qx * gR[5] - qy * gR[6] + qx * gR[7]);
    const double gqx = 2 * (qy * gR[1] + qz * gR[2] + qy * gR[3] - 2 * qx * gR[4] - qw * gR[5] + qz * gR[6] + qw * gR[7] - 2 * qx * gR[8]);
    const double gqy = 2 * (-2 * qy * gR[0] + qx * gR[1] + qw * gR[2] + qx * gR[3] + qz * gR[5] - qw * gR[6] + qz * gR[7] - 2 * qy * gR[8]);
    const double gqz = 2 * (-2 * qz * gR[0] - qw * gR[1] + qx * gR[2] + qw * gR[3] - 2 * qz * gR[4] + qy * gR[5] + qx * gR[6] + qy * gR[7]);
    const double dq = qw * gqw + qx * gqx + qy * gqy + qz * gqz;
    const double il = s->qlen > 0 ? 1 / s->qlen : 0;
    g_quats[4 * i] = (gqw - qw * dq) * il;
    g_quats[4 * i + 1] = (gqx - qx * dq) * il;
    g_quats[4 * i + 2] = (gqy - qy * dq) * il;
    g_quats[4 * i + 3] = (gqz - qz * dq) * il;
}

int orc_train_backward_f64(int64_t n, const double* means, const double* log_scales, const double* quats,
                           const double* logits, const double* sh, int K, const double* camd, int w, int h,
                           int sh_degree, double splat_scale, const double* grad_img, double* g_means,
                           double* g_log_scales, double* g_quats, double* g_logits, double* g_sh) {
    const orc_cam64 cam = cam64(camd, w, h);
    int D = sh_degree;
    if (D > 3) D = 3;
    if ((D + 1) * (D + 1) > K) return 2;
    orc_frame64 f;
    if (frame64(&cam, n, means, log_scales, quats, logits, sh, K, D, splat_scale, &f)) return 1;
    /* per-splat 2D gradients: u, v, A, B, C, o, r, g, b */
    double* g2 = (double*)calloc((n ? (size_t)n : 1) * 9, sizeof(double));
    orc_contrib* cl = (orc_contrib*)malloc((f.visible ? f.visible : 1) * sizeof(orc_contrib));
    if (!g2 || !cl) return 1;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            double col[3];
            const size_t m = pixel64(&f, x, y, cl, col);
            const double* gc = grad_img + ((size_t)y * w + x) * 3;
            double acc[3] = {0, 0, 0};
            for (size_t q = m; q-- > 0;) {
                const orc_contrib* c = &cl[q];
                const orc_sp64* s = &f.sp[c->idx];
                double* g = g2 + (size_t)c->idx * 9;
                const double wgt = c->alpha * c->T;
                double dalpha = 0;
                for (int ch = 0; ch < 3; ++ch) {
                    g[6 + ch] += gc[ch] * wgt;
                    dalpha += gc[ch] * (s->rgb[ch] * c->T - acc[ch] / (1 - c->alpha));
                    acc[ch] += s->rgb[ch] * wgt;
                }
                if (c->clamped) continue;
                /* alpha = o e^power */
                g[5] += dalpha * c->ep;
                const double dpow = dalpha * c->alpha;
                const double dx = c->dx, dy = c->dy;
                g[2] += dpow * (-0.5 * dx * dx);
                g[3] += dpow * (-dx * dy);
                g[4] += dpow * (-0.5 * dy * dy);
                g[0] += dpow * (s->A * dx + s->B * dy);  /* d power / d u */
                g[1] += dpow * (s->C * dy + s->B * dx);
            }
        }
    for (size_t k = 0; k < f.visible; ++k) {
        const uint32_t i = f.order[k];
        gauss_adjoint64(&cam, &f.sp[i], i, g2 + (size_t)i * 9, sh, K, D, g_means, g_log_scales, g_quats,
                        g_logits, g_sh);
    }
    free(g2);
    free(cl);
    free(f.sp);
    free(f.order);
    return 0;
}

/* ==== FP64 training render at full size: local queries for the gradient checks ===================
 *
 * The function of orc_train_forward_f64 / orc_train_backward_f64 (the same splat64, blending and
 * thresholds) on scenes of millions of Gaussians, where every pixel against every splat is out of
 * reach: the visible splats are kept in (depth, index) order with one list per 8x8 tile, the
 * binning of render.cpp:159-190, and each query touches only the pixels it needs.
 *   orc_big_create / orc_big_destroy   the frame: projection, depth order, tile lists
 *   orc_big_image                      the FP64 colour of a pixel window
 *   orc_big_adjoint                    the adjoint of a loss on a pixel window (dL/dcolour given
 *                                      there): the raw-parameter gradients of every Gaussian
 *   orc_big_fd                         the central difference, in one raw parameter, of the
 *                                      whole-image L2 loss against a target, evaluated on the
 *                                      pixels its Gaussian can reach (no other pixel changes), and
 *                                      whether the renderer takes the same branches at +h and -h
 *                                      (alpha cut, 0.99 clamp, early termination, depth order,
 *                                      tile rectangle, SH clamp, Jacobian clip): if not, the loss
 *                                      is not smooth on [-h, h] and the difference measures a jump.
 * Parameters are the caller's float64 arrays (orc_train_forward_f64's layout), which must outlive
 * the frame. */

typedef struct {
    double u, v, A, B, C, o, rgb[3];
    float depth32;
    uint32_t idx;
    int x0, y0, x1, y1;
} orc_bl64;

typedef struct {
    orc_cam64 cam;
    int D, K;
    double splat_scale;
    int64_t n;
    const double *means, *log_scales, *quats, *logits, *sh;
    orc_bl64* rec;          /* visible splats in (depth32, index) order */
    size_t visible;
    int tx8, ty8;
    uint64_t* tile_start;   /* tx8 * ty8 + 1 */
    uint32_t* tile_list;    /* positions in rec, ascending within each tile (= depth order) */
} orc_big64;

static void to_bl64(const orc_sp64* s, int64_t i, orc_bl64* r) {
    r->u = s->u; r->v = s->v; r->A = s->A; r->B = s->B; r->C = s->C; r->o = s->o;
    for (int c = 0; c < 3; ++c) r->rgb[c] = s->rgb[c];
    r->depth32 = s->depth32;
    r->idx = (uint32_t)i;
    r->x0 = s->x0; r->y0 = s->y0; r->x1 = s->x1; r->y1 = s->y1;
}

static int cmp_bl64(const void* a, const void* b) {
    const orc_bl64* p = (const orc_bl64*)a;
    const orc_bl64* q = (const orc_bl64*)b;
    if (p->depth32 < q->depth32) return -1;
    if (p->depth32 > q->depth32) return 1;
    return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

void orc_big_destroy(void* h) {
    orc_big64* f = (orc_big64*)h;
    if (!f) return;
    free(f->rec);
    free(f->tile_start);
    free(f->tile_list);
    free(f);
}

void* orc_big_create(int64_t n, const double* means, const double* log_scales, const double* quats,
                     const double* logits, const double* sh, int K, const double* camd, int w, int h, int sh_degree,
                     double splat_scale) {
    orc_big64* f = (orc_big64*)calloc(1, sizeof *f);
    if (!f) return NULL;
    f->cam = cam64(camd, w, h);
    f->D = sh_degree > 3 ? 3 : sh_degree;
    f->K = K;
    f->splat_scale = splat_scale;
    f->n = n;
    f->means = means; f->log_scales = log_scales; f->quats = quats; f->logits = logits; f->sh = sh;
    if ((f->D + 1) * (f->D + 1) > K) { free(f); return NULL; }
    f->rec = (orc_bl64*)malloc((n ? (size_t)n : 1) * sizeof(orc_bl64));
    f->tx8 = (w + 7) / 8;
    f->ty8 = (h + 7) / 8;
    const size_t T = (size_t)f->tx8 * f->ty8;
    f->tile_start = (uint64_t*)calloc(T + 1, sizeof(uint64_t));
    if (!f->rec || !f->tile_start) { orc_big_destroy(f); return NULL; }
    orc_sp64 s;
    for (int64_t i = 0; i < n; ++i) {
        splat64(&f->cam, means, log_scales, quats, logits, sh, K, f->D, splat_scale, i, &s);
        if (s.alive) to_bl64(&s, i, &f->rec[f->visible++]);
    }
    qsort(f->rec, f->visible, sizeof(orc_bl64), cmp_bl64);
    for (size_t k = 0; k < f->visible; ++k) {
        const orc_bl64* r = &f->rec[k];
        for (int ty = r->y0; ty <= r->y1; ++ty)
            for (int tx = r->x0; tx <= r->x1; ++tx) ++f->tile_start[(size_t)ty * f->tx8 + tx + 1];
    }
    for (size_t t = 0; t < T; ++t) f->tile_start[t + 1] += f->tile_start[t];
    f->tile_list = (uint32_t*)malloc((f->tile_start[T] ? f->tile_start[T] : 1) * sizeof(uint32_t));
    uint64_t* fill = (uint64_t*)malloc((T ? T : 1) * sizeof(uint64_t));
    if (!f->tile_list || !fill) { free(fill); orc_big_destroy(f); return NULL; }
    memcpy(fill, f->tile_start, T * sizeof(uint64_t));
    for (size_t k = 0; k < f->visible; ++k) {
        const orc_bl64* r = &f->rec[k];
        for (int ty = r->y0; ty <= r->y1; ++ty)
            for (int tx = r->x0; tx <= r->x1; ++tx) f->tile_list[fill[(size_t)ty * f->tx8 + tx]++] = (uint32_t)k;
    }
    free(fill);
    return f;
}

/* Counts of the frame: visible splats and (splat, 8x8 tile) pairs. */
void orc_big_counts(const void* h, int64_t* visible, int64_t* pairs) {
    const orc_big64* f = (const orc_big64*)h;
    *visible = (int64_t)f->visible;
    *pairs = (int64_t)f->tile_start[(size_t)f->tx8 * f->ty8];
}

static uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
    return x;
}

static int key_less64(float da, uint32_t ia, float db, uint32_t ib) { return da < db || (da == db && ia < ib); }

/* One contributor of a pixel, for the adjoint: rec position (or -1 for the variant), alpha, T before,
 * e^power, offsets, clamped. */
typedef struct { int64_t pos; double alpha, T, ep, dx, dy; int clamped; } orc_bc64;

/* Pixel (x, y) front to back (pixel64's rules). Gaussian `skip` (if >= 0) is left out and `var`
 * (if not NULL) takes part in its place at its own (depth, index) position. col: colour; sig: a
 * hash of the branches taken (applied contributors with their clamp state, the terminating
 * splat); out (may be NULL): the applied contributors. Returns their count. */
static size_t big_pixel(const orc_big64* f, int x, int y, int64_t skip, const orc_bl64* var, double* col,
                        uint64_t* sig, orc_bc64* out) {
    const double px = x + 0.5, py = y + 0.5;
    const int tx = x / 8, ty = y / 8;
    const size_t t = (size_t)ty * f->tx8 + tx;
    uint64_t q = f->tile_start[t];
    const uint64_t qe = f->tile_start[t + 1];
    int var_in = var && tx >= var->x0 && tx <= var->x1 && ty >= var->y0 && ty <= var->y1;
    double T = 1.0;
    uint64_t hsh = 0x9e3779b97f4a7c15ull;
    size_t m = 0;
    col[0] = col[1] = col[2] = 0;
    for (;;) {
        const orc_bl64* c = NULL;
        while (q < qe) {
            c = &f->rec[f->tile_list[q]];
            if ((int64_t)c->idx == skip) { ++q; c = NULL; continue; }
            break;
        }
        const orc_bl64* s;
        int64_t pos;
        if (var_in && (!c || key_less64(var->depth32, var->idx, c->depth32, c->idx))) {
            s = var; pos = -1; var_in = 0;
        } else if (c) {
            s = c; pos = (int64_t)f->tile_list[q]; ++q;
        } else {
            break;
        }
        const double dx = px - s->u, dy = py - s->v;
        const double power = -0.5 * (s->A * dx * dx + s->C * dy * dy) - s->B * dx * dy;
        if (power > 0) continue;
        const double ep = exp(power);
        const double e = s->o * ep;
        const double alpha = e < 0.99 ? e : 0.99;
        if (alpha < 1.0 / 255.0) continue;
        const double nt = T * (1 - alpha);
        if (nt < 1e-4) {
            hsh = mix64(hsh ^ (0x8000000000000000ull | s->idx));
            break;
        }
        for (int ch = 0; ch < 3; ++ch) col[ch] += s->rgb[ch] * alpha * T;
        hsh = mix64(hsh ^ ((uint64_t)s->idx << 1 | (uint64_t)!(e < 0.99)));
        if (out) {
            out[m].pos = pos; out[m].alpha = alpha; out[m].T = T; out[m].ep = ep;
            out[m].dx = dx; out[m].dy = dy; out[m].clamped = !(e < 0.99);
        }
        ++m;
        T = nt;
    }
    if (sig) *sig += mix64(hsh ^ ((uint64_t)y << 32 | (uint32_t)x));
    return m;
}

/* FP64 colour of the window [x0, x0 + ww) x [y0, y0 + wh): out ww * wh * 3 doubles. */
int orc_big_image(const void* h, int x0, int y0, int ww, int wh, double* out) {
    const orc_big64* f = (const orc_big64*)h;
    if (x0 < 0 || y0 < 0 || ww < 0 || wh < 0 || x0 + ww > f->cam.w || y0 + wh > f->cam.h) return 1;
    for (int y = 0; y < wh; ++y)
        for (int x = 0; x < ww; ++x) big_pixel(f, x0 + x, y0 + y, -1, NULL, out + ((size_t)y * ww + x) * 3, NULL, NULL);
    return 0;
}

/* The adjoint of a loss whose gradient with respect to the colour is grad (ww * wh * 3 doubles) on the
 * window and zero elsewhere: adds nothing, writes the raw-parameter gradients of every Gaussian that
 * contributes to a window pixel (the others are left as the caller set them, normally zero). */
int orc_big_adjoint(const void* h, int x0, int y0, int ww, int wh, const double* grad, double* g_means,
                    double* g_log_scales, double* g_quats, double* g_logits, double* g_sh) {
    const orc_big64* f = (const orc_big64*)h;
    if (x0 < 0 || y0 < 0 || ww < 0 || wh < 0 || x0 + ww > f->cam.w || y0 + wh > f->cam.h) return 1;
    double* g2 = (double*)calloc((f->visible ? f->visible : 1) * 9, sizeof(double));
    unsigned char* touched = (unsigned char*)calloc(f->visible ? f->visible : 1, 1);
    orc_bc64* cl = (orc_bc64*)malloc((f->visible ? f->visible : 1) * sizeof(orc_bc64));
    if (!g2 || !touched || !cl) { free(g2); free(touched); free(cl); return 2; }
    for (int y = 0; y < wh; ++y)
        for (int x = 0; x < ww; ++x) {
            double col[3];
            const size_t m = big_pixel(f, x0 + x, y0 + y, -1, NULL, col, NULL, cl);
            const double* gc = grad + ((size_t)y * ww + x) * 3;
            double acc[3] = {0, 0, 0};
            for (size_t q = m; q-- > 0;) {
                const orc_bc64* c = &cl[q];
                const orc_bl64* s = &f->rec[c->pos];
                double* g = g2 + (size_t)c->pos * 9;
                touched[c->pos] = 1;
                const double wgt = c->alpha * c->T;
                double dalpha = 0;
                for (int ch = 0; ch < 3; ++ch) {
                    g[6 + ch] += gc[ch] * wgt;
                    dalpha += gc[ch] * (s->rgb[ch] * c->T - acc[ch] / (1 - c->alpha));
                    acc[ch] += s->rgb[ch] * wgt;
                }
                if (c->clamped) continue;
                g[5] += dalpha * c->ep;
                const double dpow = dalpha * c->alpha;
                const double dx = c->dx, dy = c->dy;
                g[2] += dpow * (-0.5 * dx * dx);
                g[3] += dpow * (-dx * dy);
                g[4] += dpow * (-0.5 * dy * dy);
                g[0] += dpow * (s->A * dx + s->B * dy);
                g[1] += dpow * (s->C * dy + s->B * dx);
            }
        }
    orc_sp64 s;
    for (size_t k = 0; k < f->visible; ++k) {
        if (!touched[k]) continue;
        const int64_t i = f->rec[k].idx;
        splat64(&f->cam, f->means, f->log_scales, f->quats, f->logits, f->sh, f->K, f->D, f->splat_scale, i, &s);
        gauss_adjoint64(&f->cam, &s, i, g2 + k * 9, f->sh, f->K, f->D, g_means, g_log_scales, g_quats, g_logits,
                        g_sh);
    }
    free(g2);
    free(touched);
    free(cl);
    return 0;
}

/* The splat of Gaussian i with raw parameter (group, comp) moved by delta; group 0 means (3),
 * 1 log-scales (3), 2 quaternion (4), 3 opacity logit (1), 4 SH (K x 3). */
static void moved_splat(const orc_big64* f, int64_t i, int group, int comp, double delta, orc_sp64* s) {
    double m[3], ls[3], q[4], lg[1];
    double shv[75];
    const int K3 = f->K * 3;
    for (int k = 0; k < 3; ++k) { m[k] = f->means[3 * i + k]; ls[k] = f->log_scales[3 * i + k]; }
    for (int k = 0; k < 4; ++k) q[k] = f->quats[4 * i + k];
    lg[0] = f->logits[i];
    for (int k = 0; k < K3 && k < 75; ++k) shv[k] = f->sh[(size_t)i * K3 + k];
    double* p = group == 0 ? m : group == 1 ? ls : group == 2 ? q : group == 3 ? lg : shv;
    p[comp] += delta;
    splat64(&f->cam, m, ls, q, lg, shv, f->K, f->D, f->splat_scale, 0, s);
}

/* Central difference of L = sum over all pixels and channels of (colour - target)^2 (target: the
 * full w x h x 3 image, float32) in raw parameter (group, comp) of Gaussian i, step h:
 * *fd = (L(+h) - L(-h)) / 2h, evaluated on the tiles either moved splat touches. *smooth = 1 when
 * both evaluations take the same branches (then L is smooth on [-h, h] up to a branch flipping and
 * flipping back inside it); *pixels = the pixels evaluated. Returns nonzero on bad arguments. */
int orc_big_fd(const void* hnd, const float* target, int64_t i, int group, int comp, double step, double* fd,
               int* smooth, int64_t* pixels) {
    const orc_big64* f = (const orc_big64*)hnd;
    const int sizes[5] = {3, 3, 4, 1, f->K * 3};
    if (i < 0 || i >= f->n || group < 0 || group > 4 || comp < 0 || comp >= sizes[group] || f->K * 3 > 75) return 1;
    orc_sp64 sp, sm;
    moved_splat(f, i, group, comp, step, &sp);
    moved_splat(f, i, group, comp, -step, &sm);
    orc_bl64 bp, bm;
    if (sp.alive) to_bl64(&sp, i, &bp);
    if (sm.alive) to_bl64(&sm, i, &bm);
    int same = sp.alive == sm.alive;
    if (same && sp.alive) {
        same = sp.x0 == sm.x0 && sp.y0 == sm.y0 && sp.x1 == sm.x1 && sp.y1 == sm.y1 && sp.clx == sm.clx &&
               sp.cly == sm.cly;
        for (int c = 0; c < 3; ++c) same = same && ((sp.pre[c] > 0) == (sm.pre[c] > 0));
    }
    /* the tiles either moved splat touches (outside them both evaluations leave Gaussian i out) */
    int tx0 = f->tx8, ty0 = f->ty8, tx1 = -1, ty1 = -1;
    const orc_sp64* both[2] = {&sp, &sm};
    for (int k = 0; k < 2; ++k)
        if (both[k]->alive) {
            if (both[k]->x0 < tx0) tx0 = both[k]->x0;
            if (both[k]->y0 < ty0) ty0 = both[k]->y0;
            if (both[k]->x1 > tx1) tx1 = both[k]->x1;
            if (both[k]->y1 > ty1) ty1 = both[k]->y1;
        }
    double diff = 0;
    uint64_t sig_p = 0, sig_m = 0;
    int64_t count = 0;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx)
            for (int y = ty * 8; y < ty * 8 + 8 && y < f->cam.h; ++y)
                for (int x = tx * 8; x < tx * 8 + 8 && x < f->cam.w; ++x) {
                    double cp[3], cm[3];
                    big_pixel(f, x, y, i, sp.alive ? &bp : NULL, cp, &sig_p, NULL);
                    big_pixel(f, x, y, i, sm.alive ? &bm : NULL, cm, &sig_m, NULL);
                    const float* t = target + ((size_t)y * f->cam.w + x) * 3;
                    for (int c = 0; c < 3; ++c) diff += (cp[c] - cm[c]) * (cp[c] + cm[c] - 2.0 * (double)t[c]);
                    ++count;
                }
    *fd = diff / (2 * step);
    *smooth = same && sig_p == sig_m;
    *pixels = count;
    return 0;
}
