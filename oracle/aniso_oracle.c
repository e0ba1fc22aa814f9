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
