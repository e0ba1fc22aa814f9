/*
 * aniso_b200.h -- C ABI of the B200 (sm_100a) Gaussian-splat rasterizer.
 *
 * The drop-in boundary for the reference's CUDA renderer, class aniso::GpuRenderer
 * (include/aniso/gpu_render.h:22-37, implemented in src/gpu_render.cu). Plain pointers, sizes and
 * status codes only: every call returns ANISO_B200_OK (0) or an error code, never throws across
 * the ABI and never traps on the device; aniso_b200_last_error() gives the message. The C++ shim
 * aniso_b200/shim/gpu_render_shim.cpp rebuilds GpuRenderer's exact signatures and exception
 * convention on top of these calls.
 *
 * Threading: like GpuRenderer, one scene object is used by one host thread at a time.
 */
#ifndef ANISO_B200_H
#define ANISO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ANISO_B200_OK = 0,
    ANISO_B200_ERR_ARGUMENT = 1,       /* a null pointer, a negative size, an unsupported degree */
    ANISO_B200_ERR_CUDA = 2,           /* a CUDA runtime call failed; the message names it */
    ANISO_B200_ERR_NO_DEVICE = 3,      /* no CUDA device */
    ANISO_B200_ERR_OUT_OF_MEMORY = 4,  /* a device allocation failed */
    ANISO_B200_ERR_DEVICE_WAIT = 5     /* a bounded device-side wait gave up (never expected) */
};

/* Opaque: one uploaded scene plus the device work buffers of its renders. */
typedef struct aniso_b200_scene aniso_b200_scene;

/* aniso::Camera (include/aniso/camera.h:16-26): world-to-camera R (row-major) and t, pinhole
 * intrinsics in pixels, image size. */
typedef struct aniso_b200_camera {
    double R[9];
    double t[3];
    double fx, fy, cx, cy;
    int32_t width, height;
} aniso_b200_camera;

/* aniso::RenderOptions (include/aniso/render.h:28-33). */
typedef struct aniso_b200_options {
    int32_t sh_degree;  /* colour up to this SH degree (>= 0), clamped to the scene's and to 3 */
    float splat_scale;  /* multiplies every Gaussian's scale (1 = unchanged) */
} aniso_b200_options;

/* aniso::RenderStats (include/aniso/render.h:9-14): stage times measured with CUDA events. */
typedef struct aniso_b200_stats {
    uint64_t visible;    /* Gaussians that survived culling */
    uint64_t tile_pairs; /* splat-tile pairs at 16x16 tiles (the reference GPU path's count) */
    double project_ms;   /* projection, compaction */
    double sort_ms;      /* depth sort, duplication, tile sort, tile ranges */
    double blend_ms;     /* blending */
} aniso_b200_stats;

/* GpuRenderer::available() (gpu_render.h:33, gpu_render.cu:262-265): *available = 1 if a CUDA
 * device is present and usable, else 0. */
int aniso_b200_available(int32_t* available);

/* GpuRenderer::GpuRenderer(const Scene&) (gpu_render.h:24, gpu_render.cu:267-292).
 * gaussians: n x 11 floats, the memory of std::vector<aniso::Gaussian> (gaussian.h:21-26):
 *            position x y z, scale x y z, rotation w x y z, opacity -- already activated.
 * sh:        n x (sh_degree+1)^2 x 3 floats, [coefficient][channel] (Scene::sh, gaussian.h:33-35);
 *            sh_degree 0..4 (colour is evaluated up to degree 3).
 * The scene is copied to the device; the caller's arrays are not retained. */
int aniso_b200_scene_create(const float* gaussians, const float* sh, int64_t n, int32_t sh_degree,
                            aniso_b200_scene** out);

/* The raw (optimizer) form a 3DGS PLY stores, activated on the device as the reference loader
 * does on the host (ply_loader.cpp:124-138): xyz n x 3, f_dc n x 3, f_rest n x 3((d+1)^2-1)
 * channel-major, opacity logit n, log-scale n x 3, rot n x 4 (w first). Host pointers. */
int aniso_b200_scene_create_raw(const float* xyz, const float* f_dc, const float* f_rest, const float* opacity,
                                const float* log_scale, const float* rot, int64_t n, int32_t sh_degree,
                                aniso_b200_scene** out);

/* ~GpuRenderer (gpu_render.cu:294-297). Accepts NULL. */
/* aniso::loadPly (ply_loader.cpp:77-141) followed by the GpuRenderer constructor, with the work on
 * the device: the header is parsed on the host with the reference loader's rules and messages,
 * the vertex block is uploaded as stored (rows of float properties, any order, unknown properties
 * ignored), and one kernel de-interleaves, activates (exp, sigmoid, normalise) and reorders the SH
 * into the scene's layout. The scene's SH degree is the file's (0..4). The device exp may differ
 * from the host loader's std::exp in the last bit of an activated value. */
int aniso_b200_scene_load_ply(const char* path, aniso_b200_scene** out);

int aniso_b200_scene_destroy(aniso_b200_scene* scene);

/* GpuRenderer::render(const Camera&, RenderStats*, const RenderOptions&) (gpu_render.h:30,
 * gpu_render.cu:299-375): renders into a HOST buffer of width*height*3 bytes (RGB8, rows top to
 * bottom, image.h:10-17) and returns when it is written. options and stats may be NULL
 * (defaults: degree 3, scale 1). A page-locked buffer that the current device can address
 * (cudaHostAlloc, a pinned torch tensor) is written by the blend kernel directly, across the bus
 * while the frame blends; any other buffer receives a copy of the finished image. */
int aniso_b200_render(aniso_b200_scene* scene, const aniso_b200_camera* camera, const aniso_b200_options* options,
                      uint8_t* rgb_host, aniso_b200_stats* stats);

/* The same render, stream-ordered, into a DEVICE buffer: enqueues the kernels on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) and returns without waiting. The pair
 * buffers must already be large enough (a previous render of a similar view sizes them); a frame
 * that needed more sets the overflow status that aniso_b200_sync() reports, and should be
 * rendered again. */
int aniso_b200_render_device(aniso_b200_scene* scene, const aniso_b200_camera* camera,
                             const aniso_b200_options* options, uint8_t* rgb_device, void* stream);

/* Waits for the scene's enqueued work; reports the last frame's counts (stats may be NULL) and
 * returns ANISO_B200_ERR_ARGUMENT with message "pair capacity exceeded" if any frame since the
 * previous sync overflowed (the capacity has then been grown for the next render). */
int aniso_b200_sync(aniso_b200_scene* scene, aniso_b200_stats* stats);

/* Per-stage device timing of aniso_b200_render_device frames (no counterpart in gpu_render.h;
 * GpuRenderer times only its synchronous render, gpu_render.cu:318-373). enable = 1 clears the
 * totals and records CUDA events around each stage of every later frame on its own stream;
 * enable = 0 stops. aniso_b200_profile_read waits for the scene's work and returns the summed
 * stage times in ms and the number of frames they cover. */
int aniso_b200_profile(aniso_b200_scene* scene, int32_t enable);
int aniso_b200_profile_read(aniso_b200_scene* scene, double* project_ms, double* sort_ms, double* blend_ms,
                            int64_t* frames);

/* The number of kernels the scene's last aniso_b200_render / aniso_b200_render_device frame
 * launched (no counterpart in gpu_render.h): the library's own kernels only, not its memory
 * copies and clears. 0 before the first frame. */
int aniso_b200_frame_kernels(aniso_b200_scene* scene, int32_t* kernels);

/* Copies the last error message (NUL-terminated, truncated to len) and returns its full length. */
size_t aniso_b200_last_error(char* buf, size_t len);

/* One camera of a COLMAP sparse model: aniso::Camera (camera.h:16-26), image name included. */
typedef struct aniso_b200_colmap_camera {
    aniso_b200_camera camera;
    char image_name[256];  /* NUL-terminated */
} aniso_b200_colmap_camera;

/* aniso::loadColmapCameras (camera.h:51, camera.cpp:105-140) with COLMAP's text format added:
 * reads `folder`'s cameras.bin + images.bin when cameras.bin exists (the reference's format, its
 * rules and messages), else cameras.txt + images.txt. PINHOLE and SIMPLE_PINHOLE only (a model
 * with lens distortion is refused, camera.cpp:82-85); each image's quaternion normalised in double
 * into R; cameras sorted by image name. Host code only (no device needed). Two calls: with out ==
 * NULL only *count is set; then capacity >= *count entries of out are filled. */
int aniso_b200_colmap_load(const char* folder, aniso_b200_colmap_camera* out, int32_t capacity, int32_t* count);

/* ---- batches (no counterpart in the reference, whose multi-view caller renders views one by one
 * with two host syncs each, main.cpp:233-244): many views of several scenes rendered by one fixed
 * launch sequence. Every Gaussian is read once and projected for all views of its scene; one
 * sort orders every view's pairs; one blend launch covers every tile of every view. ---------- */

typedef struct aniso_b200_batch aniso_b200_batch;

typedef struct aniso_b200_batch_options {
    int32_t sh_degree;   /* colour up to this SH degree, clamped to each view's scene's and to 3 */
    float splat_scale;   /* as aniso_b200_options */
    int32_t tile_w;      /* tile shape: 8x8, 16x16 (the reference's, and the default for 0) or 16x32; */
    int32_t tile_h;      /*   the image is the same for every shape */
    int32_t blend_batch; /* splats staged per blend round: < 256 the smaller, >= 256 the larger set */
    int32_t use_graph;   /* 1: record the launch sequence once as a CUDA graph and replay it */
    int32_t radix_bits;  /* widest digit of the sort's tile passes: 8 (the default for 0) or 9, which
                          * takes 9-bit digits where they save a pass (depth passes are always 8-bit) */
} aniso_b200_batch_options;

/* A batch of n_views views; view k shows scene scenes[view_scene[k]]. The views of one scene must
 * be consecutive. The scenes are not copied and must outlive the batch. */
int aniso_b200_batch_create(aniso_b200_scene* const* scenes, int32_t n_scenes, const int32_t* view_scene,
                            int32_t n_views, const aniso_b200_batch_options* options, aniso_b200_batch** out);

/* Renders every view, camera k into the DEVICE RGB8 buffer rgb_device[k] (its width*height*3
 * bytes), stream-ordered, without waiting. With use_graph, the first call (and any call whose
 * image sizes differ from the recorded ones) records the graph; later calls replay it. */
int aniso_b200_batch_render(aniso_b200_batch* batch, const aniso_b200_camera* cameras, uint8_t* const* rgb_device,
                            void* stream);

/* Waits for the batch's work and reports totals over its views; as aniso_b200_sync, returns
 * ANISO_B200_ERR_ARGUMENT "pair capacity exceeded" if a render overflowed (capacity then grown). */
int aniso_b200_batch_sync(aniso_b200_batch* batch, aniso_b200_stats* stats);

int aniso_b200_batch_destroy(aniso_b200_batch* batch);

/* ---- the differentiable path (no counterpart in the reference: it has no backward pass; the
 * training pipeline it drives calls the third-party gsplat rasterizer instead,
 * pipeline/train_gsplat.py:96-102) ----------------------------------------------------------- */

/* Opaque: the work buffers of one forward and its backward. */
typedef struct aniso_b200_trainer aniso_b200_trainer;

/* The optimizer's raw tensors, DEVICE pointers, row-major float32, as train_gsplat.py:85-92 keeps
 * them: means n x 3, log-scales n x 3, quaternions n x 4 (w first, any norm), opacity logits n,
 * SH n x (sh_degree+1)^2 x 3. sh_degree is the STORED degree and must be 1 or 3 (so each
 * Gaussian's SH is whole 16-byte words); quats and sh 16-byte aligned. Activations (exp, sigmoid,
 * normalise) are applied inside the kernels. */
typedef struct aniso_b200_raw_params {
    const float* means;
    const float* log_scales;
    const float* quats;
    const float* opacity_logits;
    const float* sh;
    int64_t n;
    int32_t sh_degree;
} aniso_b200_raw_params;

/* Gradient outputs, DEVICE pointers with the shapes of aniso_b200_raw_params (quats and sh 16-byte
 * aligned). The caller zeroes them; entries of Gaussians culled in the view are left untouched.
 * The backward adds to them; with fresh = 1 (they hold only the caller's zeros) the scene's first
 * view stores its values without reading the zeros back (0 + g, the same bits). The optional
 * densification statistics (grad2d, visible) are always added to. */
typedef struct aniso_b200_raw_grads {
    float* means;
    float* log_scales;
    float* quats;
    float* opacity_logits;
    float* sh;
    /* Optional (NULL to skip), for densification: per Gaussian, the norm of dL/d(screen position)
     * in NDC units (pixels x width/2, x height/2, as gsplat's DefaultStrategy normalises it) and the
     * number of views it was visible in, both added to over the views of a backward. */
    float* grad2d;
    float* visible;
    int32_t fresh;
} aniso_b200_raw_grads;

int aniso_b200_trainer_create(aniso_b200_trainer** out);
int aniso_b200_trainer_destroy(aniso_b200_trainer* trainer);

/* Renders the float colour image (width*height*3, unclamped, the sum before the 8-bit rounding of
 * gpu_render.cu:229-231) into image_device on `stream` and keeps what the backward needs. Returns
 * after the frame has run (it reads the frame's pair count to size its buffers). */
int aniso_b200_train_forward(aniso_b200_trainer* trainer, const aniso_b200_raw_params* params,
                             const aniso_b200_camera* camera, const aniso_b200_options* options, float* image_device,
                             void* stream);

/* The adjoint of the last train_forward: given dL/d(image) (device, width*height*3), writes the
 * gradients of the 59 raw parameters per Gaussian. The params of that forward must be unchanged.
 * Deterministic: no atomics; every sum runs in a fixed order. Enqueued on `stream`. */
int aniso_b200_train_backward(aniso_b200_trainer* trainer, const float* grad_image_device,
                              const aniso_b200_raw_grads* grads, void* stream);

/* The training-step shape: n_views views of n_scenes scenes (params[s], view k of scene
 * view_scene[k], views of a scene consecutive) in one forward; images_device[k] receives view k.
 * The backward adds each view's gradient to its scene's grads[s], views in order, so the sum over
 * views is deterministic too. */
int aniso_b200_train_batch_forward(aniso_b200_trainer* trainer, const aniso_b200_raw_params* params,
                                   int32_t n_scenes, const int32_t* view_scene, const aniso_b200_camera* cameras,
                                   int32_t n_views, const aniso_b200_batch_options* options,
                                   float* const* images_device, void* stream);
int aniso_b200_train_batch_backward(aniso_b200_trainer* trainer, const float* const* grad_images_device,
                                    const aniso_b200_raw_grads* grads, void* stream);

/* ---- the optimizer step of a training loop (no counterpart in the reference: its training drives
 * one torch.optim.Adam per parameter group, pipeline/train_gsplat.py:165-167) ----------------- */

/* One parameter group: `count` floats of DEVICE arrays param / grad / exp_avg / exp_avg_sq, learning
 * rate lr and eps. Optionally the first `head` floats of every `row` floats use lr_head instead
 * (the SH tensor: coefficient 0 and the rest have different rates); head = 0 for none. */
typedef struct aniso_b200_adam_group {
    float* param;
    const float* grad;
    float* exp_avg;
    float* exp_avg_sq;
    int64_t count;
    float lr;
    float lr_head;
    int32_t row;
    int32_t head;
    float eps;
} aniso_b200_adam_group;

/* Adam (torch.optim.Adam's update, no weight decay) for step number `step` (from 1) over up to 8
 * groups in one launch, enqueued on `stream`. */
int aniso_b200_adam_step(const aniso_b200_adam_group* groups, int32_t n_groups, int32_t step, float beta1,
                         float beta2, void* stream);

/* ---- introspection used by the parity tests (no counterpart in gpu_render.h) ---------------- */

/* Runs the projection only and copies, per Gaussian, what the reference preprocess kernel
 * writes (gpu_render.cu:86-88): uv n x 2, conic_opacity n x 4, depth n, rgb n x 3, rect n x 4
 * (uint32 x0 y0 x1 y1), tiles_touched n (0 = culled). Any output may be NULL. */
int aniso_b200_debug_projection(aniso_b200_scene* scene, const aniso_b200_camera* camera,
                                const aniso_b200_options* options, float* uv, float* conic_opacity, float* depth,
                                float* rgb, uint32_t* rect, uint32_t* tiles_touched);

/* Runs projection and sort and copies the sorted pair list: tile ids and Gaussian indices
 * (capacity entries at most) and ranges (tiles_x*tiles_y x 2). *pairs receives the count; returns
 * ANISO_B200_ERR_ARGUMENT if capacity is too small. The reference's 64-bit key of pair k is
 * (tile[k] << 32) | bits(depth[value[k]]). */
int aniso_b200_debug_sorted(aniso_b200_scene* scene, const aniso_b200_camera* camera,
                            const aniso_b200_options* options, uint32_t* tiles, uint32_t* values, uint64_t capacity,
                            uint32_t* ranges, uint64_t* pairs);

/* The sort alone on a projection computed elsewhere (host arrays in the reference kernel's
 * layout: tiles_touched n, rect n x 4, depth n), for tiles_x x tiles_y tiles: the same outputs
 * as aniso_b200_debug_sorted. Needs no scene. */
int aniso_b200_sort_projection(int64_t n, const uint32_t* tiles_touched, const uint32_t* rect, const float* depth,
                               int32_t tiles_x, int32_t tiles_y, uint32_t* tiles, uint32_t* values,
                               uint64_t capacity, uint32_t* ranges, uint64_t* pairs);

/* ---- a sort that allocates nothing (no counterpart in the reference, whose GpuRenderer grows
 * its buffers with cudaFree + cudaMalloc inside render(), gpu_render.cu:24-37, 326-354) ---------
 * For callers that must not touch the CUDA allocator while they run: a render loop or a serving
 * worker that keeps all device memory in its own pool, where cudaFree would synchronise the whole
 * device and cudaMalloc could stall or fail in the middle of a frame. Same sort and outputs as
 * aniso_b200_sort_projection, but every array is a DEVICE pointer, the work is enqueued on
 * `stream` without waiting, and the work buffers are one static device array of about 20 MB per
 * device (held once the call has been used on that device), which bounds the problem size:
 *   n <= ANISO_B200_NOALLOC_MAX_GAUSSIANS (else ANISO_B200_ERR_ARGUMENT, nothing enqueued);
 *   pairs beyond min(capacity, ANISO_B200_NOALLOC_MAX_PAIRS) are not written: tiles/values are
 *   left untouched, ranges are all zero, and *pairs (device) still receives the total.
 * A rectangle outside the tile grid refuses the call on the device: *pairs = UINT64_MAX.
 * Alignment: rect and tiles 16 bytes, ranges and pairs 8 bytes (cudaMalloc'd memory is).
 * capacity 0 is a count-only call: *pairs receives the total and no pair is written.
 * The static buffers are shared: calls on one device must not overlap in time (issue them on one
 * stream, or wait for the previous one). The first call on a device looks the buffers up
 * (cudaGetSymbolAddress) and keeps the address for the life of the process, so make it before any
 * stream capture starts, and do not use the entry point on a device after cudaDeviceReset (the
 * kept address then belongs to the destroyed context). */
#define ANISO_B200_NOALLOC_MAX_GAUSSIANS 65536
#define ANISO_B200_NOALLOC_MAX_PAIRS 1048576
int aniso_b200_sort_projection_noalloc(int64_t n, const uint32_t* tiles_touched, const uint32_t* rect,
                                       const float* depth, int32_t tiles_x, int32_t tiles_y, uint32_t* tiles,
                                       uint32_t* values, uint64_t capacity, uint32_t* ranges, uint64_t* pairs,
                                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ANISO_B200_H */
