// aniso_b200_sort_projection_noalloc: the sort of aniso_b200_sort_projection on device arrays,
// for callers that must not allocate. Every work buffer lives in one file-scope __device__ array
// (g_scratch) whose address is looked up once per device; nothing here calls cudaMalloc,
// cudaFree, cudaMallocHost or a library routine that allocates. The array is sized for at most
// ANISO_B200_NOALLOC_MAX_GAUSSIANS Gaussians and ANISO_B200_NOALLOC_MAX_PAIRS splat-tile pairs
// (about 20 MB, held by each device once this file's module is loaded).
//
// What must start at zero does so without the host: the frame's control block is cleared by
// frame_begin at the start of every call, the caller's ranges are cleared with cudaMemsetAsync,
// and every other region is fully written before it is read.
//
// One g_scratch per device: two calls on one device whose work overlaps in time (different streams
// or host threads without ordering) race on it. The first call on a device resolves the array's
// address (cudaGetSymbolAddress, which may load this module), so make it before any stream
// capture begins. The address is kept for the life of the process: after cudaDeviceReset it
// belongs to a destroyed context, so the entry point must not be used on that device again.
#include <cuda_runtime.h>

#include <mutex>

#include "aniso_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace ab2 {
int report_error(int code, const char* msg);  // capi.cu: status code + aniso_b200_last_error text
}

namespace {

using namespace ab2;

constexpr size_t kG = ANISO_B200_NOALLOC_MAX_GAUSSIANS;
constexpr size_t kP = ANISO_B200_NOALLOC_MAX_PAIRS;
constexpr size_t kScratchWords = 512 * 600;         // >= sort_scratch_words(), checked at setup
constexpr size_t kSpanSums = 600;                    // >= sort_span_sums(), checked at setup
constexpr size_t kChunkWords = kP / 1024 + 2;        // >= kP / expand_chunk_pairs() + 2, checked

constexpr size_t up256(size_t x) { return (x + 255) / 256 * 256; }
// Byte offsets of the regions of g_scratch, each 256-byte aligned.
constexpr size_t kCtrl = 0;
constexpr size_t kDepthKey = up256(kCtrl + sizeof(Ctrl));
constexpr size_t kRect16 = up256(kDepthKey + 4 * kG);
constexpr size_t kVisKey0 = up256(kRect16 + 8 * kG);
constexpr size_t kVisKey1 = up256(kVisKey0 + 4 * kG);
constexpr size_t kVisIdx0 = up256(kVisKey1 + 4 * kG);
constexpr size_t kVisIdx1 = up256(kVisIdx0 + 4 * kG);
constexpr size_t kOffs = up256(kVisIdx1 + 4 * kG);
constexpr size_t kRectSorted = up256(kOffs + 4 * kG);
constexpr size_t kSort = up256(kRectSorted + 8 * kG);
constexpr size_t kSpan = up256(kSort + 4 * kScratchWords);
constexpr size_t kChunk = up256(kSpan + 8 * kSpanSums);
constexpr size_t kTables = up256(kChunk + 4 * kChunkWords);
constexpr size_t kPairKey0 = up256(kTables + 4 * 3);
constexpr size_t kPairKey1 = up256(kPairKey0 + 4 * kP);
constexpr size_t kPairVal0 = up256(kPairKey1 + 4 * kP);
constexpr size_t kPairVal1 = up256(kPairVal0 + 4 * kP);
constexpr size_t kBytes = up256(kPairVal1 + 4 * kP);

__device__ __align__(256) unsigned char g_scratch[kBytes];

constexpr unsigned kFlagBadInput = 1u << 8;  // a rectangle outside the tile grid (noalloc only)

// The one-view tables of the expansion (entry base 0, tile base 0, tiles per row), written from
// kernel arguments so no host buffer is involved.
__global__ void tables_kernel(unsigned* tables, unsigned tiles_x) {
    tables[0] = 0u;
    tables[1] = 0u;
    tables[2] = tiles_x;
}

// Every visible rectangle must lie in the tile grid (the expansion writes one pair per tile of
// it); otherwise the call is refused on the device: the overflow flag stops every later stage.
__global__ void validate_kernel(int64_t n, const unsigned* __restrict__ tiles_touched, const uint4* __restrict__ rect,
                                unsigned tiles_x, unsigned tiles_y, Ctrl* ctrl) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n || tiles_touched[i] == 0) return;
    const uint4 r = rect[i];
    if (r.x > r.z || r.y > r.w || r.z >= tiles_x || r.w >= tiles_y)
        atomicOr(&ctrl->flags, kFlagOverflow | kFlagBadInput);
}

// The caller's pair count: the frame's total, or UINT64_MAX when the input was refused.
__global__ void finish_kernel(const Ctrl* ctrl, unsigned long long* pairs) {
    *pairs = (ctrl->flags & kFlagBadInput) ? ~0ull : ctrl->pair_total;
}

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char* g_base[kMaxDevices];

int scratch_base(unsigned char** base) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return report_error(ANISO_B200_ERR_NO_DEVICE, "no usable CUDA device");
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_base[dev]) {
        if (sort_scratch_words() > kScratchWords || sort_span_sums() > kSpanSums ||
            kP / expand_chunk_pairs() + 2 > kChunkWords)
            return report_error(ANISO_B200_ERR_CUDA, "no-alloc scratch layout smaller than the sort needs");
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return report_error(ANISO_B200_ERR_CUDA, "cudaGetSymbolAddress(g_scratch) failed");
        }
        g_base[dev] = static_cast<unsigned char*>(p);
    }
    *base = g_base[dev];
    return 0;
}

int bits_for(uint32_t v) {
    int b = 0;
    while (b < 32 && (1ull << b) <= v) ++b;
    return b;
}

}  // namespace

extern "C" int aniso_b200_sort_projection_noalloc(int64_t n, const uint32_t* tiles_touched, const uint32_t* rect,
                                                  const float* depth, int32_t tiles_x, int32_t tiles_y,
                                                  uint32_t* tiles, uint32_t* values, uint64_t capacity,
                                                  uint32_t* ranges, uint64_t* pairs, void* stream) {
    if (n < 0 || static_cast<uint64_t>(n) > kG)
        return report_error(ANISO_B200_ERR_ARGUMENT, "n must be in [0, ANISO_B200_NOALLOC_MAX_GAUSSIANS]");
    if (tiles_x <= 0 || tiles_y <= 0 || tiles_x > 65535 || tiles_y > 65535 ||
        static_cast<uint64_t>(tiles_x) * static_cast<uint64_t>(tiles_y) > 0xFFFFFFFFull)
        return report_error(ANISO_B200_ERR_ARGUMENT, "tile grid must be 1..65535 on each side");
    if (!tiles || !values || !ranges || !pairs || (n > 0 && (!tiles_touched || !rect || !depth)))
        return report_error(ANISO_B200_ERR_ARGUMENT, "a device pointer is NULL");
    const auto misaligned = [](const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; };
    if (misaligned(rect, 16) || misaligned(tiles, 16) || misaligned(ranges, 8) || misaligned(pairs, 8))
        return report_error(ANISO_B200_ERR_ARGUMENT, "rect and tiles must be 16-byte aligned, ranges and pairs 8-byte");
    unsigned char* base = nullptr;
    if (const int rc = scratch_base(&base)) return rc;

    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned un = static_cast<unsigned>(n);
    const unsigned T = static_cast<unsigned>(tiles_x) * static_cast<unsigned>(tiles_y);
    const unsigned cap = static_cast<unsigned>(capacity < kP ? capacity : kP);  // pairs beyond it: not written
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(base + kCtrl);
    unsigned* depth_key = reinterpret_cast<unsigned*>(base + kDepthKey);
    auto* rect16 = reinterpret_cast<unsigned long long*>(base + kRect16);
    unsigned* vis_key[2] = {reinterpret_cast<unsigned*>(base + kVisKey0), reinterpret_cast<unsigned*>(base + kVisKey1)};
    unsigned* vis_idx[2] = {reinterpret_cast<unsigned*>(base + kVisIdx0), reinterpret_cast<unsigned*>(base + kVisIdx1)};
    unsigned* sort_scratch = reinterpret_cast<unsigned*>(base + kSort);
    unsigned* tables = reinterpret_cast<unsigned*>(base + kTables);
    unsigned* pair_key[2] = {reinterpret_cast<unsigned*>(base + kPairKey0), reinterpret_cast<unsigned*>(base + kPairKey1)};
    unsigned* pair_val[2] = {reinterpret_cast<unsigned*>(base + kPairVal0), reinterpret_cast<unsigned*>(base + kPairVal1)};
    const DupBuffers dup{reinterpret_cast<unsigned*>(base + kOffs), nullptr,
                         reinterpret_cast<unsigned long long*>(base + kRectSorted),
                         reinterpret_cast<unsigned*>(base + kChunk),
                         reinterpret_cast<unsigned long long*>(base + kSpan)};

    launch_frame_begin(ctrl, st);
    tables_kernel<<<1, 1, 0, st>>>(tables, static_cast<unsigned>(tiles_x));
    if (n > 0) {
        const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
        validate_kernel<<<blocks, 256, 0, st>>>(n, tiles_touched, reinterpret_cast<const uint4*>(rect),
                                                static_cast<unsigned>(tiles_x), static_cast<unsigned>(tiles_y), ctrl);
    }
    launch_projection_keys(n, tiles_touched, depth, reinterpret_cast<const uint4*>(rect), depth_key, rect16, st);
    for (int p = 0; p < kMaxPasses; ++p) {
        const int src = (p + 1) & 1, dst = p & 1;
        launch_radix_pass(p == 0 ? depth_key : vis_key[src], p == 0 ? nullptr : vis_idx[src],
                          p == kMaxPasses - 1 ? nullptr : vis_key[dst], vis_idx[dst], p == 0,
                          p == 0 ? SortCount::kFixed : SortCount::kVisible, un, un, p * kRadixBits, kRadixBits,
                          sort_scratch, ctrl, st);
    }
    const BatchTables tab{tables, tables + 1, tables + 2, 1u};
    launch_duplicate(vis_idx[(kMaxPasses - 1) & 1], rect16, ctrl, cap, un, tab, dup, pair_key[0], pair_val[0], st);
    const int passes = (bits_for(T - 1) + kRadixBits - 1) / kRadixBits > 1 ? (bits_for(T - 1) + kRadixBits - 1) / kRadixBits : 1;
    for (int p = 0; p < passes; ++p) {  // the last pass writes the caller's arrays
        const bool last = p == passes - 1;
        launch_radix_pass(pair_key[p & 1], pair_val[p & 1], last ? tiles : pair_key[(p + 1) & 1],
                          last ? values : pair_val[(p + 1) & 1], false, SortCount::kPairs, 0u, cap, p * kRadixBits,
                          kRadixBits, sort_scratch, ctrl, st);
    }
    cudaError_t e = cudaMemsetAsync(ranges, 0, static_cast<size_t>(T) * 2 * sizeof(uint32_t), st);
    if (e == cudaSuccess) {
        launch_ranges(tiles, ctrl, cap, reinterpret_cast<uint2*>(ranges), st);
        finish_kernel<<<1, 1, 0, st>>>(ctrl, reinterpret_cast<unsigned long long*>(pairs));
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return report_error(ANISO_B200_ERR_CUDA, cudaGetErrorString(e));
    }
    return ANISO_B200_OK;
}
