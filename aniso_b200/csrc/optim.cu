// The optimizer step of the training loop around the adjoint: Adam over every parameter group in
// one launch (the reference drives one torch.optim.Adam per group, pipeline/train_gsplat.py:165-167,
// with eps = 1e-15 and a per-group learning rate; the SH tensor's first coefficient has its own).
//
// Per element, in torch.optim.Adam's order (non-AMSGrad, no weight decay):
//   m = m + (1 - b1) (g - m)                  (lerp)
//   v = b2 v + (1 - b2) g g
//   p = p - (lr / (1 - b1^t)) m / (sqrt(v) / sqrt(1 - b2^t) + eps)
// with the bias corrections formed on the host in double, as torch does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "aniso_b200.h"

namespace ab2 {
int report_error(int code, const char* msg);
}

namespace {

constexpr int kMaxGroups = 8;

struct AdamGroupDev {
    float* param;
    const float* grad;
    float* m;
    float* v;
    unsigned long long begin;  // first element of this group in the concatenated index space
    float step_size, step_size_head;  // lr / (1 - b1^t) for the row's tail and head
    float eps;
    int row, head;                    // floats per row; leading floats of a row that use the head rate
};

struct AdamArgs {
    AdamGroupDev g[kMaxGroups];
    int n_groups;
    unsigned long long total;
    float b1c, b2, b2c;  // 1 - b1, b2, 1 - b2
    float bc2_sqrt;      // sqrt(1 - b2^t)
};

__global__ void __launch_bounds__(256) adam_kernel(AdamArgs a) {
    for (unsigned long long e = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < a.total;
         e += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        int k = 0;
        while (k + 1 < a.n_groups && a.g[k + 1].begin <= e) ++k;
        const AdamGroupDev& G = a.g[k];
        const unsigned long long i = e - G.begin;
        const float g = G.grad[i];
        const float m = fmaf(a.b1c, g - G.m[i], G.m[i]);
        const float v = fmaf(a.b2c, g * g, a.b2 * G.v[i]);
        G.m[i] = m;
        G.v[i] = v;
        const bool in_head = G.head > 0 && static_cast<int>(i % static_cast<unsigned long long>(G.row)) < G.head;
        const float step_size = in_head ? G.step_size_head : G.step_size;
        const float denom = sqrtf(v) / a.bc2_sqrt + G.eps;
        G.param[i] = fmaf(-step_size, m / denom, G.param[i]);
    }
}

}  // namespace

extern "C" int aniso_b200_adam_step(const aniso_b200_adam_group* groups, int32_t n_groups, int32_t step, float beta1,
                                    float beta2, void* stream) {
    if (!groups || n_groups <= 0 || n_groups > kMaxGroups)
        return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "n_groups must be in [1, 8]");
    if (step < 1) return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "step counts from 1");
    AdamArgs a;
    std::memset(&a, 0, sizeof a);
    a.n_groups = n_groups;
    const double bc1 = 1.0 - std::pow(static_cast<double>(beta1), step);
    const double bc2 = 1.0 - std::pow(static_cast<double>(beta2), step);
    a.b1c = 1.0f - beta1;
    a.b2 = beta2;
    a.b2c = 1.0f - beta2;
    a.bc2_sqrt = static_cast<float>(std::sqrt(bc2));
    unsigned long long total = 0;
    for (int k = 0; k < n_groups; ++k) {
        const aniso_b200_adam_group& s = groups[k];
        if (s.count < 0 || (s.count > 0 && (!s.param || !s.grad || !s.exp_avg || !s.exp_avg_sq)))
            return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "an Adam group has a NULL array or a negative count");
        if (s.head > 0 && (s.row <= 0 || s.head > s.row))
            return ab2::report_error(ANISO_B200_ERR_ARGUMENT, "an Adam group's head must fit in its row");
        AdamGroupDev& d = a.g[k];
        d.param = s.param;
        d.grad = s.grad;
        d.m = s.exp_avg;
        d.v = s.exp_avg_sq;
        d.begin = total;
        d.step_size = static_cast<float>(static_cast<double>(s.lr) / bc1);
        d.step_size_head = static_cast<float>(static_cast<double>(s.head > 0 ? s.lr_head : s.lr) / bc1);
        d.eps = s.eps;
        d.row = s.row > 0 ? s.row : 1;
        d.head = s.head;
        total += static_cast<unsigned long long>(s.count);
    }
    a.total = total;
    if (total == 0) return ANISO_B200_OK;
    const unsigned long long blocks = std::min<unsigned long long>((total + 255) / 256, 148ull * 16);
    adam_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ab2::report_error(ANISO_B200_ERR_CUDA, cudaGetErrorString(e));
    return ANISO_B200_OK;
}
