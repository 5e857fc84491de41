// hs_loss.cu -- the mean end-point-error loss of a batch of flow fields and its gradient,
// one launch each way for all pairs:
//   L = (1/n) sum_i (1/(H_i W_i)) sum_px sqrt((u-ut)^2 + (v-vt)^2 + eps)
// The sum is deterministic: fixed per-block partials in double, folded in a fixed order.
#include <algorithm>
#include <cstring>

#include "hs_common.cuh"

namespace hs {

static inline size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

constexpr int kEpeMaxPairs = 32;
constexpr int kEpeBlocks = 64;  // partial sums per pair

struct EpeTable {
    hs_epe_pair pair[kEpeMaxPairs];
    int n;
    float eps;
};

__global__ void __launch_bounds__(256) epe_partial_kernel(const __grid_constant__ EpeTable tab,
                                                          double *partials) {
    __shared__ double sh[8];
    const int i = blockIdx.y;
    const hs_epe_pair &p = tab.pair[i];
    const long n = (long)p.H * p.W;
    double s = 0.0;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const size_t o = (size_t)(e / p.W) * p.ld + (size_t)(e % p.W);
        const float a = __ldg(p.u + o) - __ldg(p.ut + o), b = __ldg(p.v + o) - __ldg(p.vt + o);
        s += (double)sqrtf(fmaf(a, a, fmaf(b, b, tab.eps)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        partials[(size_t)i * gridDim.x + blockIdx.x] = t;
    }
}

// Lane i folds pair i's partials in order (the pairs in parallel), then lane 0 adds the pairs'
// means in order: the same operations, in the same order, as one thread doing both loops.
static_assert(kEpeMaxPairs <= 32, "one lane per pair");

__global__ void epe_fold_kernel(const __grid_constant__ EpeTable tab, const double *partials,
                                float *loss) {
    __shared__ double mean[kEpeMaxPairs];
    const int i = threadIdx.x;
    if (i < tab.n) {
        double s = 0.0;
        for (int b = 0; b < kEpeBlocks; ++b) s += partials[(size_t)i * kEpeBlocks + b];
        mean[i] = s / ((double)tab.pair[i].H * (double)tab.pair[i].W);
    }
    __syncthreads();
    if (i == 0) {
        double total = 0.0;
        for (int j = 0; j < tab.n; ++j) total += mean[j];
        *loss = (float)(total / tab.n);
    }
}

__global__ void __launch_bounds__(256) epe_backward_kernel(const __grid_constant__ EpeTable tab,
                                                           const float *dloss) {
    const int i = blockIdx.y;
    const hs_epe_pair &p = tab.pair[i];
    const long n = (long)p.H * p.W;
    const float sc = __ldg(dloss) / (float)((double)tab.n * (double)n);
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const size_t o = (size_t)(e / p.W) * p.ld + (size_t)(e % p.W);
        const float a = __ldg(p.u + o) - __ldg(p.ut + o), b = __ldg(p.v + o) - __ldg(p.vt + o);
        const float r = sc * rsqrtf(fmaf(a, a, fmaf(b, b, tab.eps)));
        p.du[o] = a * r;
        p.dv[o] = b * r;
    }
}

static hs_status make_table(const hs_epe_pair *pairs, int n, float eps, bool grads, EpeTable &tab) {
    if (!pairs) HS_FAIL(HS_ERR_INVALID_ARG, "pairs is NULL");
    if (n < 1 || n > kEpeMaxPairs) HS_FAIL(HS_ERR_INVALID_ARG, "n=%d outside 1..%d", n, kEpeMaxPairs);
    if (!(eps >= 0.0f)) HS_FAIL(HS_ERR_INVALID_ARG, "eps must be >= 0");
    memset(&tab, 0, sizeof(tab));
    for (int i = 0; i < n; ++i) {
        const hs_epe_pair &p = pairs[i];
        hs_status st = check_plane_geometry(p.H, p.W, p.ld);
        if (st != HS_OK) return st;
        if (p.reserved != 0) HS_FAIL(HS_ERR_INVALID_ARG, "pair %d: reserved must be zero", i);
        const void *pl[4] = {p.u, p.v, p.ut, p.vt};
        const char *nm[4] = {"u", "v", "ut", "vt"};
        for (int q = 0; q < 4; ++q)
            if ((st = check_plane(pl[q], nm[q])) != HS_OK) return st;
        if (grads) {
            if ((st = check_plane(p.du, "du")) != HS_OK || (st = check_plane(p.dv, "dv")) != HS_OK) return st;
        }
        tab.pair[i] = p;
    }
    tab.n = n;
    tab.eps = eps;
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

size_t hs_epe_workspace_bytes(int n) {
    if (n < 1 || n > kEpeMaxPairs) return 0;
    return round256((size_t)n * kEpeBlocks * sizeof(double));
}

hs_status hs_epe_loss_batched(const hs_epe_pair *pairs, int n, float eps, float *loss,
                              void *workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    EpeTable tab;
    hs_status st = make_table(pairs, n, eps, false, tab);
    if (st != HS_OK) return st;
    if (!loss) HS_FAIL(HS_ERR_INVALID_ARG, "loss is NULL");
    if (!workspace || workspace_bytes < hs_epe_workspace_bytes(n))
        HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes, hs_epe_workspace_bytes(n));
    cudaStream_t s = (cudaStream_t)stream;
    double *part = reinterpret_cast<double *>(workspace);
    epe_partial_kernel<<<dim3(kEpeBlocks, n), 256, 0, s>>>(tab, part);
    HS_LAUNCH_CHECK("epe_partial_kernel");
    epe_fold_kernel<<<1, 32, 0, s>>>(tab, part, loss);
    HS_LAUNCH_CHECK("epe_fold_kernel");
    return HS_OK;
}

hs_status hs_epe_loss_backward_batched(const hs_epe_pair *pairs, int n, float eps,
                                       const float *dloss, void *stream) {
    clear_error();
    EpeTable tab;
    hs_status st = make_table(pairs, n, eps, true, tab);
    if (st != HS_OK) return st;
    if (!dloss) HS_FAIL(HS_ERR_INVALID_ARG, "dloss is NULL");
    long maxpx = 1;
    for (int i = 0; i < n; ++i) maxpx = std::max(maxpx, (long)pairs[i].H * pairs[i].W);
    const unsigned bx = (unsigned)std::min<long>((maxpx + 255) / 256, 4L * sm_count());
    epe_backward_kernel<<<dim3(bx, n), 256, 0, (cudaStream_t)stream>>>(tab, dloss);
    HS_LAUNCH_CHECK("epe_backward_kernel");
    return HS_OK;
}

}  // extern "C"
