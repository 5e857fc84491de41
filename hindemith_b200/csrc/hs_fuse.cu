// hs_fuse.cu -- runtime-compiled fused kernels for arbitrary Stencil / Array2D programs.
//
// The reference generates OpenCL C for each fused group of statements and compiles it at
// run time (fusion.cpp:113-303 decides the groups, lm.cpp:467-755 emits the code,
// oclgen.cpp:156-185 builds and enqueues it).  Here the front end emits the per-pixel body
// of one fused group as CUDA C; this file wraps it in a fixed kernel skeleton (pixel
// indexing, clamp-to-edge loads, deterministic block reductions for sum2d), compiles it
// with NVRTC for sm_100a into a cubin, loads it context-independently
// (cudaLibraryLoadData) and launches it.  Kernels are cached by their full source.
//
// The body sees, for the pixel (X, Y) of an H x W grid with row stride ld:
//   IN(k)          input plane k at the pixel
//   LD(k, dx, dy)  input plane k at the clamped neighbour (X+dx, Y+dy)
//   OUT(k) = v;    store to output plane k
//   S(k)           scalar parameter k
//   SUM(k, v);     add v to reduction k (accumulated in double, folded in a fixed order)
// Exact programs compile with -fmad=false (one rounding per operation, as the reference's
// statement semantics); fast programs with -fmad=true.
#include <dlfcn.h>

#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include <nvrtc.h>

#include "hs_common.cuh"

namespace hs {

constexpr int kFuseBX = 32, kFuseBY = 8;

static const char *kHead = R"(
struct hsf_args {
    const float *in[16];
    float *out[8];
    float s[64];
    int H, W, ld, nsums;
    double *sums;
    int reserved[4];
};
__device__ __forceinline__ float hsf_ld(const float *p, int x, int y, int H, int W, int ld) {
    x = x < 0 ? 0 : (x > W - 1 ? W - 1 : x);
    y = y < 0 ? 0 : (y > H - 1 ? H - 1 : y);
    return p[(size_t)y * ld + x];
}
#define IN(k) (a.in[k][o])
#define LD(k, dx, dy) hsf_ld(a.in[k], X + (dx), Y + (dy), a.H, a.W, a.ld)
#define OUT(k) a.out[k][o]
#define S(k) (a.s[k])
#define SUM(k, v) (acc[k] += (double)(v))
extern "C" __global__ void __launch_bounds__(256) hsf_kernel(const __grid_constant__ hsf_args a,
                                                             double *partials) {
    const int X = blockIdx.x * 32 + threadIdx.x, Y = blockIdx.y * 8 + threadIdx.y;
    double acc[HSF_NSUM + 1];
    for (int k = 0; k <= HSF_NSUM; ++k) acc[k] = 0.0;
    if (X < a.W && Y < a.H) {
        const size_t o = (size_t)Y * a.ld + X;
        (void)o;
)";

static const char *kTail = R"(
    }
#if HSF_NSUM > 0
    __shared__ double red[8][HSF_NSUM];
    const int lane = threadIdx.x, wy = threadIdx.y;
    for (int k = 0; k < HSF_NSUM; ++k) {
        double v = acc[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[wy][k] = v;
    }
    __syncthreads();
    if (lane == 0 && wy == 0) {
        const size_t b = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
        for (int k = 0; k < HSF_NSUM; ++k) {
            double t = 0.0;
            for (int w = 0; w < 8; ++w) t += red[w][k];
            partials[b * HSF_NSUM + k] = t;
        }
    }
#endif
}
)";

// ------------------------------------------------------------------ NVRTC, loaded on use

struct Nvrtc {
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    bool ok = false;
};

static Nvrtc &nvrtc() {
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void *h = nullptr;
        for (const char *nm : names)
            if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
        if (!h) return;
        n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
        n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
        n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
        n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
        n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
        n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
        n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
        n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    });
    return n;
}

struct Compiled {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
};

static std::mutex g_mu;
static std::unordered_map<std::string, Compiled> g_cache;

static hs_status compile_fused(const std::string &src, bool fast, Compiled &out) {
    Nvrtc &n = nvrtc();
    if (!n.ok) HS_FAIL(HS_ERR_UNSUPPORTED, "fused kernels need NVRTC (libnvrtc.so.12), which could not be loaded");
    nvrtcProgram prog;
    if (n.create(&prog, src.c_str(), "hs_fused.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        HS_FAIL(HS_ERR_CUDA, "nvrtcCreateProgram failed");
    const char *opts[] = {"-arch=sm_100a", "-std=c++17", fast ? "-fmad=true" : "-fmad=false"};
    const nvrtcResult r = n.compile(prog, 3, opts);
    if (r != NVRTC_SUCCESS) {
        size_t ls = 0;
        n.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) n.log(prog, &log[0]);
        n.destroy(&prog);
        HS_FAIL(HS_ERR_INVALID_ARG, "fused kernel does not compile: %.900s", log.c_str());
    }
    size_t cs = 0;
    n.cubin_size(prog, &cs);
    std::string cubin(cs, '\0');
    n.cubin(prog, &cubin[0]);
    n.destroy(&prog);
    HS_CUDA_CHECK(cudaLibraryLoadData(&out.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    HS_CUDA_CHECK(cudaLibraryGetKernel(&out.kernel, out.lib, "hsf_kernel"));
    return HS_OK;
}

// Fold of the per-block partials of each sum in a fixed order, the same on every run: thread t
// adds blocks t, t + kFoldThreads, ... in turn (coalesced across the block), then a
// shared-memory tree with fixed pairs.  A 1080p grid has 8100 blocks: 8 loads per thread,
// where a single thread walking them in turn took about 0.25 ms.
constexpr int kFoldThreads = 1024;

__global__ void __launch_bounds__(kFoldThreads) fuse_fold_kernel(const double *partials, int nblocks,
                                                                 int nsums, double *sums) {
    __shared__ double red[kFoldThreads];
    for (int k = 0; k < nsums; ++k) {
        double t = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += kFoldThreads) t += partials[(size_t)b * nsums + k];
        red[threadIdx.x] = t;
        __syncthreads();
        for (int h = kFoldThreads / 2; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) sums[k] = red[0];
        __syncthreads();  // red[0] is read before the next sum overwrites it
    }
}

static inline size_t fuse_blocks(int H, int W) {
    return (size_t)((W + kFuseBX - 1) / kFuseBX) * (size_t)((H + kFuseBY - 1) / kFuseBY);
}

}  // namespace hs

using namespace hs;

extern "C" {

size_t hs_fused_workspace_bytes(int H, int W, int nsums) {
    if (H < 1 || W < 1 || nsums < 0 || nsums > HS_FUSED_MAX_SUMS) return 0;
    const size_t b = nsums * fuse_blocks(H, W) * sizeof(double);
    return (b + 255) & ~(size_t)255;
}

hs_status hs_fused_launch(const char *body, int fast_math, const hs_fused_args *args,
                          void *workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    if (!body || !args) HS_FAIL(HS_ERR_INVALID_ARG, "body and args must be non-NULL");
    hs_status st = check_plane_geometry(args->H, args->W, args->ld);
    if (st != HS_OK) return st;
    if (args->nsums < 0 || args->nsums > HS_FUSED_MAX_SUMS)
        HS_FAIL(HS_ERR_INVALID_ARG, "nsums=%d outside 0..%d", args->nsums, HS_FUSED_MAX_SUMS);
    for (int i = 0; i < 4; ++i)
        if (args->reserved[i] != 0) HS_FAIL(HS_ERR_INVALID_ARG, "reserved must be zero");
    if (args->nsums > 0) {
        if (!args->sums) HS_FAIL(HS_ERR_INVALID_ARG, "sums is NULL with nsums > 0");
        if (!workspace || workspace_bytes < hs_fused_workspace_bytes(args->H, args->W, args->nsums))
            HS_FAIL(HS_ERR_WORKSPACE, "workspace %zu bytes < required %zu", workspace_bytes,
                    hs_fused_workspace_bytes(args->H, args->W, args->nsums));
    }
    for (int k = 0; k < HS_FUSED_MAX_IN; ++k)
        if (args->in[k] && (st = check_plane(args->in[k], "in")) != HS_OK) return st;
    for (int k = 0; k < HS_FUSED_MAX_OUT; ++k)
        if (args->out[k] && (st = check_plane(args->out[k], "out")) != HS_OK) return st;
    std::string src = "#define HSF_NSUM " + std::to_string(args->nsums) + "\n";
    src += kHead;
    src += body;
    src += kTail;
    const std::string key = std::string(fast_math ? "F" : "E") + src;
    Compiled kern;
    {
        std::lock_guard<std::mutex> g(g_mu);
        auto it = g_cache.find(key);
        if (it == g_cache.end()) {
            if ((st = compile_fused(src, fast_math != 0, kern)) != HS_OK) return st;
            g_cache.emplace(key, kern);
        } else {
            kern = it->second;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((unsigned)((args->W + kFuseBX - 1) / kFuseBX), (unsigned)((args->H + kFuseBY - 1) / kFuseBY));
    double *partials = reinterpret_cast<double *>(workspace);
    void *params[2] = {const_cast<hs_fused_args *>(args), &partials};
    HS_CUDA_CHECK(cudaLaunchKernel(reinterpret_cast<const void *>(kern.kernel), grid,
                                   dim3(kFuseBX, kFuseBY), params, 0, s));
    if (args->nsums > 0) {
        fuse_fold_kernel<<<1, kFoldThreads, 0, s>>>(partials, (int)fuse_blocks(args->H, args->W),
                                                    args->nsums, args->sums);
        HS_LAUNCH_CHECK("fuse_fold_kernel");
    }
    return HS_OK;
}

}  // extern "C"
