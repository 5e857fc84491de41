// hs_noalloc.cu -- hs_forward_noalloc: the plain Horn-Schunck forward for callers that
// cannot allocate device memory.
//
// Its scratch (the five planes hs_forward needs: Ix, Iy, It and the ping-pong copy of
// u, v) lives in a file-scope __device__ array of HS_NOALLOC_SCRATCH_BYTES.  The array is
// part of this library's device image: every GPU that loads the library holds it until
// the process exits, and no call here allocates or frees anything.
//
// In host code the array's name is only a host-side stand-in for the symbol, not a
// device address.  The device address is obtained once per device, with that device
// current, through cudaGetSymbolAddress, and that address is what the kernels receive.
#include <mutex>

#include "hs_common.cuh"

namespace hs {

constexpr size_t kNoAllocScratchBytes = HS_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[kMaxDevices];

// Device address of g_noalloc_scratch on the current device (set up on first use).
static hs_status noalloc_scratch(void **out) {
    int dev = 0;
    HS_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        HS_FAIL(HS_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, kMaxDevices - 1);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            HS_FAIL(HS_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d failed: %s", dev,
                    cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" hs_status hs_forward_noalloc(const float *I0, const float *I1, int H, int W, int ld,
                                        float alpha, int iters, float *u, float *v,
                                        const hs_config *cfg, void *stream) {
    clear_error();
    hs_status st = check_plane_geometry(H, W, ld);
    if (st != HS_OK) return st;
    const size_t need = hs_forward_workspace_bytes(H, W, ld);
    if (need > kNoAllocScratchBytes)
        HS_FAIL(HS_ERR_WORKSPACE,
                "H=%d ld=%d needs %zu bytes of scratch; the static scratch holds %zu bytes "
                "(at most five planes of %zu bytes each)",
                H, ld, need, kNoAllocScratchBytes, kNoAllocScratchBytes / 5 / 256 * 256);
    void *ws = nullptr;
    if ((st = noalloc_scratch(&ws)) != HS_OK) return st;
    return hs_forward(I0, I1, H, W, ld, alpha, iters, u, v, ws, kNoAllocScratchBytes, cfg, stream);
}
