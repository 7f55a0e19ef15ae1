// wig_noalloc.cu — an entry point that allocates no device memory: the
// FP64 squared norm of the pressure solve's residual, for callers that own
// every byte of device memory themselves.
//
// Why it exists: wig_fluid_create allocates the handle's scratch (the FP64
// per-block partial sums among it) with cudaMalloc.  Some hosts cannot let a
// library do that: a host that records its work into a CUDA graph while it
// runs (cudaMalloc is not allowed during stream capture), a host whose device
// memory is one pre-reserved pool carved up by its own allocator (a game or
// simulation engine, or a WebGPU bridge that imports buffers it does not
// own), and a host on a real-time path that cannot take the device-wide
// synchronisation cudaMalloc may imply.  Such a host drives the liquid's
// buffers itself and still wants to know how far the solve got.
//
// The scratch this needs, one FP64 partial per 8x8 block, lives in a
// file-scope static __device__ array of WIG_NOALLOC_MAX_BLOCKS entries
// (128 KiB): every GPU that loads this library holds it until the process
// exits.  The array's name in host code is only a host-side stand-in, so the
// host takes the array's device address once per device with
// cudaGetSymbolAddress (the first call on a device does that set-up) and
// passes it to the kernels.  That address is kept until
// wig_fluid_noalloc_forget_device, which a host that resets a device calls.  Every call shares the one array: calls whose
// work overlaps on the GPU (two streams, or two host threads) race on it.

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "wig_device.cuh"

namespace {

constexpr uint32_t MAX_DEVICES = 64;

// One FP64 partial sum per block; only the entries of the blocks worked on
// are written and read by a call, so nothing in it has to start at zero.
static __device__ __align__(256) double g_block_partials[WIG_NOALLOC_MAX_BLOCKS];

std::mutex g_mutex;
double* g_partials_of[MAX_DEVICES] = {nullptr};

int set_error(int code, const std::string& msg) {
    wig::set_last_error(msg);
    return code;
}

// Squared residual of the liquid cells of each block worked on (cg's y,
// the CG residual r, where field's z > 0), a tree of 64 per block, as the
// step's tolerance form sums it (k_cgUpdate).  The blocks worked on are
// those whose state word has ACTIVE set, the same set k_sum_partials reads,
// so no partial left from an earlier call (of this world or another) can
// enter the sum, whatever the active list holds.
__global__ void __launch_bounds__(64) k_block_r2(uint32_t W, uint32_t H, uint32_t B, uint32_t BW, const uint32_t* blocks,
                                                 const float4* field, const float4* cg, double* partials) {
    __shared__ double s[64];
    for (uint32_t n = blockIdx.x; n < B; n += gridDim.x) {
        if ((blocks[B + n] & 1u) == 0u) continue;  // not worked on (uniform in the CTA)
        const uint32_t bx = n % BW, by = n / BW;
        const uint32_t x = bx * 8u + (threadIdx.x & 7u), y = by * 8u + (threadIdx.x >> 3);
        double v = 0.0;
        if (x < W && y < H) {
            const uint32_t i = y * W + x;
            if (field[2u * i].z > 0.0f) {
                const double r = (double)cg[i].y;
                v = r * r;
            }
        }
        s[threadIdx.x] = v;
        __syncthreads();
        for (int h = 32; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[n] = s[0];
        __syncthreads();
    }
}

// One CTA of 256: the active blocks' partials in block-index order, 256
// strided runs and a tree (the step's k_norm order).
__global__ void __launch_bounds__(256) k_sum_partials(uint32_t B, const uint32_t* blocks, const double* partials, double* out) {
    __shared__ double s[256];
    double acc = 0.0;
    for (uint32_t k = threadIdx.x; k < B; k += 256u)
        if ((blocks[B + k] & 1u) != 0u) acc = acc + partials[k];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// The device address of g_block_partials on the current device, looked up
// once per device and kept for the process's life: a host that destroys and
// recreates a device's primary context (cudaDeviceReset) loads the module
// anew, so it must call wig_fluid_noalloc_forget_device afterwards.
int partials_on_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(WIG_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || (uint32_t)dev >= MAX_DEVICES) return set_error(WIG_E_ARG, "device ordinal past the ones this entry point keeps");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_partials_of[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_block_partials);
        if (e != cudaSuccess) return set_error(WIG_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_partials_of[dev] = static_cast<double*>(p);
    }
    *out = g_partials_of[dev];
    return WIG_OK;
}

}  // namespace

extern "C" {

int wig_fluid_residual_norm2_noalloc(const wig_world_desc* d, const void* field, const void* blocks, const void* cg,
                                     double* out, void* stream) {
    if (!d || !field || !blocks || !cg || !out) return set_error(WIG_E_ARG, "null argument");
    if (d->width == 0 || d->height == 0 || d->width > 32768 || d->height > 32768)
        return set_error(WIG_E_ARG, "world size out of range (1..32768 per side)");
    const uint32_t BW = (d->width + 7u) / 8u, BH = (d->height + 7u) / 8u;
    const uint64_t B = (uint64_t)BW * BH;
    if (B > WIG_NOALLOC_MAX_BLOCKS)
        return set_error(WIG_E_ARG, "world has " + std::to_string(B) + " blocks; the allocation-free entry point holds at most " +
                                        std::to_string(WIG_NOALLOC_MAX_BLOCKS) + " (a 1024 x 1024 world)");
    double* partials = nullptr;
    int rc = partials_on_current_device(&partials);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = B < 148u * 32u ? (unsigned)B : 148u * 32u;
    k_block_r2<<<grid, 64, 0, s>>>(d->width, d->height, (uint32_t)B, BW, (const uint32_t*)blocks, (const float4*)field,
                                   (const float4*)cg, partials);
    k_sum_partials<<<1, 256, 0, s>>>((uint32_t)B, (const uint32_t*)blocks, partials, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(WIG_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return WIG_OK;
}

int wig_fluid_noalloc_forget_device(void) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(WIG_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || (uint32_t)dev >= MAX_DEVICES) return set_error(WIG_E_ARG, "device ordinal past the ones this entry point keeps");
    std::lock_guard<std::mutex> lock(g_mutex);
    g_partials_of[dev] = nullptr;
    return WIG_OK;
}

}  // extern "C"
