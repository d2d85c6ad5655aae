// Allocation-free depth raster.
//
// Some hosts of this library cannot call cudaMalloc once their run has
// started: an ensemble driver that reserves all device memory up front and
// hands out fixed pools, or an application embedded in a framework that owns
// the device allocator.  For them the IDW depth raster is offered without any
// allocation: the caller passes device pointers for its inputs and its
// output, and the per-node accumulators live in a file-scope __device__ array
// of fixed size that every GPU loading this library holds until the process
// exits.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/gfsph.h"
#include "gfsph_device.cuh"

namespace {

constexpr int kNoAllocMaxNodes = GFSPH_NOALLOC_MAX_NODES;  // 1024 x 1024 DEM nodes, 16 MiB of FP64 pairs

// (sum of h/d, sum of 1/d) per DEM node.  In host code this symbol is only a
// stand-in for the device array; its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) double2 g_idw_scratch[kNoAllocMaxNodes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

__global__ void k_noalloc_clear(double2* acc, int np) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x)
        acc[k] = make_double2(0.0, 0.0);
}

// Same arithmetic as the handle's IDW raster (SPH_SW_2019.f90:14310-14400).
__global__ void k_noalloc_idw(const float2* pos, const float* rho, const int* flag, int n, int nx, int ny, float xmin,
                              float ymin, float dx, float dy, double2* acc) {
    float distg = sqrtf(dx * dx + dy * dy);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (flag && flag[i]) continue;
        float2 p = pos[i];
        float h = rho[i];
        int ipx = (int)((p.x - xmin) / dx + 1.f);
        int ipy = (int)((p.y - ymin) / dy + 1.f);
        int ix0 = max(1, ipx - 1), iy0 = max(1, ipy - 1), ix1 = min(nx, ipx + 2), iy1 = min(ny, ipy + 2);
        for (int ix = ix0; ix <= ix1; ix++)
            for (int iy = iy0; iy <= iy1; iy++) {
                int ip = (iy - 1) * nx + (ix - 1);
                float ddx = p.x - (xmin + (float)(ix - 1) * dx);
                ddx = ddx * ddx;
                float ddy = p.y - (ymin + (float)(iy - 1) * dy);
                ddy = ddy * ddy;
                float dist = sqrtf(ddx + ddy);
                dist = (1.e-6f > dist) ? 1.e-6f : dist;
                dist = dist / distg;
                atomicAdd(&acc[ip].x, (double)(h / dist));
                atomicAdd(&acc[ip].y, (double)(1.f / dist));
            }
    }
}

__global__ void k_noalloc_finish(const double2* acc, float* out, int np) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        double2 a = acc[k];
        out[k] = ((float)a.y >= 1.e-6f) ? (float)(a.x / a.y) : (float)a.x;
    }
}

// Device address of the scratch array on the current device; looked up once
// per device, on the first call made with that device current.  The cached
// address belongs to the device's primary context: it does not survive a
// cudaDeviceReset (the module is loaded again afterwards).
int scratch_address(double2** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GFSPH_ERR_NO_DEVICE;
    if (dev < 0 || dev >= kMaxDevices) return GFSPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_idw_scratch);
        if (e != cudaSuccess || !p) return GFSPH_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<double2*>(g_scratch_ptr[dev]);
    return GFSPH_OK;
}

}  // namespace

extern "C" int gfsph_raster_idw_noalloc(int n, const float* d_x, const float* d_rho, const int* d_flag, int nx,
                                        int ny, float xmin, float ymin, float dx, float dy, float* d_out,
                                        void* stream) try {
    if (n < 0 || (n > 0 && (!d_x || !d_rho)) || !d_out || nx < 2 || ny < 2 || !(dx > 0.f) || !(dy > 0.f))
        return GFSPH_ERR_ARG;
    // d_x is read as float2 (interleaved x, y): it must be 8-byte aligned;
    // the other arrays hold 4-byte elements
    if ((reinterpret_cast<uintptr_t>(d_x) & 7u) || (reinterpret_cast<uintptr_t>(d_rho) & 3u) ||
        (reinterpret_cast<uintptr_t>(d_flag) & 3u) || (reinterpret_cast<uintptr_t>(d_out) & 3u))
        return GFSPH_ERR_ARG;
    if ((long long)nx * (long long)ny > (long long)kNoAllocMaxNodes) return GFSPH_ERR_CAPACITY;
    double2* acc = nullptr;
    int st = scratch_address(&acc);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int np = nx * ny;
    int gb = (np + 255) / 256;
    if (gb > 148 * 16) gb = 148 * 16;
    k_noalloc_clear<<<gb, 256, 0, s>>>(acc, np);
    if (n > 0) {
        int pb = (n + 127) / 128;
        if (pb > 148 * 64) pb = 148 * 64;
        k_noalloc_idw<<<pb, 128, 0, s>>>(reinterpret_cast<const float2*>(d_x), d_rho, d_flag, n, nx, ny, xmin, ymin,
                                          dx, dy, acc);
    }
    k_noalloc_finish<<<gb, 256, 0, s>>>(acc, d_out, np);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GFSPH_OK : GFSPH_ERR_CUDA;
} catch (...) {  // a C++ exception never crosses the C ABI
    return GFSPH_ERR_HOST;
}
