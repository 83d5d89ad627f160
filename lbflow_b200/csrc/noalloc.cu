// noalloc.cu -- lbf_inventory_noalloc: FP64 fluid-node sums with no device allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// reduction: a service that reserved all of HBM for lattices up front and runs
// with a fixed memory budget (an allocation would fail, or evict a lattice), or
// an embedding framework whose own caching allocator owns the device memory (an
// allocation behind its back breaks its accounting).  For them this entry point
// sums caller-owned device arrays using a scratch array that lives in the
// library's static device memory, so a call performs no cudaMalloc, cudaFree or
// other allocating call.
//
// The scratch array is a file-scope __device__ array of NSLOT x NACC doubles
// (16 KiB).  Each GPU that loads the library holds one copy until the process
// exits.  Every call on a device shares it and it keeps the last call's
// partial sums, so each call clears it first; calls whose kernels overlap on the
// GPU (different streams without ordering) race on it and give wrong sums.
//
// Its device address is looked up once per device with cudaGetSymbolAddress,
// with that device current, on the first call made on that device; that first
// call also loads the four kernels below, so that no later call loads code.
// Make that first call before any stream capture starts.  The cached address
// belongs to the device's primary context: after cudaDeviceReset the next call
// must not be made (the address would be stale).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/lbflow.h"
#include "kernels.cuh"

using namespace lbf;

lbf_status lbf_internal_fail(lbf_status s, const char* msg);   // abi.cu

namespace {

static __device__ __align__(256) double g_noalloc_scratch[NSLOT * NACC];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_scratch_ptr[MAX_DEVICES] = {};

lbf_status na_fail(lbf_status s, const std::string& m) { return lbf_internal_fail(s, m.c_str()); }

__global__ void k_clear_scratch(double* scratch) {
    for (int k = threadIdx.x; k < NSLOT * NACC; k += blockDim.x) scratch[k] = 0.0;
}

// [sum rho, sum rho*u_a, sum C, sum q] over nodes whose class has no solid bit.
template <int D>
__global__ void k_inventory_class(const uint32_t* cls, long long n, const double* rho, const double* u,
                                  const double* c, const double* q, double* scratch) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < n && !(cls[i] & LBF_CLASS_SOLID)) {
        v[0] = rho[i];
        for (int a = 0; a < D; ++a) v[1 + a] = rho[i] * u[i * D + a];
        if (c) v[1 + D] = c[i];
        if (q) v[2 + D] = q[i];
    }
    block_accumulate<6>(v, scratch);
}

__global__ void k_sum_slots(const double* scratch, int nout, double* out) {
    const int k = threadIdx.x;
    if (k >= nout) return;
    double s = 0.0;
    for (int j = 0; j < NSLOT; ++j) s += scratch[j * NACC + k];
    out[k] = s;
}

// The device address of the scratch array for the current device (set-up on first use).
lbf_status scratch_for_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(LBF_EDEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return na_fail(LBF_EUNSUPPORTED, "device index beyond 63");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return na_fail(LBF_EDEVICE, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        // load every kernel of this entry point now (module loading is lazy by default)
        cudaFuncAttributes fa;
        const void* fns[4] = {(const void*)k_clear_scratch, (const void*)k_inventory_class<2>,
                              (const void*)k_inventory_class<3>, (const void*)k_sum_slots};
        for (const void* fn : fns) {
            e = cudaFuncGetAttributes(&fa, fn);
            if (e != cudaSuccess) return na_fail(LBF_EDEVICE, std::string("kernel load: ") + cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return LBF_OK;
}

}  // namespace

extern "C" lbf_status lbf_inventory_noalloc(const double* density, const double* velocity, const double* scalar,
                                            const double* q_ads, const uint32_t* node_class, int64_t n, int32_t d,
                                            double* out, void* stream) {
    if (!density || !velocity || !node_class || !out)
        return na_fail(LBF_EINVAL, "density, velocity, node_class and out must be device pointers");
    if (d != 2 && d != 3) return na_fail(LBF_EINVAL, "d must be 2 or 3");
    if (n < 1 || n > LBF_NOALLOC_MAX_NODES)
        return na_fail(LBF_EINVAL, "n must be in [1, LBF_NOALLOC_MAX_NODES = 2^31 - 1] nodes");
    double* scratch = nullptr;
    lbf_status st = scratch_for_current_device(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    k_clear_scratch<<<1, 256, 0, s>>>(scratch);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (d == 2) k_inventory_class<2><<<blocks, 256, 0, s>>>(node_class, n, density, velocity, scalar, q_ads, scratch);
    else k_inventory_class<3><<<blocks, 256, 0, s>>>(node_class, n, density, velocity, scalar, q_ads, scratch);
    k_sum_slots<<<1, 32, 0, s>>>(scratch, 3 + d, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(LBF_EDEVICE, std::string("lbf_inventory_noalloc: ") + cudaGetErrorString(e));
    return LBF_OK;
}
