// qoa_noalloc.cu — Z-string expectation values over a caller-owned device
// state vector, with no device allocation inside the library.
//
// Some callers cannot let a library call cudaMalloc: a host runtime that owns
// and accounts for every device buffer itself (for instance a VM binding that
// hands the engine memory from its own pool and must not see hidden
// allocations), or a caller on a latency-critical path where cudaMalloc's
// implicit device-wide synchronisation is not acceptable. For them this file
// provides qoa_expect_z_noalloc, a variant of the reduction behind
// qoa_expect_z whose block partial sums live in a file-scope static device
// array of fixed size instead of a buffer the handle allocates.
//
// The array is shared: every call on a device reuses it, and it keeps the last
// call's contents. Each launch writes every partial it later reads, so nothing
// in it has to start at zero. Calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on it; the caller must order them.
#include <cuda_runtime.h>

#include <mutex>
#include <stdint.h>

#include "../../include/qoa_cuda.h"

namespace qoa {
void note_global_error(const char* msg);
}

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;                    // partials per mask
constexpr int kMaxMasks = QOA_NOALLOC_MAX_MASKS;       // masks per call
constexpr int kMaxDevices = 64;

// The scratch: 8 masks x 1184 blocks x 8 bytes = 75,776 bytes on every device
// that loads the library, held until the process exits.
static __device__ __align__(256) double g_expz_scratch[kMaxMasks * kMaxBlocks];

namespace {

struct Masks {
    uint64_t m[kMaxMasks];
};

__global__ void k_expz_partials_noalloc(const double2* __restrict__ a, uint64_t len, const Masks mk, uint32_t k,
                                        double* __restrict__ partials) {
    __shared__ double sh[kMaxMasks][kThreads / 32];
    double v[kMaxMasks];
#pragma unroll
    for (int j = 0; j < kMaxMasks; ++j) v[j] = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 x = a[i];
        const double p = fma(x.x, x.x, x.y * x.y);
#pragma unroll
        for (int j = 0; j < kMaxMasks; ++j) v[j] += (__popcll(i & mk.m[j]) & 1) ? -p : p;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < kMaxMasks; ++j) {
        double x = v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[j][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double t = 0.0;
        for (int q = 0; q < kThreads / 32; ++q) t += sh[threadIdx.x][q];
        partials[(uint64_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

// One block per mask: fixed-order sum of that mask's partials.
__global__ void k_expz_reduce_noalloc(const double* __restrict__ partials, uint32_t count, double* __restrict__ out) {
    __shared__ double sh[32];
    const double* p = partials + (uint64_t)blockIdx.x * count;
    double x = 0.0;
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) x += p[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
        out[blockIdx.x] = t;
    }
}

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

extern "C" int qoa_expect_z_noalloc(const void* d_amps, size_t len, const uint64_t* masks, size_t k, double* d_out,
                                    void* stream) {
    if (!d_amps || !masks || !d_out) {
        qoa::note_global_error("qoa_expect_z_noalloc: null pointer argument");
        return QOA_E_ARG;
    }
    if (k > (size_t)kMaxMasks) {
        qoa::note_global_error("qoa_expect_z_noalloc: more than QOA_NOALLOC_MAX_MASKS (8) masks in one call; "
                               "split the masks over several calls");
        return QOA_E_ARG;
    }
    if (k == 0 || len == 0) return QOA_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        qoa::note_global_error("qoa_expect_z_noalloc: no usable current CUDA device");
        return QOA_E_NOGPU;
    }
    // Set-up, once per device with that device current: the host-side name of
    // g_expz_scratch is not a device address, so resolve the real one.
    double* scratch;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        scratch = g_scratch_ptr[dev];
        if (!scratch) {
            const cudaError_t e = cudaGetSymbolAddress((void**)&scratch, g_expz_scratch);
            if (e != cudaSuccess || !scratch) {
                qoa::note_global_error("qoa_expect_z_noalloc: cudaGetSymbolAddress of the scratch array failed");
                return QOA_E_CUDA;
            }
            g_scratch_ptr[dev] = scratch;
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t nb = (len + kThreads - 1) / kThreads;
    if (nb > (uint64_t)kMaxBlocks) nb = kMaxBlocks;
    Masks mk{};
    for (size_t j = 0; j < k; ++j) mk.m[j] = masks[j];
    k_expz_partials_noalloc<<<(unsigned)nb, kThreads, 0, st>>>((const double2*)d_amps, (uint64_t)len, mk, (uint32_t)k,
                                                               scratch);
    k_expz_reduce_noalloc<<<(unsigned)k, 1024, 0, st>>>(scratch, (uint32_t)nb, d_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        qoa::note_global_error(cudaGetErrorString(e));
        return QOA_E_CUDA;
    }
    return QOA_OK;
}
