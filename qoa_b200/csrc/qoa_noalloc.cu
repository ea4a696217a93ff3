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
//
// A __device__ array has one address per CUDA context, not per device: a
// caller may run in a context of its own (cuCtxCreate) beside the primary
// one, and cudaDeviceReset replaces the primary context. The resolved
// address is therefore cached by the current context's id (cuCtxGetId, unique
// for the life of the process), not by device number.
#include <cuda.h>  // CUcontext / CUresult types only; the two driver calls are resolved at run time
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
constexpr int kMaxContexts = 64;                       // cached (context id, address) pairs

// The scratch: 8 masks x 1184 blocks x 8 bytes = 75,776 bytes on every device
// that loads the library, held until the process exits.
static __device__ __align__(256) double g_expz_scratch[kMaxMasks * kMaxBlocks];

namespace {

struct Masks {
    uint64_t m[kMaxMasks];
};

// K masks (1..8), so a call with fewer masks accumulates only those.
template <int K>
__global__ void k_expz_partials_noalloc(const double2* __restrict__ a, uint64_t len, const Masks mk,
                                        double* __restrict__ partials) {
    __shared__ double sh[K][kThreads / 32];
    double v[K];
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 x = a[i];
        const double p = fma(x.x, x.x, x.y * x.y);
#pragma unroll
        for (int j = 0; j < K; ++j) v[j] += (__popcll(i & mk.m[j]) & 1) ? -p : p;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        double x = v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[j][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < K) {
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

const void* const kPartials[kMaxMasks + 1] = {
    nullptr,
    (const void*)k_expz_partials_noalloc<1>, (const void*)k_expz_partials_noalloc<2>,
    (const void*)k_expz_partials_noalloc<3>, (const void*)k_expz_partials_noalloc<4>,
    (const void*)k_expz_partials_noalloc<5>, (const void*)k_expz_partials_noalloc<6>,
    (const void*)k_expz_partials_noalloc<7>, (const void*)k_expz_partials_noalloc<8>,
};

// The current context's unique id, through driver entry points the runtime
// hands out (no link against libcuda). False when unavailable or when no
// context is current.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

bool current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess) ? (CtxGetCurrentFn)f : nullptr;
    }();
    static CtxGetIdFn get_id = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess) ? (CtxGetIdFn)f : nullptr;
    }();
    CUcontext c = nullptr;
    if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c) return false;
    return get_id(c, id) == CUDA_SUCCESS;
}

struct ScratchSlot {
    unsigned long long ctx_id;
    double* ptr;
};
std::mutex g_mu;
ScratchSlot g_slots[kMaxContexts];
int g_nslots = 0;

// Device address of g_expz_scratch in the current context: cached per
// context id; resolved with cudaGetSymbolAddress on a context's first call
// (and on every call if the context id cannot be read).
cudaError_t scratch_address(double** out) {
    unsigned long long id = 0;
    bool have = current_context_id(&id);
    std::lock_guard<std::mutex> lk(g_mu);
    if (have)
        for (int i = 0; i < g_nslots; ++i)
            if (g_slots[i].ctx_id == id) {
                *out = g_slots[i].ptr;
                return cudaSuccess;
            }
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_expz_scratch);
    if (e != cudaSuccess || !p) return e != cudaSuccess ? e : cudaErrorInvalidSymbol;
    if (!have) have = current_context_id(&id);  // the runtime may have just made its context current
    if (have && g_nslots < kMaxContexts) g_slots[g_nslots++] = {id, p};
    *out = p;
    return cudaSuccess;
}

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
    if (cudaGetDevice(&dev) != cudaSuccess) {
        qoa::note_global_error("qoa_expect_z_noalloc: no usable current CUDA device");
        return QOA_E_NOGPU;
    }
    // Set-up on a context's first call: the host-side name of g_expz_scratch
    // is not a device address, so resolve the real one (cached per context).
    double* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) {
        qoa::note_global_error("qoa_expect_z_noalloc: cudaGetSymbolAddress of the scratch array failed");
        return QOA_E_CUDA;
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t nb = (len + kThreads - 1) / kThreads;
    if (nb > (uint64_t)kMaxBlocks) nb = kMaxBlocks;
    Masks mk{};
    for (size_t j = 0; j < k; ++j) mk.m[j] = masks[j];
    const double2* a = (const double2*)d_amps;
    uint64_t len64 = (uint64_t)len;
    uint32_t count = (uint32_t)nb;
    // Each launch's own status (cudaLaunchKernel returns it), so an error
    // left pending by the caller's earlier work is neither reported nor cleared.
    void* pargs[] = {(void*)&a, (void*)&len64, (void*)&mk, (void*)&scratch};
    cudaError_t e = cudaLaunchKernel(kPartials[k], dim3((unsigned)nb), dim3(kThreads), pargs, 0, st);
    if (e == cudaSuccess) {
        void* rargs[] = {(void*)&scratch, (void*)&count, (void*)&d_out};
        e = cudaLaunchKernel((const void*)k_expz_reduce_noalloc, dim3((unsigned)k), dim3(1024), rargs, 0, st);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();  // this call's own launch error
        qoa::note_global_error(cudaGetErrorString(e));
        return QOA_E_CUDA;
    }
    return QOA_OK;
}
