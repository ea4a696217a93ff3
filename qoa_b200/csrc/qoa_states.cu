// qoa_states.cu — seeded random states and state comparison on the device.
//
// qoa_set_random_state draws re and im of every amplitude i.i.d. N(0,1):
// Philox4x32-10 (Salmon et al., SC'11) keyed by the seed with the amplitude
// index as counter gives two 53-bit uniforms, turned into two normals by the
// Box-Muller transform. A complex64 handle stores the complex128 draws
// rounded, so two handles seeded alike hold the same state. The stored vector
// is left unnormalised and its squared norm goes to the handle's norm2, which
// every consumer divides out (the engine's lazy renormalisation).
//
// qoa_compare reads two states of equal size (either precision) in one pass:
// the relative L2 distance and 1 - |<a|b>|^2 of the normalised vectors.
#include <cuda_runtime.h>
#include <stdint.h>

#include "qoa_kernels.cuh"

namespace qoa {

__device__ __forceinline__ void philox_dev(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

template <typename T>
__device__ __forceinline__ void store_amp(T* a, uint64_t i, double re, double im);
template <>
__device__ __forceinline__ void store_amp<double2>(double2* a, uint64_t i, double re, double im) {
    a[i] = make_double2(re, im);
}
template <>
__device__ __forceinline__ void store_amp<float2>(float2* a, uint64_t i, double re, double im) {
    a[i] = make_float2((float)re, (float)im);
}

template <typename T>
__global__ void k_random_state(T* __restrict__ a, uint64_t len, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0x73746174u, 0u};
        philox_dev(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        const uint64_t b1 = ((uint64_t)c[0] << 32) | c[1], b2 = ((uint64_t)c[2] << 32) | c[3];
        const double u1 = ((double)(b1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
        const double u2 = (double)(b2 >> 11) * (1.0 / 9007199254740992.0);          // [0, 1)
        const double r = sqrt(-2.0 * log(u1));
        double s, co;
        sincospi(2.0 * u2, &s, &co);
        store_amp<T>(a, i, r * co, r * s);
    }
}

template <typename T>
__device__ __forceinline__ double2 load_amp(const T* a, uint64_t i);
template <>
__device__ __forceinline__ double2 load_amp<double2>(const double2* a, uint64_t i) {
    return a[i];
}
template <>
__device__ __forceinline__ double2 load_amp<float2>(const float2* a, uint64_t i) {
    const float2 x = a[i];
    return make_double2(x.x, x.y);
}

// partials: [0] sum |a sa - b sb|^2, [1] Re <a|b>, [2] Im <a|b> (normalised)
template <typename TA, typename TB>
__global__ void k_compare(const TA* __restrict__ a, const TB* __restrict__ b, uint64_t len,
                          const double* __restrict__ na, const double* __restrict__ nb, double* __restrict__ partials) {
    __shared__ double sh[3][32];
    const double sa = 1.0 / sqrt(*na), sb = 1.0 / sqrt(*nb);
    double v[3] = {0.0, 0.0, 0.0};
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 x = load_amp<TA>(a, i), y = load_amp<TB>(b, i);
        const double xr = x.x * sa, xi = x.y * sa, yr = y.x * sb, yi = y.y * sb;
        const double dr = xr - yr, di = xi - yi;
        v[0] += dr * dr + di * di;
        v[1] += xr * yr + xi * yi;  // conj(x) y
        v[2] += xr * yi - xi * yr;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) sh[k][w] = t;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[threadIdx.x][k];
        partials[(uint64_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

int reduce_blocks(uint64_t len);
cudaError_t launch_reduce_sets(const double* partials, uint32_t count, uint32_t sets, double* out, cudaStream_t st);

cudaError_t launch_random_state(void* a, bool f32, uint64_t len, uint64_t seed, cudaStream_t st) {
    uint64_t blocks = (len + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (f32) k_random_state<float2><<<(unsigned)blocks, 256, 0, st>>>((float2*)a, len, seed);
    else k_random_state<double2><<<(unsigned)blocks, 256, 0, st>>>((double2*)a, len, seed);
    return cudaGetLastError();
}

cudaError_t launch_compare(const void* a, bool af32, const void* b, bool bf32, uint64_t len, const double* na,
                           const double* nb, double* partials, double* out3, cudaStream_t st) {
    const int nb_ = reduce_blocks(len);
    if (!af32 && !bf32)
        k_compare<double2, double2><<<nb_, 256, 0, st>>>((const double2*)a, (const double2*)b, len, na, nb, partials);
    else if (!af32 && bf32)
        k_compare<double2, float2><<<nb_, 256, 0, st>>>((const double2*)a, (const float2*)b, len, na, nb, partials);
    else if (af32 && !bf32)
        k_compare<float2, double2><<<nb_, 256, 0, st>>>((const float2*)a, (const double2*)b, len, na, nb, partials);
    else
        k_compare<float2, float2><<<nb_, 256, 0, st>>>((const float2*)a, (const float2*)b, len, na, nb, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce_sets(partials, (uint32_t)nb_, 3, out3, st);
}

}  // namespace qoa
