// qoa_batch.cu — many small circuits in one persistent launch.
//
// Each CTA repeatedly takes the next circuit index from a global atomic
// counter (no waiting on other CTAs), builds |0..0> of that circuit in shared
// memory, applies its gate list there, and reduces its Z-string expectation
// values straight from shared memory, so a small state never travels to HBM
// (unless the circuit is sampled afterwards: then its final state is written
// out for the sampler).
// Circuits of up to SMALL_MAX_F64 (complex128) or SMALL_MAX_F32 (complex64)
// qubits fit; larger ones go through the tile passes of the engine.
#include <cuda_runtime.h>
#include <stdint.h>

#include "qoa_kernels.cuh"

namespace qoa {

template <typename T>
struct Cx;
template <>
struct Cx<double2> {
    using R = double;
    __device__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <>
struct Cx<float2> {
    using R = float;
    __device__ static float2 make(double x, double y) { return make_float2((float)x, (float)y); }
};

template <typename T>
__device__ void small_apply(T* s, uint32_t n, const SmallOp& op) {
    using R = typename Cx<T>::R;
    const uint32_t len = 1u << n;
    const uint32_t cm = op.cmask;
    if (op.kind == SK_G1) {
        const uint32_t bit = 1u << op.t;
        const R m0x = (R)op.m[0].x, m0y = (R)op.m[0].y, m1x = (R)op.m[1].x, m1y = (R)op.m[1].y;
        const R m2x = (R)op.m[2].x, m2y = (R)op.m[2].y, m3x = (R)op.m[3].x, m3y = (R)op.m[3].y;
        for (uint32_t p = threadIdx.x; p < (len >> 1); p += blockDim.x) {
            const uint32_t i = ((p >> op.t) << (op.t + 1)) | (p & (bit - 1));
            if ((i & cm) != cm) continue;
            const uint32_t j = i | bit;
            const T a0 = s[i], a1 = s[j];
            s[i] = Cx<T>::make(m0x * a0.x - m0y * a0.y + m1x * a1.x - m1y * a1.y,
                               m0x * a0.y + m0y * a0.x + m1x * a1.y + m1y * a1.x);
            s[j] = Cx<T>::make(m2x * a0.x - m2y * a0.y + m3x * a1.x - m3y * a1.y,
                               m2x * a0.y + m2y * a0.x + m3x * a1.y + m3y * a1.x);
        }
    } else if (op.kind == SK_DIAG) {
        // factor (bit t ? m1 : m0) where (i & cmask) == cmask; t = 255: none
        const R d0x = (R)op.m[0].x, d0y = (R)op.m[0].y, d1x = (R)op.m[1].x, d1y = (R)op.m[1].y;
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
            if ((i & cm) != cm) continue;
            const bool sel = op.t < 32 && ((i >> op.t) & 1u);
            const R fx = sel ? d1x : d0x, fy = sel ? d1y : d0y;
            const T a = s[i];
            s[i] = Cx<T>::make(a.x * fx - a.y * fy, a.x * fy + a.y * fx);
        }
    } else if (op.kind == SK_SWAP) {
        const uint32_t b1 = 1u << op.t, b2 = 1u << op.t2;
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
            if ((i & (b1 | b2)) || (i & cm) != cm) continue;
            const T x = s[i | b2];
            s[i | b2] = s[i | b1];
            s[i | b1] = x;
        }
    }
    __syncthreads();
}

template <typename T>
__global__ void k_small_batch(const SmallCircuit* __restrict__ circs, uint32_t count, const SmallOp* __restrict__ ops,
                              const uint64_t* __restrict__ masks, double* __restrict__ out,
                              unsigned int* __restrict__ counter) {
    extern __shared__ unsigned char smraw[];
    T* s = reinterpret_cast<T*>(smraw);
    __shared__ uint32_t cidx;
    __shared__ double red[8 + 1][32];
    while (true) {
        if (threadIdx.x == 0) cidx = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t c = cidx;
        __syncthreads();
        if (c >= count) break;
        const SmallCircuit ci = circs[c];
        const uint32_t len = 1u << ci.n;
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) s[i] = Cx<T>::make(i == 0 ? 1.0 : 0.0, 0.0);
        __syncthreads();
        for (uint32_t k = 0; k < ci.op_count; ++k) small_apply<T>(s, ci.n, ops[ci.op_start + k]);
        if (ci.state_out)  // sampled after the run: the state goes to HBM
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) reinterpret_cast<T*>(ci.state_out)[i] = s[i];
        // <Z_mask> of the normalised state, 8 masks per sweep
        for (uint32_t m0 = 0; m0 < ci.mask_count; m0 += 8) {
            double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            uint64_t mk[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) mk[q] = (m0 + q < ci.mask_count) ? masks[ci.mask_start + m0 + q] : 0;
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
                const T a = s[i];
                const double p = (double)a.x * a.x + (double)a.y * a.y;
                v[8] += p;
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] += (__popcll((uint64_t)i & mk[q]) & 1) ? -p : p;
            }
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                double x = v[q];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 0) red[q][w] = x;
            }
            __syncthreads();
            if (threadIdx.x < 8 && m0 + threadIdx.x < ci.mask_count) {
                double t = 0.0, nrm = 0.0;
                for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { t += red[threadIdx.x][k]; nrm += red[8][k]; }
                out[ci.out_start + m0 + threadIdx.x] = t / nrm;
            }
            __syncthreads();
        }
    }
}

cudaError_t launch_small_batch(bool f32, const SmallCircuit* circs, uint32_t count, const SmallOp* ops,
                               const uint64_t* masks, double* out, unsigned int* counter, int max_n, int threads,
                               int ctas_per_sm, cudaStream_t st) {
    const size_t smem = (size_t)(f32 ? sizeof(float2) : sizeof(double2)) << max_n;
    // the attribute allows the largest state the kernel takes, the same for
    // every call: batches prepared on several host threads (the server's
    // workers) launch it concurrently with different sizes, and a smaller
    // setting made between another thread's set-up and launch fails that launch
    const int smem_cap = (int)((f32 ? sizeof(float2) : sizeof(double2)) << (f32 ? SMALL_MAX_F32 : SMALL_MAX_F64));
    if ((int)smem > smem_cap) return cudaErrorInvalidValue;
    cudaError_t e;
    if (f32) e = cudaFuncSetAttribute(k_small_batch<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap);
    else e = cudaFuncSetAttribute(k_small_batch<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    unsigned grid = (unsigned)(sms * ctas_per_sm);
    if (grid > count) grid = count ? count : 1;
    if (f32) k_small_batch<float2><<<grid, threads, smem, st>>>(circs, count, ops, masks, out, counter);
    else k_small_batch<double2><<<grid, threads, smem, st>>>(circs, count, ops, masks, out, counter);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// <Z_mask> of the arena circuits: kernel 1 sums chunks of EXPZ_CHUNK
// amplitudes of every circuit (one CTA per chunk, every mask of the circuit
// plus the squared norm); kernel 2 (one CTA per circuit) adds each slot's
// chunk sums in chunk order and divides by the norm, so results do not depend
// on the launch shape.
template <typename T>
__device__ __forceinline__ double amp_abs2(const T* a, uint64_t i) {
    const T x = a[i];
    return (double)x.x * x.x + (double)x.y * x.y;
}

template <typename T>
__global__ void __launch_bounds__(256) k_arena_expz_partials(const ExpzJob* __restrict__ jobs, uint32_t njobs,
                                                             const uint64_t* __restrict__ masks,
                                                             double* __restrict__ partials) {
    __shared__ double red[9][8];
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (jobs[mid].chunk_start <= b) lo = mid;
        else hi = mid - 1;
    }
    const ExpzJob J = jobs[lo];
    const T* a = reinterpret_cast<const T*>(J.amps);
    const uint64_t c = b - J.chunk_start;
    const uint64_t len = 1ull << J.n;
    const uint64_t begin = c * EXPZ_CHUNK;
    const uint64_t end = begin + EXPZ_CHUNK < len ? begin + EXPZ_CHUNK : len;
    const uint32_t slots = J.mask_count + 1;
    double* out = partials + J.part_start + c * slots;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t m0 = 0; m0 == 0 || m0 < J.mask_count; m0 += 8) {
        double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        uint64_t mk[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) mk[q] = (m0 + q < J.mask_count) ? masks[J.mask_start + m0 + q] : 0;
        for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
            const double p = amp_abs2<T>(a, i);
            v[8] += p;
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] += (__popcll(i & mk[q]) & 1) ? -p : p;
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            double x = v[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) red[q][w] = x;
        }
        __syncthreads();
        if (threadIdx.x < 9) {
            double t = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[threadIdx.x][k];
            const uint32_t slot = threadIdx.x < 8 ? m0 + threadIdx.x : J.mask_count;
            if (slot < J.mask_count || (threadIdx.x == 8 && m0 == 0)) out[slot] = t;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_arena_expz_final(const ExpzJob* __restrict__ jobs,
                                                          const double* __restrict__ partials,
                                                          double* __restrict__ out) {
    __shared__ double sums[EXPZ_MAX_MASKS + 1];
    const ExpzJob J = jobs[blockIdx.x];
    const uint32_t slots = J.mask_count + 1;
    const uint64_t len = 1ull << J.n;
    const uint32_t chunks = (uint32_t)((len + EXPZ_CHUNK - 1) / EXPZ_CHUNK);
    for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
        double t = 0.0;
        for (uint32_t c = 0; c < chunks; ++c) t += partials[J.part_start + (uint64_t)c * slots + s];
        sums[s] = t;
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s < J.mask_count; s += blockDim.x)
        out[J.out_start + s] = sums[s] / sums[J.mask_count];
}

cudaError_t launch_arena_expz(bool f32, const ExpzJob* jobs, uint32_t njobs, uint32_t chunks, const uint64_t* masks,
                              double* partials, double* out, cudaStream_t st) {
    if (!njobs) return cudaSuccess;
    if (f32) k_arena_expz_partials<float2><<<chunks, 256, 0, st>>>(jobs, njobs, masks, partials);
    else k_arena_expz_partials<double2><<<chunks, 256, 0, st>>>(jobs, njobs, masks, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_arena_expz_final<<<njobs, 256, 0, st>>>(jobs, partials, out);
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// Shots of sampled batch circuits: one CTA per circuit builds the marginal
// tree of its final state in global scratch (level k, 1 <= k < n, holds the
// 2^k sums over qubits k..n-1 at tree + 2^k - 2, as k_tree_leaf / k_tree_up
// lay it out), then each thread takes shots and walks the tree from qubit 0:
// the inverse-CDF rule of k_sample mode 1 (bit q = 0 while the remaining mass
// is below the marginal of that prefix). The tree is not divided by the norm:
// the states of a batch are unit vectors up to rounding, and t = u x total
// scales with it.
__device__ __forceinline__ double samp_abs2(const double2* a, uint64_t i) {
    const double2 x = a[i];
    return fma(x.x, x.x, x.y * x.y);
}
__device__ __forceinline__ double samp_abs2(const float2* a, uint64_t i) {
    const float2 x = a[i];
    return (double)x.x * x.x + (double)x.y * x.y;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_sample_jobs(const SampleJob* __restrict__ jobs, const double* __restrict__ u,
                                                      unsigned long long* __restrict__ out) {
    const SampleJob J = jobs[blockIdx.x];
    const T* a = reinterpret_cast<const T*>(J.amps);
    const uint32_t n = J.n;
    double* tree = J.tree;
    if (n >= 2) {
        const uint64_t half = 1ull << (n - 1);
        double* leaf = tree + (half - 2);
        for (uint64_t p = threadIdx.x; p < half; p += blockDim.x) leaf[p] = samp_abs2(a, p) + samp_abs2(a, p + half);
        __syncthreads();
        for (int k = (int)n - 2; k >= 1; --k) {
            const uint64_t cnt = 1ull << k;
            const double* hi = tree + ((2ull << k) - 2);
            double* lo = tree + (cnt - 2);
            for (uint64_t p = threadIdx.x; p < cnt; p += blockDim.x) lo[p] = hi[p] + hi[p + cnt];
            __syncthreads();
        }
    }
    auto h = [&](uint32_t k, uint64_t p) -> double {
        if (k == n) return samp_abs2(a, p);
        if (k == 0) return n == 1 ? samp_abs2(a, 0) + samp_abs2(a, 1) : tree[0] + tree[1];
        return tree[((1ull << k) - 2) + p];
    };
    for (uint32_t s = threadIdx.x; s < J.shots; s += blockDim.x) {
        double t = u[J.u_start + s] * h(0, 0);
        uint64_t pre = 0;
        for (uint32_t q = 0; q < n; ++q) {
            const double left = h(q + 1, pre);
            if (t < left) continue;
            t -= left;
            pre |= 1ull << q;
        }
        out[J.out_start + s] = pre;
    }
}

cudaError_t launch_sample_jobs(bool f32, const SampleJob* jobs, uint32_t njobs, const double* u,
                               unsigned long long* out, cudaStream_t st) {
    if (!njobs) return cudaSuccess;
    if (f32) k_sample_jobs<float2><<<njobs, 1024, 0, st>>>(jobs, u, out);
    else k_sample_jobs<double2><<<njobs, 1024, 0, st>>>(jobs, u, out);
    return cudaGetLastError();
}

}  // namespace qoa
