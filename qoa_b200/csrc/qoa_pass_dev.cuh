// qoa_pass_dev.cuh — device building blocks of the complex128 tile pass:
// complex arithmetic, the 2x2 forms on a register bit, conditioned X/Y and
// diagonal factors, the shared-memory swizzle, and the per-CTA angle phases
// and norm partials. Compiled twice: into the interpreter kernel (k_pass, by
// nvcc) and into the per-pass kernels generated at run time (qoa_jit.cpp, by
// NVRTC, which sees this file and qoa_kernels.cuh as in-memory headers).
#pragma once
#include "qoa_kernels.cuh"

namespace qoa {

// ------------------------------------------------------------------ helpers
// Amplitudes are complex128 (double2, the plain method) or complex64 (float2,
// the precision form's tile passes); one template serves both, arithmetic in
// the amplitude's own precision.
template <typename T> struct CT;
template <> struct CT<double2> {
    using R = double;
    __device__ __forceinline__ static double2 mk(double x, double y) { return make_double2(x, y); }
    __device__ __forceinline__ static double2 from(double2 c) { return c; }
};
template <> struct CT<float2> {
    using R = float;
    __device__ __forceinline__ static float2 mk(float x, float y) { return make_float2(x, y); }
    __device__ __forceinline__ static float2 from(double2 c) { return make_float2((float)c.x, (float)c.y); }
};

template <typename T>
__device__ __forceinline__ T c_mul(T a, T b) {
    return CT<T>::mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <typename T>
__device__ __forceinline__ T c_neg(T a) { return CT<T>::mk(-a.x, -a.y); }
__device__ __forceinline__ double c_abs2(double2 a) { return fma(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ double c_abs2(float2 a) { return (double)a.x * a.x + (double)a.y * a.y; }

// 2x2 on the amplitude pair (a0 = bit 0, a1 = bit 1). G1_H is the exact
// Hadamard (per-gate kernels); G1_HF drops its 1/sqrt2 (tile passes).
template <int SUB, typename T>
__device__ __forceinline__ void g1_pair(T& a0, T& a1, const T m0, const T m1, const T m2, const T m3) {
    using R = typename CT<T>::R;
    auto mk = [](R x, R y) { return CT<T>::mk(x, y); };
    if (SUB == G1_H) {
        const R f = m0.x;
        const R sx = a0.x + a1.x, sy = a0.y + a1.y;
        const R dx = a0.x - a1.x, dy = a0.y - a1.y;
        a0 = mk(f * sx, f * sy);
        a1 = mk(f * dx, f * dy);
    } else if (SUB == G1_HF) {
        const T t = a0;
        a0 = mk(t.x + a1.x, t.y + a1.y);
        a1 = mk(t.x - a1.x, t.y - a1.y);
    } else if (SUB == G1_X) {
        const T t = a0;
        a0 = a1;
        a1 = t;
    } else if (SUB == G1_Y) {
        const T t = a0;
        a0 = mk(a1.y, -a1.x);   // -i * a1
        a1 = mk(-t.y, t.x);     //  i * a0
    } else if (SUB == G1_RX) {
        const R c = m0.x, s = m0.y;
        const T t = a0;
        a0 = mk(fma(c, t.x, s * a1.y), fma(c, t.y, -s * a1.x));
        a1 = mk(fma(s, t.y, c * a1.x), fma(-s, t.x, c * a1.y));
    } else if (SUB == G1_RY) {
        const R c = m0.x, s = m0.y;
        const T t = a0;
        a0 = mk(fma(c, t.x, -s * a1.x), fma(c, t.y, -s * a1.y));
        a1 = mk(fma(s, t.x, c * a1.x), fma(s, t.y, c * a1.y));
    } else if (SUB == G1_RXA) {
        const R t = m0.x;
        const T u = a0;
        a0 = mk(fma(t, a1.y, u.x), fma(-t, a1.x, u.y));
        a1 = mk(fma(t, u.y, a1.x), fma(-t, u.x, a1.y));
    } else if (SUB == G1_RXB) {
        const R r = m0.x;
        const T u = a0;
        a0 = mk(fma(r, u.x, a1.y), fma(r, u.y, -a1.x));
        a1 = mk(fma(r, a1.x, u.y), fma(r, a1.y, -u.x));
    } else if (SUB == G1_RYA) {
        const R t = m0.x;
        const T u = a0;
        a0 = mk(fma(-t, a1.x, u.x), fma(-t, a1.y, u.y));
        a1 = mk(fma(t, u.x, a1.x), fma(t, u.y, a1.y));
    } else if (SUB == G1_RYB) {
        const R r = m0.x;
        const T u = a0;
        a0 = mk(fma(r, u.x, -a1.x), fma(r, u.y, -a1.y));
        a1 = mk(fma(r, a1.x, u.x), fma(r, a1.y, u.y));
    } else {
        const T t = a0;
        T r0 = c_mul(m0, t), r1 = c_mul(m2, t);
        r0.x = fma(m1.x, a1.x, r0.x); r0.x = fma(-m1.y, a1.y, r0.x);
        r0.y = fma(m1.x, a1.y, r0.y); r0.y = fma(m1.y, a1.x, r0.y);
        r1.x = fma(m3.x, a1.x, r1.x); r1.x = fma(-m3.y, a1.y, r1.x);
        r1.y = fma(m3.x, a1.y, r1.y); r1.y = fma(m3.y, a1.x, r1.y);
        a0 = r0;
        a1 = r1;
    }
}

// ------------------------------------------------- tile pass building blocks
template <int SUB, int K, typename T>
__device__ __forceinline__ void g1r(T (&a)[REGS], const T* __restrict__ m) {
    T m0 = CT<T>::mk(0, 0), m1 = m0, m2 = m0, m3 = m0;
    if (SUB != G1_HF && SUB != G1_X && SUB != G1_Y) m0 = m[0];
    if (SUB == G1_GEN) { m1 = m[1]; m2 = m[2]; m3 = m[3]; }
#pragma unroll
    for (int v = 0; v < REGS; ++v)
        if (!(v & (1 << K))) g1_pair<SUB>(a[v], a[v | (1 << K)], m0, m1, m2, m3);
}

// X / Y where every condition bit is set (tp: lane / warp / outer part)
template <int SUB, int K, typename T>
__device__ __forceinline__ void g1rc(T (&a)[REGS], bool tp, uint32_t creg) {
    if (!tp) return;
    const T z = CT<T>::mk(0, 0);
#pragma unroll
    for (int v = 0; v < REGS; ++v)
        if (!(v & (1 << K)) && (v & creg) == creg) g1_pair<SUB>(a[v], a[v | (1 << K)], z, z, z, z);
}

template <typename T>
__device__ __forceinline__ void diag_m(T (&a)[REGS], bool tp, uint32_t creg, T d) {
    if (!tp) return;
#pragma unroll
    for (int v = 0; v < REGS; ++v)
        if ((v & creg) == creg) a[v] = c_mul(a[v], d);
}

// Shared-memory position of tile index j: the low three bits are XORed with
// the three-bit folds of the higher bits, so any three tile bits with distinct
// residues mod 3 spread a quarter-warp's 16-byte accesses over all banks.
__device__ __forceinline__ uint32_t spos(uint32_t j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7u); }

// Angle phases of one CTA (tile number blk): op a sums the thetas of its
// entries whose outer condition holds, then stores e^{i sum}.
template <typename T>
__device__ __forceinline__ void pass_angles(const PassParams& P, const uint64_t blk, T* sang) {
    for (uint32_t ai = threadIdx.x; ai < P.nang; ai += PASS_THREADS) {
        double th = 0.0;
        for (uint32_t e = P.ang_start[ai]; e < P.ang_start[ai + 1]; ++e) {
            const uint64_t om = P.angles[e].omask;
            if ((blk & om) == om) th += P.angles[e].theta;
        }
        double sn, cs;
        sincos(th, &sn, &cs);
        sang[ai] = CT<T>::from(make_double2(cs, sn));
    }
}

// ------------------------------------------ streamed tiles (generated passes)
// A persistent pass CTA walks tiles blockIdx.x, +gridDim.x, ... and keeps two
// shared-memory tile buffers: while it computes one tile (that buffer also
// serves the tile's exchanges) the next tile arrives in the other by bulk
// copies (cp.async.bulk, this GPU's own memory, no multicast) that complete
// on the buffer's mbarrier.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* mb, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mb)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// the issuing thread's arrival, announcing `bytes` of copies to come
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mb, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mb)), "r"(bytes)
                 : "memory");
}
// `bytes` (a multiple of 16, both addresses 16-byte aligned) from global
// memory into shared memory, counted on mbarrier mb
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes, uint64_t* mb) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src), "r"(bytes), "r"(smem_u32(mb))
        : "memory");
}
// orders this thread's generic shared-memory accesses before later bulk
// copies into the same memory
__device__ __forceinline__ void proxy_fence_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for phase `parity` of mb to complete, for at most ~2 s: past that it
// sets bit 0 of *status (the pass's data is then not valid) and returns
// false, so that a lost copy never hangs the GPU.
__device__ __forceinline__ bool mbar_wait(uint64_t* mb, uint32_t parity, uint32_t* status) {
    const uint32_t a = smem_u32(mb);
    uint64_t t0 = 0;
    for (uint32_t i = 0;; ++i) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255u) == 0) {
            const uint64_t t = global_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > 2000000000ull) {
                atomicOr(status, 1u);
                return false;
            }
        }
    }
}

// Sum of the block's per-thread squared norms into *out (thread 0 writes).
__device__ __forceinline__ void block_norm_partial(double ss, double* red, double* out) {
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if (lane == 0) red[wid] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w2 = 0; w2 < PASS_THREADS / 32; ++w2) t += red[w2];
        *out = t;
    }
}

}  // namespace qoa
