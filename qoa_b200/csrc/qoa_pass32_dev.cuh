// qoa_pass32_dev.cuh — device building blocks of the complex64 tile pass
// with packed FP32 arithmetic (sm_100 add/sub/mul/fma .f32x2 on pairs of
// floats): packing helpers, the 2x2 forms on register bits 0..2 (both halves
// of a packed pair at once), the scalar path for register bit 3 (the pairing
// bit), conditioned X/Y and diagonal factors. Compiled into the interpreter
// kernels (qoa_pass32.cu, by nvcc) and into the per-pass kernels generated
// at run time (qoa_jit.cpp, by NVRTC).
#pragma once
#include "qoa_kernels.cuh"

namespace qoa {
namespace p32 {

typedef unsigned long long u64p;  // a packed pair of floats

__device__ __forceinline__ u64p pk(float lo, float hi) {
    return (u64p)__float_as_uint(lo) | ((u64p)__float_as_uint(hi) << 32);
}
__device__ __forceinline__ float lo(u64p a) { return __uint_as_float((unsigned)a); }
__device__ __forceinline__ float hi(u64p a) { return __uint_as_float((unsigned)(a >> 32)); }
__device__ __forceinline__ u64p bc(float x) { return pk(x, x); }

__device__ __forceinline__ u64p add2(u64p a, u64p b) {
    u64p d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64p sub2(u64p a, u64p b) {
    u64p d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64p mul2(u64p a, u64p b) {
    u64p d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64p fma2(u64p a, u64p b, u64p c) {
    u64p d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// (re, im) *= (cr, ci), componentwise complex product of packed pairs
__device__ __forceinline__ void cmul2(u64p& re, u64p& im, u64p cr, u64p ci) {
    const u64p r = fma2(cr, re, mul2(sub2(0ull, ci), im));
    im = fma2(cr, im, mul2(ci, re));
    re = r;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// 2x2 on register bit K (0..2): pairs (j, j | 1<<K), both halves at once
template <int SUB, int K>
__device__ __forceinline__ void g1p(u64p (&re)[8], u64p (&im)[8], const float2* __restrict__ m) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (j & (1 << K)) continue;
        const int k = j | (1 << K);
        u64p& r0 = re[j]; u64p& i0 = im[j]; u64p& r1 = re[k]; u64p& i1 = im[k];
        if (SUB == G1_HF) {
            const u64p a = r0, b = i0;
            r0 = add2(a, r1); i0 = add2(b, i1);
            r1 = sub2(a, r1); i1 = sub2(b, i1);
        } else if (SUB == G1_X) {
            u64p t = r0; r0 = r1; r1 = t;
            t = i0; i0 = i1; i1 = t;
        } else if (SUB == G1_Y) {  // a0' = -i a1, a1' = i a0
            const u64p a = r0, b = i0;
            r0 = i1; i0 = sub2(0ull, r1);
            r1 = sub2(0ull, b); i1 = a;
        } else if (SUB == G1_RXA) {  // a0' = a0 - i t a1, a1' = a1 - i t a0
            const u64p t = bc(m[0].x), a = r0, b = i0;
            r0 = fma2(t, i1, a); i0 = fma2(sub2(0ull, t), r1, b);
            r1 = fma2(t, b, r1); i1 = fma2(sub2(0ull, t), a, i1);
        } else if (SUB == G1_RXB) {  // a0' = r a0 - i a1, a1' = r a1 - i a0
            const u64p r = bc(m[0].x), a = r0, b = i0;
            r0 = fma2(r, a, i1); i0 = sub2(mul2(r, b), r1);
            r1 = fma2(r, r1, b); i1 = sub2(mul2(r, i1), a);
        } else if (SUB == G1_RYA) {  // a0' = a0 - t a1, a1' = a1 + t a0
            const u64p t = bc(m[0].x), nt = bc(-m[0].x), a = r0, b = i0;
            r0 = fma2(nt, r1, a); i0 = fma2(nt, i1, b);
            r1 = fma2(t, a, r1); i1 = fma2(t, b, i1);
        } else if (SUB == G1_RYB) {  // a0' = r a0 - a1, a1' = r a1 + a0
            const u64p r = bc(m[0].x), a = r0, b = i0;
            r0 = sub2(mul2(r, a), r1); i0 = sub2(mul2(r, b), i1);
            r1 = fma2(r, r1, a); i1 = fma2(r, i1, b);
        } else {  // general: a0' = m0 a0 + m1 a1, a1' = m2 a0 + m3 a1
            const float2 c0 = m[0], c1 = m[1], c2 = m[2], c3 = m[3];
            const u64p a = r0, b = i0, c = r1, d = i1;
            r0 = fma2(bc(c0.x), a, fma2(bc(-c0.y), b, fma2(bc(c1.x), c, mul2(bc(-c1.y), d))));
            i0 = fma2(bc(c0.x), b, fma2(bc(c0.y), a, fma2(bc(c1.x), d, mul2(bc(c1.y), c))));
            r1 = fma2(bc(c2.x), a, fma2(bc(-c2.y), b, fma2(bc(c3.x), c, mul2(bc(-c3.y), d))));
            i1 = fma2(bc(c2.x), b, fma2(bc(c2.y), a, fma2(bc(c3.x), d, mul2(bc(c3.y), c))));
        }
    }
}

// scalar 2x2 on a pair of complex floats (register bit 3: the two halves)
template <int SUB>
__device__ __forceinline__ void g1s(float2& a0, float2& a1, const float2* __restrict__ m) {
    if (SUB == G1_HF) {
        const float2 t = a0;
        a0 = make_float2(t.x + a1.x, t.y + a1.y);
        a1 = make_float2(t.x - a1.x, t.y - a1.y);
    } else if (SUB == G1_X) {
        const float2 t = a0; a0 = a1; a1 = t;
    } else if (SUB == G1_Y) {
        const float2 t = a0;
        a0 = make_float2(a1.y, -a1.x);
        a1 = make_float2(-t.y, t.x);
    } else if (SUB == G1_RXA) {
        const float t = m[0].x; const float2 u = a0;
        a0 = make_float2(fmaf(t, a1.y, u.x), fmaf(-t, a1.x, u.y));
        a1 = make_float2(fmaf(t, u.y, a1.x), fmaf(-t, u.x, a1.y));
    } else if (SUB == G1_RXB) {
        const float r = m[0].x; const float2 u = a0;
        a0 = make_float2(fmaf(r, u.x, a1.y), fmaf(r, u.y, -a1.x));
        a1 = make_float2(fmaf(r, a1.x, u.y), fmaf(r, a1.y, -u.x));
    } else if (SUB == G1_RYA) {
        const float t = m[0].x; const float2 u = a0;
        a0 = make_float2(fmaf(-t, a1.x, u.x), fmaf(-t, a1.y, u.y));
        a1 = make_float2(fmaf(t, u.x, a1.x), fmaf(t, u.y, a1.y));
    } else if (SUB == G1_RYB) {
        const float r = m[0].x; const float2 u = a0;
        a0 = make_float2(fmaf(r, u.x, -a1.x), fmaf(r, u.y, -a1.y));
        a1 = make_float2(fmaf(r, a1.x, u.x), fmaf(r, a1.y, u.y));
    } else {
        const float2 t = a0;
        float2 r0 = cmulf(m[0], t), r1 = cmulf(m[2], t);
        r0.x = fmaf(m[1].x, a1.x, r0.x); r0.x = fmaf(-m[1].y, a1.y, r0.x);
        r0.y = fmaf(m[1].x, a1.y, r0.y); r0.y = fmaf(m[1].y, a1.x, r0.y);
        r1.x = fmaf(m[3].x, a1.x, r1.x); r1.x = fmaf(-m[3].y, a1.y, r1.x);
        r1.y = fmaf(m[3].x, a1.y, r1.y); r1.y = fmaf(m[3].y, a1.x, r1.y);
        a0 = r0; a1 = r1;
    }
}

template <int SUB>
__device__ __forceinline__ void g1_bit3(u64p (&re)[8], u64p (&im)[8], const float2* __restrict__ m) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float2 a0 = make_float2(lo(re[j]), lo(im[j])), a1 = make_float2(hi(re[j]), hi(im[j]));
        g1s<SUB>(a0, a1, m);
        re[j] = pk(a0.x, a1.x);
        im[j] = pk(a0.y, a1.y);
    }
}

// X / Y on register bit K under register mask creg (any bits) and thread predicate
template <int SUB, int K>
__device__ __forceinline__ void g1c(u64p (&re)[8], u64p (&im)[8], bool tp, uint32_t creg) {
    if (!tp) return;
#pragma unroll
    for (int v = 0; v < 16; ++v) {
        if ((v & (1 << K)) || (v & creg) != creg) continue;
        const int w = v | (1 << K);
        const int jv = v & 7, jw = w & 7;
        const bool hv = v >= 8, hw = w >= 8;
        float2 a0 = make_float2(hv ? hi(re[jv]) : lo(re[jv]), hv ? hi(im[jv]) : lo(im[jv]));
        float2 a1 = make_float2(hw ? hi(re[jw]) : lo(re[jw]), hw ? hi(im[jw]) : lo(im[jw]));
        g1s<SUB>(a0, a1, nullptr);
        re[jv] = hv ? pk(lo(re[jv]), a0.x) : pk(a0.x, hi(re[jv]));
        im[jv] = hv ? pk(lo(im[jv]), a0.y) : pk(a0.y, hi(im[jv]));
        re[jw] = hw ? pk(lo(re[jw]), a1.x) : pk(a1.x, hi(re[jw]));
        im[jw] = hw ? pk(lo(im[jw]), a1.y) : pk(a1.y, hi(im[jw]));
    }
}

// multiply the registers v with (v & creg) == creg by d
__device__ __forceinline__ void diag_p(u64p (&re)[8], u64p (&im)[8], bool tp, uint32_t creg, float2 d) {
    if (!tp) return;
    const uint32_t cl = creg & 7u;
    const bool only_hi = (creg & 8u) != 0;
    const u64p cr = only_hi ? pk(1.f, d.x) : bc(d.x);
    const u64p ci = only_hi ? pk(0.f, d.y) : bc(d.y);
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (((uint32_t)j & cl) == cl) cmul2(re[j], im[j], cr, ci);
}

// Squared norm of a thread's 16 amplitudes: packed FP32 products summed per
// half (8 amplitudes each), the two halves added in FP64.
__device__ __forceinline__ double norm2_p(const u64p (&re)[8], const u64p (&im)[8]) {
    u64p s = 0ull;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        s = fma2(re[j], re[j], s);
        s = fma2(im[j], im[j], s);
    }
    return (double)lo(s) + (double)hi(s);
}

}  // namespace p32
}  // namespace qoa
