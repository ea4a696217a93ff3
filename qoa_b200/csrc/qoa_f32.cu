// qoa_f32.cu — the FP32-fused precision form.
//
// Complex64 amplitudes (float2), the same tile passes as the FP64 engine (the
// 5 lowest qubits plus HIGH_SLOTS high qubits per CTA tile, one HBM read and
// write per pass), but inside a pass the gates are fused on the host, in FP64,
// into dense unitaries on at most 5 tile qubits. Each such block is applied to
// the tile as a real GEMM on the tensor cores: with the block qubits as the
// row index r (32 values) and the other 6 tile bits as the column index c
// (64 values), Y = U X in complex form is
//     [Yr; Yi] = [[Ur, -Ui], [Ui, Ur]] [Xr; Xi]      (64 x 64 by 64 x 64 real)
// computed with mma.sync m16n8k8 TF32 and the 3xTF32 split a*b ~= ah*bh +
// ah*bl + al*bh (h = round-to-TF32, l = the remainder), accumulated in FP32,
// which keeps FP32-level accuracy. Diagonal gates that involve qubits outside
// the tile become, per CTA, phases on single tile bits (their outer-qubit
// condition is constant over a CTA) and are applied through two small tables.
// Norm partial sums are FP64.
#include <cuda_runtime.h>
#include <stdint.h>

#include "qoa_kernels.cuh"

namespace qoa {

constexpr int F32_THREADS = 128;
constexpr int F32_TILE = 1 << TILE_BITS;          // 2048 amplitudes, 16 KB per buffer
constexpr int F32_PER_THREAD = F32_TILE / F32_THREADS;

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pdep11(uint32_t x, uint32_t mask) {
    uint32_t r = 0;
    for (uint32_t b = 0; b < (uint32_t)TILE_BITS; ++b)
        if ((mask >> b) & 1u) {
            r |= (x & 1u) << b;
            x >>= 1;
        }
    return r;
}

// One fused block: U applied to the tile bits in `bmask` (popcount 5; fewer
// qubits are padded with tile bits the block acts on as identity).
__device__ void f32_block(const float2* __restrict__ src, float2* __restrict__ dst, uint32_t bmask,
                          const float* __restrict__ ahi, const float* __restrict__ alo, int* ro, int* co) {
    const int tid = threadIdx.x;
    const int lane = tid & 31, w = tid >> 5;
    const int gq = lane >> 2, t4 = lane & 3;
    const uint32_t cmask = ((1u << TILE_BITS) - 1) & ~bmask;
    if (tid < 32) ro[tid] = (int)pdep11((uint32_t)tid, bmask);
    if (tid < 64) co[tid] = (int)pdep11((uint32_t)tid, cmask);
    // A fragments for this warp's 16 real output rows, all 8 k-steps
    uint32_t ah[8][4], al[8][4];
    const int r0 = 16 * w + gq, r1 = r0 + 8;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        const int c0 = 8 * kk + t4, c1 = c0 + 4;
        ah[kk][0] = __float_as_uint(ahi[r0 * 64 + c0]);
        ah[kk][1] = __float_as_uint(ahi[r1 * 64 + c0]);
        ah[kk][2] = __float_as_uint(ahi[r0 * 64 + c1]);
        ah[kk][3] = __float_as_uint(ahi[r1 * 64 + c1]);
        al[kk][0] = __float_as_uint(alo[r0 * 64 + c0]);
        al[kk][1] = __float_as_uint(alo[r1 * 64 + c0]);
        al[kk][2] = __float_as_uint(alo[r0 * 64 + c1]);
        al[kk][3] = __float_as_uint(alo[r1 * 64 + c1]);
    }
    __syncthreads();
#pragma unroll 1
    for (int nt = 0; nt < 8; ++nt) {
        const int col = 8 * nt + gq;
        const int cb = co[col];
        // B rows 0..31 are Re X, rows 32..63 Im X of the same elements
        float2 x0[4], x1[4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            x0[kk] = src[ro[8 * kk + t4] | cb];
            x1[kk] = src[ro[8 * kk + t4 + 4] | cb];
        }
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const float f0 = kk < 4 ? x0[kk].x : x0[kk - 4].y;
            const float f1 = kk < 4 ? x1[kk].x : x1[kk - 4].y;
            const uint32_t bh0 = to_tf32(f0), bh1 = to_tf32(f1);
            const uint32_t bl0 = to_tf32(f0 - __uint_as_float(bh0)), bl1 = to_tf32(f1 - __uint_as_float(bh1));
            mma_tf32(acc, al[kk], bh0, bh1);
            mma_tf32(acc, ah[kk], bl0, bl1);
            mma_tf32(acc, ah[kk], bh0, bh1);
        }
        // C fragment: rows r0 (acc 0,1) and r1 (acc 2,3), cols 8nt + 2 t4 (+1)
        const int ca = co[8 * nt + 2 * t4], cbb = co[8 * nt + 2 * t4 + 1];
        if (w < 2) {  // rows 0..31: real parts
            dst[ro[r0] | ca].x = acc[0];
            dst[ro[r0] | cbb].x = acc[1];
            dst[ro[r1] | ca].x = acc[2];
            dst[ro[r1] | cbb].x = acc[3];
        } else {      // rows 32..63: imaginary parts
            dst[ro[r0 - 32] | ca].y = acc[0];
            dst[ro[r0 - 32] | cbb].y = acc[1];
            dst[ro[r1 - 32] | ca].y = acc[2];
            dst[ro[r1 - 32] | cbb].y = acc[3];
        }
    }
    __syncthreads();
}

// One CTA's tile of one FP32 pass: `blk` numbers the tile, `nrm` is the
// input's squared norm (<= 1e-12: input |0..0>, not read), `partial_out`
// (optional) receives the tile's squared norm after the pass.
__device__ __forceinline__ void f32_pass_tile(float2* __restrict__ amps, const F32PassParams& P,
                                              const float* __restrict__ mats, const F32PhaseOp* __restrict__ pops,
                                              const F32Angle* __restrict__ angles,
                                              const F32Phase* __restrict__ phases, const float2* __restrict__ tables,
                                              const double nrm, const uint64_t blk, double* __restrict__ partial_out) {
    __shared__ float2 buf[2][F32_TILE];
    __shared__ int ro[32], co[64];
    __shared__ float2 tlo[32], thi[64];
    __shared__ double alpha[TILE_BITS + 1];
    __shared__ double red[F32_THREADS / 32];
    const int tid = threadIdx.x;

    uint64_t g0 = 0;
    {
        const uint64_t b = blk;
        const int nout = (int)P.n - TILE_BITS;
        for (int k = 0; k < nout; ++k) g0 |= ((b >> k) & 1ull) << P.outer_qubits[k];
    }
    auto gidx = [&](uint32_t j) -> uint64_t {
        uint64_t g = g0 + (j & 31u);
#pragma unroll
        for (int s = 0; s < HIGH_SLOTS; ++s)
            if ((j >> (LANE_BITS + s)) & 1u) g += 1ull << P.slot_qubit[s];
        return g;
    };
    const bool valid = nrm > 1e-12;
    const float scale = valid ? (float)(1.0 / sqrt(nrm)) : 0.f;
#pragma unroll 4
    for (int i = 0; i < F32_PER_THREAD; ++i) {
        const uint32_t j = (uint32_t)(tid + F32_THREADS * i);
        const uint64_t g = gidx(j);
        float2 x = valid ? __ldcs(amps + g) : make_float2(g == 0 ? 1.f : 0.f, 0.f);
        if (valid) x = make_float2(x.x * scale, x.y * scale);
        buf[0][j] = x;
    }
    __syncthreads();

    int cur = 0;
    for (uint32_t oi = 0; oi < P.nops; ++oi) {
        const F32Op op = P.ops[oi];
        if (op.kind == 0) {  // dense block
            const float* a = mats + (size_t)op.index * 8192;
            f32_block(buf[cur], buf[cur ^ 1], op.bmask, a, a + 4096, ro, co);
            cur ^= 1;
        } else {
            const F32PhaseOp po = pops[op.index];
            // per-CTA angle of each tile bit (and of the scalar part)
            if (tid <= TILE_BITS) {
                double th = 0.0;
                for (uint32_t e = po.bit_start[tid]; e < po.bit_start[tid + 1]; ++e) {
                    const F32Angle an = angles[e];
                    if ((g0 & an.outer) == an.outer) th += an.theta;
                }
                alpha[tid] = th;
            }
            __syncthreads();
            if (tid < 32) {
                double th = alpha[TILE_BITS];
                for (int t = 0; t < LANE_BITS; ++t)
                    if ((tid >> t) & 1) th += alpha[t];
                double sn, cs;
                sincos(th, &sn, &cs);
                tlo[tid] = make_float2((float)cs, (float)sn);
            }
            if (tid < 64) {
                double th = 0.0;
                for (int t = 0; t < HIGH_SLOTS; ++t)
                    if ((tid >> t) & 1) th += alpha[LANE_BITS + t];
                double sn, cs;
                sincos(th, &sn, &cs);
                thi[tid] = make_float2((float)cs, (float)sn);
            }
            __syncthreads();
            const float2* tab = po.table >= 0 ? tables + (size_t)po.table * F32_TILE : nullptr;
            float2* s = buf[cur];
            for (int i = 0; i < F32_PER_THREAD; ++i) {
                const uint32_t j = (uint32_t)(tid + F32_THREADS * i);
                const float2 l = tlo[j & 31u], h = thi[j >> LANE_BITS];
                float2 f = make_float2(l.x * h.x - l.y * h.y, l.x * h.y + l.y * h.x);
                if (tab) {
                    const float2 u = __ldg(tab + j);
                    f = make_float2(f.x * u.x - f.y * u.y, f.x * u.y + f.y * u.x);
                }
                for (uint32_t e = 0; e < po.multi_count; ++e) {
                    const F32Phase ph = phases[po.multi_start + e];
                    if ((g0 & ph.outer) == ph.outer && (j & ph.tile) == ph.tile) {
                        const float pr = (float)ph.re, pi = (float)ph.im;
                        f = make_float2(f.x * pr - f.y * pi, f.x * pi + f.y * pr);
                    }
                }
                const float2 x = s[j];
                s[j] = make_float2(x.x * f.x - x.y * f.y, x.x * f.y + x.y * f.x);
            }
            __syncthreads();
        }
    }

    double ss = 0.0;
    for (int i = 0; i < F32_PER_THREAD; ++i) {
        const uint32_t j = (uint32_t)(tid + F32_THREADS * i);
        const float2 x = buf[cur][j];
        __stcs(amps + gidx(j), x);
        ss += (double)x.x * x.x + (double)x.y * x.y;
    }
    if (!partial_out) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((tid & 31) == 0) red[tid >> 5] = ss;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w2 = 0; w2 < F32_THREADS / 32; ++w2) t += red[w2];
        *partial_out = t;
    }
}

__global__ void __launch_bounds__(F32_THREADS, 4)
k_f32_pass(float2* __restrict__ amps, const __grid_constant__ F32PassParams P, const float* __restrict__ mats,
           const F32PhaseOp* __restrict__ pops, const F32Angle* __restrict__ angles,
           const F32Phase* __restrict__ phases, const float2* __restrict__ tables, const double* __restrict__ norm2_in,
           double* __restrict__ partials) {
    f32_pass_tile(amps, P, mats, pops, angles, phases, tables, *norm2_in, blockIdx.x, partials + blockIdx.x);
}

// Arena form: one launch runs one pass of each of many circuits (see
// k_pass_arena); every circuit's block matrices, phase groups, angle lists
// and tables lie in one shared upload, so the base pointers are common.
__global__ void __launch_bounds__(F32_THREADS, 4)
k_f32_pass_arena(const ArenaJob* __restrict__ jobs, uint32_t njobs, const uint32_t* __restrict__ tile_start,
                 const float* __restrict__ mats, const F32PhaseOp* __restrict__ pops,
                 const F32Angle* __restrict__ angles, const F32Phase* __restrict__ phases,
                 const float2* __restrict__ tables) {
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (tile_start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const ArenaJob J = jobs[lo];
    f32_pass_tile(reinterpret_cast<float2*>(J.amps), *reinterpret_cast<const F32PassParams*>(J.params), mats, pops,
                  angles, phases, tables, J.fresh ? 0.0 : 1.0, b - tile_start[lo], nullptr);
}

cudaError_t launch_f32_pass_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                                  const float* mats, const F32PhaseOp* pops, const F32Angle* angles,
                                  const F32Phase* phases, const float2* tables, cudaStream_t st) {
    if (!njobs || !tiles) return cudaSuccess;
    k_f32_pass_arena<<<tiles, F32_THREADS, 0, st>>>(jobs, njobs, tile_start, mats, pops, angles, phases, tables);
    return cudaGetLastError();
}

cudaError_t launch_f32_pass(float2* amps, const F32PassParams& P, const float* mats, const F32PhaseOp* pops,
                            const F32Angle* angles, const F32Phase* phases, const float2* tables,
                            const double* norm2_in, double* partials, cudaStream_t st) {
    const unsigned blocks = 1u << (P.n - TILE_BITS);
    k_f32_pass<<<blocks, F32_THREADS, 0, st>>>(amps, P, mats, pops, angles, phases, tables, norm2_in, partials);
    return cudaGetLastError();
}

// ---- FP32 state helpers (reductions stay FP64) -------------------------------
__global__ void k_f32_reset(float2* a, uint64_t len) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = make_float2(i == 0 ? 1.f : 0.f, 0.f);
}

__global__ void k_f32_norm_partials(const float2* __restrict__ a, uint64_t len, double* __restrict__ partials) {
    __shared__ double sh[32];
    double v = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const float2 x = a[i];
        v += (double)x.x * x.x + (double)x.y * x.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
        partials[blockIdx.x] = t;
    }
}

__global__ void k_f32_materialize(float2* __restrict__ a, uint64_t len, const double* __restrict__ norm2_in) {
    const double nrm = *norm2_in;
    const bool valid = nrm > 1e-12;
    const float s = valid ? (float)(1.0 / sqrt(nrm)) : 0.f;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        if (valid) {
            const float2 x = a[i];
            a[i] = make_float2(x.x * s, x.y * s);
        } else {
            a[i] = make_float2(i == 0 ? 1.f : 0.f, 0.f);
        }
    }
}

__global__ void k_f32_probs(const float2* __restrict__ a, uint64_t off, uint64_t cnt, const double* __restrict__ norm2_in,
                            double* __restrict__ out) {
    const double nrm = *norm2_in;
    const bool valid = nrm > 1e-12;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t g = off + i;
        if (valid) {
            const float2 x = a[g];
            out[i] = ((double)x.x * x.x + (double)x.y * x.y) / nrm;
        } else {
            out[i] = g == 0 ? 1.0 : 0.0;
        }
    }
}

__global__ void k_f32_expz_partials(const float2* __restrict__ a, uint64_t len, const ExpzMasks mk, uint32_t k,
                                    double* __restrict__ partials) {
    __shared__ double sh[8][32];
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const float2 x = a[i];
        const double p = (double)x.x * x.x + (double)x.y * x.y;
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] += (__popcll(i & mk.m[j]) & 1) ? -p : p;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        double x = v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[j][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += sh[threadIdx.x][q];
        partials[(uint64_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

int reduce_blocks(uint64_t len);
cudaError_t launch_reduce_div(const double* partials, uint32_t count, uint32_t sets, double* out, const double* divide_by,
                              cudaStream_t st);

cudaError_t launch_f32_expz(const float2* a, uint64_t len, const uint64_t* masks, uint32_t k, double* partials,
                            double* out, const double* norm2, cudaStream_t st) {
    const int nb = reduce_blocks(len);
    ExpzMasks mk{};
    for (uint32_t j = 0; j < k && j < 8; ++j) mk.m[j] = masks[j];
    k_f32_expz_partials<<<nb, 256, 0, st>>>(a, len, mk, k, partials);
    return launch_reduce_div(partials, (uint32_t)nb, k, out, norm2, st);
}

cudaError_t launch_reduce_partials(const double* partials, uint32_t count, double* out, uint32_t* status,
                                   cudaStream_t st);

static int f32_grid(uint64_t len) {
    uint64_t b = (len + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b ? b : 1);
}

cudaError_t launch_f32_reset(float2* a, uint64_t len, cudaStream_t st) {
    k_f32_reset<<<f32_grid(len), 256, 0, st>>>(a, len);
    return cudaGetLastError();
}
cudaError_t launch_f32_norm(const float2* a, uint64_t len, double* partials, double* out, uint32_t* status,
                            cudaStream_t st) {
    const int nb = reduce_blocks(len);
    k_f32_norm_partials<<<nb, 256, 0, st>>>(a, len, partials);
    return launch_reduce_partials(partials, (uint32_t)nb, out, status, st);
}
cudaError_t launch_f32_materialize(float2* a, uint64_t len, double* norm2, double* partials, uint32_t* status,
                                   cudaStream_t st) {
    k_f32_materialize<<<f32_grid(len), 256, 0, st>>>(a, len, norm2);
    return launch_f32_norm(a, len, partials, norm2, status, st);
}
cudaError_t launch_f32_probs(const float2* a, uint64_t off, uint64_t cnt, const double* norm2, double* out,
                             cudaStream_t st) {
    k_f32_probs<<<f32_grid(cnt), 256, 0, st>>>(a, off, cnt, norm2, out);
    return cudaGetLastError();
}

}  // namespace qoa
