// qoa_f32.cu — the FP32-fused precision form on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory).
//
// Complex64 amplitudes (float2), the same tile passes as the FP64 engine (the
// 5 lowest qubits plus HIGH_SLOTS high qubits per CTA tile, one HBM read and
// write per pass), but inside a pass the gates are fused on the host, in FP64,
// into dense unitaries on at most 5 tile qubits. Each such block is applied to
// the tile as one real GEMM: with the block qubits as the inner index b (32
// values) and the other 6 tile bits as the group index c (64 values), the
// tile's 64 groups are the rows of X (64 x 64: Re x_b then Im x_b) and
//     D = X U^T,   U = [[Ur, -Ui], [Ui, Ur]]     (64 x 64 real)
// gives each group's 32 outputs (Re then Im). D is computed by
// tcgen05.mma.cta_group::1.kind::tf32 (M = 64 groups, N = 64, K = 8 per
// instruction) with both operands in shared memory in the K-major canonical
// layout and the FP32 accumulator in tensor memory, with the 3xTF32 split
// a*b ~= al*bh + ah*bl + ah*bh (h = round-to-TF32, l = the rounded
// remainder), which keeps FP32-level accuracy. One thread issues the 24
// instructions and commits them to an mbarrier; the warps read D back with
// tcgen05.ld. Diagonal gates that involve qubits outside the tile become, per
// CTA, phases on single tile bits (their outer-qubit condition is constant
// over a CTA) and are applied through two small tables. Norm partial sums are
// FP64.
#include <cuda_runtime.h>
#include <stdint.h>

#include "qoa_kernels.cuh"
#include "qoa_pass_dev.cuh"

namespace qoa {

constexpr int F32_THREADS = 128;
constexpr int F32_TILE = 1 << TILE_BITS;          // 2048 amplitudes, 16 KB
constexpr int F32_PER_THREAD = F32_TILE / F32_THREADS;
// dynamic shared memory of a tensor pass CTA: the X operand (hi, lo), the
// block's U operand (hi, lo), the tile, the MMA barrier and the
// tensor-memory address
constexpr unsigned F32_TC_SMEM = 4 * 16384 + F32_TILE * 8 + 16;
constexpr uint32_t F32_TMEM_COLS = 64;            // one 64 x 64 FP32 accumulator

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
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

// Offset (in floats) of element (row, k) of a 64-row K-major operand of 64
// TF32 columns: 8 x 4 core matrices of 128 B, row groups 128 B apart, 4-column
// chunks 1 KB apart (the layout the host writes the block matrices in).
__device__ __forceinline__ uint32_t kmaj(uint32_t row, uint32_t k) {
    return (k >> 2) * 256u + (row >> 3) * 32u + (row & 7u) * 4u + (k & 3u);
}

// Shared-memory matrix descriptor: no swizzle, K-major, leading (K-chunk)
// byte offset 1024, stride (row-group) byte offset 128, sm_100 version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(1024u >> 4) << 16) | ((uint64_t)(128u >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, N = 64, M = 64.
constexpr uint32_t F32_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((64u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(F32_IDESC), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* mb) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mb))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive columns of this warp's 32 tensor-memory lanes
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,"
        "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// The CTA's accumulator: F32_TMEM_COLS tensor-memory columns allocated by
// warp 0 (address written to *slot) and freed by it at the end.
__device__ __forceinline__ void tc_alloc(uint32_t* slot) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(F32_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(F32_TMEM_COLS) : "memory");
}

struct F32Smem {
    float* xh;        // X operand, TF32 hi (64 x 64, K-major)
    float* xl;        // X operand, TF32 lo
    float* uh;        // U operand of the current block, hi
    float* ul;        // and lo (adjacent to uh, as in the host's upload)
    float2* tile;     // 2048 amplitudes
    uint64_t* mbar;   // MMA completion
    uint32_t* tslot;  // tensor-memory address
};

__device__ __forceinline__ F32Smem f32_smem(unsigned char* base) {
    F32Smem m;
    m.xh = reinterpret_cast<float*>(base);
    m.xl = m.xh + 4096;
    m.uh = m.xl + 4096;
    m.ul = m.uh + 4096;
    m.tile = reinterpret_cast<float2*>(m.ul + 4096);
    m.mbar = reinterpret_cast<uint64_t*>(m.tile + F32_TILE);
    m.tslot = reinterpret_cast<uint32_t*>(m.mbar + 1);
    return m;
}

// One fused block: U applied in place to the tile bits in `bmask` (popcount 5;
// fewer qubits are padded with tile bits the block acts on as identity).
// `nblk` counts the CTA's blocks so far (the mbarrier's phase).
__device__ void f32_block(const F32Smem& S, uint32_t taddr, uint32_t bmask, const float* __restrict__ mat,
                          uint32_t nblk, uint32_t* status) {
    const int tid = threadIdx.x;
    const int lane = tid & 31, w = tid >> 5;
    const uint32_t cmask = ((1u << TILE_BITS) - 1) & ~bmask;
    // tile index of each block state
    __shared__ uint32_t ro[32];
    if (tid < 32) ro[tid] = pdep11((uint32_t)tid, bmask);
    // the block's U (hi then lo), already in the operand layout
    {
        const uint4* src = reinterpret_cast<const uint4*>(mat);
        uint4* dst = reinterpret_cast<uint4*>(S.uh);
#pragma unroll 4
        for (int i = tid; i < 2048; i += F32_THREADS) dst[i] = __ldg(src + i);
    }
    __syncthreads();  // ro
    // X rows: thread t gathers half (16 block states) of group t >> 1
    {
        const uint32_t c = (uint32_t)tid >> 1, h = (uint32_t)tid & 1u;
        const uint32_t cb = pdep11(c, cmask);
#pragma unroll 4
        for (uint32_t i = 0; i < 16; ++i) {
            const uint32_t b = 16u * h + i;
            const float2 x = S.tile[ro[b] | cb];
            const float rh = tf32_hi(x.x), ih = tf32_hi(x.y);
            S.xh[kmaj(c, b)] = rh;
            S.xl[kmaj(c, b)] = tf32_hi(x.x - rh);
            S.xh[kmaj(c, 32u + b)] = ih;
            S.xl[kmaj(c, 32u + b)] = tf32_hi(x.y - ih);
        }
    }
    proxy_fence_async();  // the operands written above are read by the tensor cores
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
        const uint32_t xh = smem_u32(S.xh), xl = smem_u32(S.xl), uh = smem_u32(S.uh), ul = smem_u32(S.ul);
        // D = Xl Uh^T + Xh Ul^T + Xh Uh^T, K = 64 in steps of 8 (2 KB of operand per step)
#pragma unroll
        for (uint32_t s = 0; s < 8; ++s) tc_mma(taddr, smem_desc(xl + 2048u * s), smem_desc(uh + 2048u * s), s);
#pragma unroll
        for (uint32_t s = 0; s < 8; ++s) tc_mma(taddr, smem_desc(xh + 2048u * s), smem_desc(ul + 2048u * s), 1u);
#pragma unroll
        for (uint32_t s = 0; s < 8; ++s) tc_mma(taddr, smem_desc(xh + 2048u * s), smem_desc(uh + 2048u * s), 1u);
        tc_commit(S.mbar);
    }
    mbar_wait(S.mbar, nblk & 1u, status);
    tc_fence_after();
    // D row c (M = 64: rows 16w..16w+15 sit in lanes 0..15 of warp w's
    // quarter of tensor memory) -> group c's 32 amplitudes
    {
        const uint32_t base = taddr + ((uint32_t)(32 * w) << 16);
        float re[32], im[32];
        tc_ld32(base, re);
        tc_ld32(base + 32u, im);
        if (lane < 16) {
            const uint32_t c = 16u * (uint32_t)w + (uint32_t)lane;
            const uint32_t cb = pdep11(c, cmask);
#pragma unroll
            for (uint32_t b = 0; b < 32; ++b) S.tile[ro[b] | cb] = make_float2(re[b], im[b]);
        }
    }
    tc_fence_before();
    __syncthreads();
}

// One CTA's tile of one FP32 pass: `blk` numbers the tile, `nrm` is the
// input's squared norm (<= 1e-12: input |0..0>, not read), `partial_out`
// (optional) receives the tile's squared norm after the pass.
__device__ __forceinline__ void f32_pass_tile(float2* __restrict__ amps, const F32PassParams& P,
                                              const float* __restrict__ mats, const F32PhaseOp* __restrict__ pops,
                                              const F32Angle* __restrict__ angles,
                                              const F32Phase* __restrict__ phases, const float2* __restrict__ tables,
                                              const double nrm, const uint64_t blk, double* __restrict__ partial_out,
                                              uint32_t* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char f32_dsm[];
    const F32Smem S = f32_smem(f32_dsm);
    float2* const buf = S.tile;
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
        buf[j] = x;
    }
    // the tensor-memory accumulator (warp 0 allocates) and the MMA barrier
    if (tid < 32) tc_alloc(S.tslot);
    if (tid == 0) {
        mbar_init(S.mbar, 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *S.tslot;

    uint32_t nblk = 0;
    for (uint32_t oi = 0; oi < P.nops; ++oi) {
        const F32Op op = P.ops[oi];
        if (op.kind == 0) {  // dense block
            f32_block(S, taddr, op.bmask, mats + (size_t)op.index * 8192, nblk++, status);
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
            float2* s = buf;
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

    // every tensor-memory read is done (behind the last block's barrier)
    if (tid < 32) tc_dealloc(taddr);
    double ss = 0.0;
    for (int i = 0; i < F32_PER_THREAD; ++i) {
        const uint32_t j = (uint32_t)(tid + F32_THREADS * i);
        const float2 x = buf[j];
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

__global__ void __launch_bounds__(F32_THREADS, 2)
k_f32_pass(float2* __restrict__ amps, const __grid_constant__ F32PassParams P, const float* __restrict__ mats,
           const F32PhaseOp* __restrict__ pops, const F32Angle* __restrict__ angles,
           const F32Phase* __restrict__ phases, const float2* __restrict__ tables, const double* __restrict__ norm2_in,
           double* __restrict__ partials, uint32_t* __restrict__ status) {
    f32_pass_tile(amps, P, mats, pops, angles, phases, tables, *norm2_in, blockIdx.x, partials + blockIdx.x, status);
}

// Arena form: one launch runs one pass of each of many circuits (see
// k_pass_arena); every circuit's block matrices, phase groups, angle lists
// and tables lie in one shared upload, so the base pointers are common.
__global__ void __launch_bounds__(F32_THREADS, 2)
k_f32_pass_arena(const ArenaJob* __restrict__ jobs, uint32_t njobs, const uint32_t* __restrict__ tile_start,
                 const float* __restrict__ mats, const F32PhaseOp* __restrict__ pops,
                 const F32Angle* __restrict__ angles, const F32Phase* __restrict__ phases,
                 const float2* __restrict__ tables, uint32_t* __restrict__ status) {
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (tile_start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const ArenaJob J = jobs[lo];
    f32_pass_tile(reinterpret_cast<float2*>(J.amps), *reinterpret_cast<const F32PassParams*>(J.params), mats, pops,
                  angles, phases, tables, J.fresh ? 0.0 : 1.0, b - tile_start[lo], nullptr, status);
}

// The tensor pass kernels need more than the default 48 KB of dynamic shared
// memory: allowed once per device.
static cudaError_t f32_tc_setup() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    static uint64_t done = 0;  // devices set up (the set-up is idempotent, so racing threads are harmless)
    if ((__atomic_load_n(&done, __ATOMIC_ACQUIRE) >> dev) & 1) return cudaSuccess;
    e = cudaFuncSetAttribute(k_f32_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F32_TC_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_f32_pass_arena, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F32_TC_SMEM);
    if (e == cudaSuccess) __atomic_fetch_or(&done, 1ull << dev, __ATOMIC_RELEASE);
    return e;
}

cudaError_t launch_f32_pass_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                                  const float* mats, const F32PhaseOp* pops, const F32Angle* angles,
                                  const F32Phase* phases, const float2* tables, uint32_t* status, cudaStream_t st) {
    if (!njobs || !tiles) return cudaSuccess;
    const cudaError_t e = f32_tc_setup();
    if (e != cudaSuccess) return e;
    k_f32_pass_arena<<<tiles, F32_THREADS, F32_TC_SMEM, st>>>(jobs, njobs, tile_start, mats, pops, angles, phases,
                                                              tables, status);
    return cudaGetLastError();
}

cudaError_t launch_f32_pass(float2* amps, const F32PassParams& P, const float* mats, const F32PhaseOp* pops,
                            const F32Angle* angles, const F32Phase* phases, const float2* tables,
                            const double* norm2_in, double* partials, uint32_t* status, cudaStream_t st) {
    const cudaError_t e = f32_tc_setup();
    if (e != cudaSuccess) return e;
    const unsigned blocks = 1u << (P.n - TILE_BITS);
    k_f32_pass<<<blocks, F32_THREADS, F32_TC_SMEM, st>>>(amps, P, mats, pops, angles, phases, tables, norm2_in,
                                                        partials, status);
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
