// qoa_pass32.cu — the complex64 tile pass with packed FP32 arithmetic.
//
// Same tile, op stream and pass parameters as k_pass (qoa_kernels.cu), but
// each thread keeps its 16 amplitudes split by component and paired along
// register bit 3: re[j] = (Re a[j], Re a[j+8]) and im[j] = (Im a[j], Im
// a[j+8]) for j = 0..7, each pair one 64-bit register operand of the sm_100
// packed FP32 instructions (add/sub/mul/fma .f32x2). A gate on register bit
// 0..2 then updates two amplitude pairs per instruction with no shuffling of
// real and imaginary parts; a gate on register bit 3 (the pairing bit, given
// by the host to the tile bit used last) takes the scalar FP32 path. All
// rounding is single-precision round-to-nearest, as in the complex64 form of
// k_pass.
#include <cuda_runtime.h>
#include <stdint.h>

#include "qoa_kernels.cuh"
#include "qoa_pass32_dev.cuh"

namespace qoa {

namespace {

using namespace p32;

__device__ __forceinline__ uint32_t spos(uint32_t j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7u); }

__device__ __forceinline__ uint64_t tstride(const PassParams& P, uint32_t t) {
    return 1ull << (t < LANE_BITS ? t : P.slot_qubit[t - LANE_BITS]);
}

__device__ __forceinline__ void pass_tile_p32(float2* __restrict__ amps, const PassParams& P, const double nrm,
                                              const uint64_t blk, double* __restrict__ partial_out) {
    extern __shared__ __align__(16) unsigned char p32_smem[];
    float2* tile = reinterpret_cast<float2*>(p32_smem);
    __shared__ double red[PASS_THREADS / 32];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;

    uint64_t g0 = 0;
    {
        const int nout = (int)P.n - TILE_BITS;
        for (int k = 0; k < nout; ++k) g0 |= ((blk >> k) & 1ull) << P.outer_qubits[k];
    }
    const uint32_t T = (uint32_t)lane | ((uint32_t)wid << LANE_BITS) | ((uint32_t)blk << (LANE_BITS + WARP_BITS));
    const uint32_t nops = P.nops;
    uint4* sops = reinterpret_cast<uint4*>(tile + (1 << TILE_BITS));
    float2* scoef = reinterpret_cast<float2*>(sops + nops);
    {
        const uint4* gops = reinterpret_cast<const uint4*>(P.ops);
        for (uint32_t i = threadIdx.x; i < nops; i += PASS_THREADS) sops[i] = gops[i];
        for (uint32_t i = threadIdx.x; i < P.ncoef; i += PASS_THREADS)
            scoef[i] = make_float2((float)P.coef[i].x, (float)P.coef[i].y);
    }
    __shared__ float2 sang[MAX_ANG_OPS];
    for (uint32_t ai = threadIdx.x; ai < P.nang; ai += PASS_THREADS) {
        double th = 0.0;
        for (uint32_t e = P.ang_start[ai]; e < P.ang_start[ai + 1]; ++e) {
            const uint64_t om = P.angles[e].omask;
            if ((blk & om) == om) th += P.angles[e].theta;
        }
        double sn, cs;
        sincos(th, &sn, &cs);
        sang[ai] = make_float2((float)cs, (float)sn);
    }
    const bool valid = nrm > 1e-12;
    float2 pend = valid ? make_float2((float)(P.phase.x / sqrt(nrm)), (float)(P.phase.y / sqrt(nrm)))
                        : make_float2((float)P.phase.x, (float)P.phase.y);

    u64p re[8], im[8];
    {
        uint64_t tb = g0 + (uint64_t)lane;
#pragma unroll
        for (int k = 0; k < WARP_BITS; ++k)
            if ((wid >> k) & 1) tb += tstride(P, P.map0.warp[k]);
        uint64_t rst[REG_BITS];
#pragma unroll
        for (int k = 0; k < REG_BITS; ++k) rst[k] = tstride(P, P.map0.reg[k]);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            uint64_t g = tb;
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) g += rst[k];
            const uint64_t g8 = g + rst[3];
            float2 a = valid ? __ldcs(amps + g) : make_float2(g == 0 ? 1.f : 0.f, 0.f);
            float2 b = valid ? __ldcs(amps + g8) : make_float2(0.f, 0.f);
            re[j] = pk(a.x, b.x);
            im[j] = pk(a.y, b.y);
        }
    }
    __syncthreads();

    const uint32_t* ow = reinterpret_cast<const uint32_t*>(sops);
    int cur = -1;
    uint32_t w = nops ? ow[0] : 0;
    for (uint32_t oi = 0; oi < nops; ++oi) {
        const uint32_t hot = w;
        if (oi + 1 < nops) w = ow[4 * (oi + 1)];
        const uint32_t code = hot & 0xffu;
        const float2* m = scoef + (hot >> 16);
        auto conds = [&](bool& tp) -> uint32_t {
            const uint32_t cw = ow[4 * oi + 1];
            const uint32_t tm = ow[4 * oi + 2];
            tp = (T & tm) == tm;
            return cw & 0xffu;
        };
        switch (code) {
#define QOA_P3(BASE, SUB)                                           \
    case BASE + 0: g1p<SUB, 0>(re, im, m); break;                   \
    case BASE + 1: g1p<SUB, 1>(re, im, m); break;                   \
    case BASE + 2: g1p<SUB, 2>(re, im, m); break;                   \
    case BASE + 3: g1_bit3<SUB>(re, im, m); break;
            QOA_P3(PC_HF, G1_HF)
            QOA_P3(PC_RX, G1_RXA)
            QOA_P3(PC_RY, G1_RYA)
            QOA_P3(PC_RXB, G1_RXB)
            QOA_P3(PC_RYB, G1_RYB)
            QOA_P3(PC_GEN, G1_GEN)
#undef QOA_P3
#define QOA_C4(BASE, SUB)                                                                      \
    case BASE + 0: { bool tp; const uint32_t cr = conds(tp); g1c<SUB, 0>(re, im, tp, cr); } break; \
    case BASE + 1: { bool tp; const uint32_t cr = conds(tp); g1c<SUB, 1>(re, im, tp, cr); } break; \
    case BASE + 2: { bool tp; const uint32_t cr = conds(tp); g1c<SUB, 2>(re, im, tp, cr); } break; \
    case BASE + 3: { bool tp; const uint32_t cr = conds(tp); g1c<SUB, 3>(re, im, tp, cr); } break;
            QOA_C4(PC_XC, G1_X)
            QOA_C4(PC_YC, G1_Y)
#undef QOA_C4
            case PC_DIAG_T: {
                bool tp;
                conds(tp);
                if (tp) pend = cmulf(pend, m[0]);
                break;
            }
            case PC_DIAG_M: {
                bool tp;
                const uint32_t cr = conds(tp);
                diag_p(re, im, tp, cr, m[0]);
                break;
            }
            case PC_DIAG_TA: {
                bool tp;
                conds(tp);
                if (tp) pend = cmulf(pend, sang[hot >> 16]);
                break;
            }
            case PC_DIAG_MA:
                diag_p(re, im, true, ow[4 * oi + 1] & 0xffu, sang[hot >> 16]);
                break;
            case PC_DIAG_MX: {
                const uint32_t cnt = (hot >> 8) & 0xffu;
                float2 f = make_float2(1.f, 0.f);
                for (uint32_t e = 1; e <= cnt; ++e) {
                    const uint4 rec = sops[oi + e];
                    const uint32_t cw = rec.y;
                    const uint32_t tm = rec.z;
                    const bool tp = (T & tm) == tm;
                    if (tp) f = cmulf(f, scoef[rec.x >> 16]);
                    const bool last = (e == cnt) || ((cw >> 25) & 1u);
                    if (last) {
                        diag_p(re, im, true, cw & 0xffu, f);
                        f = make_float2(1.f, 0.f);
                    }
                }
                oi += cnt;
                if (oi + 1 < nops) w = ow[4 * (oi + 1)];
                break;
            }
            case PC_DIAG_TAB:
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float2 c0 = m[j], c1 = m[j + 8];
                    cmul2(re[j], im[j], pk(c0.x, c1.x), pk(c0.y, c1.y));
                }
                break;
            case PC_DIAG_TM: {
                const uint32_t cnt = (hot >> 8) & 0xffu;
                float2 f = make_float2(1.f, 0.f);
                for (uint32_t e = 1; e <= cnt; ++e) {
                    const uint4 rec = sops[oi + e];
                    const uint32_t tm = rec.z;
                    const bool tp = (T & tm) == tm;
                    if (tp) f = cmulf(f, scoef[rec.x >> 16]);
                }
                pend = cmulf(pend, f);
                oi += cnt;
                if (oi + 1 < nops) w = ow[4 * (oi + 1)];
                break;
            }
            case PC_FLUSH: {
                const u64p cr = bc(pend.x), ci = bc(pend.y);
#pragma unroll
                for (int j = 0; j < 8; ++j) cmul2(re[j], im[j], cr, ci);
                pend = make_float2(1.f, 0.f);
                break;
            }
            case PC_XCHG: {
                const TileMap& mo = cur < 0 ? P.map0 : P.xmap[cur];
                const int nxt = (int)(hot >> 16);
                const TileMap& mn = P.xmap[nxt];
                __syncthreads();
                {
                    uint32_t jb = 0;
#pragma unroll
                    for (int i = 0; i < LANE_BITS; ++i) jb |= ((uint32_t)(lane >> i) & 1u) << mo.lane[i];
#pragma unroll
                    for (int i = 0; i < WARP_BITS; ++i) jb |= ((uint32_t)(wid >> i) & 1u) << mo.warp[i];
                    const uint32_t pb = spos(jb);
                    uint32_t pr[REG_BITS];
#pragma unroll
                    for (int k = 0; k < REG_BITS; ++k) pr[k] = spos(1u << mo.reg[k]);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        uint32_t p = pb;
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            if ((j >> k) & 1) p ^= pr[k];
                        tile[p] = make_float2(lo(re[j]), lo(im[j]));
                        tile[p ^ pr[3]] = make_float2(hi(re[j]), hi(im[j]));
                    }
                }
                __syncthreads();
                {
                    uint32_t jb = 0;
#pragma unroll
                    for (int i = 0; i < LANE_BITS; ++i) jb |= ((uint32_t)(lane >> i) & 1u) << mn.lane[i];
#pragma unroll
                    for (int i = 0; i < WARP_BITS; ++i) jb |= ((uint32_t)(wid >> i) & 1u) << mn.warp[i];
                    const uint32_t pb = spos(jb);
                    uint32_t pr[REG_BITS];
#pragma unroll
                    for (int k = 0; k < REG_BITS; ++k) pr[k] = spos(1u << mn.reg[k]);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        uint32_t p = pb;
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            if ((j >> k) & 1) p ^= pr[k];
                        const float2 a = tile[p], b = tile[p ^ pr[3]];
                        re[j] = pk(a.x, b.x);
                        im[j] = pk(a.y, b.y);
                    }
                }
                cur = nxt;
                break;
            }
            default: break;
        }
    }

    double ss = 0.0;
    {
        const u64p cr = bc(pend.x), ci = bc(pend.y);
        const TileMap& mf = cur < 0 ? P.map0 : P.xmap[cur];
        uint64_t tb = g0 + (uint64_t)lane;
#pragma unroll
        for (int k = 0; k < WARP_BITS; ++k)
            if ((wid >> k) & 1) tb += 1ull << P.out_qubit[mf.warp[k]];
        uint64_t rst[REG_BITS];
#pragma unroll
        for (int k = 0; k < REG_BITS; ++k) rst[k] = 1ull << P.out_qubit[mf.reg[k]];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            uint64_t g = tb;
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) g += rst[k];
            cmul2(re[j], im[j], cr, ci);
            const float2 a = make_float2(lo(re[j]), lo(im[j])), b = make_float2(hi(re[j]), hi(im[j]));
            __stcs(amps + g, a);
            __stcs(amps + g + rst[3], b);
        }
        ss = norm2_p(re, im);
    }
    if (!partial_out) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if (lane == 0) red[wid] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w2 = 0; w2 < PASS_THREADS / 32; ++w2) t += red[w2];
        *partial_out = t;
    }
}

// Two tiles per CTA: tile b and tile b + 2^(nout-1) (they differ in the
// highest qubit outside the tile) run the same op stream side by side, so
// every dispatch, condition word and coefficient load serves 32 amplitudes
// per thread instead of 16. Conditions, angle phases and pending factors are
// kept per tile.
__device__ __forceinline__ void pass_tile_p32x2(float2* __restrict__ amps, const PassParams& P, const double nrm,
                                                const uint64_t blk0, double* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char p32x2_smem[];
    float2* tile0 = reinterpret_cast<float2*>(p32x2_smem);
    float2* tile1 = tile0 + (1 << TILE_BITS);
    __shared__ double red[2][PASS_THREADS / 32];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nout = (int)P.n - TILE_BITS;
    const uint64_t blk[2] = {blk0, blk0 | (1ull << (nout - 1))};
    // tile origins are rebuilt where they are needed (load, store) rather
    // than held in registers through the op loop
    auto origin = [&](int h) {
        uint64_t g = 0;
        for (int k = 0; k < nout; ++k) g |= ((blk[h] >> k) & 1ull) << P.outer_qubits[k];
        return g;
    };
    uint32_t T[2];
#pragma unroll
    for (int h = 0; h < 2; ++h)
        T[h] = (uint32_t)lane | ((uint32_t)wid << LANE_BITS) | ((uint32_t)blk[h] << (LANE_BITS + WARP_BITS));
    const uint32_t nops = P.nops;
    uint4* sops = reinterpret_cast<uint4*>(tile1 + (1 << TILE_BITS));
    float2* scoef = reinterpret_cast<float2*>(sops + nops);
    {
        const uint4* gops = reinterpret_cast<const uint4*>(P.ops);
        for (uint32_t i = threadIdx.x; i < nops; i += PASS_THREADS) sops[i] = gops[i];
        for (uint32_t i = threadIdx.x; i < P.ncoef; i += PASS_THREADS)
            scoef[i] = make_float2((float)P.coef[i].x, (float)P.coef[i].y);
    }
    __shared__ float2 sang[2][MAX_ANG_OPS];
    for (uint32_t x = threadIdx.x; x < 2 * P.nang; x += PASS_THREADS) {
        const uint32_t h = x / P.nang, ai = x % P.nang;
        double th = 0.0;
        for (uint32_t e = P.ang_start[ai]; e < P.ang_start[ai + 1]; ++e) {
            const uint64_t om = P.angles[e].omask;
            if ((blk[h] & om) == om) th += P.angles[e].theta;
        }
        double sn, cs;
        sincos(th, &sn, &cs);
        sang[h][ai] = make_float2((float)cs, (float)sn);
    }
    const bool valid = nrm > 1e-12;
    const float2 pend0 = valid ? make_float2((float)(P.phase.x / sqrt(nrm)), (float)(P.phase.y / sqrt(nrm)))
                               : make_float2((float)P.phase.x, (float)P.phase.y);
    float2 pend[2] = {pend0, pend0};

    u64p re[2][8], im[2][8];
    {
        uint64_t rst[REG_BITS];
#pragma unroll
        for (int k = 0; k < REG_BITS; ++k) rst[k] = tstride(P, P.map0.reg[k]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint64_t tb = origin(h) + (uint64_t)lane;
#pragma unroll
            for (int k = 0; k < WARP_BITS; ++k)
                if ((wid >> k) & 1) tb += tstride(P, P.map0.warp[k]);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                uint64_t g = tb;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if ((j >> k) & 1) g += rst[k];
                const uint64_t g8 = g + rst[3];
                float2 a = valid ? __ldcs(amps + g) : make_float2(g == 0 ? 1.f : 0.f, 0.f);
                float2 b = valid ? __ldcs(amps + g8) : make_float2(0.f, 0.f);
                re[h][j] = pk(a.x, b.x);
                im[h][j] = pk(a.y, b.y);
            }
        }
    }
    __syncthreads();

    const uint32_t* ow = reinterpret_cast<const uint32_t*>(sops);
    int cur = -1;
    uint32_t w = nops ? ow[0] : 0;
    for (uint32_t oi = 0; oi < nops; ++oi) {
        const uint32_t hot = w;
        if (oi + 1 < nops) w = ow[4 * (oi + 1)];
        const uint32_t code = hot & 0xffu;
        const float2* m = scoef + (hot >> 16);
        const uint32_t cw = ow[4 * oi + 1];
        const uint32_t tm = ow[4 * oi + 2];
        switch (code) {
#define QOA_P3(BASE, SUB)                                                              \
    case BASE + 0: g1p<SUB, 0>(re[0], im[0], m); g1p<SUB, 0>(re[1], im[1], m); break;  \
    case BASE + 1: g1p<SUB, 1>(re[0], im[0], m); g1p<SUB, 1>(re[1], im[1], m); break;  \
    case BASE + 2: g1p<SUB, 2>(re[0], im[0], m); g1p<SUB, 2>(re[1], im[1], m); break;  \
    case BASE + 3: g1_bit3<SUB>(re[0], im[0], m); g1_bit3<SUB>(re[1], im[1], m); break;
            QOA_P3(PC_HF, G1_HF)
            QOA_P3(PC_RX, G1_RXA)
            QOA_P3(PC_RY, G1_RYA)
            QOA_P3(PC_RXB, G1_RXB)
            QOA_P3(PC_RYB, G1_RYB)
            QOA_P3(PC_GEN, G1_GEN)
#undef QOA_P3
#define QOA_C4(BASE, SUB)                                                                          \
    case BASE + 0: g1c<SUB, 0>(re[0], im[0], (T[0] & tm) == tm, cw & 0xffu);                      \
                   g1c<SUB, 0>(re[1], im[1], (T[1] & tm) == tm, cw & 0xffu); break;               \
    case BASE + 1: g1c<SUB, 1>(re[0], im[0], (T[0] & tm) == tm, cw & 0xffu);                      \
                   g1c<SUB, 1>(re[1], im[1], (T[1] & tm) == tm, cw & 0xffu); break;               \
    case BASE + 2: g1c<SUB, 2>(re[0], im[0], (T[0] & tm) == tm, cw & 0xffu);                      \
                   g1c<SUB, 2>(re[1], im[1], (T[1] & tm) == tm, cw & 0xffu); break;               \
    case BASE + 3: g1c<SUB, 3>(re[0], im[0], (T[0] & tm) == tm, cw & 0xffu);                      \
                   g1c<SUB, 3>(re[1], im[1], (T[1] & tm) == tm, cw & 0xffu); break;
            QOA_C4(PC_XC, G1_X)
            QOA_C4(PC_YC, G1_Y)
#undef QOA_C4
            case PC_DIAG_T:
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    if ((T[h] & tm) == tm) pend[h] = cmulf(pend[h], m[0]);
                break;
            case PC_DIAG_M:
#pragma unroll
                for (int h = 0; h < 2; ++h) diag_p(re[h], im[h], (T[h] & tm) == tm, cw & 0xffu, m[0]);
                break;
            case PC_DIAG_TA:
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    if ((T[h] & tm) == tm) pend[h] = cmulf(pend[h], sang[h][hot >> 16]);
                break;
            case PC_DIAG_MA:
#pragma unroll
                for (int h = 0; h < 2; ++h) diag_p(re[h], im[h], true, cw & 0xffu, sang[h][hot >> 16]);
                break;
            case PC_DIAG_MX: {
                const uint32_t cnt = (hot >> 8) & 0xffu;
                float2 f[2] = {make_float2(1.f, 0.f), make_float2(1.f, 0.f)};
                for (uint32_t e = 1; e <= cnt; ++e) {
                    const uint4 rec = sops[oi + e];
                    const float2 c = scoef[rec.x >> 16];
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        if ((T[h] & rec.z) == rec.z) f[h] = cmulf(f[h], c);
                    if ((e == cnt) || ((rec.y >> 25) & 1u)) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            diag_p(re[h], im[h], true, rec.y & 0xffu, f[h]);
                            f[h] = make_float2(1.f, 0.f);
                        }
                    }
                }
                oi += cnt;
                if (oi + 1 < nops) w = ow[4 * (oi + 1)];
                break;
            }
            case PC_DIAG_TAB:
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float2 c0 = m[j], c1 = m[j + 8];
                    const u64p cr = pk(c0.x, c1.x), ci = pk(c0.y, c1.y);
                    cmul2(re[0][j], im[0][j], cr, ci);
                    cmul2(re[1][j], im[1][j], cr, ci);
                }
                break;
            case PC_DIAG_TM: {
                const uint32_t cnt = (hot >> 8) & 0xffu;
                float2 f[2] = {make_float2(1.f, 0.f), make_float2(1.f, 0.f)};
                for (uint32_t e = 1; e <= cnt; ++e) {
                    const uint4 rec = sops[oi + e];
                    const float2 c = scoef[rec.x >> 16];
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        if ((T[h] & rec.z) == rec.z) f[h] = cmulf(f[h], c);
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) pend[h] = cmulf(pend[h], f[h]);
                oi += cnt;
                if (oi + 1 < nops) w = ow[4 * (oi + 1)];
                break;
            }
            case PC_FLUSH:
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const u64p cr = bc(pend[h].x), ci = bc(pend[h].y);
#pragma unroll
                    for (int j = 0; j < 8; ++j) cmul2(re[h][j], im[h][j], cr, ci);
                    pend[h] = make_float2(1.f, 0.f);
                }
                break;
            case PC_XCHG: {
                const TileMap& mo = cur < 0 ? P.map0 : P.xmap[cur];
                const int nxt = (int)(hot >> 16);
                const TileMap& mn = P.xmap[nxt];
                __syncthreads();
                {
                    uint32_t jb = 0;
#pragma unroll
                    for (int i = 0; i < LANE_BITS; ++i) jb |= ((uint32_t)(lane >> i) & 1u) << mo.lane[i];
#pragma unroll
                    for (int i = 0; i < WARP_BITS; ++i) jb |= ((uint32_t)(wid >> i) & 1u) << mo.warp[i];
                    const uint32_t pb = spos(jb);
                    uint32_t pr[REG_BITS];
#pragma unroll
                    for (int k = 0; k < REG_BITS; ++k) pr[k] = spos(1u << mo.reg[k]);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        uint32_t p = pb;
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            if ((j >> k) & 1) p ^= pr[k];
                        tile0[p] = make_float2(lo(re[0][j]), lo(im[0][j]));
                        tile0[p ^ pr[3]] = make_float2(hi(re[0][j]), hi(im[0][j]));
                        tile1[p] = make_float2(lo(re[1][j]), lo(im[1][j]));
                        tile1[p ^ pr[3]] = make_float2(hi(re[1][j]), hi(im[1][j]));
                    }
                }
                __syncthreads();
                {
                    uint32_t jb = 0;
#pragma unroll
                    for (int i = 0; i < LANE_BITS; ++i) jb |= ((uint32_t)(lane >> i) & 1u) << mn.lane[i];
#pragma unroll
                    for (int i = 0; i < WARP_BITS; ++i) jb |= ((uint32_t)(wid >> i) & 1u) << mn.warp[i];
                    const uint32_t pb = spos(jb);
                    uint32_t pr[REG_BITS];
#pragma unroll
                    for (int k = 0; k < REG_BITS; ++k) pr[k] = spos(1u << mn.reg[k]);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        uint32_t p = pb;
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            if ((j >> k) & 1) p ^= pr[k];
                        float2 a = tile0[p], b = tile0[p ^ pr[3]];
                        re[0][j] = pk(a.x, b.x);
                        im[0][j] = pk(a.y, b.y);
                        a = tile1[p];
                        b = tile1[p ^ pr[3]];
                        re[1][j] = pk(a.x, b.x);
                        im[1][j] = pk(a.y, b.y);
                    }
                }
                cur = nxt;
                break;
            }
            default: break;
        }
    }

    double ss[2] = {0.0, 0.0};
    {
        const TileMap& mf = cur < 0 ? P.map0 : P.xmap[cur];
        uint64_t rst[REG_BITS];
#pragma unroll
        for (int k = 0; k < REG_BITS; ++k) rst[k] = 1ull << P.out_qubit[mf.reg[k]];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const u64p cr = bc(pend[h].x), ci = bc(pend[h].y);
            uint64_t tb = origin(h) + (uint64_t)lane;
#pragma unroll
            for (int k = 0; k < WARP_BITS; ++k)
                if ((wid >> k) & 1) tb += 1ull << P.out_qubit[mf.warp[k]];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                uint64_t g = tb;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if ((j >> k) & 1) g += rst[k];
                cmul2(re[h][j], im[h][j], cr, ci);
                const float2 a = make_float2(lo(re[h][j]), lo(im[h][j]));
                const float2 b = make_float2(hi(re[h][j]), hi(im[h][j]));
                __stcs(amps + g, a);
                __stcs(amps + g + rst[3], b);
            }
            ss[h] = norm2_p(re[h], im[h]);
        }
    }
    if (!partials) return;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss[h] += __shfl_xor_sync(0xffffffffu, ss[h], o);
        if (lane == 0) red[h][wid] = ss[h];
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
#pragma unroll
        for (int w2 = 0; w2 < PASS_THREADS / 32; ++w2) t += red[threadIdx.x][w2];
        partials[blk[threadIdx.x]] = t;
    }
}

#ifndef QOA_PASS_OCC32X2
#define QOA_PASS_OCC32X2 4
#endif

__global__ void __launch_bounds__(PASS_THREADS, QOA_PASS_OCC32X2)
k_pass_p32x2(float2* __restrict__ amps, const __grid_constant__ PassParams P, const double* __restrict__ norm2_in,
             double* __restrict__ partials) {
    pass_tile_p32x2(amps, P, *norm2_in, blockIdx.x, partials);
}

#ifndef QOA_PASS_OCC32
#define QOA_PASS_OCC32 7
#endif

__global__ void __launch_bounds__(PASS_THREADS, QOA_PASS_OCC32)
k_pass_p32(float2* __restrict__ amps, const __grid_constant__ PassParams P, const double* __restrict__ norm2_in,
           double* __restrict__ partials) {
    pass_tile_p32(amps, P, *norm2_in, blockIdx.x, partials + blockIdx.x);
}

__global__ void __launch_bounds__(PASS_THREADS, QOA_PASS_OCC32)
k_pass_p32_arena(const ArenaJob* __restrict__ jobs, uint32_t njobs, const uint32_t* __restrict__ tile_start) {
    const uint32_t b = blockIdx.x;
    uint32_t l = 0, h = njobs - 1;
    while (l < h) {
        const uint32_t mid = (l + h + 1) >> 1;
        if (tile_start[mid] <= b) l = mid;
        else h = mid - 1;
    }
    const ArenaJob J = jobs[l];
    pass_tile_p32(reinterpret_cast<float2*>(J.amps), *reinterpret_cast<const PassParams*>(J.params),
                  J.fresh ? 0.0 : 1.0, b - tile_start[l], nullptr);
}

}  // namespace

cudaError_t launch_pass_p32(float2* amps, const PassParams& P, const double* norm2_in, double* partials,
                            cudaStream_t st) {
    if (P.n > (uint32_t)TILE_BITS) {  // two tiles per CTA
        const int tiles_bytes = 2 * (1 << TILE_BITS) * (int)sizeof(float2);
        const int smem = tiles_bytes + (int)P.nops * 16 + (int)P.ncoef * (int)sizeof(float2);
        cudaError_t e = cudaFuncSetAttribute(k_pass_p32x2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             tiles_bytes + MAX_PASS_OPS * 16 + MAX_PASS_COEF * (int)sizeof(float2));
        if (e != cudaSuccess) return e;
        k_pass_p32x2<<<1u << (P.n - TILE_BITS - 1), PASS_THREADS, smem, st>>>(amps, P, norm2_in, partials);
        return cudaGetLastError();
    }
    const int tile_bytes = (1 << TILE_BITS) * (int)sizeof(float2);
    const int smem = tile_bytes + (int)P.nops * 16 + (int)P.ncoef * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_pass_p32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tile_bytes + MAX_PASS_OPS * 16 + MAX_PASS_COEF * (int)sizeof(float2));
    if (e != cudaSuccess) return e;
    k_pass_p32<<<1u << (P.n - TILE_BITS), PASS_THREADS, smem, st>>>(amps, P, norm2_in, partials);
    return cudaGetLastError();
}

cudaError_t launch_pass_p32_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                                  int max_nops, int max_ncoef, cudaStream_t st) {
    if (!njobs || !tiles) return cudaSuccess;
    const int tile_bytes = (1 << TILE_BITS) * (int)sizeof(float2);
    const int smem = tile_bytes + max_nops * 16 + max_ncoef * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_pass_p32_arena, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tile_bytes + MAX_PASS_OPS * 16 + MAX_PASS_COEF * (int)sizeof(float2));
    if (e != cudaSuccess) return e;
    k_pass_p32_arena<<<tiles, PASS_THREADS, smem, st>>>(jobs, njobs, tile_start);
    return cudaGetLastError();
}

}  // namespace qoa
