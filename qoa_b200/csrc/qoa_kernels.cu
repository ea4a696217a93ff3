// qoa_kernels.cu — sm_100a kernels of the state-vector engine.
//
// Hot path: k_pass, one HBM read + write of the whole state for a run of gates
// whose non-diagonal targets fall inside an 11-qubit tile (5 lane qubits that
// keep every warp access 512 contiguous bytes, 4 register qubits, 2 warp
// qubits; TILE_BITS, REG_BITS and WARP_BITS in qoa_kernels.cuh). It replaces the per-gate sweeps of src/vectorization.rs:915-1260
// plus the two normalize() sweeps that follow every gate
// (src/runtime/quantum_state.rs:839-907): the pass scales its input by the
// pending 1/||psi|| and leaves per-CTA partial sums of |a|^2 for the next one.
//
// The rest: per-gate kernels over global memory (fallback, per-gate mode and
// the vectorization.rs shims), the measurement reductions and collapse of
// quantum_state.rs:399-458, the marginal tree behind measure_all-order
// sampling (quantum_state.rs:909-918), and expectation values.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>
#include <string.h>

#include "qoa_kernels.cuh"
#include "qoa_pass_dev.cuh"

namespace qoa {

// Global index stride of tile bit t (t < 5: qubit t; else high slot t - 5).
__device__ __forceinline__ uint64_t tstride(const PassParams& P, uint32_t t) {
    return 1ull << (t < LANE_BITS ? t : P.slot_qubit[t - LANE_BITS]);
}

// ------------------------------------------------------------ the pass kernel
// One CTA's tile of one pass. `blk` numbers the tile (its bits go to the
// qubits outside the tile); `nrm` is the input's squared norm (<= 1e-12: the
// input is |0..0>, synthesised without reading); `partial_out`, when not
// null, receives the tile's squared norm after the pass. The pass's
// coefficients are built in FP64 on the host; a complex64 pass rounds them
// once when it stages them.
template <typename T>
__device__ __forceinline__ void pass_tile(T* __restrict__ amps, const PassParams& P, const double nrm,
                                          const uint64_t blk, double* __restrict__ partial_out) {
    using R = typename CT<T>::R;
    extern __shared__ __align__(16) unsigned char pass_smem[];
    T* tile = reinterpret_cast<T*>(pass_smem);
    __shared__ double red[PASS_THREADS / 32];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;

    // Global index of this CTA's tile origin: blockIdx.x deposited into the
    // qubits outside the tile.
    uint64_t g0 = 0;
    {
        const uint64_t b = blk;
        const int nout = (int)P.n - TILE_BITS;
        for (int k = 0; k < nout; ++k) g0 |= ((b >> k) & 1ull) << P.outer_qubits[k];
    }
    // the thread's condition word: lane bits, warp bits, then the tile number
    // (whose bit k is the bit of the k-th qubit outside the tile)
    const uint32_t tw = (uint32_t)lane | ((uint32_t)wid << LANE_BITS) | ((uint32_t)blk << (LANE_BITS + WARP_BITS));

    // op stream and coefficients -> shared memory (after the tile)
    const uint32_t nops = P.nops;
    uint4* sops = reinterpret_cast<uint4*>(tile + (1 << TILE_BITS));
    T* scoef = reinterpret_cast<T*>(sops + nops);
    {
        const uint4* gops = reinterpret_cast<const uint4*>(P.ops);
        for (uint32_t i = threadIdx.x; i < nops; i += PASS_THREADS) sops[i] = gops[i];
        for (uint32_t i = threadIdx.x; i < P.ncoef; i += PASS_THREADS) scoef[i] = CT<T>::from(P.coef[i]);
    }
    // angle phases of this CTA: sum the thetas whose outer condition holds
    __shared__ T sang[MAX_ANG_OPS];
    pass_angles(P, blk, sang);

    const bool valid = nrm > 1e-12;
    // The input's 1/||psi|| and the pass's factored global phase are applied
    // once, at the end, as part of the per-thread pending factor.
    T pend = valid ? CT<T>::from(make_double2(P.phase.x / sqrt(nrm), P.phase.y / sqrt(nrm)))
                   : CT<T>::from(P.phase);

    // Load with the initial mapping: lanes are tile bits 0..4 = qubits 0..4,
    // so each warp reads 32 consecutive amplitudes per register.
    T a[REGS];
    {
        uint64_t tb = g0 + (uint64_t)lane;
#pragma unroll
        for (int k = 0; k < WARP_BITS; ++k)
            if ((wid >> k) & 1) tb += tstride(P, P.map0.warp[k]);
        uint64_t rst[REG_BITS];
#pragma unroll
        for (int k = 0; k < REG_BITS; ++k) rst[k] = tstride(P, P.map0.reg[k]);
#pragma unroll
        for (int v = 0; v < REGS; ++v) {
            uint64_t g = tb;
#pragma unroll
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) g += rst[k];
            a[v] = valid ? __ldcs(amps + g) : CT<T>::mk(g == 0 ? (R)1 : (R)0, (R)0);
        }
    }
    __syncthreads();  // op stream staged

    const uint32_t* ow = reinterpret_cast<const uint32_t*>(sops);
    int cur = -1;  // mapping in force: -1 = map0, else xmap index
    uint32_t w = nops ? ow[0] : 0;
    for (uint32_t oi = 0; oi < nops; ++oi) {
        const uint32_t hot = w;
        if (oi + 1 < nops) w = ow[4 * (oi + 1)];
        const uint32_t code = hot & 0xffu;
        const T* m = scoef + (hot >> 16);
        // condition of ops that take one: register mask and thread predicate
        auto conds = [&](bool& tp) -> uint32_t {
            const uint32_t cw = ow[4 * oi + 1];
            const uint32_t tm = ow[4 * oi + 2];
            tp = (tw & tm) == tm;
            return cw & 0xffu;
        };
        switch (code) {
#define QOA_K4(BASE, ...) \
    case BASE + 0: { constexpr int K = 0; __VA_ARGS__; } break; \
    case BASE + 1: { constexpr int K = 1; __VA_ARGS__; } break; \
    case BASE + 2: { constexpr int K = 2; __VA_ARGS__; } break; \
    case BASE + 3: { constexpr int K = 3; __VA_ARGS__; } break;
            QOA_K4(PC_HF, g1r<G1_HF, K>(a, m))
            QOA_K4(PC_RX, g1r<G1_RXA, K>(a, m))
            QOA_K4(PC_RY, g1r<G1_RYA, K>(a, m))
            QOA_K4(PC_RXB, g1r<G1_RXB, K>(a, m))
            QOA_K4(PC_RYB, g1r<G1_RYB, K>(a, m))
            QOA_K4(PC_GEN, g1r<G1_GEN, K>(a, m))
            QOA_K4(PC_XC, bool tp; const uint32_t cr = conds(tp); g1rc<G1_X, K>(a, tp, cr))
            QOA_K4(PC_YC, bool tp; const uint32_t cr = conds(tp); g1rc<G1_Y, K>(a, tp, cr))
#undef QOA_K4
            case PC_DIAG_T: {
                bool tp;
                conds(tp);
                if (tp) pend = c_mul(pend, m[0]);
                break;
            }
            case PC_DIAG_M: {
                bool tp;
                const uint32_t cr = conds(tp);
                diag_m(a, tp, cr, m[0]);
                break;
            }
            case PC_DIAG_TA: {
                bool tp;
                conds(tp);
                if (tp) pend = c_mul(pend, sang[hot >> 16]);
                break;
            }
            case PC_DIAG_MA:
                diag_m(a, true, ow[4 * oi + 1] & 0xffu, sang[hot >> 16]);
                break;
            case PC_DIAG_MX: {
                // entries sorted by register mask: each run of equal masks
                // folds its thread-conditioned factors into one scalar, then
                // multiplies the matching registers once
                const uint32_t cnt = (hot >> 8) & 0xffu;
                T f = CT<T>::mk(1, 0);
                for (uint32_t e = 1; e <= cnt; ++e) {
                    const uint4 rec = sops[oi + e];
                    const uint32_t cw = rec.y;
                    const uint32_t tm = rec.z;
                    const bool tp = (tw & tm) == tm;
                    if (tp) f = c_mul(f, scoef[rec.x >> 16]);
                    const bool last = (e == cnt) || ((cw >> 25) & 1u);
                    if (last) {
                        diag_m(a, true, cw & 0xffu, f);
                        f = CT<T>::mk(1, 0);
                    }
                }
                oi += cnt;
                if (oi + 1 < nops) w = ow[4 * (oi + 1)];
                break;
            }
            case PC_DIAG_TAB:
#pragma unroll
                for (int v = 0; v < REGS; ++v) a[v] = c_mul(a[v], m[v]);
                break;
            case PC_DIAG_TM: {
                // entries oi+1 .. oi+cnt: independent factors, multiplied in
                const uint32_t cnt = (hot >> 8) & 0xffu;
                T f = CT<T>::mk(1, 0);
                for (uint32_t e = 1; e <= cnt; ++e) {
                    const uint4 rec = sops[oi + e];
                    const uint32_t tm = rec.z;
                    const bool tp = (tw & tm) == tm;
                    if (tp) f = c_mul(f, scoef[rec.x >> 16]);
                }
                pend = c_mul(pend, f);
                oi += cnt;
                if (oi + 1 < nops) w = ow[4 * (oi + 1)];
                break;
            }
            case PC_FLUSH:
#pragma unroll
                for (int v = 0; v < REGS; ++v) a[v] = c_mul(a[v], pend);
                pend = CT<T>::mk(1, 0);
                break;
            case PC_XCHG: {
                // write under the current mapping, read under the new one
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
                    for (int v = 0; v < REGS; ++v) {
                        uint32_t p = pb;
#pragma unroll
                        for (int k = 0; k < REG_BITS; ++k)
                            if ((v >> k) & 1) p ^= pr[k];
                        tile[p] = a[v];
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
                    for (int v = 0; v < REGS; ++v) {
                        uint32_t p = pb;
#pragma unroll
                        for (int k = 0; k < REG_BITS; ++k)
                            if ((v >> k) & 1) p ^= pr[k];
                        a[v] = tile[p];
                    }
                }
                cur = nxt;
                break;
            }
            default: break;
        }
    }

    // final flush of the pending factor, store, and norm partials. Tile bit t
    // goes to global qubit out_qubit[t] (its load qubit unless SWAPs in the
    // pass relabelled it); the last mapping has on lane i the tile bit stored
    // to qubit i, so the store is as coalesced as the load.
    double ss = 0.0;
    {
        const TileMap& mf = cur < 0 ? P.map0 : P.xmap[cur];
        uint64_t tb = g0 + (uint64_t)lane;
#pragma unroll
        for (int k = 0; k < WARP_BITS; ++k)
            if ((wid >> k) & 1) tb += 1ull << P.out_qubit[mf.warp[k]];
        uint64_t rst[REG_BITS];
#pragma unroll
        for (int k = 0; k < REG_BITS; ++k) rst[k] = 1ull << P.out_qubit[mf.reg[k]];
#pragma unroll
        for (int v = 0; v < REGS; ++v) {
            uint64_t g = tb;
#pragma unroll
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) g += rst[k];
            const T x = c_mul(a[v], pend);
            __stcs(amps + g, x);
            ss += c_abs2(x);
        }
    }
    if (!partial_out) return;
    block_norm_partial(ss, red, partial_out);
}

// Resident CTAs per SM: the complex128 pass needs 128 registers a thread.
// (The complex64 passes are the packed kernels of qoa_pass32.cu.)
#ifndef QOA_PASS_OCC64
#define QOA_PASS_OCC64 4
#endif
template <typename T> struct PassOcc { static constexpr int value = QOA_PASS_OCC64; };

template <typename T>
__global__ void __launch_bounds__(PASS_THREADS, PassOcc<T>::value)
k_pass(T* __restrict__ amps, const __grid_constant__ PassParams P, const double* __restrict__ norm2_in,
       double* __restrict__ partials) {
    pass_tile<T>(amps, P, *norm2_in, blockIdx.x, partials + blockIdx.x);
}

// Arena pass: one launch runs one pass of each of many circuits, whose states
// lie in one packed arena. CTA b runs tile b - tile_start[j] of job j, where
// j is the last job with tile_start[j] <= b. Squared norms are not tracked: a
// batched circuit is unitary, its start |0..0> is synthesised by its first
// pass, and its consumers normalise.
template <typename T>
__global__ void __launch_bounds__(PASS_THREADS, PassOcc<T>::value)
k_pass_arena(const ArenaJob* __restrict__ jobs, uint32_t njobs, const uint32_t* __restrict__ tile_start) {
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (tile_start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const ArenaJob J = jobs[lo];
    pass_tile<T>(reinterpret_cast<T*>(J.amps), *reinterpret_cast<const PassParams*>(J.params),
                 J.fresh ? 0.0 : 1.0, b - tile_start[lo], nullptr);
}

// ------------------------------------------------------- per-gate kernels
// Element-indexed grid-stride loops over [0, len) so that any slice length
// works, as the reference's `j < len` checks allow (vectorization.rs:920-935).
__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

template <int SUB, typename T>
__global__ void k_gate_g1(T* __restrict__ a, uint64_t len, const __grid_constant__ GGate g) {
    const uint64_t bit = 1ull << g.t;
    const T m0 = CT<T>::from(g.m[0]), m1 = CT<T>::from(g.m[1]), m2 = CT<T>::from(g.m[2]), m3 = CT<T>::from(g.m[3]);
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        if (i & bit) continue;
        const uint64_t j = i | bit;
        if (j >= len || (i & g.cmask) != g.cmask) continue;
        T x = a[i], y = a[j];
        g1_pair<SUB>(x, y, m0, m1, m2, m3);
        a[i] = x;
        a[j] = y;
    }
}

template <typename T>
__global__ void k_gate_diag(T* __restrict__ a, uint64_t len, const __grid_constant__ GGate g) {
    const bool neg = (g.sub & 0x80u) != 0;
    const bool has_sel = g.t < 64;
    const T d0 = CT<T>::from(g.m[0]), d1 = CT<T>::from(g.m[1]);
    if (!has_sel && len && !(len & (len - 1)) && g.cmask < len) {
        // a masked phase touches only the indices with every mask bit set:
        // walk those, consecutive threads on consecutive ones (compact index
        // k with a 1 inserted at each mask bit), instead of the whole state
        const uint64_t cnt = len >> __popcll(g.cmask);
        for (uint64_t k = gtid(); k < cnt; k += gstride()) {
            uint64_t i = k;
            for (uint64_t m = g.cmask; m; m &= m - 1) {
                const uint64_t b = m & (0 - m);
                i = ((i & ~(b - 1)) << 1) | b | (i & (b - 1));
            }
            a[i] = neg ? c_neg(a[i]) : c_mul(a[i], d0);
        }
        return;
    }
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        if ((i & g.cmask) != g.cmask) continue;
        if (neg) {
            a[i] = c_neg(a[i]);
        } else {
            const bool s = has_sel && ((i >> g.t) & 1ull);
            a[i] = c_mul(a[i], s ? d1 : d0);
        }
    }
}

template <typename T>
__global__ void k_gate_swap(T* __restrict__ a, uint64_t len, const __grid_constant__ GGate g) {
    const uint64_t m1 = 1ull << g.t, m2 = 1ull << g.t2;
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        if ((i & (m1 | m2)) != 0 || (i & g.cmask) != g.cmask) continue;
        const uint64_t x = i | m2, y = i | m1;
        if (x < len && y < len) {
            const T t = a[x];
            a[x] = a[y];
            a[y] = t;
        }
    }
}

template <typename T>
__global__ void k_gate_u2(T* __restrict__ a, uint64_t len, const __grid_constant__ GGate g) {
    const uint64_t ml = 1ull << g.t, mh = 1ull << g.t2;
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        if ((i & (ml | mh)) != 0) continue;
        const uint64_t idx[4] = {i, i | ml, i | mh, i | ml | mh};
        if (idx[3] >= len) continue;
        T x[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k] = a[idx[k]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            T acc = c_mul(CT<T>::from(g.m[4 * r]), x[0]);
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                const T c = CT<T>::from(g.m[4 * r + k]);
                acc.x = fma(c.x, x[k].x, acc.x); acc.x = fma(-c.y, x[k].y, acc.x);
                acc.y = fma(c.x, x[k].y, acc.y); acc.y = fma(c.y, x[k].x, acc.y);
            }
            a[idx[r]] = acc;
        }
    }
}

template <typename T>
__global__ void k_reset_all(T* __restrict__ a, uint64_t len) {
    for (uint64_t i = gtid(); i < len; i += gstride()) a[i] = CT<T>::mk(i == 0 ? 1 : 0, 0);
}

// ------------------------------------------------------------ SWAP blocks
// out[pi(i)] = in[i] for an involution pi of the qubits (disjoint SWAPs). The
// norm is unchanged, so no partial sums are written.
template <typename T>
__global__ void __launch_bounds__(256) k_swapnet(T* __restrict__ a, const __grid_constant__ PermParams P) {
    extern __shared__ __align__(16) unsigned char sw_smem[];
    const uint32_t tn = 1u << P.na;
    T* s0 = reinterpret_cast<T*>(sw_smem);
    T* s1 = s0 + tn;
    // tile index j = lo | hi << hl: its global offset and its source's tile
    // index, from two small tables each (built once per CTA)
    const uint32_t hl = P.na / 2, hh = P.na - hl;
    __shared__ uint64_t glo[64], ghi[64];
    __shared__ uint32_t slo[64], shi[64];
    for (uint32_t x = threadIdx.x; x < (1u << hh); x += blockDim.x) {
        uint64_t gl = 0, gh = 0;
        uint32_t sl = 0, sh = 0;
        for (uint32_t k = 0; k < hh; ++k) {
            if (k < hl && ((x >> k) & 1)) {
                gl |= 1ull << P.tq[k];
                sl |= 1u << P.src_bit[k];
            }
            if ((x >> k) & 1) {
                gh |= 1ull << P.tq[hl + k];
                sh |= 1u << P.src_bit[hl + k];
            }
        }
        if (x < (1u << hl)) {
            glo[x] = gl;
            slo[x] = sl;
        }
        ghi[x] = gh;
        shi[x] = sh;
    }
    // a tile number b's outer offset o, its partner's po and the partner's
    // tile number pb, each a sum over b's bytes of 256-entry tables (built
    // once per CTA; a tile's loops over its outer bits cost more than its
    // data movement)
    const uint32_t nout = P.n - P.na;
    const uint64_t ntiles = 1ull << nout;
    const uint32_t nchunk = (nout + 7) / 8;  // <= 4: the launcher checks nout <= 32
    // (the partner's offset po is the deposit of pb, so one offset table
    // serves both; 12 KB of tables keep the kernel under 48 KB of shared
    // memory with two complex128 tiles)
    __shared__ uint64_t t_o[4][256];
    __shared__ uint32_t t_pb[4][256];
    __shared__ uint8_t oidx[64];  // qubit -> its position in oq
    for (uint32_t k = threadIdx.x; k < nout; k += blockDim.x) oidx[P.oq[k]] = (uint8_t)k;
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < nchunk * 256; e += blockDim.x) {
        const uint32_t c = e >> 8, x = e & 255;
        uint64_t o = 0;
        uint32_t pb = 0;
        for (uint32_t i = 0; i < 8; ++i) {
            const uint32_t k = 8 * c + i;
            if (k >= nout || !((x >> i) & 1)) continue;
            o |= 1ull << P.oq[k];
            pb |= 1u << oidx[P.pi[P.oq[k]]];
        }
        t_o[c][x] = o;
        t_pb[c][x] = pb;
    }
    __syncthreads();
    // shared-memory slot of tile index j: its low five bits XORed with the
    // next five, so the permuted reads of a warp spread over the banks
    auto sp = [](uint32_t j) { return j ^ ((j >> 5) & 31u); };
    // persistent: CTA walks tiles b, b + gridDim.x, ...; a tile whose partner
    // (its outer bits permuted) comes first is moved by the partner's turn
    for (uint64_t b = blockIdx.x; b < ntiles; b += gridDim.x) {
        uint64_t o = 0, po = 0, pb = 0;
        for (uint32_t c = 0; c < nchunk; ++c) {
            const uint32_t x = (uint32_t)(b >> (8 * c)) & 255u;
            o |= t_o[c][x];
            pb |= (uint64_t)t_pb[c][x];
        }
        for (uint32_t c = 0; c < nchunk; ++c) po |= t_o[c][(uint32_t)(pb >> (8 * c)) & 255u];
        if (pb < b) continue;  // uniform over the CTA
        const bool two = pb != b;
        // all of the thread's loads first (tn <= 1024: at most 4 per tile),
        // so that they are in flight together
        constexpr int kMax = 1024 / 256;
        T x0[kMax], x1[kMax];
#pragma unroll
        for (int r = 0; r < kMax; ++r) {
            const uint32_t j = threadIdx.x + 256u * (uint32_t)r;
            if (j < tn) {
                const uint64_t g = glo[j & ((1u << hl) - 1)] | ghi[j >> hl];
                x0[r] = __ldcs(a + (o | g));
                if (two) x1[r] = __ldcs(a + (po | g));
            }
        }
#pragma unroll
        for (int r = 0; r < kMax; ++r) {
            const uint32_t j = threadIdx.x + 256u * (uint32_t)r;
            if (j < tn) {
                s0[sp(j)] = x0[r];
                if (two) s1[sp(j)] = x1[r];
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kMax; ++r) {
            const uint32_t j = threadIdx.x + 256u * (uint32_t)r;
            if (j < tn) {
                const uint32_t src = slo[j & ((1u << hl) - 1)] | shi[j >> hl];
                const uint64_t g = glo[j & ((1u << hl) - 1)] | ghi[j >> hl];
                __stcs(a + (po | g), s0[sp(src)]);
                if (two) __stcs(a + (o | g), s1[sp(src)]);
            }
        }
        __syncthreads();  // the buffers are reused by the next tile
    }
}

cudaError_t launch_swapnet(void* a, bool c64, const PermParams& P, cudaStream_t st) {
    // the outer-bit tables cover 32 bits; a tile holds at most 1024 amplitudes
    if (P.n - P.na > 32 || P.na > 10) return cudaErrorInvalidValue;
    const uint64_t tiles = 1ull << (P.n - P.na);
    const size_t smem = ((size_t)2 << P.na) * (c64 ? sizeof(float2) : sizeof(double2));
    // persistent: as many CTAs as are resident at once, so none waits for a
    // slot behind CTAs that walk their whole share of the tiles
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = c64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_swapnet<float2>, 256, smem)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_swapnet<double2>, 256, smem);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)std::min<uint64_t>(tiles, (uint64_t)sms * (uint64_t)std::max(per_sm, 1));
    if (c64) k_swapnet<float2><<<blocks, 256, smem, st>>>((float2*)a, P);
    else k_swapnet<double2><<<blocks, 256, smem, st>>>((double2*)a, P);
    return cudaGetLastError();
}

// --------------------------------------------------------------- reductions
template <int NB>
__device__ __forceinline__ void block_store_partials(double (&v)[NB], double* __restrict__ out, uint32_t stride) {
    __shared__ double sh[NB][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        double x = v[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[b][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < NB) {
        double t = 0.0;
        for (int k = 0; k < nw; ++k) t += sh[threadIdx.x][k];
        out[(uint64_t)threadIdx.x * stride + blockIdx.x] = t;
    }
}

// sum |a|^2 (scaled by s^2) per block
__global__ void k_norm_partials(const double2* __restrict__ a, uint64_t len, double* __restrict__ partials) {
    double v[1] = {0.0};
    for (uint64_t i = gtid(); i < len; i += gstride()) v[0] += c_abs2(a[i]);
    block_store_partials<1>(v, partials, gridDim.x);
}

// P(bit q = 0), P(bit q = 1) of the stored vector (unscaled) per block
__global__ void k_p01_partials(const double2* __restrict__ a, uint64_t len, uint32_t q, double* __restrict__ partials) {
    double v[2] = {0.0, 0.0};
    const uint64_t m = 1ull << q;
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        const double p = c_abs2(a[i]);
        if (i & m) v[1] += p;
        else v[0] += p;
    }
    block_store_partials<2>(v, partials, gridDim.x);
}

// Z-string sums for up to 8 masks per launch
struct Masks8 {
    uint64_t m[8];
};

__global__ void k_expz_partials(const double2* __restrict__ a, uint64_t len, const Masks8 mk, uint32_t k,
                                double* __restrict__ partials) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t masks[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) masks[j] = (j < (int)k) ? mk.m[j] : 0ull;
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        const double p = c_abs2(a[i]);
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] += (__popcll(i & masks[j]) & 1) ? -p : p;
    }
    block_store_partials<8>(v, partials, gridDim.x);
}

// Final reduction: out[s] = sum_k partials[s*count + k] in a fixed order (one
// block per set), then optional scaling by 1/norm2 and status bookkeeping.
__global__ void k_reduce(const double* __restrict__ partials, uint32_t count, double* __restrict__ out,
                         const double* __restrict__ divide_by, uint32_t* __restrict__ status) {
    __shared__ double sh[32];
    const double* p = partials + (uint64_t)blockIdx.x * count;
    // eight independent accumulators per thread keep eight loads in flight
    const uint32_t B = blockDim.x;
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    uint32_t i = threadIdx.x;
    for (; i + 7 * B < count; i += 8 * B) {
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += p[i + k * B];
    }
    for (; i < count; i += B) acc[0] += p[i];
    double x = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
        if (divide_by) {
            const double d = *divide_by;
            t = (d > 1e-12) ? t / d : 0.0;
        }
        out[blockIdx.x] = t;
        if (status) {
            if (t != t) atomicOr(&status[0], 1u);
            if (!(t > 1e-12)) atomicAdd(&status[2], 1u);
        }
    }
}

// Collapse for measure / reset_qubit: keep bit q == outcome scaled by `f`
// (already including the pending 1/||psi||), zero the other branch, and leave
// norm partials of the result.
__global__ void k_collapse(double2* __restrict__ a, uint64_t len, uint32_t q, uint32_t outcome, double f,
                           double* __restrict__ partials) {
    double v[1] = {0.0};
    const uint64_t m = 1ull << q;
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        const bool set = (i & m) != 0;
        double2 x;
        if (set != (outcome != 0)) x = make_double2(0.0, 0.0);
        else {
            x = a[i];
            x = make_double2(x.x * f, x.y * f);
        }
        a[i] = x;
        v[0] += c_abs2(x);
    }
    block_store_partials<1>(v, partials, gridDim.x);
}

// Materialise the pending normalisation in place (or reset to |0..0>).
__global__ void k_materialize(double2* __restrict__ a, uint64_t len, const double* __restrict__ norm2_in,
                              double* __restrict__ partials) {
    double v[1] = {0.0};
    const double nrm = *norm2_in;
    const bool valid = nrm > 1e-12;
    const double s = valid ? 1.0 / sqrt(nrm) : 0.0;
    for (uint64_t i = gtid(); i < len; i += gstride()) {
        double2 x;
        if (valid) {
            x = a[i];
            x = make_double2(x.x * s, x.y * s);
        } else {
            x = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
        }
        a[i] = x;
        v[0] += c_abs2(x);
    }
    block_store_partials<1>(v, partials, gridDim.x);
}

__global__ void k_set_scalar(double* p, double v) { *p = v; }

// Probabilities of [off, off+cnt) scaled by 1/norm2 (|0..0> when invalid).
__global__ void k_probs(const double2* __restrict__ a, uint64_t off, uint64_t cnt, const double* __restrict__ norm2_in,
                        double* __restrict__ out) {
    const double nrm = *norm2_in;
    const bool valid = nrm > 1e-12;
    const double inv = valid ? 1.0 / nrm : 0.0;
    for (uint64_t i = gtid(); i < cnt; i += gstride()) {
        const uint64_t g = off + i;
        out[i] = valid ? c_abs2(a[g]) * inv : (g == 0 ? 1.0 : 0.0);
    }
}

// --------------------------------------------------- marginal tree & shots
// Level k (1 <= k <= n-1) holds h_k[p] = sum_{i mod 2^k == p} |a_i|^2 for
// p < 2^k at offset 2^k - 2 of `tree`. Level n-1 comes from the amplitudes.
// |amplitude|^2 in FP64 for either storage precision
__device__ __forceinline__ double amp2(const double2* a, uint64_t i) { return c_abs2(a[i]); }
__device__ __forceinline__ double amp2(const float2* a, uint64_t i) {
    const float2 x = a[i];
    return (double)x.x * x.x + (double)x.y * x.y;
}

template <typename T>
__global__ void k_tree_leaf(const T* __restrict__ a, uint32_t n, const double* __restrict__ norm2_in,
                            double* __restrict__ lvl) {
    const uint64_t half = 1ull << (n - 1);
    const double nrm = *norm2_in;
    const bool valid = nrm > 1e-12;
    const double inv = valid ? 1.0 / nrm : 0.0;
    for (uint64_t p = gtid(); p < half; p += gstride()) {
        lvl[p] = valid ? (amp2(a, p) + amp2(a, p + half)) * inv : (p == 0 ? 1.0 : 0.0);
    }
}
__global__ void k_tree_up(const double* __restrict__ hi, double* __restrict__ lo, uint64_t cnt) {
    for (uint64_t p = gtid(); p < cnt; p += gstride()) lo[p] = hi[p] + hi[p + cnt];
}

// One thread per shot. mode 0: the measure_all order of the reference — qubit
// q measured with uniform u[shot*n + q] as `u < P0`, where P0 is the
// conditional probability given the earlier outcomes; a branch with
// probability <= 1e-12 zeroes the state, which normalize() then resets to
// |0..0>, so every later outcome is 0 (quantum_state.rs:424-455, 888-907).
// mode 1: inverse CDF with one uniform per shot, walking the same tree.
template <typename T>
__global__ void k_sample(const T* __restrict__ a, uint32_t n, const double* __restrict__ norm2_in,
                         const double* __restrict__ tree, const double* __restrict__ u, uint64_t shots, int mode,
                         unsigned long long* __restrict__ out) {
    const double nrm = *norm2_in;
    const bool valid = nrm > 1e-12;
    const double inv = valid ? 1.0 / nrm : 0.0;
    auto h = [&](uint32_t k, uint64_t p) -> double {
        if (k == n) return valid ? amp2(a, p) * inv : (p == 0 ? 1.0 : 0.0);
        if (k == 0) {
            if (n == 1) return valid ? (amp2(a, 0) + amp2(a, 1)) * inv : 1.0;
            return tree[0] + tree[1];
        }
        return tree[((1ull << k) - 2) + p];
    };
    for (uint64_t s = gtid(); s < shots; s += gstride()) {
        uint64_t pre = 0;
        if (mode == 0) {
            bool dead = false;
            for (uint32_t q = 0; q < n; ++q) {
                const double uq = u[s * n + q];
                if (dead) continue;  // |0..0>: P0 = 1 and u < 1
                const double tot = h(q, pre);
                const double p0 = h(q + 1, pre) / tot;
                const double p1 = h(q + 1, pre | (1ull << q)) / tot;
                const uint32_t b = (uq < p0) ? 0u : 1u;
                const double pb = b ? p1 : p0;
                pre |= (uint64_t)b << q;
                if (!(pb > 1e-12)) dead = true;
            }
        } else {
            double t = u[s] * h(0, 0);
            for (uint32_t q = 0; q < n; ++q) {
                const double left = h(q + 1, pre);
                if (t < left) continue;
                t -= left;
                pre |= 1ull << q;
            }
        }
        out[s] = pre;
    }
}

// ------------------------------------------------------------------ launchers
static int grid_for(uint64_t work, int threads, int max_blocks) {
    uint64_t b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > (uint64_t)max_blocks) b = max_blocks;
    return (int)b;
}

template <typename T>
static cudaError_t launch_pass_t(T* amps, const PassParams& P, const double* norm2_in, double* partials,
                                 cudaStream_t st) {
    const int tile_bytes = (1 << TILE_BITS) * (int)sizeof(T);
    const int smem = tile_bytes + (int)P.nops * 16 + (int)P.ncoef * (int)sizeof(T);
    cudaError_t e = cudaFuncSetAttribute(k_pass<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tile_bytes + MAX_PASS_OPS * 16 + MAX_PASS_COEF * (int)sizeof(T));
    if (e != cudaSuccess) return e;
    const unsigned blocks = 1u << (P.n - TILE_BITS);
    k_pass<T><<<blocks, PASS_THREADS, smem, st>>>(amps, P, norm2_in, partials);
    return cudaGetLastError();
}
cudaError_t launch_pass(double2* amps, const PassParams& P, const double* norm2_in, double* partials,
                        cudaStream_t st) {
    return launch_pass_t<double2>(amps, P, norm2_in, partials, st);
}
cudaError_t launch_pass_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                              int max_nops, int max_ncoef, cudaStream_t st) {
    if (!njobs || !tiles) return cudaSuccess;
    const int esz = (int)sizeof(double2);
    const int tile_bytes = (1 << TILE_BITS) * esz;
    const int smem = tile_bytes + max_nops * 16 + max_ncoef * esz;
    const int smax = tile_bytes + MAX_PASS_OPS * 16 + MAX_PASS_COEF * esz;
    cudaError_t e = cudaFuncSetAttribute(k_pass_arena<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
    if (e != cudaSuccess) return e;
    k_pass_arena<double2><<<tiles, PASS_THREADS, smem, st>>>(jobs, njobs, tile_start);
    return cudaGetLastError();
}
template <typename T>
static cudaError_t launch_gate_t(T* a, uint64_t len, const GGate& g, cudaStream_t st) {
    const int threads = 256;
    const int blocks = grid_for(len, threads, 148 * 16);
    switch (g.kind) {
        case GG_G1:
            switch (g.sub) {
                case G1_H: k_gate_g1<G1_H, T><<<blocks, threads, 0, st>>>(a, len, g); break;
                case G1_HF: k_gate_g1<G1_HF, T><<<blocks, threads, 0, st>>>(a, len, g); break;
                case G1_X: k_gate_g1<G1_X, T><<<blocks, threads, 0, st>>>(a, len, g); break;
                case G1_Y: k_gate_g1<G1_Y, T><<<blocks, threads, 0, st>>>(a, len, g); break;
                case G1_RX: k_gate_g1<G1_RX, T><<<blocks, threads, 0, st>>>(a, len, g); break;
                case G1_RY: k_gate_g1<G1_RY, T><<<blocks, threads, 0, st>>>(a, len, g); break;
                default: k_gate_g1<G1_GEN, T><<<blocks, threads, 0, st>>>(a, len, g); break;
            }
            break;
        case GG_DIAG: k_gate_diag<T><<<blocks, threads, 0, st>>>(a, len, g); break;
        case GG_SWAP: k_gate_swap<T><<<blocks, threads, 0, st>>>(a, len, g); break;
        case GG_U2: k_gate_u2<T><<<blocks, threads, 0, st>>>(a, len, g); break;
        case GG_RESET_ALL: k_reset_all<T><<<blocks, threads, 0, st>>>(a, len); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
cudaError_t launch_gate(double2* a, uint64_t len, const GGate& g, cudaStream_t st) {
    return launch_gate_t<double2>(a, len, g, st);
}
cudaError_t launch_gate_c64(float2* a, uint64_t len, const GGate& g, cudaStream_t st) {
    return launch_gate_t<float2>(a, len, g, st);
}

// Partial-sum grid: fixed per length so that reductions are deterministic.
int reduce_blocks(uint64_t len) { return grid_for(len, 256, 148 * 8); }

cudaError_t launch_norm(const double2* a, uint64_t len, double* partials, double* out, uint32_t* status,
                        cudaStream_t st) {
    const int nb = reduce_blocks(len);
    k_norm_partials<<<nb, 256, 0, st>>>(a, len, partials);
    k_reduce<<<1, 1024, 0, st>>>(partials, nb, out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t launch_p01(const double2* a, uint64_t len, uint32_t q, double* partials, double* out2,
                       const double* norm2, cudaStream_t st) {
    const int nb = reduce_blocks(len);
    k_p01_partials<<<nb, 256, 0, st>>>(a, len, q, partials);
    k_reduce<<<2, 1024, 0, st>>>(partials, nb, out2, norm2, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_expz(const double2* a, uint64_t len, const uint64_t* masks, uint32_t k, double* partials,
                        double* out, const double* norm2, cudaStream_t st) {
    const int nb = reduce_blocks(len);
    Masks8 mk{};
    for (uint32_t j = 0; j < k && j < 8; ++j) mk.m[j] = masks[j];
    k_expz_partials<<<nb, 256, 0, st>>>(a, len, mk, k, partials);
    k_reduce<<<k, 1024, 0, st>>>(partials, nb, out, norm2, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_reduce_div(const double* partials, uint32_t count, uint32_t sets, double* out, const double* divide_by,
                              cudaStream_t st) {
    k_reduce<<<sets, 1024, 0, st>>>(partials, count, out, divide_by, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_reduce_sets(const double* partials, uint32_t count, uint32_t sets, double* out, cudaStream_t st) {
    k_reduce<<<sets, 1024, 0, st>>>(partials, count, out, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_reduce_partials(const double* partials, uint32_t count, double* out, uint32_t* status,
                                   cudaStream_t st) {
    k_reduce<<<1, 1024, 0, st>>>(partials, count, out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t launch_collapse(double2* a, uint64_t len, uint32_t q, uint32_t outcome, double f, double* partials,
                            double* norm2_out, uint32_t* status, cudaStream_t st) {
    const int nb = reduce_blocks(len);
    k_collapse<<<nb, 256, 0, st>>>(a, len, q, outcome, f, partials);
    k_reduce<<<1, 1024, 0, st>>>(partials, nb, norm2_out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t launch_materialize(double2* a, uint64_t len, double* norm2, double* partials, uint32_t* status,
                               cudaStream_t st) {
    const int nb = reduce_blocks(len);
    k_materialize<<<nb, 256, 0, st>>>(a, len, norm2, partials);
    k_reduce<<<1, 1024, 0, st>>>(partials, nb, norm2, nullptr, status);
    return cudaGetLastError();
}

cudaError_t launch_set_scalar(double* p, double v, cudaStream_t st) {
    k_set_scalar<<<1, 1, 0, st>>>(p, v);
    return cudaGetLastError();
}

cudaError_t launch_probs(const double2* a, uint64_t off, uint64_t cnt, const double* norm2, double* out,
                         cudaStream_t st) {
    k_probs<<<grid_for(cnt, 256, 148 * 16), 256, 0, st>>>(a, off, cnt, norm2, out);
    return cudaGetLastError();
}

cudaError_t launch_tree(const void* a, bool f32, uint32_t n, const double* norm2, double* tree, cudaStream_t st) {
    if (n < 2) return cudaSuccess;
    double* leaf = tree + ((1ull << (n - 1)) - 2);
    const int g = grid_for(1ull << (n - 1), 256, 148 * 16);
    if (f32) k_tree_leaf<float2><<<g, 256, 0, st>>>((const float2*)a, n, norm2, leaf);
    else k_tree_leaf<double2><<<g, 256, 0, st>>>((const double2*)a, n, norm2, leaf);
    for (uint32_t k = n - 2; k >= 1; --k) {
        const uint64_t cnt = 1ull << k;
        k_tree_up<<<grid_for(cnt, 256, 148 * 16), 256, 0, st>>>(tree + ((2ull << k) - 2), tree + (cnt - 2), cnt);
    }
    return cudaGetLastError();
}

cudaError_t launch_sample(const void* a, bool f32, uint32_t n, const double* norm2, const double* tree,
                          const double* u, uint64_t shots, int mode, unsigned long long* out, cudaStream_t st) {
    const int g = grid_for(shots, 128, 148 * 16);
    if (f32) k_sample<float2><<<g, 128, 0, st>>>((const float2*)a, n, norm2, tree, u, shots, mode, out);
    else k_sample<double2><<<g, 128, 0, st>>>((const double2*)a, n, norm2, tree, u, shots, mode, out);
    return cudaGetLastError();
}

}  // namespace qoa
