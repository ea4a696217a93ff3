// qoa_kernels.cuh — descriptors shared by the host planner (qoa_engine.cpp) and
// the sm_100a kernels (qoa_kernels.cu).
//
// State layout in HBM: 2^n interleaved complex128 amplitudes (double2), index
// bit q <-> qubit q. The stored vector is kept un-normalised between kernels:
// each handle carries a device scalar `norm2` = sum |stored|^2 written by the
// last kernel that produced the vector, and every consumer reads
// logical = stored * rsqrt(norm2). A norm2 that is not above 1e-12 (or NaN)
// means the logical state is |0..0>, which is what QuantumState::normalize
// (src/runtime/quantum_state.rs:888-907) resets to.
#pragma once
#ifndef __CUDACC_RTC__  // NVRTC (run-time pass kernels) gets the integer types from its prelude
#include <stddef.h>
#include <stdint.h>
#include <vector_types.h>
#endif

namespace qoa {

// ---------------------------------------------------------------------------
// Tile pass geometry. A pass kernel CTA owns 2^TILE_BITS amplitudes: the 5
// lowest qubits are the lane bits of every warp (512 contiguous bytes per warp
// access), REG_BITS high qubits live in each thread's registers and WARP_BITS
// high qubits select the warp. Gates on register bits run in registers, gates
// on lane bits through warp shuffles; a warp-bit target needs an exchange
// through shared memory that swaps it into the registers.
// ---------------------------------------------------------------------------
constexpr int LANE_BITS = 5;
constexpr int REG_BITS = 4;
constexpr int WARP_BITS = 2;
constexpr int HIGH_SLOTS = REG_BITS + WARP_BITS;          // high qubits per pass
constexpr int TILE_BITS = LANE_BITS + HIGH_SLOTS;         // 11 -> 2048 amps, 32 KB
constexpr int PASS_THREADS = 32 << WARP_BITS;              // 128
constexpr int REGS = 1 << REG_BITS;                        // 16 amps per thread
constexpr int MAX_PASS_OPS = 640;
constexpr int MAX_PASS_COEF = 768;                         // double2 coefficients
constexpr int MAX_XCHG = 48;
// Angle phases: a phase e^{i theta} whose condition is at most one tile bit
// plus qubits outside the tile is evaluated once per CTA. Angle op a sums
// the theta of its entries angles[ang_start[a] .. ang_start[a+1]) whose
// tile-number mask is satisfied, then applies e^{i sum}.
constexpr int MAX_ANG_OPS = 64;
constexpr int MAX_PASS_ANGLES = 320;
struct PassAngle {
    uint64_t omask;  // bits of the tile number (qubits outside the tile) that must be 1
    double theta;
};

// 2x2 forms. Coefficients at coef[c..]:
//   G1_HF  (a0+a1, a0-a1): the Hadamard with its 1/sqrt2 left to the pass renormalisation
//   G1_X   swap; G1_Y (-i a1, i a0)
//   G1_RX  [[al, -i be], [-i be, al]]  al = coef.x, be = coef.y
//   G1_RY  [[al, -be], [be, al]]
//   G1_GEN general complex 2x2 (coef[c..c+3] = m00 m01 m10 m11)
//   G1_H   exact Hadamard (per-gate kernels only)
enum G1Sub : uint8_t {
    G1_HF = 0, G1_X = 1, G1_Y = 2, G1_RX = 3, G1_RY = 4, G1_GEN = 5, G1_NSUB = 6, G1_H = 7,
    // rotations with the larger of |cos|, |sin| factored out (tile passes):
    //   RXA [[1, -i t], [-i t, 1]]  RXB [[r, -i], [-i, r]]
    //   RYA [[1, -t], [t, 1]]       RYB [[r, -1], [1, r]]     (t or r = coef.x)
    G1_RXA = 8, G1_RXB = 9, G1_RYA = 10, G1_RYB = 11,
};

// Op codes of the pass interpreter (one flat jump table). Register-bit ops
// come in four copies, one per register bit k, so every pair index is a
// compile-time register name.
enum PassCode : uint8_t {
    PC_NOP = 0,
    PC_XCHG = 1,      // shared-memory exchange to mapping `coef`
    PC_FLUSH = 2,     // registers *= per-thread pending factor
    PC_DIAG_T = 3,    // pending factor *= coef[c] where the thread condition holds
    PC_DIAG_M = 4,    // registers with (v & cond_reg) == cond_reg *= coef[c] (thread condition too)
    PC_DIAG_TAB = 5,  // register v *= coef[c + v] (a product of register-only phases)
    PC_DIAG_TM = 6,   // the next k ops are PC_DIAG_T entries: pending factor *= each (one dispatch)
    PC_DIAG_MX = 7,   // the next k ops are PC_DIAG_M entries, applied in one dispatch
    PC_HF = 8,        // +k
    PC_RX = 12,       // +k
    PC_RY = 16,       // +k
    PC_GEN = 20,      // +k
    PC_XC = 24,       // +k: X on register bit k where the conditions hold (CNOT, Toffoli, X)
    PC_YC = 28,       // +k: Y likewise (CY, Y)
    PC_RXB = 32,      // +k (PC_RX carries the A form)
    PC_RYB = 36,      // +k (PC_RY carries the A form)
    PC_DIAG_TA = 40,  // pending factor *= angle phase `coef` where the thread condition holds
    PC_DIAG_MA = 41,  // registers with (v & cond_reg) == cond_reg *= angle phase `coef`
    PC_NCODES = 42,
};

// One op of a pass (16 bytes). The first 32-bit word (code, k, coef) is all
// the interpreter loop reads; the condition words are read only by ops that
// take conditions. Conditions: every listed bit must be 1 (controls of CNOT /
// Toffoli / CY; masks of phase gates, CZ, CPHASE).
// 16-byte aligned: the pass kernels stage the op stream with 16-byte loads.
struct alignas(16) PassOp {
    uint8_t code;
    uint8_t k;          // register bit of the op
    uint16_t coef;      // index into PassParams::coef; PC_XCHG: mapping index
    uint8_t cond_reg;   // register-bit mask
    uint8_t cond_lane;  // lane-bit mask
    uint8_t cond_warp;  // warp-bit mask
    uint8_t has_tp;     // bit 0: any lane / warp / outer condition; bit 1: last entry of a phase run
    uint64_t tmask;     // thread condition over T = lane | warp << 5 | (tile number) << 7
                        // (kernels read the low 32 bits; passes need n <= 36): every set
                        // bit of tmask must be set in the thread's T
};
static_assert(sizeof(PassOp) == 16, "k_pass reads a PassOp as 32/64-bit words");

// A register / lane / warp assignment of the tile's TILE_BITS index bits.
// Tile bit t < 5 is qubit t; tile bit 5 + s is high slot s.
struct TileMap {
    uint8_t lane[LANE_BITS];
    uint8_t reg[REG_BITS];
    uint8_t warp[WARP_BITS];
};

// Everything a pass kernel launch needs, passed by value (__grid_constant__);
// each CTA copies the op stream and coefficients into shared memory once.
struct PassParams {
    uint32_t n;                       // qubits
    uint32_t nops;
    uint32_t ncoef;
    uint32_t pad_;
    double2 phase;                    // global phase of the factored gates of this pass
    uint8_t slot_qubit[HIGH_SLOTS];   // global qubit of each high slot (at load)
    uint8_t out_qubit[TILE_BITS];     // global qubit each tile bit is stored to (SWAPs relabel tile bits)
    uint8_t outer_qubits[64];         // qubits outside the tile, ascending (n - TILE_BITS of them)
    TileMap map0;                     // mapping at load (lanes = tile bits 0..4)
    TileMap xmap[MAX_XCHG];           // mappings after each exchange
    uint16_t nang;                    // angle ops
    uint16_t ang_start[MAX_ANG_OPS + 1];
    PassOp ops[MAX_PASS_OPS];
    double2 coef[MAX_PASS_COEF];
    PassAngle angles[MAX_PASS_ANGLES];
};
static_assert(sizeof(PassParams) <= 32000, "PassParams travels as a kernel parameter (32 KB limit)");

#ifndef __CUDACC_RTC__
static_assert(offsetof(PassParams, ops) % 16 == 0 && offsetof(PassParams, coef) % 16 == 0,
              "the op stream and coefficients are staged with 16-byte loads");
#endif

// One circuit's pass inside an arena launch: its state, the pass's parameters
// (PassParams for complex128, F32PassParams for complex64), and whether this
// is the circuit's first pass (input |0..0>, not read).
struct ArenaJob {
    void* amps;
    const void* params;
    uint32_t fresh;
    uint32_t pad_;
};

// ---------------------------------------------------------------------------
// FP32-fused precision passes (qoa_f32.cu)
// ---------------------------------------------------------------------------
constexpr int MAX_F32_OPS = 256;

struct ExpzMasks {
    uint64_t m[8];
};

struct F32Op {
    uint32_t kind;   // 0 = dense block, 1 = phase group
    uint32_t bmask;  // kind 0: the 5 tile bits the block acts on
    uint32_t index;  // kind 0: matrix index; kind 1: F32PhaseOp index
    uint32_t count;
};

// Multiply by (re, im) where the global index has every bit of `outer` and
// the tile index every bit of `tile`.
struct F32Phase {
    uint64_t outer;
    uint32_t tile;
    uint32_t pad_;
    double re, im;
};

// A phase group (F32Op kind 1). Every phase is e^{i theta}. The part that does
// not depend on the CTA is a host-made table over the 2048 tile indices; the
// CTA-dependent part with at most one tile bit is a list of (outer mask,
// angle) per tile bit t (t = TILE_BITS: no tile bit), summed per CTA; the
// rest (two or more tile bits and an outer condition) is checked per
// amplitude.
struct F32Angle {
    uint64_t outer;
    double theta;
};
struct F32PhaseOp {
    int32_t table;                      // index of a 2048-entry float2 table, or -1
    uint32_t bit_start[TILE_BITS + 2];  // F32Angle ranges per tile bit (and scalar)
    uint32_t multi_start, multi_count;  // F32Phase entries checked per amplitude
};

struct F32PassParams {
    uint32_t n;
    uint32_t nops;
    uint8_t slot_qubit[HIGH_SLOTS];
    uint8_t outer_qubits[64];
    F32Op ops[MAX_F32_OPS];
};

// ---------------------------------------------------------------------------
// Batched small circuits (qoa_batch.cu): whole state in shared memory
// ---------------------------------------------------------------------------
constexpr int SMALL_MAX_F64 = 12;  // 2^12 complex128 = 64 KB
constexpr int SMALL_MAX_F32 = 13;  // 2^13 complex64 = 64 KB

enum SmallKind : uint8_t { SK_G1 = 0, SK_DIAG = 1, SK_SWAP = 2 };

struct SmallOp {
    uint8_t kind;
    uint8_t sub;
    uint8_t t;       // target / selector (255: none)
    uint8_t t2;
    uint32_t cmask;  // condition: every bit set
    double2 m[4];    // SK_G1: m00 m01 m10 m11; SK_DIAG: d0, d1
};

// Arena circuits' <Z_mask>: chunk partial sums, then one CTA per circuit.
constexpr uint32_t EXPZ_CHUNK = 4096;
constexpr uint32_t EXPZ_MAX_MASKS = 255;
struct ExpzJob {
    const void* amps;
    uint32_t n;
    uint32_t mask_start, mask_count;
    uint32_t out_start;
    uint32_t chunk_start;  // first partials-kernel CTA of this circuit
    uint32_t pad_;
    uint64_t part_start;   // first partial (chunks x (mask_count + 1) of them)
};

struct SmallCircuit {
    uint32_t n;
    uint32_t op_start, op_count;
    uint32_t mask_start, mask_count;
    uint32_t out_start;
    void* state_out;  // where the final state is written (circuits that are sampled), else null
};

// A batch circuit sampled after the run (qoa_batch.cu, k_sample_jobs): its
// final state, scratch for its marginal tree (2^n - 2 doubles), and its shots'
// uniforms and outcomes (inverse CDF, one uniform per shot).
struct SampleJob {
    const void* amps;
    double* tree;
    uint32_t n;
    uint32_t shots;
    uint64_t u_start;
    uint64_t out_start;
};

// ---------------------------------------------------------------------------
// Per-gate kernels over global memory (fallback / per-gate mode / shims).
// ---------------------------------------------------------------------------
enum GGKind : uint8_t {
    GG_G1 = 0,        // 2x2 (sub = G1Sub) on target t, condition cmask
    GG_DIAG = 1,      // factor (bit t ? d1 : d0) where (i & cmask) == cmask; t = 64 -> no selector
    GG_SWAP = 2,      // swap bits t and t2 where (i & cmask) == cmask
    GG_U2 = 3,        // 4x4 on (lo = t, hi = t2), basis 2*bit(hi) + bit(lo)
    GG_COLLAPSE = 4,  // keep bit t == outcome (scaled by d0.x), zero the rest
    GG_RESET_ALL = 5, // |0..0>
    GG_SCALE = 6,     // materialise: multiply by the pending scale only
};

// A block of disjoint SWAPs applied as one in-place permutation of the
// amplitudes (k_swapnet): pi maps each qubit to its partner (or itself). The
// tile qubits tq (qubits 0..4 first, then the partners of 0..4) are closed
// under pi; CTA b handles the tile whose outside bits are b deposited into
// oq, together with its partner tile, so every CTA writes only what it read.
struct PermParams {
    uint32_t n;
    uint32_t na;       // tile qubits
    uint8_t tq[16];
    uint8_t oq[48];
    uint8_t pi[64];
    uint8_t src_bit[16];  // tile bit k of an output index reads tile bit src_bit[k] of its source
};

struct GGate {
    uint8_t kind;
    uint8_t sub;
    uint8_t t;
    uint8_t t2;
    uint32_t outcome;
    uint64_t cmask;
    double2 m[16];
};

}  // namespace qoa
