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
#include <stdint.h>
#include <vector_types.h>

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
constexpr int WARP_BITS = 3;
constexpr int HIGH_SLOTS = REG_BITS + WARP_BITS;          // high qubits per pass
constexpr int TILE_BITS = LANE_BITS + HIGH_SLOTS;         // 12 -> 4096 amps, 64 KB
constexpr int PASS_THREADS = 32 << WARP_BITS;              // 256
constexpr int REGS = 1 << REG_BITS;                        // 16 amps per thread
constexpr int MAX_PASS_OPS = 320;
constexpr int MAX_PASS_COEF = 640;                         // double2 coefficients

// Op kinds inside a pass.
enum PassOpKind : uint8_t {
    PK_G1_REG = 0,   // 2x2 on register bit t0
    PK_G1_LANE = 1,  // 2x2 on lane bit t0 (qubit t0 < 5), via shuffles
    PK_DIAG = 2,     // diagonal factor: (sel ? d1 : d0) where the condition holds
    PK_XCHG = 3,     // shared-memory exchange to a new register/warp mapping
};

// 2x2 specialisations (sub field). Coefficients at coef[c..c+3] = m00 m01 m10 m11.
enum G1Sub : uint8_t {
    G1_GEN = 0,  // general complex 2x2
    G1_H = 1,    // (a+b)*f, (a-b)*f with real f = coef[c].x
    G1_X = 2,    // swap
    G1_Y = 3,    // (-i a1, i a0)
    G1_RX = 4,   // [[c, -is], [-is, c]] with c = coef[c].x, s = coef[c].y
    G1_RY = 5,   // [[c, -s], [s, c]]
};

// Location of the selector bit of a PK_DIAG op.
enum SelLoc : uint8_t { SEL_NONE = 0, SEL_REG = 1, SEL_LANE = 2, SEL_WARP = 3, SEL_OUTER = 4 };

// One op of a pass. Conditions: every listed bit must be 1 (control masks of
// CNOT / Toffoli / CY, and the CZ / CPHASE / phase-gate masks).
struct PassOp {
    uint8_t kind;
    uint8_t sub;        // G1Sub, or SelLoc for PK_DIAG
    uint8_t t0;         // register bit / lane bit / selector index
    uint8_t reg_free;   // PK_DIAG: 1 when the factor is constant over a thread's registers
    uint16_t coef;      // index into PassParams::coef
    uint8_t cond_reg;   // register-bit mask
    uint8_t cond_lane;  // lane-bit mask
    uint8_t cond_warp;  // warp-bit mask
    uint8_t xreg[REG_BITS];   // PK_XCHG: slot held by each register bit afterwards
    uint8_t xwarp[WARP_BITS]; // PK_XCHG: slot held by each warp bit afterwards
    uint64_t cond_outer;      // mask over global index bits outside the tile
};

// Everything a pass kernel launch needs, passed by value (__grid_constant__):
// kernel parameters live in the constant bank, so every warp reads the op
// stream with broadcast loads and concurrent launches never share it.
struct PassParams {
    uint32_t n;                  // qubits
    uint32_t nops;
    uint32_t ncoef;
    uint8_t slot_qubit[HIGH_SLOTS];   // global qubit of each high slot
    uint8_t reg_slot0[REG_BITS];      // initial mapping: slot of each register bit
    uint8_t warp_slot0[WARP_BITS];    // initial mapping: slot of each warp bit
    uint8_t outer_qubits[64];         // qubits outside the tile, ascending (n - TILE_BITS of them)
    PassOp ops[MAX_PASS_OPS];
    double2 coef[MAX_PASS_COEF];
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
