/*
 * qoa_cuda.h — C ABI of the B200 (sm_100a) state-vector engine that replaces the
 * gate-application hot path of the QOA executor.
 *
 * Two layers are exported:
 *
 *  (i)  The handle API (qoa_create ... qoa_last_error). It replaces the amplitude
 *       ownership of `QuantumState` (src/runtime/quantum_state.rs:38-53) and the
 *       per-gate methods that call into src/vectorization.rs. The amplitudes live
 *       in HBM for the lifetime of the handle; gates are submitted as an op list
 *       that uses the reference's opcode numbers (src/instructions.rs:631-830).
 *
 *  (ii) Slice-level shims (qoa_vec_*). One per `pub fn apply_*_vectorized` in
 *       src/vectorization.rs:16-902, with the same argument meaning: the caller
 *       owns a host `&mut [Complex64]` (interleaved re/im f64, `len` complex
 *       elements) that is updated in place. Each call copies host->device,
 *       runs one kernel and copies back, so they exist for line-for-line
 *       compatibility, not speed.
 *
 * Conventions
 *   - Every entry point returns an int status: QOA_OK (0) or a QOA_E_* code.
 *     No C++ exception crosses the ABI.
 *   - Amplitude layout: interleaved {re, im} complex128 (num-complex
 *     `Complex64` is #[repr(C)]), index bit q <-> qubit q (qubit 0 = LSB),
 *     exactly as src/vectorization.rs:920-935 indexes it.
 *   - Each handle owns one CUDA stream. Distinct handles may be used from
 *     distinct threads; one handle must not be used from two threads at once
 *     (the reference's QuantumState is not shared across threads either).
 *   - Gate ops whose qubits are out of range (or equal where they must be
 *     distinct) are skipped, the way QuantumState prints and no-ops them
 *     (e.g. quantum_state.rs:189-195, 318-321); qoa_apply then returns
 *     QOA_E_RANGE after applying every valid op, and qoa_last_error() names
 *     the first skipped op.
 *   - After every gate the reference renormalises (apply_noise -> normalize,
 *     quantum_state.rs:839-907). The engine keeps that contract: the state that
 *     any read observes is normalised, and a state whose squared norm is not
 *     above 1e-12 (or is NaN) is reset to |0...0>, as normalize() does.
 */
#ifndef QOA_CUDA_H
#define QOA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define QOA_OK        0
#define QOA_E_RANGE   1  /* qubit index out of range / equal qubits: op skipped, state untouched */
#define QOA_E_ARG     2  /* null pointer, size mismatch, bad enum value */
#define QOA_E_OPCODE  3  /* opcode not supported by the engine */
#define QOA_E_CUDA    4  /* a CUDA runtime call failed */
#define QOA_E_OOM     5  /* device allocation failed */
#define QOA_E_STATE   6  /* numerical status: NaN/Inf seen (see qoa_status) */
#define QOA_E_NOGPU   7  /* no CUDA device visible */

/* ---- precision -------------------------------------------------------- */
#define QOA_PREC_F64  0  /* complex128 amplitudes: the plain (drop-in) method */
/* complex64 amplitudes: the same fused tile passes as complex128 (pass
 * coefficients built in FP64 on the host, arithmetic in FP32, half the HBM
 * bytes), or with QOA_FLAG_F32_TENSOR gates fused into dense blocks of up to
 * 5 qubits on the tensor cores (3xTF32). Norms, probabilities and sampling
 * stay FP64. Unitary ops only. */
#define QOA_PREC_F32  1

/* ---- handle flags ------------------------------------------------------ */
/* CZ / CPHASE condition mask. The reference's QuantumState passes the raw
 * qubit INDICES into apply_cz_vectorized / apply_controlled_phase_rotation_
 * vectorized, whose parameters are MASKS (quantum_state.rs:338,356-361 ->
 * vectorization.rs:745,788), so the phase lands on every i with
 * (i & (c|t)) == (c|t). With this flag the engine reproduces that; without it
 * the mask is (1<<c)|(1<<t), the physical CZ. */
#define QOA_FLAG_COMPAT_MASK_QUIRK  0x1u
/* One kernel launch per gate (no multi-gate passes). For comparison runs. */
#define QOA_FLAG_PER_GATE           0x2u
/* Record a CUDA event pair around every launch (qoa_launch_times). */
#define QOA_FLAG_PROFILE            0x4u
/* Depolarising noise only on the qubits the gate touched (the reference
 * applies it to every qubit after every gate, quantum_state.rs:872-885). */
#define QOA_FLAG_NOISE_GATE_QUBITS  0x8u
/* complex64 handles: fuse gates into dense <=5-qubit blocks applied on the
 * tensor cores (3xTF32) instead of the default complex64 tile passes; needs
 * n >= 11 */
#define QOA_FLAG_F32_TENSOR         0x10u
/* Plan every op list with the pass scheduler's slot search, whatever the
 * state size (states of 26 or more qubits always plan with it). Results do
 * not depend on it beyond rounding; it exercises the deeper passes that
 * large states run, on states small enough to check against the CPU. */
#define QOA_FLAG_SLOT_SEARCH        0x20u

/* ---- opcodes: the reference byte code numbers (src/instructions.rs) ---- */
#define QOA_OP_APPLYGATE   0x02  /* q[0]=qubit, q[1]= 'H','X','Y','Z','T','S' (execute_arithmetic APPLYGATE) */
#define QOA_OP_QINIT       0x04  /* q[0]=qubit count: state re-created as max(n,1) qubits in |0..0> */
#define QOA_OP_H           0x05
#define QOA_OP_Z           0x06
#define QOA_OP_X           0x07
#define QOA_OP_P           0x08  /* PHASESHIFT(q, angle) */
#define QOA_OP_RESET       0x0A
#define QOA_OP_SWAP        0x0B
#define QOA_OP_CSWAP       0x0C  /* q = {control, t1, t2} */
#define QOA_OP_T           0x0D
#define QOA_OP_S           0x0E
#define QOA_OP_RZ          0x0F
#define QOA_OP_ENTANGLE    0x11  /* = CNOT(q0,q1) */
#define QOA_OP_EBELL       0x12  /* H(q0); CNOT(q0,q1) */
#define QOA_OP_EMULTI      0x13  /* H(first); CNOT(first, q) for the rest (list op) */
#define QOA_OP_ECLUSTER    0x14  /* H on all; CZ on neighbour pairs (list op) */
#define QOA_OP_ESWAP       0x15  /* CNOT(a,c); CNOT(b,d); SWAP(c,d) */
#define QOA_OP_ESWAPM      0x16  /* ESWAP then MEASURE c, MEASURE d */
#define QOA_OP_CNOT        0x17
#define QOA_OP_ECFB        0x19  /* = CNOT(q0,q1) */
#define QOA_OP_EDIST       0x1A  /* no-op (placeholder in the reference) */
#define QOA_OP_MEASB       0x1B  /* q[1] = 'X','Y','Z' basis */
#define QOA_OP_RESETALL    0x1C
#define QOA_OP_SETPHASE    0x1D  /* = PHASESHIFT */
#define QOA_OP_CZ          0x1E
#define QOA_OP_RX          0x22
#define QOA_OP_RY          0x23
#define QOA_OP_PHASE       0x24  /* = PHASESHIFT */
#define QOA_OP_MEASURE     0x32
#define QOA_OP_ROT         0x33  /* q[1] = 'X','Y','Z' axis */
#define QOA_OP_CPHASE      0x35
/* Engine extensions in the opcode range the reference leaves unused
 * (0xF0-0xFE; 0xFF is HALT). Each names the QuantumState method it exposes. */
#define QOA_OP_Y           0xF0  /* apply_y (quantum_state.rs:213) */
#define QOA_OP_U1          0xF1  /* apply_custom_unitary: matrix = 4 complex (8 doubles), row-major */
#define QOA_OP_U2          0xF2  /* apply_two_qubit_unitary(q0,q1): 16 complex (32 doubles) */
#define QOA_OP_TOFFOLI     0xF3  /* apply_toffoli(c1,c2,t) */
#define QOA_OP_CY          0xF4  /* apply_controlled_y(c,t) */

/* One instruction. `nq` operands are in q[0..3]; list ops (EMULTI/ECLUSTER)
 * with more than 4 qubits pass them through `qlist` instead. `matrix` is read
 * only by U1/U2. */
typedef struct qoa_op {
    uint32_t opcode;
    uint32_t nq;
    uint32_t q[4];
    double angle;
    const uint32_t* qlist;
    const double* matrix;
} qoa_op;

typedef struct qoa_state_s* qoa_state_t;

/* Numerical status flags (Status{nan, div_by_zero, overflow},
 * quantum_state.rs:27-35, plus the normalize() reset counter). */
typedef struct qoa_status_t {
    uint32_t nan_seen;
    uint32_t inf_seen;
    uint32_t zero_norm_resets;  /* times normalize() found norm^2 <= 1e-12 and reset to |0..0> */
    uint32_t copy_timeouts;     /* nonzero: a streamed pass gave up waiting (~2 s) for a tile's
                                   copy into shared memory; the state is not valid */
} qoa_status_t;

/* ---- (i) handle API ----------------------------------------------------- */

/* QuantumState::new (quantum_state.rs:56-90): n = max(n,1) qubits in |0..0>. */
int qoa_create(uint32_t n, int precision, uint32_t flags, qoa_state_t* out);
int qoa_destroy(qoa_state_t s);
int qoa_num_qubits(qoa_state_t s, uint32_t* n);
/* apply_reset_all (quantum_state.rs:183-186). */
int qoa_reset_all(qoa_state_t s);
/* The per-gate methods (quantum_state.rs:171-397) and execute_arithmetic's
 * instruction dispatch (quantum_state.rs:460-565), for a list of ops. Work is
 * queued on the handle's stream; MEASURE-type ops synchronise. */
int qoa_apply(qoa_state_t s, const qoa_op* ops, size_t nops);
/* measure (quantum_state.rs:399-458) with a caller-supplied uniform u in
 * [0,1): outcome = (u < P0) ? 0 : 1. A negative u draws from the handle's
 * counter-based RNG (qoa_seed). complex128 handles only (the complex64 form
 * takes unitary ops; sample it with qoa_sample). */
int qoa_measure(qoa_state_t s, uint32_t q, double u, uint32_t* outcome);
/* Shots. mode 0 = measure_all order (quantum_state.rs:909-918): qubits 0..n-1
 * measured one after another, n uniforms per shot (u[shot*n + q]); mode 1 =
 * inverse-CDF over the full distribution, one uniform per shot. out[shot]
 * holds the outcome bits (bit q = qubit q). The state is left unchanged, as
 * measure_all measures a clone. */
int qoa_sample(qoa_state_t s, const double* u, size_t shots, int mode, uint64_t* out);
/* get_probabilities (quantum_state.rs:128-133): 2^n doubles. */
int qoa_probabilities(qoa_state_t s, double* out);
/* <Z_mask> = sum_i (-1)^popcount(i & mask) |a_i|^2 for k masks (FP64 sums,
 * either precision). */
int qoa_expect_z(qoa_state_t s, const uint64_t* masks, size_t k, double* out);
/* get_state_vector / set_state_vector (quantum_state.rs:1129-1145); set
 * renormalises. bytes must be 2^n * 16 (complex128), or 2^n * 8 (complex64)
 * for a QOA_PREC_F32 handle. */
int qoa_get_state(qoa_state_t s, void* host, size_t bytes);
int qoa_set_state(qoa_state_t s, const void* host, size_t bytes);
/* No reference counterpart: a seeded Gaussian state (re, im of every
 * amplitude i.i.d. N(0,1), Philox4x32-10 + Box-Muller), normalised. Handles of
 * either precision seeded alike hold the same state (complex64 = rounded). */
int qoa_set_random_state(qoa_state_t s, uint64_t seed);
/* No reference counterpart: relative L2 distance and 1 - |<a|b>|^2 of the
 * normalised states of two handles of equal size (either precision). */
int qoa_compare(qoa_state_t a, qoa_state_t b, double* rel_l2, double* infidelity);
/* seed_rng (quantum_state.rs:956): seeds the handle's Philox4x32-10 stream. */
int qoa_seed(qoa_state_t s, uint64_t seed);
/* NoiseConfig (quantum_state.rs:15-24): mode 0 Ideal, 1 Fixed(p), 2 Random;
 * mode 3 = no config at all (the Option's None, a fresh handle's state: no
 * noise, like Ideal, but saved as null in the JSON checkpoint). */
int qoa_set_noise(qoa_state_t s, int mode, double p);
/* Selects the Philox stream of the noise and MEASURE draws (one per Pauli
 * trajectory) and restarts its event counter. No reference counterpart: the
 * reference's StdRng stream is not addressable (quantum_state.rs:76). */
int qoa_set_trajectory(qoa_state_t s, uint64_t trajectory);
int qoa_status(qoa_state_t s, qoa_status_t* out);
/* Blocks until the handle's queued work is done. */
int qoa_sync(qoa_state_t s);
/* The handle's cudaStream_t, so a caller can order its own work against it. */
int qoa_stream(qoa_state_t s, void** stream);
/* Kernel launches issued by this handle since creation. */
int qoa_launch_count(qoa_state_t s, uint64_t* count);
/* With QOA_FLAG_PROFILE: per-launch device times (ms) and algorithmic bytes of
 * the launches since the last call; returns the count in *n (<= cap). */
int qoa_launch_times(qoa_state_t s, double* ms, double* bytes, int* kind, size_t cap, size_t* n);
const char* qoa_last_error(qoa_state_t s);
const char* qoa_strerror(int code);

/* ---- batching form (no reference counterpart) ---------------------------- */
/* Many circuits run together: circuits of up to tune.small_max_n qubits (at
 * most 12 for complex128, 13 for complex64) run whole-state in shared memory
 * in one persistent launch; larger ones run as tile passes on views into one
 * packed arena, spread over tune.streams streams. The first qoa_batch_run
 * launches eagerly; the second captures the whole batch into a CUDA graph and
 * launches it; later runs replay the graph. Results: <Z_mask> of each circuit's final state for the masks
 * given at qoa_batch_add, in order of addition. Unitary ops only. */
typedef struct qoa_batch_s* qoa_batch_t;
typedef struct qoa_batch_tuning {
    uint32_t small_max_n;       /* shared-memory kernel up to this many qubits */
    uint32_t small_threads;     /* threads per CTA of that kernel (multiple of 32) */
    uint32_t small_ctas_per_sm; /* its persistent grid = SMs x this */
    uint32_t streams;           /* streams the larger circuits spread over */
    uint32_t pass_gate_budget;  /* max gates per tile pass (fusion width); 0 = default */
    uint32_t f32_tensor;        /* complex64 batches: 1 = dense tensor-core blocks, 0 = tile passes */
    uint32_t jit;               /* tile passes as generated kernels, one per pass structure:
                                   QOA_JIT_OFF, QOA_JIT_ASYNC (default: compiled in the background,
                                   the graph is captured again once they are loaded), QOA_JIT_SYNC */
} qoa_batch_tuning;
int qoa_batch_create(int precision, uint32_t flags, qoa_batch_t* out);
int qoa_batch_add(qoa_batch_t b, uint32_t n, const qoa_op* ops, size_t nops, const uint64_t* zmasks, size_t nmasks,
                  uint32_t* id);
int qoa_batch_set_tuning(qoa_batch_t b, const qoa_batch_tuning* t);
int qoa_batch_get_tuning(qoa_batch_t b, qoa_batch_tuning* t);
int qoa_batch_run(qoa_batch_t b);
/* Replays the captured graph on the batch's stream without waiting. */
int qoa_batch_launch(qoa_batch_t b);
/* The stream the batch runs on (its graph launches and joins there). */
int qoa_batch_stream(qoa_batch_t b, void** stream);
int qoa_batch_results(qoa_batch_t b, double* out, size_t count);
int qoa_batch_info(qoa_batch_t b, uint32_t* circuits, uint32_t* small, uint32_t* large, uint32_t* graph_ready);
/* Generated arena kernels: distinct pass structures, how many are loaded,
 * and whether the captured graph launches them (1) or the interpreter (0). */
int qoa_batch_jit_info(qoa_batch_t b, uint32_t* structures, uint32_t* ready, uint32_t* graph_uses);
/* Algorithmic bytes of one run's arena tile passes (each pass reads and
 * writes its circuit's state once) and the number of pass rounds. */
int qoa_batch_traffic(qoa_batch_t b, double* arena_pass_bytes, uint32_t* rounds);
/* Trajectory `trajectory` of a noisy circuit as a batch circuit, sampled
 * after the run: the ops expanded with the depolarising draws that qoa_apply
 * makes on a state given qoa_seed(seed), qoa_set_noise(1, noise_p) and
 * qoa_set_trajectory(trajectory) (noise_p = 0: none), then `shots` outcomes
 * of the final state by the inverse-CDF rule of qoa_sample mode 1, one
 * uniform each from u. Unitary ops only (QOA_E_OPCODE otherwise). Returns
 * QOA_E_RANGE, with the circuit added, where qoa_apply would skip an op. The
 * serving form runs a request's trajectories this way. */
int qoa_batch_add_trajectory(qoa_batch_t b, uint32_t n, const qoa_op* ops, size_t nops, uint64_t seed,
                             double noise_p, uint64_t trajectory, const double* u, uint32_t shots, uint32_t* id);
/* The outcomes of circuit id (count = its shots) after qoa_batch_run. */
int qoa_batch_shots(qoa_batch_t b, uint32_t id, uint64_t* out, size_t count);
/* Empties a batch for reuse: its circuits and device buffers go, its streams
 * and tuning stay. */
int qoa_batch_reset(qoa_batch_t b);
/* Host threads that plan the batch's circuits (0, the default: all cores). */
int qoa_batch_set_host_threads(qoa_batch_t b, uint32_t threads);
/* *unitary = 1 when every op expands to unitary gates (no measurement,
 * reset or QINIT), i.e. the ops can run as batch circuits. */
int qoa_ops_unitary(uint32_t n, uint32_t flags, const qoa_op* ops, size_t nops, int* unitary);
const char* qoa_batch_last_error(qoa_batch_t b);
int qoa_batch_destroy(qoa_batch_t b);

/* ---- serving form (no reference counterpart) ----------------------------- */
/* A request loop with continuous batching. Each request is a circuit with
 * depolarising noise p per gate (QuantumState::apply_noise semantics,
 * quantum_state.rs:839-885) run as `trajectories` stochastic Pauli
 * trajectories of `shots_per_trajectory` inverse-CDF shots each. Trajectory t
 * of a request with seed s draws its noise from counter-based stream t and
 * its shot uniforms from stream t ^ 0x73686f74, so its result does not depend
 * on scheduling or on the other requests. Worker threads (one trajectory each,
 * one stream each) take the next trajectory of the oldest admitted request; a
 * request is admitted when a worker is free and its state fits the HBM budget
 * beside the states in use. States stay resident for reuse. With precision
 * QOA_PREC_F32 and QOA_FLAG_F32_TENSOR, requests under 11 qubits run in
 * complex128. */
typedef struct qoa_server_s* qoa_server_t;
typedef struct qoa_server_config {
    int precision;             /* QOA_PREC_F64 / QOA_PREC_F32 */
    uint32_t flags;            /* handle flags (QOA_FLAG_COMPAT_MASK_QUIRK, ...) */
    uint64_t hbm_budget_bytes; /* states + sampling scratch held at once */
    uint32_t workers;          /* host threads = trajectories in flight */
} qoa_server_config;
typedef struct qoa_request {
    uint32_t n;
    const qoa_op* ops;         /* copied at submission */
    size_t nops;
    double noise_p;            /* depolarising probability per qubit per gate; 0 = ideal */
    uint32_t trajectories;
    uint32_t shots_per_trajectory;
    uint64_t seed;
} qoa_request;
typedef struct qoa_request_result {
    uint64_t id;
    int status;                /* QOA_OK or the first error of its trajectories */
    uint32_t n;
    int precision;             /* precision it ran in */
    double t_submit, t_admit, t_start, t_done; /* seconds on the server's clock */
    uint64_t shots;            /* trajectories x shots_per_trajectory */
} qoa_request_result;
typedef struct qoa_server_stats {
    uint64_t submitted, done, queued, admitted, trajectories_running, states_resident;
    uint64_t bytes_reserved, peak_bytes_reserved;
    uint64_t trajectories_batched;  /* trajectories that ran in batch chunks */
} qoa_server_stats;
int qoa_server_create(const qoa_server_config* cfg, qoa_server_t* out);
int qoa_server_submit(qoa_server_t s, const qoa_request* req, uint64_t* id);
/* Finished requests (up to cap); waits up to timeout_ms (<0: forever) for one. */
int qoa_server_poll(qoa_server_t s, qoa_request_result* out, size_t cap, size_t* got, int timeout_ms);
/* Outcomes of a finished request in (trajectory, shot) order; releases them. */
int qoa_server_take_shots(qoa_server_t s, uint64_t id, uint64_t* out, size_t cap);
int qoa_server_get_stats(qoa_server_t s, qoa_server_stats* out);
double qoa_server_now(qoa_server_t s);
/* Waits for every submitted request, then stops the workers. */
int qoa_server_destroy(qoa_server_t s);

/* The engine's counter-based uniform in [0,1): Philox4x32-10 keyed by seed,
 * counter (event lo, event hi, slot, stream); noise draws of trajectory t use
 * stream t, slots 2q+1 (hit test) and 2q+2 (Pauli type) of gate event e. */
double qoa_philox_uniform(uint64_t seed, uint32_t stream, uint64_t event, uint32_t slot);
/* The hit tests of gate event `event` on trajectory `stream`: bit q (q < n <=
 * 64) set where qoa_philox_uniform(seed, stream, event, 2q + 1) < p, i.e.
 * the qubits that receive a Pauli (its type: slot 2q + 2, < 1/3 X, < 2/3 Y,
 * else Z). */
uint64_t qoa_noise_hits(uint64_t seed, uint32_t stream, uint64_t event, uint32_t n, double p);

/* ---- bytecode front-end: .qexe / .qx programs -------------------------- */
/* File = 4-byte magic ("QEXE","OEXE","QOX ","XEXE","QEX ","QX\0\0"), version
 * byte, u32 LE payload length, payload (parse_exe_file, main.rs:1711-1745). */
typedef struct qoa_exe_info {
    char kind[8];              /* "qexe", "oexe", "qox", "xexe", "qex", "qx" */
    uint32_t version;
    uint32_t inferred_qubits;  /* `qoa run`'s qubit count: largest qubit byte + 1 (main.rs:3844-4226) */
    uint64_t payload_offset;
    uint64_t payload_len;
} qoa_exe_info;
typedef struct qoa_exe_result {
    uint64_t instructions;     /* executed */
    uint64_t gates;            /* quantum ops sent to the engine */
    uint64_t measurements;
    uint64_t chars_out;        /* CHAROUT */
    uint64_t range_errors;     /* ops skipped for out-of-range qubits (printed, ignored upstream) */
    uint64_t loop_errors;      /* LOOPEND without a pushed LOOPSTART */
    uint64_t unknown_opcodes;  /* advanced by one byte, as upstream */
    uint64_t unsupported;      /* QGATE names / rotation axes the executor skips */
    uint32_t halted;           /* HALT or EXITCODE reached */
    int32_t exit_code;
    double registers[24];
} qoa_exe_result;
#define QOA_EXE_LOOPS 0x1      /* LOOPSTART n pushes n iterations (upstream pushes none) */
/* Header + qubit-count scan; host only. */
int qoa_exe_parse(const uint8_t* file, size_t len, qoa_exe_info* info);
/* Runs a program on a complex128 handle (run_exe, main.rs:2314-3722); quantum
 * instructions are batched into qoa_apply calls between measurements. Printed
 * text (PRINT / PRINTLN / PRINTF / CHAROUT / DUMPREGS) goes to out_text
 * (NUL-terminated, truncated to out_cap; *out_len = full length). max_steps
 * bounds executed instructions (0 = none). */
int qoa_exe_run(qoa_state_t s, const uint8_t* file, size_t len, uint32_t flags, uint64_t max_steps,
                qoa_exe_result* res, char* out_text, size_t out_cap, size_t* out_len);
/* The same interpreter without a state (host only): the op list a run would
 * send, with every measurement outcome taken as 0. */
int qoa_exe_trace(const uint8_t* file, size_t len, uint32_t flags, uint64_t max_steps, qoa_op* ops, size_t cap,
                  size_t* nops, qoa_exe_result* res, char* out_text, size_t out_cap, size_t* out_len);

/* ---- checkpoint I/O ------------------------------------------------------- */
/* Binary: the stored amplitudes and norm2 exactly ("QOAS" version 2,
 * checksummed), any size or precision, with the handle's generator state
 * (seed, noise trajectory and draw counters, measurement draws), noise
 * configuration and status words, so that a loaded handle continues the same
 * trajectory; a save/load round trip is bit-exact. Version-1 files (amplitudes
 * and norm2 only) still load, with a fresh handle's generator state. */
int qoa_state_save(qoa_state_t s, const char* path);
int qoa_state_load(const char* path, uint32_t flags, qoa_state_t* out);
/* JSON in the reference's --save-state / --load-state layout: serde_json of
 * (QuantumState, Vec<f64> registers) (main.rs:3800-3830, 4290-4300); up to
 * 26 qubits. Loading makes a complex128 handle with the file's noise config
 * and returns the registers. */
int qoa_state_save_json(qoa_state_t s, const double* regs, size_t nregs, const char* path);
int qoa_state_load_json(const char* path, uint32_t flags, qoa_state_t* out, double* regs, size_t regs_cap,
                        size_t* nregs);
int qoa_get_noise(qoa_state_t s, int* mode, double* p);
int qoa_get_precision(qoa_state_t s, int* precision);

/* ---- plan introspection (host only, no GPU needed) ---------------------- */
/* Runs the pass scheduler on an op list for an n-qubit state and writes, for
 * each expanded gate in submission order, the index of the pass that applies
 * it (pass_of[i]) and the order within the pass (order[i]); *npasses receives
 * the pass count and *ngates the expanded gate count (<= cap). */
/* Plans with the scheduler's slot search at any size (states of 26 or more
 * qubits always plan with it); for tests of the plans. */
#define QOA_PLAN_SLOT_SEARCH 0x100u
int qoa_plan(uint32_t n, uint32_t flags, const qoa_op* ops, size_t nops, size_t cap,
             int32_t* pass_of, int32_t* order, int32_t* gate_kind, uint32_t* gate_qubits,
             double* gate_matrix, size_t* ngates, size_t* npasses);

/* ---- generated pass kernels ------------------------------------------------ */
/* No counterpart in the reference (its gates are fixed shaders / CPU loops).
 * A complex128 tile pass can run as the interpreter kernel (k_pass, which
 * reads the pass's op stream) or as a kernel generated for that pass: CUDA
 * C++ with every register bit, condition and exchange address a literal,
 * compiled at run time by NVRTC for sm_100a. Coefficients stay parameters, so
 * one compiled kernel serves every pass of the same structure (repeated
 * circuits, angle sweeps); compiled kernels are cached for the process.
 * complex128 and complex64 (non-tensor) handles both have the form.
 * Results are identical either way. Per handle:
 *   QOA_JIT_OFF    interpret every pass
 *   QOA_JIT_ASYNC  (default) a pass structure seen for the second time is
 *                  compiled on background threads; passes interpret until
 *                  their kernel is ready (one-off structures, such as a
 *                  noisy trajectory's Pauli draws, are never compiled)
 *   QOA_JIT_SYNC   compile before the first launch
 * States below min_qubits (default 20) always interpret. At most 8192
 * kernels are loaded per process (environment QOA_JIT_MAX_KERNELS); further
 * structures interpret. */
#define QOA_JIT_OFF   0
#define QOA_JIT_ASYNC 1
#define QOA_JIT_SYNC  2
int qoa_set_jit(qoa_state_t s, int mode, uint32_t min_qubits);
/* Blocks until every compile requested so far has finished. */
int qoa_jit_wait(void);
typedef struct qoa_jit_stats {
    uint64_t kernels;    /* compiled pass kernels in the process cache */
    uint64_t hits;       /* pass requests served from the cache */
    uint64_t misses;     /* pass requests that were compiled */
    uint64_t failures;   /* kernels whose compile or load failed (see qoa_last_error(NULL)) */
    uint64_t launches;   /* generated-kernel passes run by this handle (0 when s is NULL) */
    double compile_ms;   /* total compile + load time */
} qoa_jit_stats;
int qoa_jit_stats_get(qoa_state_t s, qoa_jit_stats* out);
/* Host only, no GPU needed: plans an op list for an n-qubit state of the
 * given precision (QOA_PREC_F64 / QOA_PREC_F32 tile passes) and writes the
 * generated source of each pass's kernel (concatenated, NUL terminated,
 * truncated to cap; *len = full length) and the pass count. compile bit 0:
 * also compile it with NVRTC (nothing is loaded; QOA_E_ARG and the compiler
 * log when it does not compile); bit 1: the batch (arena) form of each
 * kernel instead of the single-state form. */
int qoa_jit_translate(uint32_t n, int precision, uint32_t flags, const qoa_op* ops, size_t nops, int compile,
                      char* out, size_t cap, size_t* len, size_t* npasses);

/* ---- allocation-free entry point ----------------------------------------- */
/* No counterpart in the reference. <Z_mask> = sum_i (-1)^popcount(i & mask)
 * |a_i|^2 over a state vector the CALLER owns in device memory (`d_amps`,
 * `len` interleaved complex128 values, used as given, not renormalised), for
 * k <= QOA_NOALLOC_MAX_MASKS masks; the k results go to the caller's device
 * array `d_out`. Work is queued on the caller's cudaStream_t `stream` (NULL =
 * legacy default stream) and the call returns without waiting.
 * It calls no cudaMalloc, cudaFree or other allocating routine, for callers
 * that cannot allow one: a host runtime that owns and accounts for every
 * device buffer itself, or a latency-critical caller that cannot accept
 * cudaMalloc's implicit synchronisation. Its scratch is one fixed static
 * device array of 75,776 bytes that every device loading the library holds
 * until exit. The first call in each CUDA context (a device's primary
 * context, or one the caller made with cuCtxCreate) resolves that array's
 * address in that context (cudaGetSymbolAddress); make that first call before
 * any stream capture. All calls share the array, so calls that overlap on the
 * GPU race: order them. More than QOA_NOALLOC_MAX_MASKS masks -> QOA_E_ARG
 * (see qoa_last_error(NULL)); a failed launch of its own -> QOA_E_CUDA (an
 * error left pending by earlier work of the caller is neither reported nor
 * cleared). */
#define QOA_NOALLOC_MAX_MASKS 8
int qoa_expect_z_noalloc(const void* d_amps, size_t len, const uint64_t* masks, size_t k, double* d_out,
                         void* stream);

/* ---- (ii) slice-level shims: src/vectorization.rs pub fns ---------------- */
/* `amps` points to `len` interleaved complex128 values in host memory. */
int qoa_vec_apply_hadamard(double* amps, size_t len, double norm_re, double norm_im, size_t mask_bit); /* vectorization.rs:16 */
int qoa_vec_apply_x(double* amps, size_t len, size_t mask_bit);                                         /* vectorization.rs:69 */
int qoa_vec_apply_y(double* amps, size_t len, size_t mask_bit);                                         /* vectorization.rs:118 */
int qoa_vec_apply_z(double* amps, size_t len, size_t mask_bit);                                         /* vectorization.rs:173 */
int qoa_vec_apply_t(double* amps, size_t len, size_t mask_bit);                                         /* vectorization.rs:217 */
int qoa_vec_apply_s(double* amps, size_t len, size_t mask_bit);                                         /* vectorization.rs:262 */
int qoa_vec_apply_phaseshift(double* amps, size_t len, size_t mask_bit, double angle);                  /* vectorization.rs:307 */
int qoa_vec_apply_reset(double* amps, size_t len, size_t mask_bit);                                     /* vectorization.rs:352 */
int qoa_vec_apply_swap(double* amps, size_t len, size_t q1, size_t q2);                                 /* vectorization.rs:421 */
int qoa_vec_apply_controlled_swap(double* amps, size_t len, size_t control, size_t target1, size_t target2); /* vectorization.rs:469 */
int qoa_vec_apply_rx(double* amps, size_t len, size_t mask_bit, double angle);                          /* vectorization.rs:528 */
int qoa_vec_apply_ry(double* amps, size_t len, size_t mask_bit, double angle);                          /* vectorization.rs:588 */
int qoa_vec_apply_rz(double* amps, size_t len, size_t mask_bit, double angle);                          /* vectorization.rs:648 */
int qoa_vec_apply_cnot(double* amps, size_t len, size_t control, size_t target);                        /* vectorization.rs:699 */
int qoa_vec_apply_cz(double* amps, size_t len, size_t control_mask, size_t target_mask);                /* vectorization.rs:745 */
int qoa_vec_apply_controlled_phase_rotation(double* amps, size_t len, size_t control_mask,
                                            size_t target_mask, double angle);                          /* vectorization.rs:788 */
int qoa_vec_apply_reset_all(double* amps, size_t len);                                                  /* vectorization.rs:857 */

#ifdef __cplusplus
}
#endif
#endif /* QOA_CUDA_H */
