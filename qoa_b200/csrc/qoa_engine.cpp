// qoa_engine.cpp — host side of the engine: the C ABI of include/qoa_cuda.h,
// instruction expansion with QuantumState's semantics, the pass scheduler that
// groups gates into single-sweep tile passes, and the vectorization.rs shims.
//
// Reference correspondence (paths inside planetryan/qoa):
//   QuantumState gate methods      src/runtime/quantum_state.rs:171-397
//   execute_arithmetic dispatch    src/runtime/quantum_state.rs:460-705
//   measure / measure_all          src/runtime/quantum_state.rs:399-458, 909-918
//   apply_noise / normalize        src/runtime/quantum_state.rs:839-907
//   matrix set-up per gate         src/vectorization.rs:16-902
#include <cuda_runtime.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <algorithm>
#include <memory>
#include <deque>
#include <thread>
#include <functional>
#include <atomic>
#include <unordered_map>
#include <complex>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <array>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qoa_cuda.h"
#include "qoa_kernels.cuh"
#include "qoa_jit.h"

namespace qoa {
cudaError_t launch_pass(double2* amps, const PassParams& P, const double* norm2_in, double* partials, cudaStream_t st);
cudaError_t launch_gate(double2* a, uint64_t len, const GGate& g, cudaStream_t st);
cudaError_t launch_swapnet(void* a, bool c64, const PermParams& P, cudaStream_t st);
int reduce_blocks(uint64_t len);
cudaError_t launch_norm(const double2* a, uint64_t len, double* partials, double* out, uint32_t* status, cudaStream_t st);
cudaError_t launch_p01(const double2* a, uint64_t len, uint32_t q, double* partials, double* out2, const double* norm2,
                       cudaStream_t st);
cudaError_t launch_expz(const double2* a, uint64_t len, const uint64_t* masks, uint32_t k, double* partials, double* out,
                        const double* norm2, cudaStream_t st);
cudaError_t launch_reduce_partials(const double* partials, uint32_t count, double* out, uint32_t* status, cudaStream_t st);
cudaError_t launch_collapse(double2* a, uint64_t len, uint32_t q, uint32_t outcome, double f, double* partials,
                            double* norm2_out, uint32_t* status, cudaStream_t st);
cudaError_t launch_materialize(double2* a, uint64_t len, double* norm2, double* partials, uint32_t* status, cudaStream_t st);
cudaError_t launch_set_scalar(double* p, double v, cudaStream_t st);
cudaError_t launch_probs(const double2* a, uint64_t off, uint64_t cnt, const double* norm2, double* out, cudaStream_t st);
cudaError_t launch_tree(const void* a, bool f32, uint32_t n, const double* norm2, double* tree, cudaStream_t st);
cudaError_t launch_sample(const void* a, bool f32, uint32_t n, const double* norm2, const double* tree,
                          const double* u, uint64_t shots, int mode, unsigned long long* out, cudaStream_t st);
cudaError_t launch_f32_pass(float2* amps, const F32PassParams& P, const float* mats, const F32PhaseOp* pops,
                            const F32Angle* angles, const F32Phase* phases, const float2* tables,
                            const double* norm2_in, double* partials, uint32_t* status, cudaStream_t st);
cudaError_t launch_f32_reset(float2* a, uint64_t len, cudaStream_t st);
cudaError_t launch_f32_norm(const float2* a, uint64_t len, double* partials, double* out, uint32_t* status,
                            cudaStream_t st);
cudaError_t launch_f32_materialize(float2* a, uint64_t len, double* norm2, double* partials, uint32_t* status,
                                   cudaStream_t st);
cudaError_t launch_f32_probs(const float2* a, uint64_t off, uint64_t cnt, const double* norm2, double* out,
                             cudaStream_t st);
cudaError_t launch_random_state(void* a, bool f32, uint64_t len, uint64_t seed, cudaStream_t st);
cudaError_t launch_f32_expz(const float2* a, uint64_t len, const uint64_t* masks, uint32_t k, double* partials,
                            double* out, const double* norm2, cudaStream_t st);
cudaError_t launch_pass_p32(float2* amps, const PassParams& P, const double* norm2_in, double* partials,
                            cudaStream_t st);
cudaError_t launch_pass_p32_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                                  int max_nops, int max_ncoef, cudaStream_t st);
cudaError_t launch_gate_c64(float2* a, uint64_t len, const GGate& g, cudaStream_t st);
cudaError_t launch_pass_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                              int max_nops, int max_ncoef, cudaStream_t st);
cudaError_t launch_f32_pass_arena(const ArenaJob* jobs, uint32_t njobs, const uint32_t* tile_start, uint32_t tiles,
                                  const float* mats, const F32PhaseOp* pops, const F32Angle* angles,
                                  const F32Phase* phases, const float2* tables, uint32_t* status, cudaStream_t st);
cudaError_t launch_arena_expz(bool f32, const ExpzJob* jobs, uint32_t njobs, uint32_t chunks, const uint64_t* masks,
                              double* partials, double* out, cudaStream_t st);
cudaError_t launch_sample_jobs(bool f32, const SampleJob* jobs, uint32_t njobs, const double* u,
                               unsigned long long* out, cudaStream_t st);
cudaError_t launch_small_batch(bool f32, const SmallCircuit* circs, uint32_t count, const SmallOp* ops,
                               const uint64_t* masks, double* out, unsigned int* counter, int max_n, int threads,
                               int ctas_per_sm, cudaStream_t st);
cudaError_t launch_compare(const void* a, bool af32, const void* b, bool bf32, uint64_t len, const double* na,
                           const double* nb, double* partials, double* out3, cudaStream_t st);
}  // namespace qoa

using namespace qoa;

namespace {
std::mutex g_err_mu;
std::string g_err;  // errors before a handle exists
}  // namespace

namespace qoa {
// Records an error for qoa_last_error(NULL) (entry points without a handle).
void note_global_error(const char* msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
}
}  // namespace qoa

namespace {

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). Draw (seed; stream,
// event, slot) -> uniform double in [0,1) from the top 53 bits of words 0-1.
void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
double uniform01(uint64_t seed, uint64_t stream, uint64_t event, uint32_t slot) {
    uint32_t c[4] = {(uint32_t)event, (uint32_t)(event >> 32), slot, (uint32_t)stream};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t bits = ((uint64_t)c[0] << 32) | c[1];
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}
const uint64_t kMeasStreamXor = 0x6d656173ull;

// The hit tests of one gate event: bit q of the result is set when
// uniform01(seed, stream, event, 2q + 1) < p, for q < n (n <= 64). The same
// draws as one uniform01 call per qubit, computed W counters at a time
// in structure-of-arrays form so that the rounds vectorise (AVX-512 or AVX2
// where the host has it: a noisy circuit draws one uniform per qubit per
// gate).
template <int W>
inline uint64_t hits8(uint32_t k0, uint32_t k1, uint32_t e0, uint32_t e1, uint32_t st, uint32_t q0, uint32_t n,
                      double p) {
    uint32_t c0[W], c1[W], c2[W], c3[W];
    for (int i = 0; i < W; ++i) {
        c0[i] = e0;
        c1[i] = e1;
        c2[i] = 2u * (q0 + (uint32_t)i) + 1u;
        c3[i] = st;
    }
    for (int r = 0; r < 10; ++r) {
        for (int i = 0; i < W; ++i) {
            const uint64_t p0 = (uint64_t)0xD2511F53u * c0[i];
            const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2[i];
            const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1[i] ^ k0;
            const uint32_t n1 = (uint32_t)p1;
            const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3[i] ^ k1;
            const uint32_t n3 = (uint32_t)p0;
            c0[i] = n0; c1[i] = n1; c2[i] = n2; c3[i] = n3;
        }
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    uint64_t h = 0;
    for (int i = 0; i < W; ++i) {
        const uint64_t bits = ((uint64_t)c0[i] << 32) | c1[i];
        const double r = (double)(bits >> 11) * (1.0 / 9007199254740992.0);
        if (q0 + (uint32_t)i < n && r < p) h |= 1ull << (q0 + (uint32_t)i);
    }
    return h;
}
uint64_t noise_hits_generic(uint64_t seed, uint64_t stream, uint64_t event, uint32_t n, double p) {
    uint64_t h = 0;
    for (uint32_t q0 = 0; q0 < n; q0 += 8)
        h |= hits8<8>((uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)event, (uint32_t)(event >> 32),
                      (uint32_t)stream, q0, n, p);
    return h;
}
#if defined(__x86_64__) && defined(__GNUC__)
__attribute__((target("avx2"))) uint64_t noise_hits_avx2(uint64_t seed, uint64_t stream, uint64_t event, uint32_t n,
                                                         double p) {
    uint64_t h = 0;
    for (uint32_t q0 = 0; q0 < n; q0 += 8)
        h |= hits8<8>((uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)event, (uint32_t)(event >> 32),
                      (uint32_t)stream, q0, n, p);
    return h;
}
// Sixteen counters per 512-bit register, one 32-bit word of each: a round's
// 32 x 32 -> 64-bit products come from two even-lane multiplies (the odd
// lanes shifted down), their high and low words blended back into lanes.
// The hit test compares the 53-bit mantissa source m = (w0:w1) >> 11 with
// U = ceil(p * 2^53) as the pair (w0, w1 >> 11) against (U >> 21, U mod
// 2^21): m * 2^-53 < p exactly when m < U, for an integer m.
__attribute__((target("avx512f"))) inline __m512i philox_hi(__m512i a, __m512i m) {
    const __m512i ev = _mm512_mul_epu32(a, m);
    const __m512i od = _mm512_mul_epu32(_mm512_srli_epi64(a, 32), m);
    return _mm512_mask_blend_epi32((__mmask16)0xAAAA, _mm512_srli_epi64(ev, 32), od);
}
__attribute__((target("avx512f"))) inline __m512i philox_lo(__m512i a, __m512i m) {
    return _mm512_mullo_epi32(a, m);
}
__attribute__((target("avx512f"))) uint64_t noise_hits_avx512(uint64_t seed, uint64_t stream, uint64_t event,
                                                              uint32_t n, double p) {
    const double T = std::ceil(p * 9007199254740992.0);  // 2^53
    if (!(T > 0.0)) return 0;
    const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1);
    if (T >= 9007199254740992.0) return all;  // p >= 1: every draw hits
    const uint64_t U = (uint64_t)T;
    const __m512i uh = _mm512_set1_epi32((int)(uint32_t)(U >> 21));
    const __m512i ul = _mm512_set1_epi32((int)(uint32_t)(U & ((1u << 21) - 1)));
    const __m512i M0 = _mm512_set1_epi32((int)0xD2511F53u), M1 = _mm512_set1_epi32((int)0xCD9E8D57u);
    const __m512i lane = _mm512_set_epi32(15, 14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 0);
    uint64_t h = 0;
    for (uint32_t q0 = 0; q0 < n; q0 += 16) {
        __m512i c0 = _mm512_set1_epi32((int)(uint32_t)event);
        __m512i c1 = _mm512_set1_epi32((int)(uint32_t)(event >> 32));
        // slot 2(q0 + i) + 1 of lane i
        __m512i c2 = _mm512_add_epi32(_mm512_slli_epi32(_mm512_add_epi32(lane, _mm512_set1_epi32((int)q0)), 1),
                                      _mm512_set1_epi32(1));
        __m512i c3 = _mm512_set1_epi32((int)(uint32_t)stream);
        uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
        for (int r = 0; r < 10; ++r) {
            const __m512i h0 = philox_hi(c0, M0), l0 = philox_lo(c0, M0);
            const __m512i h1 = philox_hi(c2, M1), l1 = philox_lo(c2, M1);
            const __m512i n0 = _mm512_xor_si512(_mm512_xor_si512(h1, c1), _mm512_set1_epi32((int)k0));
            const __m512i n2 = _mm512_xor_si512(_mm512_xor_si512(h0, c3), _mm512_set1_epi32((int)k1));
            c0 = n0; c1 = l1; c2 = n2; c3 = l0;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const __mmask16 lt = _mm512_cmplt_epu32_mask(c0, uh);
        const __mmask16 eq = _mm512_cmpeq_epi32_mask(c0, uh);
        const __mmask16 lo = _mm512_cmplt_epu32_mask(_mm512_srli_epi32(c1, 11), ul);
        const uint64_t m16 = (uint64_t)(uint16_t)(lt | (eq & lo));
        h |= m16 << q0;
    }
    return h & all;
}
#endif
uint64_t noise_hits(uint64_t seed, uint64_t stream, uint64_t event, uint32_t n, double p) {
#if defined(__x86_64__) && defined(__GNUC__)
    static const int isa = __builtin_cpu_supports("avx512f") ? 2 : __builtin_cpu_supports("avx2") ? 1 : 0;
    if (isa == 2) return noise_hits_avx512(seed, stream, event, n, p);
    if (isa == 1) return noise_hits_avx2(seed, stream, event, n, p);
#endif
    return noise_hits_generic(seed, stream, event, n, p);
}

// ------------------------------------------------------------------ gates
enum GateKind { K_G1 = 0, K_DIAG = 1, K_SWAP = 2, K_U2 = 3, K_MEASURE = 4, K_RESET = 5, K_RESETALL = 6, K_QINIT = 7,
                K_PERM = 8 /* a block of disjoint SWAPs, made by the executor */ };

struct Gate {
    int kind = K_G1;
    int sub = G1_GEN;
    int t = 0, t2 = 0;      // target(s); K_DIAG: selector qubit or -1
    uint64_t cmask = 0;     // condition mask over global qubits
    bool neg = false;       // K_DIAG: factor -1
    double2 m[16];
    uint64_t nmask = 0;     // qubits acted on non-diagonally
    uint64_t dmask = 0;     // qubits acted on diagonally (controls, phase masks, selector)
    int src = -1;           // source op index
    double u = -1.0;        // K_MEASURE: uniform
    uint8_t pi[64];         // K_PERM: partner of each qubit (itself if unpaired)
};

inline double2 d2(double x, double y) { double2 r; r.x = x; r.y = y; return r; }
inline double2 from_polar(double r, double t) { return d2(r * std::cos(t), r * std::sin(t)); }

// Tile passes take every diagonal gate and the 2x2 gates; a controlled 2x2
// must be X or Y (CNOT, Toffoli, CY), which is all the instruction set makes.
bool is_pass_gate(const Gate& g) {
    if (g.kind == K_DIAG) return true;
    if (g.kind == K_SWAP) return g.cmask == 0;  // a relabelling of two tile bits
    return g.kind == K_G1 && (g.cmask == 0 || g.sub == G1_X || g.sub == G1_Y);
}
bool is_barrier(const Gate& g) { return g.kind >= K_MEASURE; }

// Algorithmic bytes of one per-gate application, S = 2^n * 16.
double gate_bytes(const Gate& g, uint32_t n) {
    const double S = std::ldexp(16.0, (int)n);
    auto pc = [](uint64_t x) { return (double)__builtin_popcountll(x); };
    switch (g.kind) {
        case K_G1: return 2.0 * S / std::ldexp(1.0, (int)pc(g.cmask));
        case K_DIAG: return g.t >= 0 ? 2.0 * S : 2.0 * S / std::ldexp(1.0, (int)pc(g.cmask));
        case K_SWAP: return S / std::ldexp(1.0, (int)pc(g.cmask));
        case K_U2: return 2.0 * S;
        default: return 2.0 * S;
    }
}

}  // namespace

// ------------------------------------------------------------------ handle
struct qoa_state_s {
    uint32_t n = 1;
    uint32_t flags = 0;
    int precision = QOA_PREC_F64;
    void* f32_mats = nullptr;        // FP32 passes: upload arena (device bytes)
    size_t f32_mats_cap = 0;
    std::vector<F32PassParams> f32_passes;  // prepared FP32 passes
    size_t f32_off[5] = {0, 0, 0, 0, 0};    // arena sections: mats, pops, angles, phases, tables
    bool view = false;               // batch view: amps / scal / status / partials / stream not owned
    int pass_budget = 0;             // max gates per tile pass (0: the default)
    F32Phase* f32_phases = nullptr;  // FP32 passes: phase entries (device)
    size_t f32_phases_cap = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    double2* amps = nullptr;
    double* scal = nullptr;       // [0] norm2, [1] P0, [2] P1, [3..] scratch
    uint32_t* status = nullptr;   // device status words
    double* partials = nullptr;
    size_t partials_cap = 0;
    double* host_scal = nullptr;  // pinned mirror of scal
    uint64_t seed = 0;
    uint64_t noise_stream = 0;
    uint64_t noise_event = 0;
    uint64_t meas_draws = 0;
    int noise_mode = 0;
    double noise_p = 0.0;
    uint64_t launches = 0;
    uint32_t host_resets = 0;     // normalize() resets decided on the host
    // The reference's serde JSON view that the engine does not otherwise
    // keep: noise_config None (never set) as opposed to Some(Ideal), the
    // Status.div_by_zero flag, and the QuantumState's own registers
    // (complex pairs), restored by a JSON load and written back on save.
    bool noise_none = true;
    bool div_by_zero = false;
    std::vector<double> json_regs;
    std::shared_ptr<void> plans;    // PlanCache: plans of repeated op lists
    int jit_mode = QOA_JIT_ASYNC;   // generated complex128 pass kernels (qoa_jit.cpp)
    uint32_t jit_min_qubits = 20;   // smaller states interpret their passes
    uint64_t jit_launches = 0;
    std::string err;
    // profiling
    struct Rec { cudaEvent_t a, b; double bytes; int kind; };
    std::vector<Rec> recs;
};

namespace {

int set_err(qoa_state_t s, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    else {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_err = buf;
    }
    return code;
}

// A failed call's error is also the thread's "last error"; it is cleared
// here (when it is not sticky) so that the next launch check does not
// report it again.
#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            cudaGetLastError();                                                           \
            return set_err(s, e_ == cudaErrorMemoryAllocation ? QOA_E_OOM : QOA_E_CUDA,   \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
        }                                                                                 \
    } while (0)

uint64_t state_len(const qoa_state_t s) { return 1ull << s->n; }

size_t partials_needed(uint32_t n) {
    size_t a = (n >= (uint32_t)TILE_BITS) ? (size_t)1 << (n - TILE_BITS) : 1;
    size_t b = (size_t)8 * (size_t)reduce_blocks(1ull << n);
    return std::max(a, b);
}

// Device buffers of batches come from one stream-ordered memory pool per
// device that keeps freed memory for the next batch (a batch of thousands of
// circuits holds tens of GB; mapping that afresh for every batch, or
// synchronising the device on every free, costs more than the batch's
// launches). A state allocation that finds the device full first returns the
// pools' unused memory and tries again.
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

cudaMemPool_t batch_pool(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

// Returns the batch pools' unused memory to the device (after the work that
// freed it has finished).
void trim_batch_pools() {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    bool any = false;
    for (cudaMemPool_t p : g_pools) any = any || p;
    if (!any) return;
    cudaDeviceSynchronize();
    for (cudaMemPool_t p : g_pools)
        if (p) cudaMemPoolTrimTo(p, 0);
}

// cudaMalloc, retried once after trimming the batch pools
cudaError_t device_alloc(void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        trim_batch_pools();
        e = cudaMalloc(p, bytes);
    }
    return e;
}

int alloc_state(qoa_state_t s, uint32_t n) {
    if (s->amps) { cudaFree(s->amps); s->amps = nullptr; }
    if (s->partials) { cudaFree(s->partials); s->partials = nullptr; }
    s->n = n;
    CK(device_alloc((void**)&s->amps, (s->precision == QOA_PREC_F32 ? sizeof(float2) : sizeof(double2)) << n));
    s->partials_cap = partials_needed(n);
    CK(device_alloc((void**)&s->partials, s->partials_cap * sizeof(double)));
    return QOA_OK;
}

struct Timer {
    qoa_state_t s;
    cudaEvent_t a = nullptr;
    double bytes;
    int kind;
    Timer(qoa_state_t st, double b, int k) : s(st), bytes(b), kind(k) {
        if (s->flags & QOA_FLAG_PROFILE) {
            cudaEventCreate(&a);
            cudaEventRecord(a, s->stream);
        }
    }
    ~Timer() {
        if (a) {
            cudaEvent_t b;
            cudaEventCreate(&b);
            cudaEventRecord(b, s->stream);
            s->recs.push_back({a, b, bytes, kind});
        }
    }
};

// -------------------------------------------------------------- expansion
struct Expander {
    uint32_t n;
    uint32_t flags;
    qoa_state_t s;                 // for noise draws (may be null in plan mode)
    std::vector<Gate> out;
    int first_err = QOA_OK;
    std::string err;
    int cur = -1;

    void skip(int code, const char* what) {
        if (first_err == QOA_OK) {
            first_err = code;
            char b[256];
            snprintf(b, sizeof b, "op %d skipped: %s", cur, what);
            err = b;
        }
    }

    // QuantumState::apply_noise (quantum_state.rs:839-869) after a gate event:
    // depolarising draws become explicit X / Y / Z gates.
    void noise_event(uint64_t touched) {
        if (!s || s->noise_mode == 0) return;
        const uint64_t ev = s->noise_event++;
        double p = s->noise_p;
        if (s->noise_mode == 2) p = 0.1 + 0.9 * uniform01(s->seed, s->noise_stream, ev, 0);
        if (s->noise_mode == 1 && !(p > 0.0)) return;
        uint64_t hit = noise_hits(s->seed, s->noise_stream, ev, n, p);
        if (flags & QOA_FLAG_NOISE_GATE_QUBITS) hit &= touched;
        for (; hit; hit &= hit - 1) {  // hit qubits in ascending order, each with its Pauli type draw
            const uint32_t q = (uint32_t)__builtin_ctzll(hit);
            const double u2 = uniform01(s->seed, s->noise_stream, ev, 2 * q + 2);
            int e = (int)(u2 * 3.0);
            if (e > 2) e = 2;
            Gate g;
            g.src = cur;
            if (e == 0) g1(g, q, G1_X, d2(0, 0), d2(0, 0), d2(0, 0), d2(0, 0), 0);
            else if (e == 1) g1(g, q, G1_Y, d2(0, 0), d2(0, 0), d2(0, 0), d2(0, 0), 0);
            else diag_neg(g, 1ull << q);
            out.push_back(g);
        }
    }

    static void g1(Gate& g, uint32_t t, int sub, double2 m0, double2 m1, double2 m2, double2 m3, uint64_t cm) {
        g.kind = K_G1; g.sub = sub; g.t = (int)t; g.cmask = cm;
        g.m[0] = m0; g.m[1] = m1; g.m[2] = m2; g.m[3] = m3;
        g.nmask = 1ull << t; g.dmask = cm;
    }
    static void diag_neg(Gate& g, uint64_t mask) {
        g.kind = K_DIAG; g.t = -1; g.neg = true; g.cmask = mask; g.m[0] = g.m[1] = d2(-1, 0);
        g.nmask = 0; g.dmask = mask;
    }
    static void diag_phase(Gate& g, uint64_t mask, double2 f) {
        g.kind = K_DIAG; g.t = -1; g.neg = false; g.cmask = mask; g.m[0] = g.m[1] = f;
        g.nmask = 0; g.dmask = mask;
    }

    void push(Gate g, uint64_t touched) {
        g.src = cur;
        out.push_back(g);
        noise_event(touched);
    }

    // ---- QuantumState methods (bounds-checked; out of range -> no-op) ----
    void h(uint32_t q) {
        if (q >= n) return skip(QOA_E_RANGE, "H qubit out of range");
        Gate g;
        // apply_h: norm_factor = Complex64::new(1.0 / SQRT_2, 0.0) (quantum_state.rs:196)
        g1(g, q, G1_H, d2(1.0 / M_SQRT2, 0.0), d2(0, 0), d2(0, 0), d2(0, 0), 0);
        push(g, 1ull << q);
    }
    void x(uint32_t q) {
        if (q >= n) return skip(QOA_E_RANGE, "X qubit out of range");
        Gate g; g1(g, q, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), 0); push(g, 1ull << q);
    }
    void y(uint32_t q) {
        if (q >= n) return skip(QOA_E_RANGE, "Y qubit out of range");
        Gate g; g1(g, q, G1_Y, d2(0, 0), d2(0, -1), d2(0, 1), d2(0, 0), 0); push(g, 1ull << q);
    }
    void z(uint32_t q) {
        if (q >= n) return skip(QOA_E_RANGE, "Z qubit out of range");
        Gate g; diag_neg(g, 1ull << q); push(g, 1ull << q);
    }
    void phase(uint32_t q, double2 f) {
        if (q >= n) return skip(QOA_E_RANGE, "phase qubit out of range");
        Gate g; diag_phase(g, 1ull << q, f); push(g, 1ull << q);
    }
    void rx(uint32_t q, double a) {
        if (q >= n) return skip(QOA_E_RANGE, "RX qubit out of range");
        const double c = std::cos(a / 2.0), sn = std::sin(a / 2.0);
        Gate g; g1(g, q, G1_RX, d2(c, sn), d2(0, -sn), d2(0, -sn), d2(c, 0), 0); push(g, 1ull << q);
    }
    void ry(uint32_t q, double a) {
        if (q >= n) return skip(QOA_E_RANGE, "RY qubit out of range");
        const double c = std::cos(a / 2.0), sn = std::sin(a / 2.0);
        Gate g; g1(g, q, G1_RY, d2(c, sn), d2(-sn, 0), d2(sn, 0), d2(c, 0), 0); push(g, 1ull << q);
    }
    void rz(uint32_t q, double a) {
        if (q >= n) return skip(QOA_E_RANGE, "RZ qubit out of range");
        Gate g;
        g.kind = K_DIAG; g.t = (int)q; g.cmask = 0;
        g.m[0] = from_polar(1.0, -a / 2.0);
        g.m[1] = from_polar(1.0, a / 2.0);
        g.nmask = 0; g.dmask = 1ull << q;
        push(g, 1ull << q);
    }
    void cnot(uint32_t c, uint32_t t) {
        if (c >= n || t >= n) return skip(QOA_E_RANGE, "CNOT qubit out of range");
        if (c == t) return skip(QOA_E_RANGE, "CNOT control == target");
        Gate g; g1(g, t, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), 1ull << c); push(g, (1ull << c) | (1ull << t));
    }
    uint64_t cz_mask(uint32_t c, uint32_t t) const {
        return (flags & QOA_FLAG_COMPAT_MASK_QUIRK) ? ((uint64_t)c | (uint64_t)t) : ((1ull << c) | (1ull << t));
    }
    void cz(uint32_t c, uint32_t t) {
        if (c >= n || t >= n) return skip(QOA_E_RANGE, "CZ qubit out of range");
        if (c == t) return skip(QOA_E_RANGE, "CZ control == target");
        Gate g; diag_neg(g, cz_mask(c, t)); push(g, (1ull << c) | (1ull << t));
    }
    void cphase(uint32_t c, uint32_t t, double a) {
        if (c >= n || t >= n) return skip(QOA_E_RANGE, "CPHASE qubit out of range");
        if (c == t) return skip(QOA_E_RANGE, "CPHASE control == target");
        Gate g; diag_phase(g, cz_mask(c, t), from_polar(1.0, a)); push(g, (1ull << c) | (1ull << t));
    }
    void swap(uint32_t a, uint32_t b, int ctrl) {
        if (a >= n || b >= n || (ctrl >= 0 && (uint32_t)ctrl >= n)) return skip(QOA_E_RANGE, "SWAP qubit out of range");
        if (a == b || (ctrl >= 0 && ((uint32_t)ctrl == a || (uint32_t)ctrl == b)))
            return skip(QOA_E_RANGE, "SWAP qubits not distinct");
        Gate g;
        g.kind = K_SWAP; g.t = (int)a; g.t2 = (int)b;
        g.cmask = ctrl >= 0 ? 1ull << ctrl : 0;
        g.nmask = (1ull << a) | (1ull << b); g.dmask = g.cmask;
        push(g, g.nmask | g.cmask);
    }
    void toffoli(uint32_t c1, uint32_t c2, uint32_t t) {
        if (c1 >= n || c2 >= n || t >= n) return skip(QOA_E_RANGE, "TOFFOLI qubit out of range");
        if (c1 == c2 || c1 == t || c2 == t) return skip(QOA_E_RANGE, "TOFFOLI qubits not distinct");
        Gate g; g1(g, t, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), (1ull << c1) | (1ull << c2));
        push(g, (1ull << c1) | (1ull << c2) | (1ull << t));
    }
    void cy(uint32_t c, uint32_t t) {
        if (c >= n || t >= n) return skip(QOA_E_RANGE, "CY qubit out of range");
        if (c == t) return skip(QOA_E_RANGE, "CY control == target");
        Gate g; g1(g, t, G1_Y, d2(0, 0), d2(0, -1), d2(0, 1), d2(0, 0), 1ull << c); push(g, (1ull << c) | (1ull << t));
    }
    void u1(uint32_t q, const double* m) {
        if (q >= n) return skip(QOA_E_RANGE, "U1 qubit out of range");
        if (!m) return skip(QOA_E_ARG, "U1 without matrix");
        Gate g; g1(g, q, G1_GEN, d2(m[0], m[1]), d2(m[2], m[3]), d2(m[4], m[5]), d2(m[6], m[7]), 0);
        push(g, 1ull << q);
    }
    void u2(uint32_t q1, uint32_t q2, const double* m) {
        if (q1 >= n || q2 >= n) return skip(QOA_E_RANGE, "U2 qubit out of range");
        if (q1 == q2) return skip(QOA_E_RANGE, "U2 qubits equal");
        if (!m) return skip(QOA_E_ARG, "U2 without matrix");
        Gate g;
        g.kind = K_U2; g.t = (int)std::min(q1, q2); g.t2 = (int)std::max(q1, q2);
        for (int k = 0; k < 16; ++k) g.m[k] = d2(m[2 * k], m[2 * k + 1]);
        g.nmask = (1ull << q1) | (1ull << q2);
        push(g, g.nmask);
    }
    void measure(uint32_t q) {
        if (q >= n) return skip(QOA_E_RANGE, "MEASURE qubit out of range");
        Gate g; g.kind = K_MEASURE; g.t = (int)q; g.nmask = ~0ull;
        push(g, 1ull << q);
    }
    void reset(uint32_t q) {
        if (q >= n) return skip(QOA_E_RANGE, "RESET qubit out of range");
        Gate g; g.kind = K_RESET; g.t = (int)q; g.nmask = ~0ull;
        push(g, 1ull << q);
    }
    void reset_all() {
        Gate g; g.kind = K_RESETALL; g.nmask = ~0ull;
        push(g, 0);
    }

    uint32_t qat(const qoa_op& op, uint32_t k) const { return (op.nq > 4 && op.qlist) ? op.qlist[k] : op.q[k]; }

    // execute_arithmetic (quantum_state.rs:460-705)
    void op(const qoa_op& o) {
        const uint32_t q0 = o.q[0], q1 = o.q[1], q2 = o.q[2], q3 = o.q[3];
        const double a = o.angle;
        switch (o.opcode) {
            case QOA_OP_QINIT: {
                Gate g; g.kind = K_QINIT; g.t = (int)std::max<uint32_t>(q0, 1); g.nmask = ~0ull; g.src = cur;
                out.push_back(g);
                n = (uint32_t)g.t;
                break;
            }
            case QOA_OP_RESET: reset(q0); break;
            case QOA_OP_RESETALL: reset_all(); break;
            case QOA_OP_H: h(q0); break;
            case QOA_OP_X: x(q0); break;
            case QOA_OP_Y: y(q0); break;
            case QOA_OP_Z: z(q0); break;
            case QOA_OP_T: phase(q0, from_polar(1.0, M_PI / 4.0)); break;   // vectorization.rs:218
            case QOA_OP_S: phase(q0, from_polar(1.0, M_PI / 2.0)); break;   // vectorization.rs:263
            case QOA_OP_P: case QOA_OP_SETPHASE: case QOA_OP_PHASE: phase(q0, from_polar(1.0, a)); break;
            case QOA_OP_RX: rx(q0, a); break;
            case QOA_OP_RY: ry(q0, a); break;
            case QOA_OP_RZ: rz(q0, a); break;
            case QOA_OP_CNOT: case QOA_OP_ENTANGLE: case QOA_OP_ECFB: cnot(q0, q1); break;
            case QOA_OP_CZ: cz(q0, q1); break;
            case QOA_OP_CPHASE: cphase(q0, q1, a); break;
            case QOA_OP_EBELL: h(q0); cnot(q0, q1); break;
            case QOA_OP_EMULTI: {
                if (o.nq == 0) { skip(QOA_E_ARG, "empty qubit list for entanglemulti"); break; }
                const uint32_t first = qat(o, 0);
                h(first);
                for (uint32_t k = 1; k < o.nq; ++k) cnot(first, qat(o, k));
                break;
            }
            case QOA_OP_ECLUSTER:
                for (uint32_t k = 0; k < o.nq; ++k) h(qat(o, k));
                for (uint32_t k = 0; k + 1 < o.nq; ++k) cz(qat(o, k), qat(o, k + 1));
                break;
            case QOA_OP_APPLYGATE:
                switch (q1) {
                    case 'H': h(q0); break;
                    case 'X': x(q0); break;
                    case 'Y': y(q0); break;
                    case 'Z': z(q0); break;
                    case 'T': phase(q0, from_polar(1.0, M_PI / 4.0)); break;
                    case 'S': phase(q0, from_polar(1.0, M_PI / 2.0)); break;
                    default: skip(QOA_E_OPCODE, "unknown gate name for applygate");
                }
                break;
            case QOA_OP_ESWAP: cnot(q0, q2); cnot(q1, q3); swap(q2, q3, -1); break;
            case QOA_OP_ESWAPM: cnot(q0, q2); cnot(q1, q3); swap(q2, q3, -1); measure(q2); measure(q3); break;
            case QOA_OP_EDIST: break;
            case QOA_OP_MEASB:
                if (q0 >= n) { skip(QOA_E_RANGE, "MEASB qubit out of range"); break; }
                if (q1 == 'X') { h(q0); measure(q0); h(q0); }
                else if (q1 == 'Y') {
                    phase(q0, from_polar(1.0, M_PI / 2.0)); h(q0); measure(q0); h(q0);
                    phase(q0, from_polar(1.0, M_PI / 2.0)); z(q0);
                } else if (q1 == 'Z') measure(q0);
                else skip(QOA_E_OPCODE, "unsupported measurement basis");
                break;
            case QOA_OP_MEASURE: measure(q0); break;
            case QOA_OP_ROT:
                if (q1 == 'X') rx(q0, a);
                else if (q1 == 'Y') ry(q0, a);
                else if (q1 == 'Z') rz(q0, a);
                else skip(QOA_E_OPCODE, "unsupported rotation axis");
                break;
            case QOA_OP_SWAP: swap(q0, q1, -1); break;
            case QOA_OP_CSWAP: swap(q1, q2, (int)q0); break;
            case QOA_OP_TOFFOLI: toffoli(q0, q1, q2); break;
            case QOA_OP_U1: u1(q0, o.matrix); break;
            case QOA_OP_U2: u2(q0, q1, o.matrix); break;
            case QOA_OP_CY: cy(q0, q1); break;
            default: skip(QOA_E_OPCODE, "unsupported opcode");
        }
    }
};

// -------------------------------------------------------------- scheduler
// A step is either a tile pass (a set of K_G1 / K_DIAG gates) or a single
// gate that runs on its own kernel (SWAP, U2, barriers).
struct Step {
    bool pass = false;
    std::vector<int> gates;        // indices into the gate list, in application order
    std::vector<int> slots;        // pass: high qubits of the tile (HIGH_SLOTS)
};

// Plans of repeated op lists (per state): a list seen for the second time
// keeps its schedule, its built pass parameters and its generated kernel
// texts, so that a circuit executed again (benchmark steps, shot or
// trajectory loops, a VM loop body) skips the host planning. Keyed by two
// independent hashes of every gate field the plan depends on.
struct PlanEntry {
    uint64_t h1 = 0, h2 = 0;
    std::vector<Step> steps;
    bool prebuilt = false;
    std::vector<PassParams> built;
    std::vector<int> built_of;
    std::vector<std::string> bodies;
};
struct PlanCache {
    static constexpr size_t kEntries = 8;
    std::deque<PlanEntry> entries;                 // most recent last
    std::unordered_map<uint64_t, uint8_t> seen;    // op lists seen once
};

void plan_hash(const std::vector<Gate>& G, uint64_t key, uint64_t& h1, uint64_t& h2) {
    h1 = 1469598103934665603ull ^ key;
    h2 = 0x9e3779b97f4a7c15ull ^ (key * 0xff51afd7ed558ccdull);
    auto mix = [&](const void* p, size_t nb) {
        const unsigned char* c = (const unsigned char*)p;
        for (size_t i = 0; i < nb; ++i) {
            h1 = (h1 ^ c[i]) * 1099511628211ull;
            h2 = (h2 ^ c[i]) * 0x100000001b3ull + (h2 >> 29);
        }
    };
    for (const Gate& g : G) {
        mix(&g.kind, sizeof g.kind);
        mix(&g.sub, sizeof g.sub);
        mix(&g.t, sizeof g.t);
        mix(&g.t2, sizeof g.t2);
        mix(&g.cmask, sizeof g.cmask);
        const uint8_t neg = g.neg;
        mix(&neg, 1);
        mix(g.m, sizeof g.m);
        mix(&g.nmask, sizeof g.nmask);
        mix(&g.dmask, sizeof g.dmask);
        mix(&g.u, sizeof g.u);
        if (g.kind == K_PERM) mix(g.pi, sizeof g.pi);
    }
}

// Greedy list scheduling. Gate g may run in the current pass when every
// earlier gate still waiting commutes with it: for each shared qubit both act
// diagonally (controls, phases). Non-diagonal targets must be in the tile:
// qubits 0..4 always are; up to HIGH_SLOTS higher qubits are claimed in the
// order gates ask for them.
// FP32 passes fuse gates into dense blocks, so a non-diagonal gate needs all
// of its qubits (controls included) in the tile, and SWAP / U2 can join too.
bool is_pass_gate_f32(const Gate& g) { return g.kind <= K_U2; }
uint64_t tile_need(const Gate& g, bool f32) {
    if (!f32) return g.nmask;
    return g.kind == K_DIAG ? 0 : (g.nmask | g.dmask);
}

// slot_weight 0: in-order greedy only; w > 0: slot search scoring a
// diagonal gate 1 and any other gate w.
std::vector<Step> schedule_pass_order(const std::vector<Gate>& G, uint32_t n, bool per_gate, bool f32,
                                      int gate_budget, int slot_weight) {
    const bool slot_search = slot_weight > 0;
    std::vector<Step> steps;
    const size_t N = G.size();
    std::vector<char> done(N, 0);
    size_t first = 0;
    const bool tiles = !per_gate && n >= (uint32_t)TILE_BITS;
    while (true) {
        while (first < N && done[first]) ++first;
        if (first >= N) break;
        const Gate& g0 = G[first];
        if (!tiles || !(f32 ? is_pass_gate_f32(g0) : is_pass_gate(g0))) {
            Step st;
            st.gates.push_back((int)first);
            done[first] = 1;
            steps.push_back(st);
            continue;
        }
        Step st;
        st.pass = true;
        // Gates of the pass from `first` on, in order, each joining when its
        // qubits are not blocked by a waiting gate and its non-diagonal
        // qubits are in the tile (claiming free high slots as needed, unless
        // the tile is given whole). Returns the tile.
        auto fill = [&](uint64_t tile, int nslots, std::vector<int>& out) -> uint64_t {
            uint64_t bN = 0, bD = 0;  // qubits blocked by waiting gates (non-diagonal / diagonal action)
            int budget_ops = MAX_PASS_OPS / 3;  // room for the exchanges and flushes
            if (gate_budget > 0 && gate_budget < budget_ops) budget_ops = gate_budget;
            int budget_coef = MAX_PASS_COEF - 8;
            for (size_t i = first; i < N; ++i) {
                if (done[i]) continue;
                const Gate& g = G[i];
                if (is_barrier(g)) break;
                bool ok = (f32 ? is_pass_gate_f32(g) : is_pass_gate(g)) && !(g.nmask & (bN | bD)) && !(g.dmask & bN);
                if (ok) {
                    const uint64_t need = tile_need(g, f32) & ~tile;
                    const int k = __builtin_popcountll(need);
                    const int nc = g.kind == K_G1 ? 4 : 2;  // a selector diagonal becomes two phase ops
                    if (nslots + k > HIGH_SLOTS || budget_ops < 1 || budget_coef < nc) ok = false;
                    else {
                        tile |= need;
                        nslots += k;
                        budget_ops -= 1;
                        budget_coef -= nc;
                    }
                }
                if (ok) {
                    out.push_back((int)i);
                } else {
                    bN |= g.nmask;
                    bD |= g.dmask;
                    const uint64_t full = (n >= 64) ? ~0ull : ((1ull << n) - 1);
                    if ((bN & full) == full) break;  // every qubit blocked: nothing else can join
                }
            }
            return tile;
        };
        uint64_t tile = fill(0x1Full, 0, st.gates);
        // Slot search: the greedy claims slots for the first gates that need
        // them; swapping one slot qubit for another, with the tile then
        // fixed, often admits more gates. Hill-climb while it does.
        if (slot_search && n > (uint32_t)TILE_BITS && __builtin_popcountll(tile) == TILE_BITS) {
            auto score = [&](const std::vector<int>& v) {
                long sc = 0;
                for (int gi : v) sc += G[gi].kind == K_DIAG ? 1 : slot_weight;
                return sc;
            };
            std::vector<int> best_gates = st.gates, trial;
            uint64_t best_tile = tile;
            for (int round = 0; round < 6; ++round) {
                bool improved = false;
                uint64_t cand_tile = best_tile;
                std::vector<int> cand_gates;
                for (uint32_t a = LANE_BITS; a < n; ++a) {
                    if (!((best_tile >> a) & 1)) continue;
                    for (uint32_t q = LANE_BITS; q < n; ++q) {
                        if ((best_tile >> q) & 1) continue;
                        const uint64_t t2 = (best_tile & ~(1ull << a)) | (1ull << q);
                        trial.clear();
                        fill(t2, HIGH_SLOTS, trial);
                        if (score(trial) > std::max(score(best_gates), score(cand_gates))) {
                            cand_gates = trial;
                            cand_tile = t2;
                        }
                    }
                }
                if (score(cand_gates) > score(best_gates)) {
                    best_gates = cand_gates;
                    best_tile = cand_tile;
                    improved = true;
                }
                if (!improved) break;
            }
            st.gates = best_gates;
            tile = best_tile;
        }
        for (int gi : st.gates) done[gi] = 1;
        // the tile's high slots: claimed qubits, padded with unused ones >= 5
        for (uint32_t q = LANE_BITS; q < n; ++q)
            if ((tile >> q) & 1) st.slots.push_back((int)q);
        for (uint32_t q = LANE_BITS; q < n && (int)st.slots.size() < HIGH_SLOTS; ++q)
            if (!((tile >> q) & 1)) st.slots.push_back((int)q);
        steps.push_back(st);
    }
    return steps;
}

// The pass plan of a gate list: the in-order greedy, and (when `search`)
// the same with the slot search scoring all gates alike or non-diagonal
// ones double; the one with the fewest steps (the search is per pass, so
// any of them can win overall). The search costs ~5x the host time of the
// greedy (~25 us per gate at 28 qubits) and saves about a quarter of the
// passes, which pays for itself from ~26 qubits on (a pass over 2^26
// complex128 amplitudes takes ~0.5 ms).
// QOA_SCHED_SEARCH=0 keeps the greedy alone.
bool slot_search_pays(uint32_t n) { return n >= 26; }

std::vector<Step> schedule(const std::vector<Gate>& G, uint32_t n, bool per_gate, bool f32 = false,
                           int gate_budget = 0, bool search_wanted = false) {
    static const bool search_on = [] {
        const char* v = getenv("QOA_SCHED_SEARCH");
        return !(v && v[0] == '0');
    }();
    std::vector<Step> best = schedule_pass_order(G, n, per_gate, f32, gate_budget, 0);
    if (!search_wanted || !search_on || per_gate || n <= (uint32_t)TILE_BITS || best.size() < 2) return best;
    for (int w : {1, 2}) {
        std::vector<Step> t = schedule_pass_order(G, n, per_gate, f32, gate_budget, w);
        if (t.size() < best.size()) best.swap(t);
    }
    return best;
}

// Builds the kernel op stream of a pass. The tile's TILE_BITS index bits
// (tile bit t < 5 = qubit t, tile bit 5 + s = high slot s) are assigned to
// lane / register / warp roles; every 2x2 gate must act on a register bit, so
// an exchange through shared memory re-assigns roles when its target is not
// one (Belady: keep the bits needed soonest). The load and the store need the
// lanes on tile bits 0..4 (coalesced), so a pass that moved them ends with an
// exchange back. Gates are rewritten into cheaper equivalents up to a scalar:
//   H  -> (a0+a1, a0-a1): the 1/sqrt2 is restored by the pass renormalisation;
//   RZ -> e^{-i t/2} * diag(1, e^{i t}): the global phase joins P.phase;
//   Z, CZ -> phase -1.
// Diagonal factors that are constant over a thread's registers accumulate in
// a per-thread pending factor, flushed only before an exchange that moves
// amplitudes between threads whose factors may differ.
// pair_pin (complex64 passes): register bit 3, along which the packed FP32
// kernels pair amplitudes, holds one tile bit for the whole pass (one that
// no 2x2 gate of the pass targets where there is one), so that every
// exchange moves whole packed pairs.
int build_pass(const std::vector<Gate>& G, const Step& st, uint32_t n, PassParams& P, bool pair_pin) {
    // thread conditions are 32-bit words: lane, warp and tile-number bits
    if (n > 32 - (LANE_BITS + WARP_BITS) + TILE_BITS) return -1;
    memset(&P, 0, sizeof P);
    P.n = n;
    P.phase = d2(1.0, 0.0);
    int slot_of[64];
    for (int q = 0; q < 64; ++q) slot_of[q] = -1;
    for (int s = 0; s < HIGH_SLOTS; ++s) {
        P.slot_qubit[s] = (uint8_t)st.slots[s];
        slot_of[st.slots[s]] = s;
    }
    int no = 0;
    for (uint32_t q = LANE_BITS; q < n; ++q)
        if (slot_of[q] < 0) P.outer_qubits[no++] = (uint8_t)q;
    // Tile bit holding each qubit (-1: outside the tile). A SWAP of two tile
    // qubits moves no data: it exchanges their tile bits here and the store
    // writes each tile bit to the qubit it ends up holding (out_qubit).
    int tb_of[64];
    for (int q = 0; q < 64; ++q) tb_of[q] = q < LANE_BITS ? q : (slot_of[q] < 0 ? -1 : LANE_BITS + slot_of[q]);
    auto tbit = [&](int q) -> int { return tb_of[q]; };
    auto relabel = [](int* tb, const Gate& g) { std::swap(tb[g.t], tb[g.t2]); };

    // register demand per gate (tile bit of each 2x2 target)
    const int ng = (int)st.gates.size();
    std::vector<int> need(ng, -1);
    int final_q[TILE_BITS];  // qubit each tile bit is stored to
    {
        int tb_sim[64];
        std::memcpy(tb_sim, tb_of, sizeof tb_of);
        for (int i = 0; i < ng; ++i) {
            const Gate& g = G[st.gates[i]];
            if (g.kind == K_G1) need[i] = tb_sim[g.t];
            else if (g.kind == K_SWAP) relabel(tb_sim, g);
        }
        for (int q = 0; q < 64; ++q)
            if (tb_sim[q] >= 0) final_q[tb_sim[q]] = q;
    }
    // the pinned pairing bit: a high tile bit stored outside the lanes, the
    // least used as a 2x2 target (ties: first used latest)
    int pin = -1;
    if (pair_pin) {
        int best_uses = 1 << 30, best_first = -1;
        for (int t = LANE_BITS; t < TILE_BITS; ++t) {
            if (final_q[t] < LANE_BITS) continue;
            int uses = 0, first = 1 << 30;
            for (int i = 0; i < ng; ++i)
                if (need[i] == t) { ++uses; first = std::min(first, i); }
            if (uses < best_uses || (uses == best_uses && first > best_first)) {
                best_uses = uses; best_first = first; pin = t;
            }
        }
    }
    // next_use(from, t): the first gate at or after `from` that needs tile
    // bit t in a register (1 << 30: none), tabled by a backward sweep
    std::vector<std::array<int, TILE_BITS>> nu((size_t)ng + 1);
    nu[ng].fill(1 << 30);
    for (int i = ng - 1; i >= 0; --i) {
        nu[i] = nu[i + 1];
        if (need[i] >= 0) nu[i][need[i]] = i;
    }
    auto next_use = [&](int from, int t) { return from >= ng ? (1 << 30) : nu[from][t]; };

    TileMap m;  // mapping in force
    // initial mapping: lanes on tile bits 0..4; registers = the four high
    // tile bits needed soonest; warps = the other two
    {
        for (int i = 0; i < LANE_BITS; ++i) m.lane[i] = (uint8_t)i;
        std::vector<std::pair<int, int>> c;
        for (int t = LANE_BITS; t < TILE_BITS; ++t) c.push_back({t == pin ? -1 : next_use(0, t), t});
        std::sort(c.begin(), c.end());
        for (int k = 0; k < REG_BITS; ++k) m.reg[k] = (uint8_t)c[k].second;
        for (int k = 0; k < WARP_BITS; ++k) m.warp[k] = (uint8_t)c[REG_BITS + k].second;
        if (pin >= 0) {  // the pinned bit on register bit 3
            for (int k = 0; k < REG_BITS - 1; ++k)
                if (m.reg[k] == pin) std::swap(m.reg[k], m.reg[REG_BITS - 1]);
        }
    }
    P.map0 = m;

    int nops = 0, ncoef = 0, nx = 0;
    // T positions (lane bits 0..4, warp bits 5..6) the pending factor depends on
    uint32_t dirty = 0;
    auto new_op = [&]() -> PassOp* {
        if (nops >= MAX_PASS_OPS) return nullptr;
        PassOp* o = &P.ops[nops++];
        memset(o, 0, sizeof *o);
        return o;
    };
    // Deferred diagonal factors (they commute with everything up to the next
    // 2x2 on one of their register bits, or the next exchange):
    //   tab[v]  product of the register-only phases, per register index v
    //   tm      thread-only phases (lane / warp / outer conditions), emitted as
    //           one PC_DIAG_TM group
    double2 tab[REGS];
    uint32_t tab_bits = 0;
    int tab_count = 0;
    PassOp tab_last;
    double2 tab_last_d = d2(1, 0);
    std::vector<std::pair<PassOp, double2>> tm;
    std::vector<std::pair<PassOp, double2>> mx;  // register x thread phases
    uint32_t mx_bits = 0;
    // angle phases (one tile bit at most, plus qubits outside the tile): per
    // register bit, or per thread condition; summed once per CTA in the kernel
    typedef std::vector<std::pair<uint64_t, double>> AngList;
    AngList ang_reg[REG_BITS];
    std::map<uint64_t, AngList> ang_thr;
    uint32_t ang_reg_bits = 0;
    int ang_used = 0, ang_pending = 0;
    auto emit_ang = [&](AngList& ent, uint8_t code, uint32_t creg, uint64_t tm) -> bool {
        if (ent.empty()) return true;
        if (P.nang >= MAX_ANG_OPS || ang_used + (int)ent.size() > MAX_PASS_ANGLES) return false;
        PassOp* o = new_op();
        if (!o) return false;
        o->code = code;
        o->cond_reg = (uint8_t)creg;
        o->tmask = tm;
        o->has_tp = tm ? 1 : 0;
        o->coef = P.nang;
        P.ang_start[P.nang] = (uint16_t)ang_used;
        for (const auto& e : ent) {
            P.angles[ang_used].omask = e.first;
            P.angles[ang_used].theta = e.second;
            ++ang_used;
        }
        P.nang++;
        P.ang_start[P.nang] = (uint16_t)ang_used;
        ang_pending -= (int)ent.size();
        ent.clear();
        return true;
    };
    auto flush_ang_reg = [&](uint32_t bits) -> bool {
        for (int k = 0; k < REG_BITS; ++k)
            if ((bits >> k) & 1) {
                if (!emit_ang(ang_reg[k], PC_DIAG_MA, 1u << k, 0)) return false;
                ang_reg_bits &= ~(1u << k);
            }
        return true;
    };
    auto flush_ang_thr = [&]() -> bool {
        for (auto& kv : ang_thr)
            if (!emit_ang(kv.second, PC_DIAG_TA, 0, kv.first)) return false;
        ang_thr.clear();
        return true;
    };
    auto ang_keys_pending = [&]() -> int {
        int c = (int)ang_thr.size();
        for (int k = 0; k < REG_BITS; ++k) c += ang_reg[k].empty() ? 0 : 1;
        return c;
    };
    uint32_t tab_touched = 0;  // registers whose table factor is not exactly 1
    auto tab_reset = [&]() {
        for (int v = 0; v < REGS; ++v) tab[v] = d2(1, 0);
        tab_bits = 0;
        tab_count = 0;
        tab_touched = 0;
    };
    tab_reset();
    auto flush_tab = [&]() -> bool {
        if (tab_count == 0) return true;
        PassOp* o = new_op();
        if (!o) return false;
        if (tab_count == 1) {  // one phase: the masked form touches fewer registers
            *o = tab_last;
            if (ncoef >= MAX_PASS_COEF) return false;
            o->coef = (uint16_t)ncoef;
            P.coef[ncoef++] = tab_last_d;
        } else {
            if (ncoef + REGS > MAX_PASS_COEF) return false;
            o->code = PC_DIAG_TAB;
            o->coef = (uint16_t)ncoef;
            // the registers whose factor is not exactly 1 (the generated
            // kernels multiply only those; the interpreter multiplies all)
            o->tmask = tab_touched;
            for (int v = 0; v < REGS; ++v) P.coef[ncoef++] = tab[v];
        }
        tab_reset();
        return true;
    };
    // a group header followed by its entry records (one dispatch)
    auto emit_group = [&](std::vector<std::pair<PassOp, double2>>& list, uint8_t code) -> bool {
        size_t at = 0;
        while (at < list.size()) {
            const size_t cnt = std::min<size_t>(255, list.size() - at);
            PassOp* h = new_op();
            if (!h) return false;
            h->code = code;
            h->k = (uint8_t)cnt;
            for (size_t e = 0; e < cnt; ++e) {
                PassOp* r = new_op();
                if (!r || ncoef >= MAX_PASS_COEF) return false;
                *r = list[at + e].first;
                r->code = PC_NOP;
                r->coef = (uint16_t)ncoef;
                P.coef[ncoef++] = list[at + e].second;
            }
            at += cnt;
        }
        list.clear();
        return true;
    };
    auto flush_tm = [&]() -> bool { return emit_group(tm, PC_DIAG_TM); };
    auto flush_mx = [&]() -> bool {
        mx_bits = 0;
        if (mx.size() == 1) {  // a lone entry needs no group header
            PassOp* e = new_op();
            if (!e || ncoef >= MAX_PASS_COEF) return false;
            *e = mx[0].first;
            e->code = PC_DIAG_M;
            e->coef = (uint16_t)ncoef;
            P.coef[ncoef++] = mx[0].second;
            mx.clear();
            return true;
        }
        // runs of equal register masks share one register multiply in the kernel;
        // the last entry of each run carries the flag that triggers it
        std::stable_sort(mx.begin(), mx.end(), [](const std::pair<PassOp, double2>& x,
                                                  const std::pair<PassOp, double2>& y) {
            return x.first.cond_reg < y.first.cond_reg;
        });
        for (size_t e = 0; e < mx.size(); ++e)
            if (e + 1 == mx.size() || mx[e + 1].first.cond_reg != mx[e].first.cond_reg) mx[e].first.has_tp |= 2;
        return emit_group(mx, PC_DIAG_MX);
    };
    // lane positions 0..2 carry a quarter-warp: give them tile bits with
    // distinct residues mod 3 where the lane set allows (bank-conflict-free).
    // With a pinned pairing bit the exchanges index the tile without that
    // bit, so a tile bit above it counts one position lower.
    auto order_lanes = [&](TileMap& t) {
        int best[LANE_BITS];
        for (int i = 0; i < LANE_BITS; ++i) best[i] = t.lane[i];
        int seen[3] = {-1, -1, -1};
        std::vector<int> first, rest;
        for (int i = 0; i < LANE_BITS; ++i) {
            const int r = (pin >= 0 && best[i] > pin ? best[i] - 1 : best[i]) % 3;
            if (seen[r] < 0) { seen[r] = best[i]; first.push_back(best[i]); }
            else rest.push_back(best[i]);
        }
        int k = 0;
        for (int x : first) t.lane[k++] = (uint8_t)x;
        for (int x : rest) t.lane[k++] = (uint8_t)x;
    };
    auto exchange_to = [&](const TileMap& nm) -> bool {
        if (!flush_tab() || !flush_mx() || !flush_tm() || !flush_ang_reg(0xfu) || !flush_ang_thr()) return false;
        // The pending factor stays with the thread across the exchange when
        // every lane / warp position it depends on keeps its tile bit: each
        // amplitude the thread receives then came from a thread with the
        // same bits there, so it owes the same factor. Otherwise flush it
        // into the registers first.
        uint32_t moved = 0;
        for (int i = 0; i < LANE_BITS; ++i)
            if (nm.lane[i] != m.lane[i]) moved |= 1u << i;
        for (int k = 0; k < WARP_BITS; ++k)
            if (nm.warp[k] != m.warp[k]) moved |= 1u << (LANE_BITS + k);
        if (dirty & moved) {
            PassOp* f = new_op();
            if (!f) return false;
            f->code = PC_FLUSH;
            dirty = 0;
        }
        if (nx >= MAX_XCHG) return false;
        PassOp* x = new_op();
        if (!x) return false;
        x->code = PC_XCHG;
        x->coef = (uint16_t)nx;
        P.xmap[nx++] = nm;
        m = nm;
        return true;
    };
    // bring tile bit `must` into the registers
    auto make_reg = [&](int i, int must) -> bool {
        std::vector<std::pair<int, int>> c;
        for (int t = 0; t < TILE_BITS; ++t) c.push_back({t == must ? -1 : (t == pin ? -2 : next_use(i, t)), t});
        std::sort(c.begin(), c.end());
        bool want[TILE_BITS] = {};
        for (int k = 0; k < REG_BITS; ++k) want[c[k].second] = true;
        TileMap nm = m;
        // outgoing register bits take the positions the incoming bits leave
        std::vector<int> outgoing;
        for (int k = 0; k < REG_BITS; ++k)
            if (!want[m.reg[k]]) outgoing.push_back(m.reg[k]);
        std::vector<int> incoming;
        for (int t = 0; t < TILE_BITS; ++t) {
            if (!want[t]) continue;
            bool held = false;
            for (int k = 0; k < REG_BITS; ++k) held |= m.reg[k] == t;
            if (!held) incoming.push_back(t);
        }
        size_t oi = 0;
        for (int t : incoming) {
            const int o = outgoing[oi++];
            for (int k = 0; k < REG_BITS; ++k)
                if (nm.reg[k] == o) nm.reg[k] = (uint8_t)t;
            for (int k = 0; k < LANE_BITS; ++k)
                if (m.lane[k] == t) nm.lane[k] = (uint8_t)o;
            for (int k = 0; k < WARP_BITS; ++k)
                if (m.warp[k] == t) nm.warp[k] = (uint8_t)o;
        }
        // register positions by next use: the last register bit goes to the
        // tile bit needed last (the complex64 pass pairs amplitudes along it)
        auto key = [&](uint8_t x) { return x == pin ? (1 << 30) + 1 : (x == must ? -1 : next_use(i, x)); };
        std::stable_sort(nm.reg, nm.reg + REG_BITS, [&](uint8_t x, uint8_t y) { return key(x) < key(y); });
        if (!getenv("QOA_NO_ORDER_LANES")) order_lanes(nm);
        return exchange_to(nm);
    };
    int outer_k[64];  // position of each outer qubit among outer_qubits (-1: in the tile)
    for (int q = 0; q < 64; ++q) outer_k[q] = -1;
    for (int k = 0; k < no; ++k) outer_k[P.outer_qubits[k]] = k;
    auto cond = [&](uint64_t mask, PassOp& op) {
        for (uint64_t mm = mask; mm; mm &= mm - 1) {
            const int q = __builtin_ctzll(mm);
            const int t = tbit(q);
            if (t < 0) {  // outside the tile: the CTA's tile-number bit of that qubit
                if (outer_k[q] >= 0) op.tmask |= 1ull << (LANE_BITS + WARP_BITS + outer_k[q]);
                continue;
            }
            for (int k = 0; k < LANE_BITS; ++k)
                if (m.lane[k] == t) op.cond_lane |= (uint8_t)(1u << k);
            for (int k = 0; k < REG_BITS; ++k)
                if (m.reg[k] == t) op.cond_reg |= (uint8_t)(1u << k);
            for (int k = 0; k < WARP_BITS; ++k)
                if (m.warp[k] == t) op.cond_warp |= (uint8_t)(1u << k);
        }
        for (int k = 0; k < LANE_BITS; ++k)
            if ((op.cond_lane >> k) & 1) op.tmask |= 1ull << k;
        for (int k = 0; k < WARP_BITS; ++k)
            if ((op.cond_warp >> k) & 1) op.tmask |= 1ull << (LANE_BITS + k);
        op.has_tp = op.tmask ? 1 : 0;
    };
    auto phase_op = [&](uint64_t mask, double2 d) -> bool {
        if (mask == 0) {  // global factor
            P.phase = d2(P.phase.x * d.x - P.phase.y * d.y, P.phase.x * d.y + P.phase.y * d.x);
            return true;
        }
        PassOp o;
        memset(&o, 0, sizeof o);
        cond(mask, o);
        {
            const int tb = LANE_BITS + WARP_BITS;
            const uint64_t thr = o.tmask & ((1ull << tb) - 1), outer = o.tmask >> tb;
            const bool one_bit = (__builtin_popcount(o.cond_reg) == 1 && !thr) ||
                                 (!o.cond_reg && __builtin_popcountll(thr) <= 1);
            const bool room = ang_used + ang_pending < MAX_PASS_ANGLES && (int)P.nang + ang_keys_pending() + 1 < MAX_ANG_OPS;
            if (outer && one_bit && room && std::fabs(d.x * d.x + d.y * d.y - 1.0) < 1e-14) {
                const double th = std::atan2(d.y, d.x);
                if (o.cond_reg) {
                    const int k = __builtin_ctz(o.cond_reg);
                    ang_reg[k].push_back({outer, th});
                    ang_reg_bits |= 1u << k;
                } else {
                    ang_thr[thr].push_back({outer, th});
                    dirty |= (uint32_t)thr;
                }
                ++ang_pending;
                return true;
            }
        }
        if (o.cond_reg == 0) {  // thread-only: joins the pending factor
            o.code = PC_DIAG_T;
            dirty |= (uint32_t)(o.tmask & ((1ull << (LANE_BITS + WARP_BITS)) - 1));
            tm.push_back({o, d});
            return true;
        }
        if (!o.has_tp) {  // register-only: joins the table
            for (int v = 0; v < REGS; ++v)
                if (((uint32_t)v & o.cond_reg) == o.cond_reg) {
                    tab[v] = d2(tab[v].x * d.x - tab[v].y * d.y, tab[v].x * d.y + tab[v].y * d.x);
                    tab_touched |= 1u << v;
                }
            tab_bits |= o.cond_reg;
            o.code = PC_DIAG_M;
            tab_last = o;
            tab_last_d = d;
            ++tab_count;
            return true;
        }
        mx.push_back({o, d});  // register and thread conditions together
        mx_bits |= o.cond_reg;
        return true;
    };

    for (int i = 0; i < ng; ++i) {
        const Gate& g = G[st.gates[i]];
        if (g.kind == K_SWAP) {
            if (g.cmask || tbit(g.t) < 0 || tbit(g.t2) < 0) return -1;
            relabel(tb_of, g);
            continue;
        }
        if (g.kind == K_G1) {
            const int t = tbit(g.t);
            int k = -1;
            for (int j = 0; j < REG_BITS; ++j)
                if (m.reg[j] == t) k = j;
            if (k < 0) {
                if (!make_reg(i, t)) return -1;
                for (int j = 0; j < REG_BITS; ++j)
                    if (m.reg[j] == t) k = j;
            }
            // deferred register phases on this bit or on a control bit must land first
            uint32_t touch = 1u << k;
            {
                PassOp c;
                memset(&c, 0, sizeof c);
                cond(g.cmask, c);
                touch |= c.cond_reg;
            }
            if ((tab_bits & touch) && !flush_tab()) return -1;
            if ((mx_bits & touch) && !flush_mx()) return -1;
            if ((ang_reg_bits & touch) && !flush_ang_reg(ang_reg_bits & touch)) return -1;
            PassOp* o = new_op();
            if (!o) return -1;
            cond(g.cmask, *o);
            o->k = (uint8_t)k;
            const bool controlled = o->has_tp || o->cond_reg;
            const int sub = g.sub == G1_H ? G1_HF : g.sub;
            switch (sub) {
                case G1_X: o->code = (uint8_t)(PC_XC + k); break;
                case G1_Y: o->code = (uint8_t)(PC_YC + k); break;
                case G1_HF: o->code = (uint8_t)(PC_HF + k); break;
                case G1_RX: o->code = (uint8_t)(PC_RX + k); break;
                case G1_RY: o->code = (uint8_t)(PC_RY + k); break;
                default: o->code = (uint8_t)(PC_GEN + k); break;
            }
            if (controlled && sub != G1_X && sub != G1_Y) return -1;
            if (ncoef + 4 > MAX_PASS_COEF) return -1;
            o->coef = (uint16_t)ncoef;
            for (int j = 0; j < 4; ++j) P.coef[ncoef++] = g.m[j];
            if (sub == G1_RX || sub == G1_RY) {
                // factor out the larger of |cos|, |sin|: its sign joins the
                // global phase, its magnitude the renormalisation
                const double c = g.m[0].x, sn = g.m[0].y;
                const bool a_form = std::fabs(c) >= std::fabs(sn);
                const double f = a_form ? c : sn;
                P.coef[o->coef] = d2(a_form ? sn / c : c / sn, 0.0);
                if (f < 0) P.phase = d2(-P.phase.x, -P.phase.y);
                if (!a_form) o->code = (uint8_t)((sub == G1_RX ? PC_RXB : PC_RYB) + k);
            }
        } else {  // K_DIAG
            if (g.neg) {
                if (!phase_op(g.cmask, d2(-1, 0))) return -1;
            } else if (g.t < 0) {
                if (!phase_op(g.cmask, g.m[0])) return -1;
            } else {
                // (bit t ? d1 : d0) under cmask = d0 under cmask, then d1/d0 under cmask|t
                const double2 d0 = g.m[0], d1 = g.m[1];
                const double2 r = d2(d1.x * d0.x + d1.y * d0.y, d1.y * d0.x - d1.x * d0.y);  // d1 * conj(d0)
                const double s2 = d0.x * d0.x + d0.y * d0.y;
                if (!phase_op(g.cmask, d0)) return -1;
                if (!phase_op(g.cmask | (1ull << g.t), d2(r.x / s2, r.y / s2))) return -1;
            }
        }
    }
    if (!flush_tab() || !flush_mx() || !flush_tm() || !flush_ang_reg(0xfu) || !flush_ang_thr()) return -1;
    // where each tile bit is stored: the qubit it holds after the pass's SWAPs
    int lane_tb[LANE_BITS];
    for (int q = 0; q < 64; ++q) {
        const int t = tb_of[q];
        if (t < 0) continue;
        P.out_qubit[t] = (uint8_t)q;
        if (q < LANE_BITS) lane_tb[q] = t;
    }
    // lanes on the tile bits stored to qubits 0..4, in order, for the coalesced store
    bool canonical = true;
    for (int i = 0; i < LANE_BITS; ++i) canonical &= m.lane[i] == lane_tb[i];
    if (!canonical) {
        TileMap nm;
        bool is_lane[TILE_BITS] = {};
        for (int i = 0; i < LANE_BITS; ++i) {
            nm.lane[i] = (uint8_t)lane_tb[i];
            is_lane[lane_tb[i]] = true;
        }
        std::vector<int> high;  // the other tile bits keep registers where they can
        for (int k = 0; k < REG_BITS; ++k)
            if (!is_lane[m.reg[k]]) high.push_back(m.reg[k]);
        for (int k = 0; k < WARP_BITS; ++k)
            if (!is_lane[m.warp[k]]) high.push_back(m.warp[k]);
        for (int k = 0; k < LANE_BITS; ++k)
            if (!is_lane[m.lane[k]]) high.push_back(m.lane[k]);
        if (pin >= 0 && !is_lane[pin]) {  // the pinned bit stays on register bit 3
            high.erase(std::find(high.begin(), high.end(), pin));
            high.insert(high.begin() + (REG_BITS - 1), pin);
        }
        for (int k = 0; k < REG_BITS; ++k) nm.reg[k] = (uint8_t)high[k];
        for (int k = 0; k < WARP_BITS; ++k) nm.warp[k] = (uint8_t)high[REG_BITS + k];
        if (!exchange_to(nm)) return -1;
    }
    P.nops = (uint32_t)nops;
    P.ncoef = (uint32_t)ncoef;
    return 0;
}

// ------------------------------------------------------- FP32 fused passes
using cplx = std::complex<double>;

// The exact 2x2 of a K_G1 gate (the forms of Expander).
void g1_exact(const Gate& g, cplx (&m)[4]) {
    switch (g.sub) {
        case G1_H: {
            const double f = g.m[0].x;
            m[0] = f; m[1] = f; m[2] = f; m[3] = -f;
            break;
        }
        case G1_X: m[0] = 0; m[1] = 1; m[2] = 1; m[3] = 0; break;
        case G1_Y: m[0] = 0; m[1] = cplx(0, -1); m[2] = cplx(0, 1); m[3] = 0; break;
        case G1_RX: {
            const double c = g.m[0].x, sn = g.m[0].y;
            m[0] = c; m[1] = cplx(0, -sn); m[2] = cplx(0, -sn); m[3] = c;
            break;
        }
        case G1_RY: {
            const double c = g.m[0].x, sn = g.m[0].y;
            m[0] = c; m[1] = -sn; m[2] = sn; m[3] = c;
            break;
        }
        default:
            for (int k = 0; k < 4; ++k) m[k] = cplx(g.m[k].x, g.m[k].y);
    }
}

// Applies gate g to a vector over the 5-qubit block space whose bit i is the
// block's i-th qubit bq[i] (global qubit indices).
void block_apply(const Gate& g, const int* bq, cplx* v) {
    auto bit = [&](int q) -> uint32_t {
        for (int i = 0; i < 5; ++i)
            if (bq[i] == q) return 1u << i;
        return 0;
    };
    auto bmask = [&](uint64_t m) -> uint32_t {
        uint32_t r = 0;
        for (int q = 0; q < 64; ++q)
            if ((m >> q) & 1) r |= bit(q);
        return r;
    };
    const uint32_t cm = bmask(g.cmask);
    if (g.kind == K_G1) {
        cplx m[4];
        g1_exact(g, m);
        const uint32_t tb = bit(g.t);
        for (uint32_t r = 0; r < 32; ++r) {
            if ((r & tb) || (r & cm) != cm) continue;
            const cplx a0 = v[r], a1 = v[r | tb];
            v[r] = m[0] * a0 + m[1] * a1;
            v[r | tb] = m[2] * a0 + m[3] * a1;
        }
    } else if (g.kind == K_DIAG) {
        const uint32_t sb = g.t >= 0 ? bit(g.t) : 0;
        for (uint32_t r = 0; r < 32; ++r) {
            if ((r & cm) != cm) continue;
            if (g.neg) v[r] = -v[r];
            else v[r] *= (sb && (r & sb)) ? cplx(g.m[1].x, g.m[1].y) : cplx(g.m[0].x, g.m[0].y);
        }
    } else if (g.kind == K_SWAP) {
        const uint32_t b1 = bit(g.t), b2 = bit(g.t2);
        for (uint32_t r = 0; r < 32; ++r) {
            if ((r & (b1 | b2)) || (r & cm) != cm) continue;
            std::swap(v[r | b2], v[r | b1]);
        }
    } else if (g.kind == K_U2) {
        const uint32_t bl = bit(g.t), bh = bit(g.t2);
        for (uint32_t r = 0; r < 32; ++r) {
            if (r & (bl | bh)) continue;
            const uint32_t idx[4] = {r, r | bl, r | bh, r | bl | bh};
            cplx x[4], y[4];
            for (int k = 0; k < 4; ++k) x[k] = v[idx[k]];
            for (int row = 0; row < 4; ++row) {
                y[row] = 0;
                for (int k = 0; k < 4; ++k) y[row] += cplx(g.m[4 * row + k].x, g.m[4 * row + k].y) * x[k];
            }
            for (int k = 0; k < 4; ++k) v[idx[k]] = y[k];
        }
    }
}

uint64_t gate_qubits(const Gate& g) {
    uint64_t m = g.nmask | g.dmask;
    if (g.kind == K_DIAG && g.t >= 0) m |= 1ull << g.t;
    return m;
}

// TF32 of x, rounded to nearest (ties away from zero), as mma consumes it.
float tf32_round(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    if ((b & 0x7f800000u) != 0x7f800000u) {
        b += 0x1000u;
        b &= 0xffffe000u;
    }
    float r;
    memcpy(&r, &b, 4);
    return r;
}

// Fuses a pass's gates into dense blocks of <= 5 tile qubits (FP64 unitaries,
// rounded for the tensor cores) and phase groups.
struct F32Upload {
    std::vector<float> mats;
    std::vector<F32PhaseOp> pops;
    std::vector<F32Angle> angles;
    std::vector<F32Phase> phases;
    std::vector<float2> tables;
};

int build_f32_pass(const std::vector<Gate>& G, const Step& st, uint32_t n, F32PassParams& P, F32Upload& up) {
    std::vector<float>& mats = up.mats;
    memset(&P, 0, sizeof P);
    P.n = n;
    int slot_of[64];
    for (int q = 0; q < 64; ++q) slot_of[q] = -1;
    for (int s = 0; s < HIGH_SLOTS; ++s) {
        P.slot_qubit[s] = (uint8_t)st.slots[s];
        slot_of[st.slots[s]] = s;
    }
    int no = 0;
    for (uint32_t q = LANE_BITS; q < n; ++q)
        if (slot_of[q] < 0) P.outer_qubits[no++] = (uint8_t)q;
    uint64_t tile = 0x1Full;
    for (int s = 0; s < HIGH_SLOTS; ++s) tile |= 1ull << st.slots[s];
    auto tbit = [&](int q) -> int { return q < LANE_BITS ? q : LANE_BITS + slot_of[q]; };

    int nops = 0;
    uint64_t B = 0;                 // qubits of the open block
    std::vector<const Gate*> blk;   // its gates, in order
    std::vector<const Gate*> pend;  // deferred diagonal gates
    uint64_t pend_q = 0;

    auto close_block = [&]() -> bool {
        if (blk.empty()) return true;
        if (nops >= MAX_F32_OPS) return false;
        // block qubits: B padded to 5 with other tile qubits, ascending tile bit
        std::vector<std::pair<int, int>> bq;
        for (int q = 0; q < 64; ++q)
            if ((B >> q) & 1) bq.push_back({tbit(q), q});
        for (int q = 0; q < 64 && bq.size() < 5; ++q)
            if (((tile >> q) & 1) && !((B >> q) & 1)) bq.push_back({tbit(q), q});
        std::sort(bq.begin(), bq.end());
        int qs[5];
        uint32_t bm = 0;
        for (int i = 0; i < 5; ++i) { qs[i] = bq[i].second; bm |= 1u << bq[i].first; }
        cplx U[32][32];
        for (int c = 0; c < 32; ++c) {
            cplx v[32];
            for (int r = 0; r < 32; ++r) v[r] = (r == c) ? 1.0 : 0.0;
            for (const Gate* g : blk) block_apply(*g, qs, v);
            for (int r = 0; r < 32; ++r) U[r][c] = v[r];
        }
        // real embedding [[Ur, -Ui], [Ui, Ur]] (row r = output, column c =
        // input), split into TF32 hi / lo, each stored as the tensor cores'
        // K-major operand: 8-row x 4-element core matrices of 128 bytes, the
        // 8 row groups of one 4-column chunk adjacent, chunks 1 KB apart
        const size_t base = mats.size();
        mats.resize(base + 8192);
        for (int r = 0; r < 64; ++r)
            for (int c = 0; c < 64; ++c) {
                const cplx u = U[r & 31][c & 31];
                double x;
                if (r < 32) x = (c < 32) ? u.real() : -u.imag();
                else x = (c < 32) ? u.imag() : u.real();
                const float h = tf32_round((float)x);
                const float l = tf32_round((float)(x - (double)h));
                const size_t off = (size_t)(c >> 2) * 256 + (size_t)(r >> 3) * 32 + (size_t)(r & 7) * 4 + (c & 3);
                mats[base + off] = h;
                mats[base + 4096 + off] = l;
            }
        F32Op& op = P.ops[nops++];
        op.kind = 0;
        op.bmask = bm;
        op.index = (uint32_t)(base / 8192);
        blk.clear();
        B = 0;
        return true;
    };
    // pending diagonal gates -> one phase group: unit factors d = e^{i theta}
    // where every bit of a mask is set, split by how they depend on the CTA
    auto flush_pend = [&]() -> bool {
        if (pend.empty()) return true;
        if (nops >= MAX_F32_OPS) return false;
        std::vector<std::vector<F32Angle>> lists(TILE_BITS + 1);
        std::vector<cplx> table;
        std::vector<F32Phase> multi;
        auto entry = [&](uint64_t mask, cplx d) {
            uint32_t tl = 0;
            uint64_t outer = 0;
            for (int q = 0; q < 64; ++q) {
                if (!((mask >> q) & 1)) continue;
                if ((tile >> q) & 1) tl |= 1u << tbit(q);
                else outer |= 1ull << q;
            }
            if (outer == 0) {  // the same in every CTA: into the tile table
                if (table.empty()) table.assign(1u << TILE_BITS, cplx(1.0, 0.0));
                for (uint32_t j = 0; j < (1u << TILE_BITS); ++j)
                    if ((j & tl) == tl) table[j] *= d;
            } else if (__builtin_popcount(tl) <= 1) {
                const int t = tl ? __builtin_ctz(tl) : TILE_BITS;
                lists[t].push_back(F32Angle{outer, std::atan2(d.imag(), d.real())});
            } else {
                F32Phase e;
                memset(&e, 0, sizeof e);
                e.outer = outer;
                e.tile = tl;
                e.re = d.real();
                e.im = d.imag();
                multi.push_back(e);
            }
        };
        for (const Gate* g : pend) {
            if (g->neg) entry(g->cmask, -1.0);
            else if (g->t < 0) entry(g->cmask, cplx(g->m[0].x, g->m[0].y));
            else {
                const cplx d0(g->m[0].x, g->m[0].y), d1(g->m[1].x, g->m[1].y);
                entry(g->cmask, d0);
                entry(g->cmask | (1ull << g->t), d1 / d0);
            }
        }
        F32PhaseOp po;
        memset(&po, 0, sizeof po);
        po.table = -1;
        for (int t = 0; t <= TILE_BITS; ++t) {
            po.bit_start[t] = (uint32_t)up.angles.size();
            up.angles.insert(up.angles.end(), lists[t].begin(), lists[t].end());
        }
        po.bit_start[TILE_BITS + 1] = (uint32_t)up.angles.size();
        if (!table.empty()) {
            po.table = (int32_t)(up.tables.size() >> TILE_BITS);
            for (const cplx& c : table) {
                float2 f;
                f.x = (float)c.real();
                f.y = (float)c.imag();
                up.tables.push_back(f);
            }
        }
        po.multi_start = (uint32_t)up.phases.size();
        po.multi_count = (uint32_t)multi.size();
        up.phases.insert(up.phases.end(), multi.begin(), multi.end());
        F32Op& op = P.ops[nops++];
        op.kind = 1;
        op.index = (uint32_t)up.pops.size();
        up.pops.push_back(po);
        pend.clear();
        pend_q = 0;
        return true;
    };

    for (int gi : st.gates) {
        const Gate& g = G[gi];
        const uint64_t Q = gate_qubits(g);
        if (g.kind == K_DIAG) {
            if (!blk.empty() && (Q & ~tile) == 0 && __builtin_popcountll(B | Q) <= 5) {
                blk.push_back(&g);
                B |= Q;
            } else {
                pend.push_back(&g);
                pend_q |= Q;
            }
            continue;
        }
        // non-diagonal: every qubit is a tile qubit (the scheduler claimed them)
        if (pend_q & g.nmask) {
            if (!close_block() || !flush_pend()) return -1;
        }
        if (__builtin_popcountll(B | Q) > 5) {
            if (!close_block()) return -1;
        }
        blk.push_back(&g);
        B |= Q;
    }
    if (!close_block() || !flush_pend()) return -1;
    P.nops = (uint32_t)nops;
    return 0;
}

// ------------------------------------------------------------- execution
GGate to_ggate(const Gate& g) {
    GGate k;
    memset(&k, 0, sizeof k);
    k.cmask = g.cmask;
    if (g.kind == K_G1) {
        k.kind = GG_G1; k.sub = (uint8_t)g.sub; k.t = (uint8_t)g.t;
        for (int j = 0; j < 4; ++j) k.m[j] = g.m[j];
    } else if (g.kind == K_DIAG) {
        k.kind = GG_DIAG; k.sub = g.neg ? 0x80 : 0; k.t = g.t >= 0 ? (uint8_t)g.t : 64;
        k.m[0] = g.m[0]; k.m[1] = g.m[1];
    } else if (g.kind == K_SWAP) {
        k.kind = GG_SWAP; k.t = (uint8_t)g.t; k.t2 = (uint8_t)g.t2;
    } else if (g.kind == K_U2) {
        k.kind = GG_U2; k.t = (uint8_t)g.t; k.t2 = (uint8_t)g.t2;
        for (int j = 0; j < 16; ++j) k.m[j] = g.m[j];
    }
    return k;
}

int run_gate(qoa_state_t s, const Gate& g) {
    const GGate k = to_ggate(g);
    Timer tm(s, gate_bytes(g, s->n) * (s->precision == QOA_PREC_F32 ? 0.5 : 1.0), 1);
    if (s->precision == QOA_PREC_F32) CK(launch_gate_c64((float2*)s->amps, state_len(s), k, s->stream));
    else CK(launch_gate(s->amps, state_len(s), k, s->stream));
    s->launches++;
    return QOA_OK;
}

int run_pass(qoa_state_t s, const std::vector<Gate>& G, const Step& st) {
    static thread_local PassParams P;
    if (build_pass(G, st, s->n, P, s->precision == QOA_PREC_F32) != 0) {
        // op stream too long for one launch: fall back to per-gate kernels
        for (int gi : st.gates) {
            int rc = run_gate(s, G[gi]);
            if (rc) return rc;
        }
        return QOA_OK;
    }
    if (s->precision == QOA_PREC_F32) {
        Timer tm(s, 2.0 * std::ldexp(8.0, (int)s->n), 3);
        CK(launch_pass_p32((float2*)s->amps, P, s->scal, s->partials, s->stream));
    } else {
        Timer tm(s, 2.0 * std::ldexp(16.0, (int)s->n), 0);
        CK(launch_pass(s->amps, P, s->scal, s->partials, s->stream));
    }
    CK(launch_reduce_partials(s->partials, 1u << (s->n - TILE_BITS), s->scal, s->status, s->stream));
    s->launches += 2;
    return QOA_OK;
}

// A complex128 pass whose parameters were built ahead (with its generated
// kernel requested): the generated kernel when it is ready, else k_pass.
int run_pass_built(qoa_state_t s, const PassParams& P, const JitKernel& jk) {
    const bool c64 = s->precision == QOA_PREC_F32;
    {
        Timer tm(s, 2.0 * std::ldexp(c64 ? 8.0 : 16.0, (int)s->n), c64 ? 3 : 0);
        cudaError_t je = cudaErrorNotReady;
        if (jk.ready()) {
            je = jk.launch(s->amps, P, s->scal, s->partials, s->status + 3, s->stream);
            if (je == cudaSuccess) s->jit_launches++;
            else if (je != cudaErrorNotSupported) CK(je);
        }
        if (je != cudaSuccess) {  // not compiled yet, or its launch set-up unavailable: the interpreter
            if (c64) CK(launch_pass_p32((float2*)s->amps, P, s->scal, s->partials, s->stream));
            else CK(launch_pass(s->amps, P, s->scal, s->partials, s->stream));
        }
    }
    CK(launch_reduce_partials(s->partials, 1u << (s->n - TILE_BITS), s->scal, s->status, s->stream));
    s->launches += 2;
    return QOA_OK;
}

// Reads norm2, P0, P1 of qubit q (logical probabilities) to the host.
int read_p01(qoa_state_t s, uint32_t q, double& p0, double& p1, double& norm2) {
    CK(launch_p01(s->amps, state_len(s), q, s->partials, s->scal + 1, s->scal, s->stream));
    s->launches += 2;
    CK(cudaMemcpyAsync(s->host_scal, s->scal, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    norm2 = s->host_scal[0];
    if (!(norm2 > 1e-12)) {  // logical state is |0..0>
        p0 = 1.0; p1 = 0.0;
    } else {
        p0 = s->host_scal[1]; p1 = s->host_scal[2];
    }
    return QOA_OK;
}

int do_reset_all(qoa_state_t s) {
    if (s->precision == QOA_PREC_F32) {
        CK(launch_f32_reset((float2*)s->amps, state_len(s), s->stream));
        CK(launch_set_scalar(s->scal, 1.0, s->stream));
        s->launches += 2;
        return QOA_OK;
    }
    GGate k;
    memset(&k, 0, sizeof k);
    k.kind = GG_RESET_ALL;
    CK(launch_gate(s->amps, state_len(s), k, s->stream));
    CK(launch_set_scalar(s->scal, 1.0, s->stream));
    s->launches += 2;
    return QOA_OK;
}

// measure (quantum_state.rs:399-458) with uniform u
int do_measure(qoa_state_t s, uint32_t q, double u, uint32_t* outcome) {
    double p0, p1, norm2;
    int rc = read_p01(s, q, p0, p1, norm2);
    if (rc) return rc;
    const uint32_t res = (u < p0) ? 0u : 1u;
    const double p = res ? p1 : p0;
    if (outcome) *outcome = res;
    if (!(p > 1e-12)) {
        // normalization_factor 0 zeroes the state; normalize() then resets it
        // to |0..0> (quantum_state.rs:431-443, 895-906)
        s->host_resets++;
        return do_reset_all(s);
    }
    const double f = 1.0 / std::sqrt(p);
    if (!(norm2 > 1e-12)) {
        rc = do_reset_all(s);
        if (rc) return rc;
        norm2 = 1.0;
    }
    CK(launch_collapse(s->amps, state_len(s), q, res, f / std::sqrt(norm2), s->partials, s->scal, s->status,
                       s->stream));
    s->launches += 2;
    return QOA_OK;
}

// apply_reset_simd (vectorization.rs:1020-1056)
int do_reset_qubit(qoa_state_t s, uint32_t q) {
    double p0, p1, norm2;
    int rc = read_p01(s, q, p0, p1, norm2);
    if (rc) return rc;
    if (!(norm2 > 1e-12)) return do_reset_all(s);
    if (p0 > 1e-12) {
        CK(launch_collapse(s->amps, state_len(s), q, 0, (1.0 / std::sqrt(p0)) / std::sqrt(norm2), s->partials,
                           s->scal, s->status, s->stream));
        s->launches += 2;
        return QOA_OK;
    }
    return do_reset_all(s);
}

double next_meas_uniform(qoa_state_t s) {
    return uniform01(s->seed, s->noise_stream ^ kMeasStreamXor, s->meas_draws++, 0);
}

// Packs an FP32 upload (block matrices, phase groups, angle lists, phases,
// tables) into one 256-byte-aligned image; off[] receives the offsets.
std::vector<unsigned char> f32_pack(const F32Upload& up, size_t off[5]) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    off[0] = 0;
    off[1] = al(off[0] + up.mats.size() * sizeof(float));
    off[2] = al(off[1] + up.pops.size() * sizeof(F32PhaseOp));
    off[3] = al(off[2] + up.angles.size() * sizeof(F32Angle));
    off[4] = al(off[3] + up.phases.size() * sizeof(F32Phase));
    const size_t total = al(off[4] + up.tables.size() * sizeof(float2)) + 256;
    std::vector<unsigned char> host(total, 0);
    auto put = [&](size_t o, const void* src, size_t bytes) { if (bytes) memcpy(host.data() + o, src, bytes); };
    put(off[0], up.mats.data(), up.mats.size() * sizeof(float));
    put(off[1], up.pops.data(), up.pops.size() * sizeof(F32PhaseOp));
    put(off[2], up.angles.data(), up.angles.size() * sizeof(F32Angle));
    put(off[3], up.phases.data(), up.phases.size() * sizeof(F32Phase));
    put(off[4], up.tables.data(), up.tables.size() * sizeof(float2));
    return host;
}

// FP32 precision form: every step must be a fused pass. Prepare builds all
// passes of an op list and uploads their block matrices and phases at once
// (synchronously); launch only enqueues kernels, so it can be captured.
int f32_prepare(qoa_state_t s, std::vector<Gate>& G) {
    for (const Gate& g : G)
        if (g.kind > K_U2)
            return set_err(s, QOA_E_OPCODE, "the FP32 precision form takes unitary ops only");
    if (s->n < (uint32_t)TILE_BITS) return set_err(s, QOA_E_ARG, "the FP32 precision form needs n >= %d", TILE_BITS);
    std::vector<Step> steps = schedule(G, s->n, false, true, s->pass_budget);
    s->f32_passes.assign(steps.size(), F32PassParams());
    F32Upload up;
    for (size_t i = 0; i < steps.size(); ++i) {
        if (!steps[i].pass) return set_err(s, QOA_E_OPCODE, "gate outside an FP32 pass");
        if (build_f32_pass(G, steps[i], s->n, s->f32_passes[i], up) != 0)
            return set_err(s, QOA_E_ARG, "FP32 pass %zu does not fit one launch", i);
    }
    std::vector<unsigned char> host = f32_pack(up, s->f32_off);
    const size_t total = host.size();
    CK(cudaStreamSynchronize(s->stream));
    if (total > s->f32_mats_cap) {
        if (s->f32_mats) cudaFree(s->f32_mats);
        s->f32_mats = nullptr;
        CK(cudaMalloc(&s->f32_mats, total));
        s->f32_mats_cap = total;
    }
    CK(cudaMemcpy(s->f32_mats, host.data(), total, cudaMemcpyHostToDevice));
    return QOA_OK;
}

int f32_launch(qoa_state_t s) {
    unsigned char* dev = (unsigned char*)s->f32_mats;
    const size_t* o = s->f32_off;
    for (const F32PassParams& P : s->f32_passes) {
        {
            Timer tm(s, 2.0 * std::ldexp(8.0, (int)s->n), 2);
            CK(launch_f32_pass((float2*)s->amps, P, (const float*)(dev + o[0]), (const F32PhaseOp*)(dev + o[1]),
                               (const F32Angle*)(dev + o[2]), (const F32Phase*)(dev + o[3]),
                               (const float2*)(dev + o[4]), s->scal, s->partials, s->status + 3, s->stream));
        }
        CK(launch_reduce_partials(s->partials, 1u << (s->n - TILE_BITS), s->scal, s->status, s->stream));
        s->launches += 2;
    }
    return QOA_OK;
}

int execute_f32(qoa_state_t s, std::vector<Gate>& G) {
    int rc = f32_prepare(s, G);
    if (rc) return rc;
    return f32_launch(s);
}

// Runs of at least three consecutive disjoint SWAPs (a QFT's final swap
// network) become one K_PERM step: a single in-place permutation pass instead
// of several tile passes that only relabel.
void merge_swap_blocks(std::vector<Gate>& G) {
    std::vector<Gate> out;
    out.reserve(G.size());
    size_t i = 0;
    while (i < G.size()) {
        size_t j = i;
        uint64_t used = 0;
        while (j < G.size() && G[j].kind == K_SWAP && G[j].cmask == 0 &&
               !(used & ((1ull << G[j].t) | (1ull << G[j].t2)))) {
            used |= (1ull << G[j].t) | (1ull << G[j].t2);
            ++j;
        }
        if (j - i >= 3) {
            Gate p;
            p.kind = K_PERM;
            for (int q = 0; q < 64; ++q) p.pi[q] = (uint8_t)q;
            for (size_t k = i; k < j; ++k) {
                p.pi[G[k].t] = (uint8_t)G[k].t2;
                p.pi[G[k].t2] = (uint8_t)G[k].t;
            }
            p.nmask = used;
            p.src = G[i].src;
            out.push_back(p);
            i = j;
        } else {
            out.push_back(G[i]);
            ++i;
        }
    }
    G.swap(out);
}

int run_perm(qoa_state_t s, const Gate& g) {
    const uint32_t n = s->n;
    PermParams P;
    memset(&P, 0, sizeof P);
    P.n = n;
    bool in_a[64] = {};
    const uint32_t low = std::min<uint32_t>(LANE_BITS, n);
    for (uint32_t q = 0; q < low; ++q) {
        P.tq[P.na++] = (uint8_t)q;
        in_a[q] = true;
    }
    for (uint32_t q = low; q < n; ++q)  // partners of the lane qubits, ascending
        for (uint32_t l = 0; l < low; ++l)
            if (g.pi[l] == q && !in_a[q]) {
                P.tq[P.na++] = (uint8_t)q;
                in_a[q] = true;
            }
    uint32_t no = 0;
    for (uint32_t q = 0; q < n; ++q)
        if (!in_a[q]) P.oq[no++] = (uint8_t)q;
    for (uint32_t q = 0; q < n; ++q) P.pi[q] = g.pi[q];
    for (uint32_t k = 0; k < P.na; ++k)
        for (uint32_t k2 = 0; k2 < P.na; ++k2)
            if (P.tq[k2] == g.pi[P.tq[k]]) P.src_bit[k] = (uint8_t)k2;
    const double bytes = 2.0 * std::ldexp(s->precision == QOA_PREC_F32 ? 8.0 : 16.0, (int)n);
    Timer tm(s, bytes, 4);
    CK(launch_swapnet(s->amps, s->precision == QOA_PREC_F32, P, s->stream));
    s->launches++;
    return QOA_OK;
}

// Max gates per tile pass of a state: its own setting, else QOA_PASS_GATES
// (tuning), else the scheduler's default.
int state_pass_budget(qoa_state_t s) {
    static const int env = [] {
        const char* v = getenv("QOA_PASS_GATES");
        return v ? std::max(0, atoi(v)) : 0;
    }();
    return s->pass_budget ? s->pass_budget : env;
}

int execute(qoa_state_t s, std::vector<Gate>& G) {
    const bool c64 = s->precision == QOA_PREC_F32;
    if (c64 && (s->flags & QOA_FLAG_F32_TENSOR)) return execute_f32(s, G);
    if (c64)
        for (const Gate& g : G)
            if (g.kind > K_U2 && g.kind != K_RESETALL)
                return set_err(s, QOA_E_OPCODE, "the FP32 precision form takes unitary ops only");
    const bool per_gate = (s->flags & QOA_FLAG_PER_GATE) != 0;
    // Split at QINIT (changes n) and run each segment through the scheduler.
    size_t i = 0;
    while (i < G.size()) {
        size_t j = i;
        while (j < G.size() && G[j].kind != K_QINIT) ++j;
        std::vector<Gate> seg(G.begin() + i, G.begin() + j);
        if (!per_gate) merge_swap_blocks(seg);
        const bool prebuild = !per_gate && s->jit_mode != QOA_JIT_OFF && s->n >= s->jit_min_qubits;
        // a repeated op list reuses its plan
        PlanEntry local;
        PlanEntry* pe = &local;
        bool cache_it = false;
        if (!per_gate && s->n > (uint32_t)TILE_BITS) {
            if (!s->plans) s->plans = std::make_shared<PlanCache>();
            PlanCache& pc = *static_cast<PlanCache*>(s->plans.get());
            const uint64_t key = (uint64_t)s->n | ((uint64_t)c64 << 8) | ((uint64_t)prebuild << 9) |
                                 ((uint64_t)(uint32_t)state_pass_budget(s) << 16);
            plan_hash(seg, key, local.h1, local.h2);
            for (auto& e : pc.entries)
                if (e.h1 == local.h1 && e.h2 == local.h2) pe = &e;
            if (pe == &local) {
                if (pc.seen.size() > 4096) pc.seen.clear();
                cache_it = pc.seen[local.h1]++ > 0;
            }
        }
        const bool fresh = pe == &local;
        if (fresh) {
            // the plan depends on the op list and the size only, so a list
            // executed again gives bit-identical results
            pe->steps = schedule(seg, s->n, per_gate, false, state_pass_budget(s),
                                 slot_search_pays(s->n) || (s->flags & QOA_FLAG_SLOT_SEARCH));
            pe->built_of.assign(pe->steps.size(), -1);
            // tile passes of a large state: built ahead, and their generated
            // kernels requested from the compile cache
            if (prebuild) {
                size_t np = 0;
                for (const Step& st : pe->steps) np += st.pass ? 1 : 0;
                pe->built.resize(np);
                size_t b = 0;
                for (size_t k = 0; k < pe->steps.size(); ++k) {
                    if (!pe->steps[k].pass || build_pass(seg, pe->steps[k], s->n, pe->built[b], c64) != 0) continue;
                    pe->built_of[k] = (int)b;
                    pe->bodies.push_back(c64 ? jit_pass32_body(pe->built[b]) : jit_pass_body(pe->built[b]));
                    ++b;
                }
                pe->prebuilt = true;
            }
            if (cache_it) {
                PlanCache& pc = *static_cast<PlanCache*>(s->plans.get());
                if (pc.entries.size() >= PlanCache::kEntries) pc.entries.pop_front();
                pc.entries.push_back(std::move(local));
                pe = &pc.entries.back();
            }
        }
        const std::vector<Step>& steps = pe->steps;
        const std::vector<PassParams>& built = pe->built;
        const std::vector<int>& built_of = pe->built_of;
        std::vector<JitKernel> jk;
        if (pe->prebuilt)
            jk = jit_request(pe->bodies, s->jit_mode == QOA_JIT_SYNC ? JitWhen::WAIT : JitWhen::SECOND_SIGHTING);
        for (size_t k = 0; k < steps.size(); ++k) {
            const Step& st = steps[k];
            int rc;
            if (st.pass && built_of[k] >= 0) rc = run_pass_built(s, built[built_of[k]], jk[built_of[k]]);
            else if (st.pass) rc = run_pass(s, seg, st);
            else {
                const Gate& g = seg[st.gates[0]];
                switch (g.kind) {
                    case K_MEASURE: {
                        const double u = g.u >= 0 ? g.u : next_meas_uniform(s);
                        rc = do_measure(s, (uint32_t)g.t, u, nullptr);
                        break;
                    }
                    case K_RESET: rc = do_reset_qubit(s, (uint32_t)g.t); break;
                    case K_RESETALL: rc = do_reset_all(s); break;
                    case K_PERM: rc = run_perm(s, g); break;
                    default: rc = run_gate(s, g);
                }
            }
            if (rc) return rc;
        }
        if (j < G.size()) {  // QINIT
            const uint32_t nn = (uint32_t)G[j].t;
            if (nn != s->n) {
                CK(cudaStreamSynchronize(s->stream));
                int rc = alloc_state(s, nn);
                if (rc) return rc;
            }
            int rc = do_reset_all(s);
            if (rc) return rc;
            ++j;
        }
        i = j;
    }
    return QOA_OK;
}

int check_handle(qoa_state_t s) {
    if (!s) return set_err(nullptr, QOA_E_ARG, "null handle");
    if (cudaSetDevice(s->device) != cudaSuccess) return set_err(s, QOA_E_CUDA, "cudaSetDevice failed");
    return QOA_OK;
}

// -------------------------------------------------------------- shims
std::mutex g_shim_mu;
double2* g_shim_buf = nullptr;
size_t g_shim_cap = 0;
double* g_shim_scr = nullptr;
cudaStream_t g_shim_stream = nullptr;
int g_shim_dev = -1;

int shim_begin(double* amps, size_t len, double2** dev) {
    qoa_state_t s = nullptr;
    if (!amps && len) return set_err(nullptr, QOA_E_ARG, "null amps");
    int dev_id = 0;
    CK(cudaGetDevice(&dev_id));
    if (g_shim_dev != dev_id) {
        g_shim_buf = nullptr; g_shim_cap = 0; g_shim_scr = nullptr; g_shim_stream = nullptr;
        g_shim_dev = dev_id;
    }
    if (!g_shim_stream) CK(cudaStreamCreateWithFlags(&g_shim_stream, cudaStreamNonBlocking));
    if (len > g_shim_cap) {
        if (g_shim_buf) cudaFree(g_shim_buf);
        if (g_shim_scr) cudaFree(g_shim_scr);
        g_shim_buf = nullptr; g_shim_scr = nullptr; g_shim_cap = 0;
        CK(cudaMalloc(&g_shim_buf, len * sizeof(double2)));
        CK(cudaMalloc(&g_shim_scr, (size_t)(2 * reduce_blocks(len) + 8) * sizeof(double)));
        g_shim_cap = len;
    }
    if (len) CK(cudaMemcpyAsync(g_shim_buf, amps, len * sizeof(double2), cudaMemcpyHostToDevice, g_shim_stream));
    *dev = g_shim_buf;
    return QOA_OK;
}
int shim_end(double* amps, size_t len) {
    qoa_state_t s = nullptr;
    if (len) CK(cudaMemcpyAsync(amps, g_shim_buf, len * sizeof(double2), cudaMemcpyDeviceToHost, g_shim_stream));
    CK(cudaStreamSynchronize(g_shim_stream));
    return QOA_OK;
}
int shim_gate(double* amps, size_t len, const GGate& k) {
    std::lock_guard<std::mutex> lk(g_shim_mu);
    qoa_state_t s = nullptr;
    double2* dev;
    int rc = shim_begin(amps, len, &dev);
    if (rc) return rc;
    if (len) CK(launch_gate(dev, len, k, g_shim_stream));
    return shim_end(amps, len);
}
GGate shim_g1(size_t t, int sub, double2 m0, double2 m1, double2 m2, double2 m3, uint64_t cm) {
    GGate k;
    memset(&k, 0, sizeof k);
    k.kind = GG_G1; k.sub = (uint8_t)sub; k.t = (uint8_t)t; k.cmask = cm;
    k.m[0] = m0; k.m[1] = m1; k.m[2] = m2; k.m[3] = m3;
    return k;
}
GGate shim_diag(int sel, double2 d0, double2 d1, uint64_t cm, bool neg) {
    GGate k;
    memset(&k, 0, sizeof k);
    k.kind = GG_DIAG; k.sub = neg ? 0x80 : 0; k.t = sel >= 0 ? (uint8_t)sel : 64; k.cmask = cm;
    k.m[0] = d0; k.m[1] = d1;
    return k;
}
// A bit index >= 64 makes every reference loop a no-op (no index has it).
inline bool shim_bit_ok(size_t b) { return b < 64; }

}  // namespace

// ================================================================ batching
// Many circuits in one go, by three routes:
//  - small: whole state in one CTA's shared memory; all such circuits in one
//    persistent launch (k_small_batch);
//  - arena: n >= the tile size and every step a tile pass; states packed in
//    one arena, and round r is ONE launch of k_pass_arena / k_f32_pass_arena
//    over the r-th pass of every circuit that has one (a circuit's first pass
//    synthesises |0..0>, so there is no reset launch);
//  - view: anything else (per-gate steps) runs through the engine's own
//    executor on a handle that views its slice of the arena, round-robin
//    over a pool of streams.
// All <Z_mask> results of the arena and view circuits come from one pair of
// launches over the arena. The first run executes eagerly and captures
// everything into a CUDA graph; later runs replay it.
enum BatchRoute { R_SMALL = 0, R_ARENA = 1, R_VIEW = 2 };
constexpr int kRoundStreams = 4;  // extra streams of a round's generated launches

struct qoa_batch_s {
    int precision = QOA_PREC_F64;
    uint32_t flags = 0;
    int device = 0;
    qoa_batch_tuning tune{};
    struct Circ {
        uint32_t n;
        std::vector<Gate> gates;
        std::vector<uint64_t> masks;
        uint32_t out_start;
        int route;
        size_t state_off;  // arena / view (and sampled small circuits): offset of the state in the arena
        uint32_t shots = 0;        // inverse-CDF shots of the final state
        uint64_t shot_start = 0;   // its uniforms in shot_u and its outcomes in the shot output
    };
    std::vector<Circ> circs;
    uint32_t nresults = 0;
    std::vector<double> shot_u;    // every sampled circuit's uniforms, in order of addition
    unsigned host_threads = 0;     // planning threads (0: all host cores)
    bool prepared = false;
    uint64_t runs = 0;
    // device
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    void* arena = nullptr;
    SmallCircuit* d_small = nullptr;
    SmallOp* d_ops = nullptr;
    uint64_t* d_masks = nullptr;   // every circuit's masks, in order of addition
    double* d_out = nullptr;
    unsigned int* d_counter = nullptr;
    uint32_t nsmall = 0;
    uint32_t small_max_n_used = 0;
    // arena route
    void* d_params = nullptr;      // PassParams[] or F32PassParams[]
    void* d_f32 = nullptr;         // FP32 upload shared by all arena circuits
    size_t f32_off[5] = {};
    ArenaJob* d_jobs = nullptr;
    uint32_t* d_tstart = nullptr;
    // one launch of a generated arena kernel: njobs jobs of one structure
    // from job_off, 2^lt tiles each
    struct Group { uint32_t job_off, njobs, lt; int kernel; int stream; };
    struct Round { uint32_t job_off, njobs, tiles; int max_nops, max_ncoef; std::vector<Group> groups; };
    std::vector<Round> rounds;
    std::vector<JitKernel> jit_kernels;  // by structure
    // a round's generated launches spread over stream 0 and these
    // (small groups would leave most SMs idle one after another)
    std::vector<cudaStream_t> rstreams;
    std::vector<cudaEvent_t> revents;    // [0] fork, [1 + i] join of rstreams[i]
    bool graph_jit = false;              // the captured graph launches the generated kernels
    double arena_pass_bytes = 0;   // algorithmic bytes of one run's arena passes
    uint32_t narena = 0;
    // expectation values of arena and view circuits
    ExpzJob* d_ejobs = nullptr;
    uint32_t n_ejobs = 0, e_chunks = 0;
    double* d_epart = nullptr;
    // sampled circuits (qoa_batch_add_trajectory)
    double* d_shot_u = nullptr;
    unsigned long long* d_shot_out = nullptr;
    SampleJob* d_sjobs = nullptr;
    double* d_trees = nullptr;
    uint32_t n_sjobs = 0;
    // host copy of the arena passes' parameters, kept (growing only) across
    // the batch's prepares: pinned for large batches, whose upload is then one
    // DMA at link speed rather than a staged pageable copy; pageable below
    // kPinnedMinPasses passes, where pinning pages (per batch handle, e.g.
    // each server worker's) costs more than the copy it speeds up
    PassParams* h_params = nullptr;
    size_t h_params_cap = 0;
    std::vector<PassParams> h_pageable;
    // view route
    std::vector<qoa_state_t> views;
    std::vector<int> view_circ;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string err;
};

namespace {

int bset_err(qoa_batch_t b, int code, const char* msg) {
    if (b) b->err = msg;
    note_global_error(msg);
    return code;
}

#define BCK(call)                                                                   \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            cudaGetLastError();                                                     \
            return bset_err(b, e_ == cudaErrorMemoryAllocation ? QOA_E_OOM : QOA_E_CUDA, \
                            cudaGetErrorString(e_));                                \
        }                                                                           \
    } while (0)

bool small_ok(const Gate& g) { return g.kind == K_G1 || g.kind == K_DIAG || g.kind == K_SWAP; }

SmallOp to_small(const Gate& g) {
    SmallOp o;
    memset(&o, 0, sizeof o);
    o.cmask = (uint32_t)g.cmask;
    if (g.kind == K_G1) {
        o.kind = SK_G1;
        o.t = (uint8_t)g.t;
        cplx m[4];
        g1_exact(g, m);
        for (int k = 0; k < 4; ++k) o.m[k] = d2(m[k].real(), m[k].imag());
    } else if (g.kind == K_DIAG) {
        o.kind = SK_DIAG;
        o.t = g.t >= 0 ? (uint8_t)g.t : 255;
        if (g.neg) o.m[0] = o.m[1] = d2(-1, 0);
        else {
            o.m[0] = g.m[0];
            o.m[1] = g.t >= 0 ? g.m[1] : g.m[0];
        }
    } else {
        o.kind = SK_SWAP;
        o.t = (uint8_t)g.t;
        o.t2 = (uint8_t)g.t2;
    }
    return o;
}

template <typename T>
void dfree(T*& p, cudaStream_t st) {
    if (p) cudaFreeAsync((void*)p, st);  // stream-ordered: no device-wide synchronisation
    p = nullptr;
}

// Pinned host buffers for batches' pass parameters, kept when a batch goes
// so that the next one (a fresh batch per request, a server chunk) skips the
// page pinning: up to four, the smallest dropped first.
std::mutex g_hp_mu;
std::vector<std::pair<PassParams*, size_t>> g_hp_free;
constexpr size_t kPinnedMinPasses = 16384;  // ~460 MB of pass parameters

cudaError_t pinned_params_take(size_t n, PassParams*& p, size_t& cap) {
    {
        std::lock_guard<std::mutex> lk(g_hp_mu);
        size_t best = g_hp_free.size();
        for (size_t i = 0; i < g_hp_free.size(); ++i)
            if (g_hp_free[i].second >= n && (best == g_hp_free.size() || g_hp_free[i].second < g_hp_free[best].second))
                best = i;
        if (best < g_hp_free.size()) {
            p = g_hp_free[best].first;
            cap = g_hp_free[best].second;
            g_hp_free.erase(g_hp_free.begin() + (long)best);
            return cudaSuccess;
        }
    }
    const cudaError_t e = cudaMallocHost((void**)&p, n * sizeof(PassParams));
    cap = e == cudaSuccess ? n : 0;
    if (e != cudaSuccess) p = nullptr;
    return e;
}

void pinned_params_give(PassParams* p, size_t cap) {
    PassParams* drop = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_hp_mu);
        g_hp_free.push_back({p, cap});
        if (g_hp_free.size() > 4) {
            size_t small = 0;
            for (size_t i = 1; i < g_hp_free.size(); ++i)
                if (g_hp_free[i].second < g_hp_free[small].second) small = i;
            drop = g_hp_free[small].first;
            g_hp_free.erase(g_hp_free.begin() + (long)small);
        }
    }
    if (drop) cudaFreeHost(drop);
}

// Device buffers of a batch: stream-ordered on the batch's first stream, from
// the device's batch pool (a freed batch's memory goes back to the pool
// without synchronising the device and serves the next batch, which matters
// when many batches come and go, as in the server's trajectory chunks).
template <typename T>
cudaError_t dalloc(qoa_batch_t b, T*& dst, size_t bytes) {
    void* p = nullptr;
    cudaMemPool_t pool = batch_pool(b->device);
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, b->streams[0])
                         : cudaMallocAsync(&p, bytes, b->streams[0]);
    if (e == cudaErrorMemoryAllocation && pool) {  // memory held elsewhere: retry once after a trim
        cudaGetLastError();
        trim_batch_pools();
        e = cudaMallocFromPoolAsync(&p, bytes, pool, b->streams[0]);
    }
    dst = static_cast<T*>(p);
    return e;
}

void batch_free_device(qoa_batch_t b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    for (qoa_state_t v : b->views) qoa_destroy(v);
    b->views.clear();
    b->view_circ.clear();
    // every stream of a run is joined into stream 0, so frees ordered there
    // follow all of the batch's work
    cudaStream_t st = b->streams.empty() ? nullptr : b->streams[0];
    dfree(b->arena, st); dfree(b->d_small, st); dfree(b->d_ops, st); dfree(b->d_masks, st); dfree(b->d_out, st);
    dfree(b->d_counter, st); dfree(b->d_params, st); dfree(b->d_f32, st); dfree(b->d_jobs, st); dfree(b->d_tstart, st);
    dfree(b->d_ejobs, st); dfree(b->d_epart, st);
    dfree(b->d_shot_u, st); dfree(b->d_shot_out, st); dfree(b->d_sjobs, st); dfree(b->d_trees, st);
    b->n_sjobs = 0;
    b->rounds.clear();
    b->jit_kernels.clear();
    b->graph_jit = false;
    b->arena_pass_bytes = 0;
    b->nsmall = b->narena = b->n_ejobs = b->e_chunks = 0;
    b->prepared = false;
    b->runs = 0;
}

template <typename T>
int upload(qoa_batch_t b, T*& dst, const std::vector<T>& src) {
    BCK(dalloc(b, dst, std::max<size_t>(1, src.size()) * sizeof(T)));
    if (!src.empty())
        BCK(cudaMemcpyAsync((void*)dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, b->streams[0]));
    return QOA_OK;
}

// fn(0) .. fn(count - 1) on `threads` host threads (0: all host cores, at
// most 64; 1: this thread)
void parallel_for(size_t count, const std::function<void(size_t)>& fn, unsigned threads = 0) {
    unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
    if (threads) nt = std::min(nt, threads);
    if (nt == 1 || count <= 1) {
        for (size_t k = 0; k < count; ++k) fn(k);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (size_t k; (k = next.fetch_add(1)) < count;) fn(k);
        });
    for (auto& th : pool) th.join();
}

// The parts of a PassParams that its generated kernel depends on (all but
// the coefficient values, the global phase and the angle values): passes
// that agree here share one generated kernel. build_pass zeroes unused
// fields, so whole arrays compare.
struct PassShape {
    const PassParams* P;
    size_t nangles() const { return P->nang ? P->ang_start[P->nang] : 0; }
    // the factored form of a rotation follows its angle: one shape for both
    static PassOp canon(PassOp o) {
        if (o.code >= PC_RXB && o.code < PC_RXB + 4) o.code = (uint8_t)(PC_RX + (o.code - PC_RXB));
        else if (o.code >= PC_RYB && o.code < PC_RYB + 4) o.code = (uint8_t)(PC_RY + (o.code - PC_RYB));
        return o;
    }
    uint64_t hash() const {
        uint64_t h = 1469598103934665603ull;
        auto mix = [&](const void* p, size_t nb) {
            const unsigned char* c = (const unsigned char*)p;
            for (size_t i = 0; i < nb; ++i) { h ^= c[i]; h *= 1099511628211ull; }
        };
        mix(&P->n, 3 * sizeof(uint32_t));
        mix(P->slot_qubit, offsetof(PassParams, ops) - offsetof(PassParams, slot_qubit));
        for (uint32_t k = 0; k < P->nops; ++k) {
            const PassOp o = canon(P->ops[k]);
            mix(&o, sizeof o);
        }
        for (size_t e = 0; e < nangles(); ++e) mix(&P->angles[e].omask, sizeof(uint64_t));
        return h;
    }
    bool operator==(const PassShape& o) const {
        const PassParams &a = *P, &b = *o.P;
        if (a.n != b.n || a.nops != b.nops || a.ncoef != b.ncoef) return false;
        if (memcmp(a.slot_qubit, b.slot_qubit, offsetof(PassParams, ops) - offsetof(PassParams, slot_qubit))) return false;
        for (uint32_t k = 0; k < a.nops; ++k) {
            const PassOp x = canon(a.ops[k]), y = canon(b.ops[k]);
            if (memcmp(&x, &y, sizeof x)) return false;
        }
        for (size_t e = 0; e < nangles(); ++e)
            if (a.angles[e].omask != b.angles[e].omask) return false;
        return true;
    }
};

int batch_prepare(qoa_batch_t b) {
    // streams first: the device buffers are allocated in stream 0's order
    const uint32_t nstreams = std::max<uint32_t>(1, b->tune.streams);
    while (b->streams.size() < nstreams) {
        cudaStream_t st;
        BCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        b->streams.push_back(st);
        cudaEvent_t ev;
        BCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->events.push_back(ev);
    }
    const bool f32 = b->precision == QOA_PREC_F32;
    const uint32_t cap = f32 ? SMALL_MAX_F32 : SMALL_MAX_F64;
    const uint32_t smax = std::min<uint32_t>(b->tune.small_max_n, cap);
    const int budget = (int)b->tune.pass_gate_budget;
    const size_t esz = f32 ? sizeof(float2) : sizeof(double2);
    const bool tensor = f32 && b->tune.f32_tensor;  // dense tensor-core blocks, else tile passes
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };

    std::vector<SmallCircuit> sc;
    std::vector<SmallOp> sops;
    std::vector<uint64_t> masks;
    std::vector<uint32_t> mask_start(b->circs.size());
    for (size_t i = 0; i < b->circs.size(); ++i) {
        mask_start[i] = (uint32_t)masks.size();
        masks.insert(masks.end(), b->circs[i].masks.begin(), b->circs[i].masks.end());
    }
    // arena route: every pass of every circuit, built on the host
    struct {
        PassParams* p = nullptr;
        size_t n = 0;
        size_t size() const { return n; }
        bool empty() const { return n == 0; }
        PassParams& operator[](size_t i) const { return p[i]; }
        const PassParams* data() const { return p; }
    } p64;
    std::vector<F32PassParams> p32;
    F32Upload up;
    std::vector<std::vector<uint32_t>> pass_idx(b->circs.size());
    uint32_t maxn = 1;
    size_t total = 0;  // arena bytes
    const size_t NC = b->circs.size();
    std::vector<char> is_small(NC, 0);
    for (size_t i = 0; i < NC; ++i) {
        const auto& c = b->circs[i];
        bool small = c.n <= smax || (tensor && c.n < (uint32_t)TILE_BITS);
        for (const Gate& g : c.gates) small = small && small_ok(g);
        is_small[i] = small;
    }
    // Tile-pass route, planned on all host cores: schedule every candidate
    // circuit, then build all passes into their final slots.
    std::vector<std::vector<Step>> steps_of(NC);
    std::vector<char> all_pass(NC, 0), built_ok(NC, 0);
    std::vector<size_t> pbase(NC, 0);
    if (!tensor) {
        parallel_for(NC, [&](size_t i) {
            const auto& c = b->circs[i];
            if (is_small[i] || c.n < (uint32_t)TILE_BITS || c.gates.empty()) return;
            steps_of[i] = schedule(c.gates, c.n, false, false, budget);
            bool ok = true;
            for (const Step& st : steps_of[i]) ok = ok && st.pass;
            all_pass[i] = ok;
        }, b->host_threads);
        size_t np = 0;
        std::vector<std::pair<size_t, size_t>> jobs;  // (circuit, step)
        for (size_t i = 0; i < NC; ++i)
            if (all_pass[i]) {
                pbase[i] = np;
                for (size_t k = 0; k < steps_of[i].size(); ++k) jobs.push_back({i, k});
                np += steps_of[i].size();
            }
        if (np >= kPinnedMinPasses) {
            if (np > b->h_params_cap) {
                if (b->h_params) pinned_params_give(b->h_params, b->h_params_cap);
                b->h_params = nullptr;
                b->h_params_cap = 0;
                BCK(pinned_params_take(np, b->h_params, b->h_params_cap));
            }
            p64.p = b->h_params;
        } else {
            if (b->h_pageable.size() < np) b->h_pageable.resize(np);
            p64.p = b->h_pageable.data();
        }
        p64.n = np;
        std::vector<char> step_ok(jobs.size(), 0);
        parallel_for(jobs.size(), [&](size_t x) {
            const size_t i = jobs[x].first, k = jobs[x].second;
            step_ok[x] = build_pass(b->circs[i].gates, steps_of[i][k], b->circs[i].n, p64[pbase[i] + k],
                                    b->precision == QOA_PREC_F32) == 0;
        }, b->host_threads);
        for (size_t i = 0; i < NC; ++i) built_ok[i] = all_pass[i];
        for (size_t x = 0; x < jobs.size(); ++x)
            if (!step_ok[x]) built_ok[jobs[x].first] = 0;
    }
    for (size_t i = 0; i < NC; ++i) {
        auto& c = b->circs[i];
        const bool small = is_small[i];
        if (small) {
            if (c.n > cap) return bset_err(b, QOA_E_ARG, "circuit too large for the shared-memory kernel");
            c.route = R_SMALL;
            SmallCircuit d;
            d.n = c.n;
            d.op_start = (uint32_t)sops.size();
            for (const Gate& g : c.gates) sops.push_back(to_small(g));
            d.op_count = (uint32_t)c.gates.size();
            d.mask_start = mask_start[i];
            d.mask_count = (uint32_t)c.masks.size();
            d.out_start = c.out_start;
            d.state_out = nullptr;  // set once the arena exists
            sc.push_back(d);
            maxn = std::max(maxn, c.n);
            if (c.shots) {  // its final state is sampled from the arena
                c.state_off = total;
                total = al(total + (esz << c.n));
            }
            continue;
        }
        if (tensor && c.n < (uint32_t)TILE_BITS)
            return bset_err(b, QOA_E_ARG, "circuit below the FP32 tile size with a gate the small kernel lacks");
        c.route = R_VIEW;
        if (!tensor) {
            if (built_ok[i]) {
                for (size_t k = 0; k < steps_of[i].size(); ++k) pass_idx[i].push_back((uint32_t)(pbase[i] + k));
                c.route = R_ARENA;
            }
        } else if (c.n >= (uint32_t)TILE_BITS && !c.gates.empty()) {
            std::vector<Step> steps = schedule(c.gates, c.n, false, tensor, budget);
            bool ok = true;
            for (const Step& st : steps) ok = ok && st.pass;
            if (ok) {
                const size_t base = p32.size();
                p32.resize(base + steps.size());
                for (size_t k = 0; k < steps.size(); ++k)
                    if (build_f32_pass(c.gates, steps[k], c.n, p32[base + k], up) != 0)
                        return bset_err(b, QOA_E_ARG, "FP32 pass does not fit one launch");
                for (size_t k = 0; k < steps.size(); ++k) pass_idx[i].push_back((uint32_t)(base + k));
            } else {
                return bset_err(b, QOA_E_OPCODE, "gate outside an FP32 pass");
            }
            c.route = R_ARENA;
        }
        c.state_off = total;
        total = al(total + (esz << c.n));
    }
    // view scratch (partials, scalars, status) after the states
    std::vector<size_t> view_off;
    for (auto& c : b->circs) {
        if (c.route != R_VIEW) continue;
        view_off.push_back(total);
        total = al(total + partials_needed(c.n) * sizeof(double));
        total = al(total + 16 * sizeof(double));
        total = al(total + 4 * sizeof(uint32_t));
    }
    // sampled circuits: marginal-tree scratch (2^n - 2 doubles each)
    std::vector<size_t> tree_off(NC, 0);
    size_t tree_total = 0;
    uint64_t shot_total = 0;
    for (size_t i = 0; i < NC; ++i) {
        const auto& c = b->circs[i];
        if (!c.shots) continue;
        tree_off[i] = tree_total;
        tree_total += c.n >= 2 ? (1ull << c.n) - 2 : 1;
        shot_total = std::max<uint64_t>(shot_total, c.shot_start + c.shots);
    }
    b->nsmall = (uint32_t)sc.size();
    b->small_max_n_used = maxn;
    BCK(dalloc(b, b->d_out, std::max<size_t>(1, b->nresults) * sizeof(double)));
    // [0] the small-circuit ticket counter, [1] the tensor passes' status word
    BCK(dalloc(b, b->d_counter, 2 * sizeof(unsigned int)));
    BCK(cudaMemsetAsync(b->d_counter, 0, 2 * sizeof(unsigned int), b->streams[0]));
    int rc;
    if ((rc = upload(b, b->d_masks, masks))) return rc;
    if (total) BCK(dalloc(b, b->arena, total));
    unsigned char* arena = (unsigned char*)b->arena;
    if (!sc.empty()) {
        size_t k = 0;
        for (size_t i = 0; i < NC; ++i) {
            if (b->circs[i].route != R_SMALL) continue;
            if (b->circs[i].shots) sc[k].state_out = arena + b->circs[i].state_off;
            ++k;
        }
        if ((rc = upload(b, b->d_small, sc))) return rc;
        if ((rc = upload(b, b->d_ops, sops))) return rc;
    }
    if (shot_total) {
        std::vector<SampleJob> sj;
        BCK(dalloc(b, b->d_trees, std::max<size_t>(1, tree_total) * sizeof(double)));
        for (size_t i = 0; i < NC; ++i) {
            const auto& c = b->circs[i];
            if (!c.shots) continue;
            SampleJob J;
            memset(&J, 0, sizeof J);
            J.amps = arena + c.state_off;
            J.tree = b->d_trees + tree_off[i];
            J.n = c.n;
            J.shots = c.shots;
            J.u_start = c.shot_start;
            J.out_start = c.shot_start;
            sj.push_back(J);
        }
        if ((rc = upload(b, b->d_sjobs, sj))) return rc;
        if ((rc = upload(b, b->d_shot_u, b->shot_u))) return rc;
        BCK(dalloc(b, b->d_shot_out, shot_total * sizeof(unsigned long long)));
        b->n_sjobs = (uint32_t)sj.size();
    }

    // arena rounds
    const size_t psz = tensor ? sizeof(F32PassParams) : sizeof(PassParams);
    if (tensor ? !p32.empty() : !p64.empty()) {
        BCK(dalloc(b, b->d_params, (tensor ? p32.size() : p64.size()) * psz));
        BCK(cudaMemcpyAsync(b->d_params, tensor ? (const void*)p32.data() : (const void*)p64.data(),
                            (tensor ? p32.size() : p64.size()) * psz, cudaMemcpyHostToDevice, b->streams[0]));
    }
    if (tensor && !p32.empty()) {
        std::vector<unsigned char> img = f32_pack(up, b->f32_off);
        BCK(dalloc(b, b->d_f32, img.size()));
        BCK(cudaMemcpyAsync(b->d_f32, img.data(), img.size(), cudaMemcpyHostToDevice, b->streams[0]));
    }
    std::vector<ArenaJob> jobs;
    std::vector<uint32_t> tstart;
    size_t maxp = 0;
    for (auto& v : pass_idx) maxp = std::max(maxp, v.size());
    // generated arena kernels: every distinct pass structure gets one; a
    // round's jobs are ordered by structure so that each structure's jobs
    // are one contiguous launch
    bool jit = !tensor && b->tune.jit != QOA_JIT_OFF && !p64.empty();
    std::vector<int> shape_of(p64.size(), -1);
    std::vector<uint32_t> reps;  // representative pass of each structure
    if (jit) {
        std::vector<uint64_t> hs(p64.size());
        parallel_for(p64.size(), [&](size_t k) { hs[k] = PassShape{&p64[k]}.hash(); }, b->host_threads);
        std::unordered_map<uint64_t, std::vector<int>> by_hash;
        for (auto& v : pass_idx)
            for (uint32_t pi : v) {
                auto& cands = by_hash[hs[pi]];
                int found = -1;
                for (int sid : cands)
                    if (PassShape{&p64[reps[sid]]} == PassShape{&p64[pi]}) { found = sid; break; }
                if (found < 0) {
                    found = (int)reps.size();
                    reps.push_back(pi);
                    cands.push_back(found);
                }
                shape_of[pi] = found;
            }
        // in the default mode a structure must serve at least 8 passes of
        // the batch to be worth its compile (~0.3 s of host time)
        size_t npass = 0;
        for (auto& v : pass_idx) npass += v.size();
        if (b->tune.jit == QOA_JIT_ASYNC && reps.size() * 8 > npass) jit = false;
    }
    if (jit) {
        std::vector<std::string> bodies(reps.size());
        parallel_for(reps.size(), [&](size_t k) {
            bodies[k] = f32 ? jit_pass32_body(p64[reps[k]], true) : jit_pass_body(p64[reps[k]], true);
        }, b->host_threads);
        b->jit_kernels = jit_request(bodies, b->tune.jit == QOA_JIT_SYNC ? JitWhen::WAIT : JitWhen::NOW);
    }
    for (size_t r = 0; r < maxp; ++r) {
        qoa_batch_s::Round R{(uint32_t)jobs.size(), 0, 0, 0, 0, {}};
        std::vector<size_t> order;
        for (size_t i = 0; i < b->circs.size(); ++i)
            if (pass_idx[i].size() > r) order.push_back(i);
        if (jit)
            std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
                return shape_of[pass_idx[x][r]] < shape_of[pass_idx[y][r]];
            });
        for (size_t i : order) {
            const auto& c = b->circs[i];
            const uint32_t pi = pass_idx[i][r];
            if (jit) {
                if (R.groups.empty() || R.groups.back().kernel != shape_of[pi])
                    R.groups.push_back({(uint32_t)jobs.size(), 0, c.n - (uint32_t)TILE_BITS, shape_of[pi], 0});
                R.groups.back().njobs++;
            }
            ArenaJob J;
            J.amps = arena + c.state_off;
            J.params = (const unsigned char*)b->d_params + (size_t)pi * psz;
            J.fresh = r == 0;
            J.pad_ = 0;
            jobs.push_back(J);
            tstart.push_back(R.tiles);
            R.tiles += 1u << (c.n - TILE_BITS);
            b->arena_pass_bytes += 2.0 * (double)esz * std::ldexp(1.0, (int)c.n);
            R.njobs++;
            if (!tensor) {
                R.max_nops = std::max(R.max_nops, (int)p64[pi].nops);
                R.max_ncoef = std::max(R.max_ncoef, (int)p64[pi].ncoef);
            }
        }
        if (R.groups.size() > 1) {
            // longest-processing-time-first over 1 + kRoundStreams streams
            std::vector<size_t> idx(R.groups.size());
            for (size_t g = 0; g < idx.size(); ++g) idx[g] = g;
            auto work = [&](size_t g) { return (double)R.groups[g].njobs * std::ldexp(1.0, (int)R.groups[g].lt); };
            std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return work(x) > work(y); });
            double load[1 + kRoundStreams] = {};
            for (size_t g : idx) {
                int best = 0;
                for (int k = 1; k <= kRoundStreams; ++k)
                    if (load[k] < load[best]) best = k;
                R.groups[g].stream = best;
                load[best] += work(g);
            }
        }
        b->rounds.push_back(R);
    }
    for (auto& v : pass_idx) b->narena += v.empty() ? 0u : 1u;
    if (!jobs.empty()) {
        if ((rc = upload(b, b->d_jobs, jobs))) return rc;
        if ((rc = upload(b, b->d_tstart, tstart))) return rc;
    }

    // expectation values of every arena and view circuit
    std::vector<ExpzJob> ej;
    uint32_t chunks = 0;
    uint64_t parts = 0;
    for (size_t i = 0; i < b->circs.size(); ++i) {
        const auto& c = b->circs[i];
        if (c.route == R_SMALL || c.masks.empty()) continue;
        if (c.masks.size() > EXPZ_MAX_MASKS) return bset_err(b, QOA_E_ARG, "more than 255 masks on one circuit");
        ExpzJob J;
        memset(&J, 0, sizeof J);
        J.amps = arena + c.state_off;
        J.n = c.n;
        J.mask_start = mask_start[i];
        J.mask_count = (uint32_t)c.masks.size();
        J.out_start = c.out_start;
        J.chunk_start = chunks;
        J.part_start = parts;
        const uint32_t nch = (uint32_t)(((1ull << c.n) + EXPZ_CHUNK - 1) / EXPZ_CHUNK);
        chunks += nch;
        parts += (uint64_t)nch * (J.mask_count + 1);
        ej.push_back(J);
    }
    b->n_ejobs = (uint32_t)ej.size();
    b->e_chunks = chunks;
    if (!ej.empty()) {
        if ((rc = upload(b, b->d_ejobs, ej))) return rc;
        BCK(dalloc(b, b->d_epart, parts * sizeof(double)));
    }

    if (jit && b->rstreams.empty()) {
        cudaEvent_t ev;
        BCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->revents.push_back(ev);
        for (int k = 0; k < kRoundStreams; ++k) {
            cudaStream_t st;
            BCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            b->rstreams.push_back(st);
            BCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            b->revents.push_back(ev);
        }
    }

    const uint32_t ns = (uint32_t)b->streams.size();

    // view handles
    size_t k = 0;
    for (size_t i = 0; i < b->circs.size(); ++i) {
        auto& c = b->circs[i];
        if (c.route != R_VIEW) continue;
        unsigned char* base = arena + view_off[k];
        qoa_state_t v = new qoa_state_s();
        v->view = true;
        v->n = c.n;
        v->flags = (b->flags & QOA_FLAG_COMPAT_MASK_QUIRK) | (tensor ? QOA_FLAG_F32_TENSOR : 0u);
        v->precision = b->precision;
        v->device = b->device;
        v->pass_budget = budget;
        v->stream = b->streams[k % ns];
        v->amps = (double2*)(arena + c.state_off);
        size_t o = 0;
        v->partials = (double*)(base + o);
        v->partials_cap = partials_needed(c.n);
        o = al(o + v->partials_cap * sizeof(double));
        v->scal = (double*)(base + o);
        o = al(o + 16 * sizeof(double));
        v->status = (uint32_t*)(base + o);
        BCK(cudaMemsetAsync(v->status, 0, 4 * sizeof(uint32_t), b->streams[0]));
        if (tensor) {
            rc = f32_prepare(v, c.gates);
            if (rc) { std::string m = v->err; qoa_destroy(v); return bset_err(b, rc, m.c_str()); }
        }
        b->views.push_back(v);
        b->view_circ.push_back((int)i);
        ++k;
    }
    b->prepared = true;
    return QOA_OK;
}

// Enqueues one full batch on stream 0 (forking to the pool and joining).
int batch_enqueue(qoa_batch_t b) {
    const bool f32 = b->precision == QOA_PREC_F32;
    cudaStream_t s0 = b->streams[0];
    const uint32_t ns = (uint32_t)b->streams.size();
    BCK(cudaEventRecord(b->events[0], s0));
    for (uint32_t i = 1; i < ns; ++i) BCK(cudaStreamWaitEvent(b->streams[i], b->events[0], 0));
    // small circuits beside the arena rounds
    if (b->nsmall) {
        BCK(launch_small_batch(f32, b->d_small, b->nsmall, b->d_ops, b->d_masks, b->d_out, b->d_counter,
                               (int)b->small_max_n_used, (int)b->tune.small_threads, (int)b->tune.small_ctas_per_sm,
                               b->streams[ns > 1 ? 1 : 0]));
    }
    for (size_t k = 0; k < b->views.size(); ++k) {
        qoa_state_t v = b->views[k];
        auto& c = b->circs[b->view_circ[k]];
        int rc = do_reset_all(v);
        if (!rc) rc = (v->flags & QOA_FLAG_F32_TENSOR) ? f32_launch(v) : execute(v, c.gates);
        if (rc) return bset_err(b, rc, v->err.c_str());
    }
    const unsigned char* fb = (const unsigned char*)b->d_f32;
    const bool tensor = f32 && b->tune.f32_tensor;
    bool all_ready = !b->jit_kernels.empty();
    for (const auto& k : b->jit_kernels) all_ready = all_ready && k.ready();
    for (const auto& R : b->rounds) {
        if (all_ready && !R.groups.empty()) {
            const bool fork = R.groups.size() > 1 && !b->rstreams.empty();
            if (fork) {
                BCK(cudaEventRecord(b->revents[0], s0));
                for (cudaStream_t st : b->rstreams) BCK(cudaStreamWaitEvent(st, b->revents[0], 0));
            }
            for (const auto& Gp : R.groups) {
                cudaStream_t st = (fork && Gp.stream > 0) ? b->rstreams[Gp.stream - 1] : s0;
                BCK(b->jit_kernels[Gp.kernel].launch_arena(b->d_jobs + Gp.job_off, Gp.njobs, Gp.lt, st));
            }
            if (fork)
                for (size_t k = 0; k < b->rstreams.size(); ++k) {
                    BCK(cudaEventRecord(b->revents[1 + k], b->rstreams[k]));
                    BCK(cudaStreamWaitEvent(s0, b->revents[1 + k], 0));
                }
            continue;
        }
        if (tensor)
            BCK(launch_f32_pass_arena(b->d_jobs + R.job_off, R.njobs, b->d_tstart + R.job_off, R.tiles,
                                      (const float*)(fb + b->f32_off[0]), (const F32PhaseOp*)(fb + b->f32_off[1]),
                                      (const F32Angle*)(fb + b->f32_off[2]), (const F32Phase*)(fb + b->f32_off[3]),
                                      (const float2*)(fb + b->f32_off[4]), b->d_counter + 1, s0));
        else if (f32)
            BCK(launch_pass_p32_arena(b->d_jobs + R.job_off, R.njobs, b->d_tstart + R.job_off, R.tiles,
                                      R.max_nops, R.max_ncoef, s0));
        else
            BCK(launch_pass_arena(b->d_jobs + R.job_off, R.njobs, b->d_tstart + R.job_off, R.tiles,
                                  R.max_nops, R.max_ncoef, s0));
    }
    for (uint32_t i = 1; i < ns; ++i) {
        BCK(cudaEventRecord(b->events[i], b->streams[i]));
        BCK(cudaStreamWaitEvent(s0, b->events[i], 0));
    }
    BCK(launch_arena_expz(f32, b->d_ejobs, b->n_ejobs, b->e_chunks, b->d_masks, b->d_epart, b->d_out, s0));
    BCK(launch_sample_jobs(f32, b->d_sjobs, b->n_sjobs, b->d_shot_u, b->d_shot_out, s0));
    b->graph_jit = all_ready;
    return QOA_OK;
}

bool batch_jit_all_ready(qoa_batch_t b) {
    if (b->jit_kernels.empty()) return false;
    for (const auto& k : b->jit_kernels)
        if (!k.ready()) return false;
    return true;
}

// Drops a graph captured with interpreter passes once the generated kernels
// are all loaded (the next run captures again).
int batch_refresh_graph(qoa_batch_t b) {
    if (!b->exec || b->graph_jit || !batch_jit_all_ready(b)) return QOA_OK;
    BCK(cudaStreamSynchronize(b->streams[0]));
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    return QOA_OK;
}

}  // namespace

// ==================================================================== C ABI
namespace qoa {
// The serde-only fields above, for qoa_checkpoint.cpp.
struct JsonExtras {
    bool noise_none;
    bool div_by_zero;
    std::vector<double> regs;
};
JsonExtras json_extras(qoa_state_t s) { return JsonExtras{s->noise_none, s->div_by_zero, s->json_regs}; }
int set_json_extras(qoa_state_t s, const JsonExtras& x, bool nan, bool overflow) {
    s->noise_none = x.noise_none;
    s->div_by_zero = x.div_by_zero;
    s->json_regs = x.regs;
    const uint32_t w[2] = {nan ? 1u : 0u, overflow ? 1u : 0u};
    CK(cudaMemcpyAsync(s->status, w, sizeof w, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return QOA_OK;
}
}  // namespace qoa

extern "C" {

const char* qoa_strerror(int code) {
    switch (code) {
        case QOA_OK: return "ok";
        case QOA_E_RANGE: return "qubit index out of range (op skipped)";
        case QOA_E_ARG: return "invalid argument";
        case QOA_E_OPCODE: return "unsupported opcode";
        case QOA_E_CUDA: return "CUDA error";
        case QOA_E_OOM: return "device out of memory";
        case QOA_E_STATE: return "numerical status";
        case QOA_E_NOGPU: return "no CUDA device";
        default: return "unknown";
    }
}

const char* qoa_last_error(qoa_state_t s) {
    if (s) return s->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_err.c_str();
}

int qoa_create(uint32_t n, int precision, uint32_t flags, qoa_state_t* out) {
    qoa_state_t s = nullptr;
    if (!out) return set_err(nullptr, QOA_E_ARG, "null out");
    *out = nullptr;
    if (precision != QOA_PREC_F64 && precision != QOA_PREC_F32)
        return set_err(nullptr, QOA_E_ARG, "unsupported precision %d", precision);
    if (precision == QOA_PREC_F32 && (flags & QOA_FLAG_F32_TENSOR) && n < (uint32_t)TILE_BITS)
        return set_err(nullptr, QOA_E_ARG, "the tensor-core block form needs n >= %d", TILE_BITS);
    if (n < 1) n = 1;
    if (n > 40) return set_err(nullptr, QOA_E_ARG, "n=%u qubits exceeds the engine limit", n);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(nullptr, QOA_E_NOGPU, "no CUDA device");
    s = new qoa_state_s();
    s->flags = flags;
    s->precision = precision;
    cudaGetDevice(&s->device);
    auto fail = [&](int rc) {
        cudaGetLastError();  // do not leave the failure as this thread's last error
        std::string m = s->err;
        qoa_destroy(s);
        set_err(nullptr, rc, "%s", m.c_str());
        return rc;
    };
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_err(s, QOA_E_CUDA, "stream create failed"));
    if (cudaMalloc(&s->scal, 16 * sizeof(double)) != cudaSuccess) return fail(set_err(s, QOA_E_OOM, "scalar alloc"));
    if (cudaMalloc(&s->status, 4 * sizeof(uint32_t)) != cudaSuccess) return fail(set_err(s, QOA_E_OOM, "status alloc"));
    if (cudaMemsetAsync(s->status, 0, 4 * sizeof(uint32_t), s->stream) != cudaSuccess)
        return fail(set_err(s, QOA_E_CUDA, "status memset"));
    if (cudaMallocHost(&s->host_scal, 16 * sizeof(double)) != cudaSuccess) return fail(set_err(s, QOA_E_OOM, "pinned alloc"));
    int rc = alloc_state(s, n);
    if (rc) return fail(rc);
    rc = do_reset_all(s);
    if (rc) return fail(rc);
    *out = s;
    return QOA_OK;
}

int qoa_destroy(qoa_state_t s) {
    if (!s) return QOA_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->view) {  // batch view: only its own FP32 arena
        if (s->f32_mats) cudaFree(s->f32_mats);
        delete s;
        return QOA_OK;
    }
    for (auto& r : s->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    if (s->amps) cudaFree(s->amps);
    if (s->f32_mats) cudaFree(s->f32_mats);
    if (s->f32_phases) cudaFree(s->f32_phases);
    if (s->partials) cudaFree(s->partials);
    if (s->scal) cudaFree(s->scal);
    if (s->status) cudaFree(s->status);
    if (s->host_scal) cudaFreeHost(s->host_scal);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return QOA_OK;
}

int qoa_num_qubits(qoa_state_t s, uint32_t* n) {
    if (!s || !n) return set_err(s, QOA_E_ARG, "null argument");
    *n = s->n;
    return QOA_OK;
}

int qoa_reset_all(qoa_state_t s) {
    int rc = check_handle(s);
    if (rc) return rc;
    return do_reset_all(s);
}

int qoa_apply(qoa_state_t s, const qoa_op* ops, size_t nops) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (!ops && nops) return set_err(s, QOA_E_ARG, "null ops");
    Expander ex;
    ex.n = s->n;
    ex.flags = s->flags;
    ex.s = s;
    ex.out.reserve(nops * 2 + 8);
    for (size_t i = 0; i < nops; ++i) {
        ex.cur = (int)i;
        ex.op(ops[i]);
    }
    rc = execute(s, ex.out);
    if (rc) return rc;
    if (ex.first_err != QOA_OK) return set_err(s, ex.first_err, "%s", ex.err.c_str());
    return QOA_OK;
}

int qoa_measure(qoa_state_t s, uint32_t q, double u, uint32_t* outcome) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (s->precision == QOA_PREC_F32) return set_err(s, QOA_E_ARG, "not available for an FP32 handle");
    if (q >= s->n) return set_err(s, QOA_E_RANGE, "qubit index %u out of bounds", q);
    if (u < 0) u = next_meas_uniform(s);
    rc = do_measure(s, q, u, outcome);
    if (rc) return rc;
    // apply_noise after the measurement (quantum_state.rs:455)
    Expander ex;
    ex.n = s->n; ex.flags = s->flags; ex.s = s; ex.cur = -1;
    ex.noise_event(1ull << q);
    return execute(s, ex.out);
}

int qoa_sample(qoa_state_t s, const double* u, size_t shots, int mode, uint64_t* out) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (!u || !out || (mode != 0 && mode != 1)) return set_err(s, QOA_E_ARG, "bad sample arguments");
    if (shots == 0) return QOA_OK;
    const uint32_t n = s->n;
    const size_t nu = mode == 0 ? shots * n : shots;
    double* d_tree = nullptr;
    double* d_u = nullptr;
    unsigned long long* d_out = nullptr;
    const size_t tree_len = (n >= 2) ? ((1ull << n) - 2) : 1;
    CK(cudaMallocAsync(&d_tree, tree_len * sizeof(double), s->stream));
    CK(cudaMallocAsync(&d_u, nu * sizeof(double), s->stream));
    CK(cudaMallocAsync(&d_out, shots * sizeof(unsigned long long), s->stream));
    CK(cudaMemcpyAsync(d_u, u, nu * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    const bool f32 = s->precision == QOA_PREC_F32;
    CK(launch_tree(s->amps, f32, n, s->scal, d_tree, s->stream));
    CK(launch_sample(s->amps, f32, n, s->scal, d_tree, d_u, shots, mode, d_out, s->stream));
    s->launches += (n >= 2 ? (n - 1) : 0) + 1;
    CK(cudaMemcpyAsync(out, d_out, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaFreeAsync(d_tree, s->stream));
    CK(cudaFreeAsync(d_u, s->stream));
    CK(cudaFreeAsync(d_out, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return QOA_OK;
}

int qoa_probabilities(qoa_state_t s, double* out) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (!out) return set_err(s, QOA_E_ARG, "null out");
    const uint64_t len = state_len(s);
    const uint64_t chunk = std::min<uint64_t>(len, 1ull << 24);
    double* d = nullptr;
    CK(cudaMallocAsync(&d, chunk * sizeof(double), s->stream));
    for (uint64_t off = 0; off < len; off += chunk) {
        const uint64_t cnt = std::min(chunk, len - off);
        if (s->precision == QOA_PREC_F32)
            CK(launch_f32_probs((const float2*)s->amps, off, cnt, s->scal, d, s->stream));
        else
            CK(launch_probs(s->amps, off, cnt, s->scal, d, s->stream));
        s->launches++;
        CK(cudaMemcpyAsync(out + off, d, cnt * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    }
    CK(cudaFreeAsync(d, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return QOA_OK;
}

int qoa_expect_z(qoa_state_t s, const uint64_t* masks, size_t k, double* out) {
    int rc = check_handle(s);
    if (rc) return rc;
    if ((!masks || !out) && k) return set_err(s, QOA_E_ARG, "null argument");
    for (size_t i = 0; i < k; i += 8) {
        const uint32_t kk = (uint32_t)std::min<size_t>(8, k - i);
        if (s->precision == QOA_PREC_F32)  // FP64 sums over the complex64 state
            CK(launch_f32_expz((const float2*)s->amps, state_len(s), masks + i, kk, s->partials, s->scal + 8,
                               s->scal, s->stream));
        else
            CK(launch_expz(s->amps, state_len(s), masks + i, kk, s->partials, s->scal + 8, s->scal, s->stream));
        s->launches += 2;
        CK(cudaMemcpyAsync(s->host_scal + 8, s->scal + 8, kk * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        for (uint32_t j = 0; j < kk; ++j) out[i + j] = s->host_scal[8 + j];
    }
    return QOA_OK;
}

int qoa_get_state(qoa_state_t s, void* host, size_t bytes) {
    int rc = check_handle(s);
    if (rc) return rc;
    const size_t esz = s->precision == QOA_PREC_F32 ? sizeof(float2) : sizeof(double2);
    if (!host || bytes != state_len(s) * esz)
        return set_err(s, QOA_E_ARG, "get_state needs %llu bytes", (unsigned long long)(state_len(s) * esz));
    if (s->precision == QOA_PREC_F32)
        CK(launch_f32_materialize((float2*)s->amps, state_len(s), s->scal, s->partials, s->status, s->stream));
    else
        CK(launch_materialize(s->amps, state_len(s), s->scal, s->partials, s->status, s->stream));
    s->launches += 2;
    CK(cudaMemcpyAsync(host, s->amps, bytes, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return QOA_OK;
}

int qoa_set_state(qoa_state_t s, const void* host, size_t bytes) {
    int rc = check_handle(s);
    if (rc) return rc;
    const size_t esz = s->precision == QOA_PREC_F32 ? sizeof(float2) : sizeof(double2);
    if (!host || bytes != state_len(s) * esz)
        return set_err(s, QOA_E_ARG, "set_state needs %llu bytes", (unsigned long long)(state_len(s) * esz));
    CK(cudaMemcpyAsync(s->amps, host, bytes, cudaMemcpyHostToDevice, s->stream));
    if (s->precision == QOA_PREC_F32)
        CK(launch_f32_norm((const float2*)s->amps, state_len(s), s->partials, s->scal, nullptr, s->stream));
    else
        CK(launch_norm(s->amps, state_len(s), s->partials, s->scal, nullptr, s->stream));
    s->launches += 2;
    // set_state_vector normalises at once (quantum_state.rs:1143): a zero or
    // NaN vector becomes |0..0> before any gate sees it.
    CK(cudaMemcpyAsync(s->host_scal, s->scal, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (!(s->host_scal[0] > 1e-12)) {
        s->host_resets++;
        return do_reset_all(s);
    }
    return QOA_OK;
}

int qoa_set_random_state(qoa_state_t s, uint64_t seed) {
    int rc = check_handle(s);
    if (rc) return rc;
    const bool f32 = s->precision == QOA_PREC_F32;
    CK(launch_random_state(s->amps, f32, state_len(s), seed, s->stream));
    if (f32) CK(launch_f32_norm((const float2*)s->amps, state_len(s), s->partials, s->scal, nullptr, s->stream));
    else CK(launch_norm(s->amps, state_len(s), s->partials, s->scal, nullptr, s->stream));
    s->launches += 3;
    CK(cudaStreamSynchronize(s->stream));
    return QOA_OK;
}

int qoa_compare(qoa_state_t a, qoa_state_t b, double* rel_l2, double* infidelity) {
    qoa_state_t s = a;  // error reporting
    int rc = check_handle(a);
    if (rc) return rc;
    if (!b || a->n != b->n || a->device != b->device) return set_err(a, QOA_E_ARG, "states differ in size or device");
    CK(cudaStreamSynchronize(b->stream));
    CK(launch_compare(a->amps, a->precision == QOA_PREC_F32, b->amps, b->precision == QOA_PREC_F32, state_len(a),
                      a->scal, b->scal, a->partials, a->scal + 8, a->stream));
    a->launches += 2;
    double h[3];
    CK(cudaMemcpyAsync(h, a->scal + 8, sizeof h, cudaMemcpyDeviceToHost, a->stream));
    CK(cudaStreamSynchronize(a->stream));
    if (rel_l2) *rel_l2 = std::sqrt(std::max(h[0], 0.0));
    if (infidelity) *infidelity = 1.0 - (h[1] * h[1] + h[2] * h[2]);
    return QOA_OK;
}

int qoa_seed(qoa_state_t s, uint64_t seed) {
    if (!s) return set_err(nullptr, QOA_E_ARG, "null handle");
    s->seed = seed;
    s->noise_event = 0;
    s->meas_draws = 0;
    return QOA_OK;
}

int qoa_set_noise(qoa_state_t s, int mode, double p) {
    if (!s) return set_err(nullptr, QOA_E_ARG, "null handle");
    if (mode < 0 || mode > 3 || (mode == 1 && !(p >= 0.0 && p <= 1.0))) return set_err(s, QOA_E_ARG, "bad noise config");
    s->noise_none = mode == 3;  // Option::None: no noise, like Ideal
    s->noise_mode = mode == 3 ? 0 : mode;
    s->noise_p = mode == 1 ? p : 0.0;
    return QOA_OK;
}

int qoa_set_trajectory(qoa_state_t s, uint64_t stream) {
    if (!s) return set_err(nullptr, QOA_E_ARG, "null handle");
    s->noise_stream = stream;
    s->noise_event = 0;
    return QOA_OK;
}

int qoa_status(qoa_state_t s, qoa_status_t* out) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (!out) return set_err(s, QOA_E_ARG, "null out");
    uint32_t h[4];
    CK(cudaMemcpyAsync(h, s->status, sizeof h, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    out->nan_seen = h[0];
    out->inf_seen = h[1];
    out->zero_norm_resets = h[2] + s->host_resets;
    out->copy_timeouts = h[3];
    return QOA_OK;
}

int qoa_sync(qoa_state_t s) {
    int rc = check_handle(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    return QOA_OK;
}

int qoa_stream(qoa_state_t s, void** stream) {
    if (!s || !stream) return set_err(s, QOA_E_ARG, "null argument");
    *stream = (void*)s->stream;
    return QOA_OK;
}

int qoa_launch_count(qoa_state_t s, uint64_t* count) {
    if (!s || !count) return set_err(s, QOA_E_ARG, "null argument");
    *count = s->launches;
    return QOA_OK;
}

int qoa_launch_times(qoa_state_t s, double* ms, double* bytes, int* kind, size_t cap, size_t* n) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (!n) return set_err(s, QOA_E_ARG, "null n");
    CK(cudaStreamSynchronize(s->stream));
    size_t k = 0;
    for (auto& r : s->recs) {
        if (k < cap) {
            float t = 0.f;
            cudaEventElapsedTime(&t, r.a, r.b);
            if (ms) ms[k] = t;
            if (bytes) bytes[k] = r.bytes;
            if (kind) kind[k] = r.kind;
            ++k;
        }
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    s->recs.clear();
    *n = k;
    return QOA_OK;
}

int qoa_plan(uint32_t n, uint32_t flags, const qoa_op* ops, size_t nops, size_t cap, int32_t* pass_of,
             int32_t* order, int32_t* gate_kind, uint32_t* gate_qubits, double* gate_matrix, size_t* ngates,
             size_t* npasses) {
    if ((!ops && nops) || !ngates || !npasses) return set_err(nullptr, QOA_E_ARG, "null argument");
    Expander ex;
    ex.n = std::max<uint32_t>(n, 1);
    ex.flags = flags;
    ex.s = nullptr;
    for (size_t i = 0; i < nops; ++i) {
        ex.cur = (int)i;
        ex.op(ops[i]);
    }
    const std::vector<Gate>& G = ex.out;
    for (const Gate& g : G)
        if (g.kind == K_QINIT) return set_err(nullptr, QOA_E_ARG, "qoa_plan does not take QINIT");
    std::vector<Step> steps = schedule(G, ex.n, (flags & QOA_FLAG_PER_GATE) != 0, false, 0,
                                       slot_search_pays(ex.n) || (flags & QOA_PLAN_SLOT_SEARCH));
    *ngates = G.size();
    *npasses = steps.size();
    if (G.size() > cap) return set_err(nullptr, QOA_E_ARG, "cap too small: %zu gates", G.size());
    for (size_t si = 0; si < steps.size(); ++si) {
        for (size_t k = 0; k < steps[si].gates.size(); ++k) {
            const int gi = steps[si].gates[k];
            if (pass_of) pass_of[gi] = (int32_t)si;
            if (order) order[gi] = (int32_t)k;
        }
        if (steps[si].pass) {  // make sure the kernel op stream builds
            static thread_local PassParams P;
            if (build_pass(G, steps[si], ex.n, P, false) != 0)
                return set_err(nullptr, QOA_E_ARG, "pass %zu does not fit one launch", si);
            if (getenv("QOA_PLAN_STATS")) {  // op mix of each pass, for tuning
                int cnt[PC_NCODES] = {};
                for (uint32_t o = 0; o < P.nops; ++o) cnt[P.ops[o].code < PC_NCODES ? P.ops[o].code : 0]++;
                int g1 = 0;
                for (int c = PC_HF; c < PC_DIAG_TA; ++c) g1 += cnt[c];
                const int disp = (int)P.nops - cnt[PC_NOP];
                fprintf(stderr, "pass %zu: gates %zu dispatches %d g1 %d tm %d mx %d (entries %d) tab %d diag_m %d xchg %d flush %d ang_ops %d (entries %d)\n",
                        si, steps[si].gates.size(), disp, g1, cnt[PC_DIAG_TM], cnt[PC_DIAG_MX], cnt[PC_NOP],
                        cnt[PC_DIAG_TAB], cnt[PC_DIAG_M], cnt[PC_XCHG], cnt[PC_FLUSH], (int)P.nang,
                        (int)P.ang_start[P.nang]);
            }
        }
    }
    for (size_t gi = 0; gi < G.size(); ++gi) {
        const Gate& g = G[gi];
        if (gate_kind) gate_kind[gi] = g.kind * 16 + (g.kind == K_G1 ? g.sub : (g.neg ? 1 : 0));
        if (gate_qubits) {
            gate_qubits[4 * gi + 0] = (uint32_t)g.t;
            gate_qubits[4 * gi + 1] = (uint32_t)g.t2;
            gate_qubits[4 * gi + 2] = (uint32_t)g.cmask;
            gate_qubits[4 * gi + 3] = (uint32_t)(g.cmask >> 32);
        }
        if (gate_matrix)
            for (int k = 0; k < 16; ++k) {
                gate_matrix[32 * gi + 2 * k] = g.m[k].x;
                gate_matrix[32 * gi + 2 * k + 1] = g.m[k].y;
            }
    }
    return QOA_OK;
}


// ---- batching form ------------------------------------------------------------
int qoa_batch_create(int precision, uint32_t flags, qoa_batch_t* out) {
    if (!out) return set_err(nullptr, QOA_E_ARG, "null out");
    *out = nullptr;
    if (precision != QOA_PREC_F64 && precision != QOA_PREC_F32)
        return set_err(nullptr, QOA_E_ARG, "unsupported precision %d", precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(nullptr, QOA_E_NOGPU, "no CUDA device");
    qoa_batch_t b = new qoa_batch_s();
    b->precision = precision;
    b->flags = flags;
    cudaGetDevice(&b->device);
    b->tune.small_max_n = precision == QOA_PREC_F32 ? SMALL_MAX_F32 : SMALL_MAX_F64;
    b->tune.small_threads = 256;
    b->tune.small_ctas_per_sm = 2;
    b->tune.streams = 8;
    b->tune.pass_gate_budget = 0;
    b->tune.f32_tensor = 0;
    b->tune.jit = QOA_JIT_ASYNC;
    *out = b;
    return QOA_OK;
}

int qoa_batch_add(qoa_batch_t b, uint32_t n, const qoa_op* ops, size_t nops, const uint64_t* zmasks, size_t nmasks,
                  uint32_t* id) {
    if (!b || (!ops && nops) || (!zmasks && nmasks)) return bset_err(b, QOA_E_ARG, "null argument");
    if (b->prepared) return bset_err(b, QOA_E_ARG, "batch already ran; create a new batch to add circuits");
    if (n < 1 || n > 40) return bset_err(b, QOA_E_ARG, "bad qubit count");
    Expander ex;
    ex.n = n;
    ex.flags = b->flags;
    ex.s = nullptr;
    for (size_t i = 0; i < nops; ++i) {
        ex.cur = (int)i;
        ex.op(ops[i]);
    }
    if (ex.first_err != QOA_OK) return bset_err(b, ex.first_err, ex.err.c_str());
    for (const Gate& g : ex.out)
        if (g.kind > K_U2) return bset_err(b, QOA_E_OPCODE, "batched circuits take unitary ops only");
    if (nmasks > EXPZ_MAX_MASKS) return bset_err(b, QOA_E_ARG, "more than 255 masks on one circuit");
    qoa_batch_s::Circ c;
    c.n = n;
    c.gates = std::move(ex.out);
    c.masks.assign(zmasks, zmasks + nmasks);
    c.out_start = b->nresults;
    c.route = R_VIEW;
    c.state_off = 0;
    b->nresults += (uint32_t)nmasks;
    if (id) *id = (uint32_t)b->circs.size();
    b->circs.push_back(std::move(c));
    return QOA_OK;
}

int qoa_batch_add_trajectory(qoa_batch_t b, uint32_t n, const qoa_op* ops, size_t nops, uint64_t seed,
                             double noise_p, uint64_t trajectory, const double* u, uint32_t shots, uint32_t* id) {
    if (!b || (!ops && nops) || (!u && shots)) return bset_err(b, QOA_E_ARG, "null argument");
    if (b->prepared) return bset_err(b, QOA_E_ARG, "batch already ran; reset it to add circuits");
    if (n < 1 || n > 40) return bset_err(b, QOA_E_ARG, "bad qubit count");
    if (!(noise_p >= 0.0 && noise_p <= 1.0)) return bset_err(b, QOA_E_ARG, "bad noise level");
    // the noise draws of a state seeded `seed` on trajectory `trajectory` with
    // qoa_set_noise(mode 1, noise_p): the same Expander over a host-only
    // noise context, so the gates are those qoa_apply would insert
    qoa_state_s ctx;
    ctx.n = n;
    ctx.flags = b->flags;
    ctx.seed = seed;
    ctx.noise_mode = noise_p > 0.0 ? 1 : 0;
    ctx.noise_p = noise_p;
    ctx.noise_stream = trajectory;
    ctx.noise_event = 0;
    Expander ex;
    ex.n = n;
    ex.flags = b->flags;
    ex.s = &ctx;
    ex.out.reserve(nops * 2 + 8);
    for (size_t i = 0; i < nops; ++i) {
        ex.cur = (int)i;
        ex.op(ops[i]);
    }
    if (ex.first_err != QOA_OK && ex.first_err != QOA_E_RANGE) return bset_err(b, ex.first_err, ex.err.c_str());
    for (const Gate& g : ex.out)
        if (g.kind > K_U2) return bset_err(b, QOA_E_OPCODE, "batched circuits take unitary ops only");
    qoa_batch_s::Circ c;
    c.n = n;
    c.gates = std::move(ex.out);
    c.out_start = b->nresults;
    c.route = R_VIEW;
    c.state_off = 0;
    c.shots = shots;
    c.shot_start = b->shot_u.size();
    b->shot_u.insert(b->shot_u.end(), u, u + shots);
    if (id) *id = (uint32_t)b->circs.size();
    b->circs.push_back(std::move(c));
    if (ex.first_err == QOA_E_RANGE) {  // the op was skipped, the circuit added (qoa_apply's rule)
        bset_err(b, QOA_E_RANGE, ex.err.c_str());
        return QOA_E_RANGE;
    }
    return QOA_OK;
}

int qoa_batch_shots(qoa_batch_t b, uint32_t id, uint64_t* out, size_t count) {
    if (!b || (!out && count)) return bset_err(b, QOA_E_ARG, "null argument");
    if (id >= b->circs.size()) return bset_err(b, QOA_E_ARG, "no such circuit");
    if (count != b->circs[id].shots) return bset_err(b, QOA_E_ARG, "count must equal the circuit's shots");
    if (!b->prepared || !b->runs) return bset_err(b, QOA_E_ARG, "run the batch first");
    cudaSetDevice(b->device);
    BCK(cudaStreamSynchronize(b->streams[0]));
    if (count)
        BCK(cudaMemcpy(out, b->d_shot_out + b->circs[id].shot_start, count * sizeof(uint64_t),
                       cudaMemcpyDeviceToHost));
    return QOA_OK;
}

int qoa_batch_reset(qoa_batch_t b) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    cudaSetDevice(b->device);
    for (cudaStream_t st : b->streams) BCK(cudaStreamSynchronize(st));
    for (cudaStream_t st : b->rstreams) BCK(cudaStreamSynchronize(st));
    batch_free_device(b);
    b->circs.clear();
    b->nresults = 0;
    b->shot_u.clear();
    return QOA_OK;
}

int qoa_batch_set_host_threads(qoa_batch_t b, uint32_t threads) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    b->host_threads = threads;
    return QOA_OK;
}

int qoa_ops_unitary(uint32_t n, uint32_t flags, const qoa_op* ops, size_t nops, int* unitary) {
    if ((!ops && nops) || !unitary) return set_err(nullptr, QOA_E_ARG, "null argument");
    if (n < 1 || n > 40) return set_err(nullptr, QOA_E_ARG, "bad qubit count");
    Expander ex;
    ex.n = n;
    ex.flags = flags;
    ex.s = nullptr;  // noise adds Paulis only: unitary either way
    for (size_t i = 0; i < nops; ++i) {
        ex.cur = (int)i;
        ex.op(ops[i]);
    }
    bool ok = ex.first_err == QOA_OK || ex.first_err == QOA_E_RANGE;
    for (const Gate& g : ex.out) ok = ok && g.kind <= K_U2;
    *unitary = ok ? 1 : 0;
    return QOA_OK;
}

int qoa_batch_set_tuning(qoa_batch_t b, const qoa_batch_tuning* t) {
    if (!b || !t) return bset_err(b, QOA_E_ARG, "null argument");
    if (t->small_threads < 32 || t->small_threads > 1024 || (t->small_threads & 31) || t->small_ctas_per_sm < 1 ||
        t->streams < 1 || t->streams > 64 || t->jit > QOA_JIT_SYNC)
        return bset_err(b, QOA_E_ARG, "bad tuning values");
    if (b->prepared) {
        cudaSetDevice(b->device);
        for (cudaStream_t st : b->streams) cudaStreamSynchronize(st);
        for (cudaStream_t st : b->rstreams) cudaStreamSynchronize(st);
        batch_free_device(b);
    }
    b->tune = *t;
    return QOA_OK;
}

int qoa_batch_get_tuning(qoa_batch_t b, qoa_batch_tuning* t) {
    if (!b || !t) return bset_err(b, QOA_E_ARG, "null argument");
    *t = b->tune;
    return QOA_OK;
}

int qoa_batch_run(qoa_batch_t b) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    if (cudaSetDevice(b->device) != cudaSuccess) return bset_err(b, QOA_E_CUDA, "cudaSetDevice failed");
    if (!b->prepared) {
        int rc = batch_prepare(b);
        if (rc) return rc;
    }
    if (b->runs == 0) {
        // first run: eager launches (a batch that runs once never pays for a graph)
        int rc = batch_enqueue(b);
        if (rc) return rc;
        BCK(cudaStreamSynchronize(b->streams[0]));
        b->runs++;
        return QOA_OK;
    }
    int rrc = batch_refresh_graph(b);
    if (rrc) return rrc;
    if (!b->exec) {
        // second run: capture the same launches into a graph, then replay it
        BCK(cudaStreamBeginCapture(b->streams[0], cudaStreamCaptureModeThreadLocal));
        int rc = batch_enqueue(b);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->streams[0], &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        BCK(e);
        b->graph = g;
        BCK(cudaGraphInstantiate(&b->exec, g, 0));
    }
    BCK(cudaGraphLaunch(b->exec, b->streams[0]));
    BCK(cudaStreamSynchronize(b->streams[0]));
    b->runs++;
    return QOA_OK;
}

int qoa_batch_launch(qoa_batch_t b) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    if (!b->exec) return bset_err(b, QOA_E_ARG, "qoa_batch_launch replays the graph that the second qoa_batch_run makes");
    if (cudaSetDevice(b->device) != cudaSuccess) return bset_err(b, QOA_E_CUDA, "cudaSetDevice failed");
    if (!b->graph_jit && batch_jit_all_ready(b)) {
        // the generated kernels arrived after the capture: capture again
        int rc = batch_refresh_graph(b);
        if (rc) return rc;
        BCK(cudaStreamBeginCapture(b->streams[0], cudaStreamCaptureModeThreadLocal));
        rc = batch_enqueue(b);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->streams[0], &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        BCK(e);
        b->graph = g;
        BCK(cudaGraphInstantiate(&b->exec, g, 0));
    }
    BCK(cudaGraphLaunch(b->exec, b->streams[0]));
    return QOA_OK;
}

int qoa_batch_stream(qoa_batch_t b, void** stream) {
    if (!b || !stream) return bset_err(b, QOA_E_ARG, "null argument");
    if (b->streams.empty()) return bset_err(b, QOA_E_ARG, "the batch has not run yet");
    *stream = (void*)b->streams[0];
    return QOA_OK;
}

int qoa_batch_results(qoa_batch_t b, double* out, size_t count) {
    if (!b || (!out && count)) return bset_err(b, QOA_E_ARG, "null argument");
    if (count != b->nresults) return bset_err(b, QOA_E_ARG, "count must equal the number of masks added");
    if (!b->prepared) return bset_err(b, QOA_E_ARG, "run the batch first");
    cudaSetDevice(b->device);
    BCK(cudaStreamSynchronize(b->streams[0]));
    if (count) BCK(cudaMemcpy(out, b->d_out, count * sizeof(double), cudaMemcpyDeviceToHost));
    return QOA_OK;
}

int qoa_batch_info(qoa_batch_t b, uint32_t* circuits, uint32_t* small, uint32_t* large, uint32_t* graph_ready) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    if (circuits) *circuits = (uint32_t)b->circs.size();
    if (small) *small = b->nsmall;
    if (large) *large = b->narena + (uint32_t)b->views.size();
    if (graph_ready) *graph_ready = b->exec ? 1u : 0u;
    return QOA_OK;
}

int qoa_batch_jit_info(qoa_batch_t b, uint32_t* structures, uint32_t* ready, uint32_t* graph_uses) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    uint32_t r = 0;
    for (const auto& k : b->jit_kernels) r += k.ready() ? 1u : 0u;
    if (structures) *structures = (uint32_t)b->jit_kernels.size();
    if (ready) *ready = r;
    if (graph_uses) *graph_uses = (b->exec && b->graph_jit) ? 1u : 0u;
    return QOA_OK;
}

int qoa_batch_traffic(qoa_batch_t b, double* arena_pass_bytes, uint32_t* rounds) {
    if (!b) return bset_err(nullptr, QOA_E_ARG, "null batch");
    if (arena_pass_bytes) *arena_pass_bytes = b->arena_pass_bytes;
    if (rounds) *rounds = (uint32_t)b->rounds.size();
    return QOA_OK;
}

double qoa_philox_uniform(uint64_t seed, uint32_t stream, uint64_t event, uint32_t slot) {
    return uniform01(seed, stream, event, slot);
}

uint64_t qoa_noise_hits(uint64_t seed, uint32_t stream, uint64_t event, uint32_t n, double p) {
    return n > 64 ? 0 : noise_hits(seed, stream, event, n, p);
}

// ---- checkpoint I/O: exact binary dump of a handle's stored state ------------
// Layout (little endian): "QOAS", u32 version 1, u32 precision, u32 n,
// f64 norm2 (the stored vector's squared norm: the logical state is
// stored / sqrt(norm2)), u64 amplitude bytes, the stored amplitudes, u64
// checksum (sum of the payload's u64 words after mixing each with its index).
// Saving does not normalise on the device and loading restores norm2 as it
// was, so a round trip gives the same logical state bit for bit.
namespace {
constexpr size_t kCkptChunk = 64ull << 20;
uint64_t ckpt_mix(uint64_t w, uint64_t i) {
    uint64_t x = w ^ (i * 0x9E3779B97F4A7C15ull);
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    return x ^ (x >> 29);
}

// The version-2 header fields, mixed into the checksum ahead of the amplitudes.
uint64_t ckpt_header_sum(const uint64_t (&rng)[4], const int32_t (&mode)[2], double noise_p,
                         const uint32_t (&words)[6], uint64_t& word) {
    uint64_t sum = 0, bits = 0;
    for (uint64_t x : rng) sum += ckpt_mix(x, word++);
    sum += ckpt_mix((uint64_t)(uint32_t)mode[0] | ((uint64_t)(uint32_t)mode[1] << 32), word++);
    std::memcpy(&bits, &noise_p, 8);
    sum += ckpt_mix(bits, word++);
    for (int k = 0; k < 6; k += 2) sum += ckpt_mix((uint64_t)words[k] | ((uint64_t)words[k + 1] << 32), word++);
    return sum;
}
}  // namespace

int qoa_state_save(qoa_state_t s, const char* path) {
    int rc = check_handle(s);
    if (rc) return rc;
    if (!path) return set_err(s, QOA_E_ARG, "null path");
    FILE* f = std::fopen(path, "wb");
    if (!f) return set_err(s, QOA_E_ARG, "cannot open %s for writing", path);
    const size_t esz = s->precision == QOA_PREC_F32 ? sizeof(float2) : sizeof(double2);
    const uint64_t bytes = state_len(s) * esz;
    CK(cudaMemcpyAsync(s->host_scal, s->scal, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double norm2 = s->host_scal[0];
    // version 2: after the amplitudes' header, the handle's noise and
    // measurement generator state and its status words, so that a loaded
    // handle continues the same trajectory and reports the same status
    uint32_t status[4];
    CK(cudaMemcpyAsync(status, s->status, sizeof status, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const uint32_t hdr[4] = {0x53414f51u /* "QOAS" */, 2u, (uint32_t)s->precision, s->n};
    const uint64_t rng[4] = {s->seed, s->noise_stream, s->noise_event, s->meas_draws};
    const int32_t mode[2] = {s->noise_mode, s->noise_none ? 1 : 0};
    const uint32_t words[6] = {status[0], status[1], status[2], status[3], s->host_resets, 0u};
    bool ok = std::fwrite(hdr, sizeof hdr, 1, f) == 1 && std::fwrite(&norm2, 8, 1, f) == 1 &&
              std::fwrite(&bytes, 8, 1, f) == 1 && std::fwrite(rng, sizeof rng, 1, f) == 1 &&
              std::fwrite(mode, sizeof mode, 1, f) == 1 && std::fwrite(&s->noise_p, 8, 1, f) == 1 &&
              std::fwrite(words, sizeof words, 1, f) == 1;
    void* stage = nullptr;
    if (ok && cudaMallocHost(&stage, kCkptChunk) != cudaSuccess) {
        std::fclose(f);
        return set_err(s, QOA_E_OOM, "pinned staging buffer");
    }
    uint64_t sum = 0, word = 0;
    sum += ckpt_header_sum(rng, mode, s->noise_p, words, word);
    for (uint64_t off = 0; ok && off < bytes; off += kCkptChunk) {
        const size_t k = (size_t)std::min<uint64_t>(kCkptChunk, bytes - off);
        if (cudaMemcpyAsync(stage, (const unsigned char*)s->amps + off, k, cudaMemcpyDeviceToHost, s->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess) {
            ok = false;
            break;
        }
        const uint64_t* w = (const uint64_t*)stage;
        for (size_t j = 0; j < k / 8; ++j) sum += ckpt_mix(w[j], word++);
        ok = std::fwrite(stage, 1, k, f) == k;
    }
    if (stage) cudaFreeHost(stage);
    ok = ok && std::fwrite(&sum, 8, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return set_err(s, QOA_E_ARG, "writing %s failed", path);
    return QOA_OK;
}

int qoa_state_load(const char* path, uint32_t flags, qoa_state_t* out) {
    if (!path || !out) return set_err(nullptr, QOA_E_ARG, "null argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return set_err(nullptr, QOA_E_ARG, "cannot open %s", path);
    uint32_t hdr[4];
    double norm2 = 0;
    uint64_t bytes = 0;
    if (std::fread(hdr, sizeof hdr, 1, f) != 1 || hdr[0] != 0x53414f51u || (hdr[1] != 1u && hdr[1] != 2u) ||
        std::fread(&norm2, 8, 1, f) != 1 || std::fread(&bytes, 8, 1, f) != 1) {
        std::fclose(f);
        return set_err(nullptr, QOA_E_ARG, "%s is not a state checkpoint (version 1 or 2)", path);
    }
    // version 2 carries the generator state and status words (version 1:
    // a fresh handle's, i.e. seed 0, noise off, clear status)
    uint64_t rng[4] = {0, 0, 0, 0};
    int32_t mode[2] = {0, 0};
    double noise_p = 0.0;
    uint32_t words[6] = {0, 0, 0, 0, 0, 0};
    if (hdr[1] == 2u && (std::fread(rng, sizeof rng, 1, f) != 1 || std::fread(mode, sizeof mode, 1, f) != 1 ||
                         std::fread(&noise_p, 8, 1, f) != 1 || std::fread(words, sizeof words, 1, f) != 1 ||
                         mode[0] < 0 || mode[0] > 2)) {
        std::fclose(f);
        return set_err(nullptr, QOA_E_ARG, "%s: truncated checkpoint header", path);
    }
    const int prec = (int)hdr[2];
    const uint32_t n = hdr[3];
    const size_t esz = prec == QOA_PREC_F32 ? sizeof(float2) : sizeof(double2);
    if ((prec != QOA_PREC_F64 && prec != QOA_PREC_F32) || n < 1 || n > 40 || bytes != (esz << n)) {
        std::fclose(f);
        return set_err(nullptr, QOA_E_ARG, "%s: inconsistent checkpoint header", path);
    }
    qoa_state_t s = nullptr;
    int rc = qoa_create(n, prec, flags, &s);
    if (rc) {
        std::fclose(f);
        return rc;
    }
    void* stage = nullptr;
    if (cudaMallocHost(&stage, kCkptChunk) != cudaSuccess) {
        std::fclose(f);
        qoa_destroy(s);
        return set_err(nullptr, QOA_E_OOM, "pinned staging buffer");
    }
    uint64_t sum = 0, word = 0, want = 0;
    if (hdr[1] == 2u) sum += ckpt_header_sum(rng, mode, noise_p, words, word);
    bool ok = true;
    for (uint64_t off = 0; ok && off < bytes; off += kCkptChunk) {
        const size_t k = (size_t)std::min<uint64_t>(kCkptChunk, bytes - off);
        ok = std::fread(stage, 1, k, f) == k;
        if (!ok) break;
        const uint64_t* w = (const uint64_t*)stage;
        for (size_t j = 0; j < k / 8; ++j) sum += ckpt_mix(w[j], word++);
        ok = cudaMemcpyAsync((unsigned char*)s->amps + off, stage, k, cudaMemcpyHostToDevice, s->stream) ==
                 cudaSuccess &&
             cudaStreamSynchronize(s->stream) == cudaSuccess;
    }
    cudaFreeHost(stage);
    ok = ok && std::fread(&want, 8, 1, f) == 1 && want == sum;
    std::fclose(f);
    if (!ok) {
        qoa_destroy(s);
        return set_err(nullptr, QOA_E_ARG, "%s: truncated or corrupt checkpoint", path);
    }
    s->host_scal[0] = norm2;
    if (cudaMemcpyAsync(s->scal, s->host_scal, sizeof(double), cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaMemcpyAsync(s->status, words, 4 * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess) {
        qoa_destroy(s);
        return set_err(nullptr, QOA_E_CUDA, "restoring norm2 and status failed");
    }
    s->seed = rng[0];
    s->noise_stream = rng[1];
    s->noise_event = rng[2];
    s->meas_draws = rng[3];
    s->noise_mode = mode[0];
    s->noise_p = noise_p;
    s->noise_none = mode[1] != 0;
    s->host_resets = words[4];
    *out = s;
    return QOA_OK;
}


int qoa_get_noise(qoa_state_t s, int* mode, double* p) {
    if (!s || !mode || !p) return set_err(s, QOA_E_ARG, "null argument");
    *mode = s->noise_mode;
    *p = s->noise_p;
    return QOA_OK;
}

int qoa_get_precision(qoa_state_t s, int* precision) {
    if (!s || !precision) return set_err(s, QOA_E_ARG, "null argument");
    *precision = s->precision;
    return QOA_OK;
}

int qoa_set_jit(qoa_state_t s, int mode, uint32_t min_qubits) {
    if (!s) return set_err(nullptr, QOA_E_ARG, "null handle");
    if (mode != QOA_JIT_OFF && mode != QOA_JIT_ASYNC && mode != QOA_JIT_SYNC)
        return set_err(s, QOA_E_ARG, "unknown jit mode %d", mode);
    s->jit_mode = mode;
    s->jit_min_qubits = std::max<uint32_t>(min_qubits, TILE_BITS);
    return QOA_OK;
}

int qoa_jit_wait(void) {
    jit_wait_all();
    return QOA_OK;
}

int qoa_jit_stats_get(qoa_state_t s, qoa_jit_stats* out) {
    if (!out) return set_err(s, QOA_E_ARG, "null argument");
    const JitStats j = jit_stats();
    out->kernels = j.kernels;
    out->hits = j.hits;
    out->misses = j.misses;
    out->failures = j.failures;
    out->compile_ms = j.compile_ms;
    out->launches = s ? s->jit_launches : 0;
    if (j.failures) set_err(nullptr, QOA_E_CUDA, "%s", jit_last_error().c_str());
    return QOA_OK;
}

int qoa_jit_translate(uint32_t n, int precision, uint32_t flags, const qoa_op* ops, size_t nops, int compile,
                      char* out, size_t cap, size_t* len, size_t* npasses) {
    if ((!ops && nops) || (!out && cap)) return set_err(nullptr, QOA_E_ARG, "null argument");
    if (precision != QOA_PREC_F64 && precision != QOA_PREC_F32) return set_err(nullptr, QOA_E_ARG, "bad precision");
    if (n < (uint32_t)TILE_BITS || n > 36) return set_err(nullptr, QOA_E_ARG, "tile passes need 11..36 qubits");
    Expander ex;
    ex.n = n;
    ex.flags = flags;
    ex.s = nullptr;
    for (size_t i = 0; i < nops; ++i) {
        ex.cur = (int)i;
        ex.op(ops[i]);
    }
    std::vector<Gate>& G = ex.out;
    for (const Gate& g : G)
        if (g.kind == K_QINIT) return set_err(nullptr, QOA_E_ARG, "qoa_jit_translate does not take QINIT");
    merge_swap_blocks(G);
    std::vector<Step> steps = schedule(G, n, false, false, 0, slot_search_pays(n));
    std::vector<std::string> bodies;
    static thread_local PassParams P;
    for (const Step& st : steps) {
        if (!st.pass) continue;
        if (build_pass(G, st, n, P, precision == QOA_PREC_F32) != 0)
            return set_err(nullptr, QOA_E_ARG, "a pass does not fit one launch");
        const bool arena = (compile & 2) != 0;
        bodies.push_back(precision == QOA_PREC_F32 ? jit_pass32_body(P, arena) : jit_pass_body(P, arena));
    }
    if (npasses) *npasses = bodies.size();
    const std::string text = jit_program(bodies);
    if (len) *len = text.size();
    if (cap) {
        const size_t k = std::min(cap - 1, text.size());
        memcpy(out, text.data(), k);
        out[k] = '\0';
    }
    if ((compile & 1) && !bodies.empty()) {
        std::string err;
        if (!jit_compile_only(bodies, err)) return set_err(nullptr, QOA_E_ARG, "%s", err.c_str());
    }
    return QOA_OK;
}

const char* qoa_batch_last_error(qoa_batch_t b) { return b ? b->err.c_str() : qoa_last_error(nullptr); }

int qoa_batch_destroy(qoa_batch_t b) {
    if (!b) return QOA_OK;
    cudaSetDevice(b->device);
    for (cudaStream_t st : b->streams) cudaStreamSynchronize(st);
    for (cudaStream_t st : b->rstreams) cudaStreamSynchronize(st);
    batch_free_device(b);
    if (b->h_params) pinned_params_give(b->h_params, b->h_params_cap);
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    for (cudaStream_t st : b->streams) cudaStreamDestroy(st);
    for (cudaEvent_t e : b->revents) cudaEventDestroy(e);
    for (cudaStream_t st : b->rstreams) cudaStreamDestroy(st);
    delete b;
    return QOA_OK;
}

// ---- vectorization.rs shims ------------------------------------------------
int qoa_vec_apply_hadamard(double* amps, size_t len, double nre, double nim, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    // norm_factor * (a +/- b); a real factor takes the exact (a+b)*f form
    const double2 f = d2(nre, nim);
    if (nim == 0.0) return shim_gate(amps, len, shim_g1(bit, G1_H, f, d2(0, 0), d2(0, 0), d2(0, 0), 0));
    return shim_gate(amps, len, shim_g1(bit, G1_GEN, f, f, f, d2(-f.x, -f.y), 0));
}
int qoa_vec_apply_x(double* amps, size_t len, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    return shim_gate(amps, len, shim_g1(bit, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), 0));
}
int qoa_vec_apply_y(double* amps, size_t len, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    return shim_gate(amps, len, shim_g1(bit, G1_Y, d2(0, 0), d2(0, -1), d2(0, 1), d2(0, 0), 0));
}
int qoa_vec_apply_z(double* amps, size_t len, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    return shim_gate(amps, len, shim_diag(-1, d2(-1, 0), d2(-1, 0), 1ull << bit, true));
}
int qoa_vec_apply_t(double* amps, size_t len, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    const double2 f = from_polar(1.0, M_PI / 4.0);
    return shim_gate(amps, len, shim_diag(-1, f, f, 1ull << bit, false));
}
int qoa_vec_apply_s(double* amps, size_t len, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    const double2 f = from_polar(1.0, M_PI / 2.0);
    return shim_gate(amps, len, shim_diag(-1, f, f, 1ull << bit, false));
}
int qoa_vec_apply_phaseshift(double* amps, size_t len, size_t bit, double angle) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    const double2 f = from_polar(1.0, angle);
    return shim_gate(amps, len, shim_diag(-1, f, f, 1ull << bit, false));
}
int qoa_vec_apply_reset(double* amps, size_t len, size_t bit) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    std::lock_guard<std::mutex> lk(g_shim_mu);
    qoa_state_t s = nullptr;
    double2* dev;
    int rc = shim_begin(amps, len, &dev);
    if (rc) return rc;
    if (len) {
        CK(launch_p01(dev, len, (uint32_t)bit, g_shim_scr + 8, g_shim_scr, nullptr, g_shim_stream));
        double p[2];
        CK(cudaMemcpyAsync(p, g_shim_scr, sizeof p, cudaMemcpyDeviceToHost, g_shim_stream));
        CK(cudaStreamSynchronize(g_shim_stream));
        if (p[0] > 1e-12) {
            CK(launch_collapse(dev, len, (uint32_t)bit, 0, 1.0 / std::sqrt(p[0]), g_shim_scr + 8, g_shim_scr + 2,
                               nullptr, g_shim_stream));
        } else {
            GGate k;
            memset(&k, 0, sizeof k);
            k.kind = GG_RESET_ALL;
            CK(launch_gate(dev, len, k, g_shim_stream));
        }
    }
    return shim_end(amps, len);
}
int qoa_vec_apply_swap(double* amps, size_t len, size_t q1, size_t q2) {
    if (!shim_bit_ok(q1) || !shim_bit_ok(q2)) return QOA_OK;
    GGate k;
    memset(&k, 0, sizeof k);
    k.kind = GG_SWAP; k.t = (uint8_t)q1; k.t2 = (uint8_t)q2;
    return shim_gate(amps, len, k);
}
int qoa_vec_apply_controlled_swap(double* amps, size_t len, size_t c, size_t t1, size_t t2) {
    if (!shim_bit_ok(c) || !shim_bit_ok(t1) || !shim_bit_ok(t2)) return QOA_OK;
    // apply_controlled_swap_simd (vectorization.rs:1200-1232): for base i with
    // control, t1, t2 all 0, swap i|c|t2 <-> i|c|t1. With coinciding indices
    // that degenerates to a controlled X (or to nothing), reproduced here.
    if (t1 == t2) return QOA_OK;
    if (c == t1) return shim_gate(amps, len, shim_g1(t2, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), 1ull << c));
    if (c == t2) return shim_gate(amps, len, shim_g1(t1, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), 1ull << c));
    GGate k;
    memset(&k, 0, sizeof k);
    k.kind = GG_SWAP; k.t = (uint8_t)t1; k.t2 = (uint8_t)t2; k.cmask = 1ull << c;
    return shim_gate(amps, len, k);
}
int qoa_vec_apply_rx(double* amps, size_t len, size_t bit, double angle) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    const double c = std::cos(angle / 2.0), sn = std::sin(angle / 2.0);
    return shim_gate(amps, len, shim_g1(bit, G1_RX, d2(c, sn), d2(0, -sn), d2(0, -sn), d2(c, 0), 0));
}
int qoa_vec_apply_ry(double* amps, size_t len, size_t bit, double angle) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    const double c = std::cos(angle / 2.0), sn = std::sin(angle / 2.0);
    return shim_gate(amps, len, shim_g1(bit, G1_RY, d2(c, sn), d2(-sn, 0), d2(sn, 0), d2(c, 0), 0));
}
int qoa_vec_apply_rz(double* amps, size_t len, size_t bit, double angle) {
    if (!shim_bit_ok(bit)) return QOA_OK;
    return shim_gate(amps, len, shim_diag((int)bit, from_polar(1.0, -angle / 2.0), from_polar(1.0, angle / 2.0), 0, false));
}
int qoa_vec_apply_cnot(double* amps, size_t len, size_t control, size_t target) {
    if (!shim_bit_ok(control) || !shim_bit_ok(target)) return QOA_OK;
    if (control == target) return QOA_OK;  // (i & cm) == cm && (i & tm) == 0 never holds
    return shim_gate(amps, len, shim_g1(target, G1_X, d2(0, 0), d2(1, 0), d2(1, 0), d2(0, 0), 1ull << control));
}
int qoa_vec_apply_cz(double* amps, size_t len, size_t control_mask, size_t target_mask) {
    return shim_gate(amps, len, shim_diag(-1, d2(-1, 0), d2(-1, 0), (uint64_t)(control_mask | target_mask), true));
}
int qoa_vec_apply_controlled_phase_rotation(double* amps, size_t len, size_t control_mask, size_t target_mask,
                                            double angle) {
    const double2 f = from_polar(1.0, angle);
    return shim_gate(amps, len, shim_diag(-1, f, f, (uint64_t)(control_mask | target_mask), false));
}
int qoa_vec_apply_reset_all(double* amps, size_t len) {
    GGate k;
    memset(&k, 0, sizeof k);
    k.kind = GG_RESET_ALL;
    return shim_gate(amps, len, k);
}

}  // extern "C"
