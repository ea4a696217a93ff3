// qoa_jit.cpp — complex128 tile passes generated as CUDA C++ and compiled at
// run time with NVRTC for sm_100a.
//
// The generated kernel does exactly what k_pass does for the same
// PassParams (qoa_kernels.cu: load under map0, the op stream, exchanges
// through shared memory, the pending factor, the store under out_qubit and
// the norm partials), with the interpreter's run-time decisions resolved on
// the host: each op becomes a call of the same device building block
// (qoa_pass_dev.cuh) with its register bit, condition masks and coefficient
// slot as literals, and each exchange a list of 16 shared-memory stores and
// loads at literal swizzled offsets from one per-thread base. What the
// interpreter pays per op — fetching and decoding the op, the indirect jump,
// staging coefficients in shared memory, forming exchange addresses from
// run-time mappings — disappears, and the compiler schedules across gates.
#include "qoa_jit.h"

#include <dlfcn.h>
#include <nvrtc.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <algorithm>
#include <array>
#include <functional>

namespace qoa {

namespace {

const char kTypesHeader[] =
#include "qoa_kernels.cuh.inc"
    ;
const char kDevHeader[] =
#include "qoa_pass_dev.cuh.inc"
    ;
const char kDev32Header[] =
#include "qoa_pass32_dev.cuh.inc"
    ;

// Marker of the streamed form in a kernel body (launch and compile options
// depend on it).
const char kStreamMark[] = "/*qoa:streamed*/";

// NVRTC has no C library headers: the fixed-width types the headers use.
const char kPrelude[] =
    "typedef unsigned char uint8_t;\n"
    "typedef unsigned short uint16_t;\n"
    "typedef unsigned int uint32_t;\n"
    "typedef int int32_t;\n"
    "typedef unsigned long long uint64_t;\n"
    "#include \"qoa_pass_dev.cuh\"\n"
    "#include \"qoa_pass32_dev.cuh\"\n";

// Resident CTAs per SM of a generated pass (128 threads): complex128 the
// same register budget as k_pass (128), complex64 up to 80 registers.
constexpr int JIT_OCC = 4;
constexpr int JIT_OCC32 = 6;

// QOA_JIT_OCC / QOA_JIT_OCC32 override the resident-CTA targets (tuning).
int occ_target(bool c64) {
    const char* v = getenv(c64 ? "QOA_JIT_OCC32" : "QOA_JIT_OCC");
    const int d = c64 ? JIT_OCC32 : JIT_OCC;
    if (!v) return d;
    const int k = atoi(v);
    return (k >= 1 && k <= 16) ? k : d;
}

// Resident CTAs per SM of a streamed pass (two tile buffers each: 64 KB for
// complex128, 32 KB for complex64); QOA_JIT_OCC_STREAMED overrides.
int occ_streamed(bool c64) {
    const int d = c64 ? 6 : 3;
    const char* v = getenv("QOA_JIT_OCC_STREAMED");
    const int k = v ? atoi(v) : d;
    return (k >= 1 && k <= d) ? k : d;
}

// Which generated single-state passes take the streamed (persistent,
// double-buffered) form: QOA_JIT_STREAM=0/1/2/3 = neither (the default) /
// complex128 / complex64 / both. Measured on B200, the streamed form loses
// for both precisions: the passes are bound by FP64 (complex128) or
// instruction issue (complex64), not by their loads, and the second tile
// buffer lowers residency (complex128: 3 CTAs per SM instead of 4; 30-qubit
// layered circuit 13.6 against 10.6 ms a pass; complex64 QFT at 32 qubits
// 156 against 151 ms).
int stream_mode() {
    const char* v = getenv("QOA_JIT_STREAM");  // read at each pass's generation (cheap, and tests switch it)
    return v ? atoi(v) : 0;
}
bool stream_f64() { return (stream_mode() & 1) != 0; }
bool stream_f32() { return (stream_mode() & 2) != 0; }

uint32_t spos_host(uint32_t j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7u); }

struct Emit {
    std::string s;
    void line(const char* fmt, ...) __attribute__((format(printf, 2, 3))) {
        char buf[512];
        va_list ap, ap2;
        va_start(ap, fmt);
        va_copy(ap2, ap);
        const int k = vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        if (k >= (int)sizeof buf) {  // a long line (e.g. many outer-qubit runs): format again in full
            std::string big((size_t)k + 1, '\0');
            vsnprintf(&big[0], big.size(), fmt, ap2);
            big.resize((size_t)k);
            s += big;
        } else if (k > 0) {
            s += buf;
        }
        va_end(ap2);
        s += '\n';
    }
};

const char* g1_name(int code) {
    switch (code & ~3) {
        case PC_HF: return "G1_HF";
        case PC_RX: return "G1_RXA";
        case PC_RY: return "G1_RYA";
        case PC_RXB: return "G1_RXB";
        case PC_RYB: return "G1_RYB";
        case PC_GEN: return "G1_GEN";
        default: return nullptr;
    }
}

// RX / RY ops in either factored form (A: cos factored out, B: sin)
bool rotation(int code) {
    const int b = code & ~3;
    return b == PC_RX || b == PC_RY || b == PC_RXB || b == PC_RYB;
}
bool rot_x(int code) {
    const int b = code & ~3;
    return b == PC_RX || b == PC_RXB;
}

// "(tw & m) == m" or "true"
std::string tcond(uint32_t tm) {
    if (!tm) return "true";
    char b[64];
    snprintf(b, sizeof b, "((tw & 0x%xu) == 0x%xu)", tm, tm);
    return b;
}

// Both mappings put the same tile bits on the warp bits: an exchange between
// them moves data only among the threads of each warp.
bool same_warps(const TileMap& a, const TileMap& b) {
    for (int k = 0; k < WARP_BITS; ++k)
        if (a.warp[k] != b.warp[k]) return false;
    return true;
}

// Tile index (shared-memory bits) of this thread's register 0 under map m:
// lane bit i sits at tile bit m.lane[i], warp bit i at m.warp[i].
std::string tile_base(const TileMap& m) {
    std::string e = "0u";
    char b[96];
    for (int i = 0; i < LANE_BITS; ++i) {
        snprintf(b, sizeof b, " | ((((uint32_t)lane >> %d) & 1u) << %d)", i, m.lane[i]);
        e += b;
    }
    for (int i = 0; i < WARP_BITS; ++i) {
        snprintf(b, sizeof b, " | ((((uint32_t)wid >> %d) & 1u) << %d)", i, m.warp[i]);
        e += b;
    }
    return e;
}

// Swizzled offset of register v's tile-index part under map m (spos is
// linear over XOR, and lane/warp and register bits are disjoint).
uint32_t reg_part(const TileMap& m, int v) {
    uint32_t j = 0;
    for (int k = 0; k < REG_BITS; ++k)
        if ((v >> k) & 1) j |= 1u << m.reg[k];
    return spos_host(j);
}

// Pair exchanges (complex64, pairing bit r3 fixed): a tile bit t sits at
// position t (t < r3) or t - 1 (t > r3) of the 10-bit pair index.
int pair_pos(int t, int r3) { return t < r3 ? t : t - 1; }

// Shared-memory layout of one exchange: index bit t of a 16-byte unit's
// index keeps its place, except that the low three bits are XORed with A[t]
// for every set bit t >= 3 (a linear bijection, like spos). A quarter-warp
// (lanes 0..7) touches 8 units that differ in the index bits of lane bits
// 0..2; they fall in 8 distinct bank groups when those three bits' low-3
// images are linearly independent. Each exchange picks its own A so that
// this holds for the mapping it stores under and the one it loads under.
struct Swizzle {
    int nbits = TILE_BITS;
    uint32_t A[16] = {};
    uint32_t img(int t) const { return t < 3 ? 1u << t : A[t]; }
    uint32_t f(uint32_t j) const {
        uint32_t g = 0;
        for (int t = 3; t < nbits; ++t)
            if ((j >> t) & 1) g ^= A[t];
        return j ^ g;
    }
};

bool independent3(uint32_t a, uint32_t b, uint32_t c) {
    return a && b && c && a != b && c != a && c != b && c != (a ^ b);
}

// so[i] / sn[i]: index positions of lane bits 0..2 under the store and the
// load mapping
Swizzle make_swizzle(const int (&so)[3], const int (&sn)[3], int nbits) {
    Swizzle z;
    z.nbits = nbits;
    for (int t = 3; t < nbits; ++t) z.A[t] = 1u << (t % 3);  // the spos choice
    std::vector<int> vars;
    for (int i = 0; i < 3; ++i) {
        if (so[i] >= 3 && std::find(vars.begin(), vars.end(), so[i]) == vars.end()) vars.push_back(so[i]);
        if (sn[i] >= 3 && std::find(vars.begin(), vars.end(), sn[i]) == vars.end()) vars.push_back(sn[i]);
    }
    auto ok = [&]() {
        return independent3(z.img(so[0]), z.img(so[1]), z.img(so[2])) &&
               independent3(z.img(sn[0]), z.img(sn[1]), z.img(sn[2]));
    };
    if (ok()) return z;
    // at most six free images of 7 values each: exhaustive, spos-like first
    std::function<bool(size_t)> search = [&](size_t k) -> bool {
        if (k == vars.size()) return ok();
        const int t = vars[k];
        const uint32_t first = 1u << (t % 3);
        for (uint32_t d = 0; d < 7; ++d) {
            z.A[t] = ((first - 1 + d) % 7) + 1;
            if (search(k + 1)) return true;
        }
        z.A[t] = first;
        return false;
    };
    if (!search(0))
        for (int t = 3; t < nbits; ++t) z.A[t] = 1u << (t % 3);  // no such layout: keep spos
    return z;
}

// One layout for every exchange of a pass: each lane triple (index
// positions of lane bits 0..2 under a mapping the pass stores or loads
// under) must get independent low-3 images. With one layout, a thread
// stores each exchange's data exactly where it loaded the previous
// exchange's, so the barrier that otherwise separates the previous loads
// from the next stores is not needed. False when no layout is found within
// a bounded search.
bool pass_swizzle(const std::vector<std::array<int, 3>>& triples, int nbits, Swizzle& z) {
    z = Swizzle();
    z.nbits = nbits;
    for (int t = 3; t < nbits; ++t) z.A[t] = 1u << (t % 3);
    int freq[16] = {};
    for (const auto& tr : triples)
        for (int p : tr)
            if (p >= 3) freq[p]++;
    std::vector<int> vars;
    for (int t = 3; t < nbits; ++t)
        if (freq[t]) vars.push_back(t);
    std::sort(vars.begin(), vars.end(), [&](int a, int b) { return freq[a] > freq[b]; });
    int rank[16];
    for (int t = 0; t < 16; ++t) rank[t] = -1;
    for (size_t k = 0; k < vars.size(); ++k) rank[vars[k]] = (int)k;
    // a triple is checked once its last variable is assigned
    std::vector<std::vector<int>> due(vars.size() + 1);
    for (size_t i = 0; i < triples.size(); ++i) {
        int last = -1;
        for (int p : triples[i]) last = std::max(last, p >= 3 ? rank[p] : -1);
        due[last + 1].push_back((int)i);
    }
    auto holds = [&](int i) {
        const auto& tr = triples[i];
        return independent3(z.img(tr[0]), z.img(tr[1]), z.img(tr[2]));
    };
    for (int i : due[0])
        if (!holds(i)) return false;
    long nodes = 0;
    std::function<bool(size_t)> search = [&](size_t k) -> bool {
        if (k == vars.size()) return true;
        if (++nodes > 200000) return false;
        const int t = vars[k];
        const uint32_t first = 1u << (t % 3);
        for (uint32_t d = 0; d < 7; ++d) {
            z.A[t] = ((first - 1 + d) % 7) + 1;
            bool good = true;
            for (int i : due[k + 1]) good = good && holds(i);
            if (good && search(k + 1)) return true;
        }
        z.A[t] = first;
        return false;
    };
    return search(0);
}

// f(index of this thread's unit 0) as an XOR of constants selected by the
// lane and warp bits (pos[t]: index position of tile bit t)
std::string swz_base(const Swizzle& z, const TileMap& m, const int* pos) {
    std::string e = "0u";
    char b[112];
    for (int i = 0; i < LANE_BITS; ++i) {
        snprintf(b, sizeof b, " ^ ((0u - (((uint32_t)lane >> %d) & 1u)) & 0x%xu)", i, z.f(1u << pos[m.lane[i]]));
        e += b;
    }
    for (int i = 0; i < WARP_BITS; ++i) {
        snprintf(b, sizeof b, " ^ ((0u - (((uint32_t)wid >> %d) & 1u)) & 0x%xu)", i, z.f(1u << pos[m.warp[i]]));
        e += b;
    }
    return e;
}

// The swizzled accesses arr[pb ^ K] of one exchange half, K the register
// parts. pb is an XOR of constants selected by the lane and warp bits; above
// the low three bits those constants and the K are different tile bits, so
// pb ^ K = (pb ^ (K & 7)) + (K & ~7): one pointer per distinct K & 7, the
// rest a constant offset that each load or store takes as its immediate
// instead of an address computation per access. `pb_hi` is the OR of pb's
// possible constants; where it overlaps a K (no such layout is made) the
// accesses keep the XOR form. Returns the access expression of each K and
// emits the pointers (named pfx0..pfx7) as it goes.
std::vector<std::string> swz_access(Emit& E, const char* arr, const char* pfx, uint32_t pb_hi,
                                    const std::vector<uint32_t>& ks) {
    bool disjoint = true;
    uint32_t lows = 0;
    for (uint32_t k : ks) {
        disjoint = disjoint && !(pb_hi & k & ~7u);
        lows |= 1u << (k & 7u);
    }
    std::vector<std::string> out;
    char b[96];
    if (!disjoint) {
        for (uint32_t k : ks) {
            snprintf(b, sizeof b, "%s[pb ^ %uu]", arr, k);
            out.push_back(b);
        }
        return out;
    }
    for (uint32_t m = 0; m < 8; ++m)
        if ((lows >> m) & 1) E.line("auto* const %s%u = %s + (pb ^ %uu);", pfx, m, arr, m);
    for (uint32_t k : ks) {
        snprintf(b, sizeof b, "%s%u[%uu]", pfx, k & 7u, k & ~7u);
        out.push_back(b);
    }
    return out;
}

// OR of the constants swz_base may XOR into pb (lane and warp bits)
uint32_t swz_base_bits(const Swizzle& z, const TileMap& m, const int* pos) {
    uint32_t r = 0;
    for (int i = 0; i < LANE_BITS; ++i) r |= z.f(1u << pos[m.lane[i]]);
    for (int i = 0; i < WARP_BITS; ++i) r |= z.f(1u << pos[m.warp[i]]);
    return r;
}

}  // namespace

// Kernel head shared by both precisions: the signature, shared memory, the
// thread's lane / warp / tile number, the amplitude pointer, the pass
// parameters P and the input's squared norm nrm. Single-state form: P is the
// __grid_constant__ parameter, one CTA per tile. Arena form: CTA b runs tile
// b % 2^(n - 11) of job b / 2^(n - 11) (every job of the launch has this
// structure), P is the job's PassParams in global memory and its
// coefficients are staged in shared memory (scoef).
void emit_head(Emit& E, const PassParams& P, bool c64, bool arena) {
    const char* T = c64 ? "float2" : "double2";
    if (arena) {
        E.line("(const qoa::ArenaJob* __restrict__ jobs) {");
    } else {
        E.line("(%s* __restrict__ amps, const __grid_constant__ qoa::PassParams P,", T);
        E.line(" const double* __restrict__ norm2_in, double* __restrict__ partials) {");
    }
    E.line("using namespace qoa;");
    if (c64) E.line("using namespace qoa::p32;");
    E.line("typedef %s T;", T);
    E.line("__shared__ __align__(16) T tile[1 << TILE_BITS];");
    if (!arena) E.line("__shared__ double red[PASS_THREADS / 32];");
    if (c64 || arena) E.line("__shared__ __align__(16) T scoef[%u];", P.ncoef ? P.ncoef : 1);
    if (P.nang) E.line("__shared__ T sang[%u];", P.nang);
    E.line("const int lane = threadIdx.x & 31;");
    E.line("const int wid = threadIdx.x >> 5;");
    if (arena) {
        const int lt = (int)P.n - TILE_BITS;
        E.line("const qoa::ArenaJob J = jobs[blockIdx.x >> %d];", lt);
        E.line("const uint64_t blk = blockIdx.x & 0x%xu;", (1u << lt) - 1);
        E.line("T* __restrict__ amps = reinterpret_cast<T*>(J.amps);");
        E.line("const PassParams& P = *reinterpret_cast<const PassParams*>(J.params);");
        E.line("const double nrm = J.fresh ? 0.0 : 1.0;");
    } else {
        E.line("const uint64_t blk = blockIdx.x;");
        E.line("const double nrm = *norm2_in;");
    }
    E.line("const uint32_t tw = (uint32_t)lane | ((uint32_t)wid << %d) | ((uint32_t)blk << %d);", LANE_BITS,
           LANE_BITS + WARP_BITS);
    // tile origin: the tile number's bits deposited into the outer qubits,
    // one shift per run of consecutive qubits
    {
        std::string g = "0ull";
        const int nout = (int)P.n - TILE_BITS;
        char b[128];
        for (int k = 0; k < nout;) {
            int len = 1;
            while (k + len < nout && P.outer_qubits[k + len] == P.outer_qubits[k] + len) ++len;
            snprintf(b, sizeof b, " | (((blk >> %d) & 0x%llxull) << %d)", k,
                     (unsigned long long)((len >= 64) ? ~0ull : ((1ull << len) - 1)), P.outer_qubits[k]);
            g += b;
            k += len;
        }
        E.line("const uint64_t g0 = %s;", g.c_str());
    }
    if (c64)
        E.line("for (uint32_t i = threadIdx.x; i < %uu; i += PASS_THREADS) scoef[i] = make_float2((float)P.coef[i].x, (float)P.coef[i].y);",
               P.ncoef);
    else if (arena)
        E.line("for (uint32_t i = threadIdx.x; i < %uu; i += PASS_THREADS) scoef[i] = P.coef[i];", P.ncoef);
    if (P.nang) E.line("pass_angles(P, blk, sang);");
}

// The op stream of a complex128 pass (gates, diagonal factors, exchanges
// through the shared-memory array `tile`), emitted as straight-line code;
// returns the mapping in force at its end.
const TileMap* emit_ops128(Emit& E, const PassParams& P, bool arena, const char* cf) {
    // one exchange layout for the whole pass where one exists
    Swizzle zp;
    bool shared_layout = false;
    {
        std::vector<std::array<int, 3>> tr;
        const TileMap* m = &P.map0;
        for (uint32_t oi = 0; oi < P.nops; ++oi) {
            const PassOp& op = P.ops[oi];
            if (op.code == PC_DIAG_MX || op.code == PC_DIAG_TM) { oi += op.k; continue; }
            if (op.code != PC_XCHG) continue;
            const TileMap& mn = P.xmap[op.coef];
            tr.push_back({m->lane[0], m->lane[1], m->lane[2]});
            tr.push_back({mn.lane[0], mn.lane[1], mn.lane[2]});
            m = &mn;
        }
        shared_layout = !tr.empty() && pass_swizzle(tr, TILE_BITS, zp);
    }
    int nxchg = 0;

    const TileMap* cur = &P.map0;
    const uint32_t* ow = reinterpret_cast<const uint32_t*>(P.ops);
    for (uint32_t oi = 0; oi < P.nops; ++oi) {
        const PassOp& op = P.ops[oi];
        const int code = op.code;
        const uint32_t c = op.coef;
        const uint32_t cr = op.cond_reg;
        const uint32_t tm = ow[4 * oi + 2];
        if (arena && rotation(code)) {
            // RX / RY in the batch form: which of |cos|, |sin| was factored
            // out is a property of the angle, read from the op at run time,
            // so that circuits differing only in angles share the kernel
            // (the single-state form keeps the branch out of the code)
            const bool x = rot_x(code);
            E.line("if (P.ops[%u].code >= %d) g1r<%s, %d>(a, %s + %u); else g1r<%s, %d>(a, %s + %u);", oi,
                   x ? PC_RXB : PC_RYB, x ? "G1_RXB" : "G1_RYB", code & 3, cf, c, x ? "G1_RXA" : "G1_RYA", code & 3,
                   cf, c);
        } else if (code >= PC_HF && code < PC_XC) {
            E.line("g1r<%s, %d>(a, %s + %u);", g1_name(code), code & 3, cf, c);
        } else if (code >= PC_RXB && code < PC_DIAG_TA) {
            E.line("g1r<%s, %d>(a, %s + %u);", g1_name(code), code & 3, cf, c);
        } else if (code >= PC_XC && code < PC_RXB) {
            E.line("g1rc<%s, %d>(a, %s, 0x%xu);", (code & ~3) == PC_XC ? "G1_X" : "G1_Y", code & 3,
                   tcond(tm).c_str(), cr);
        } else {
            switch (code) {
                case PC_DIAG_T:
                    if (tm) E.line("if (%s) pend = c_mul(pend, %s[%u]);", tcond(tm).c_str(), cf, c);
                    else E.line("pend = c_mul(pend, %s[%u]);", cf, c);
                    break;
                case PC_DIAG_M:
                    E.line("diag_m(a, %s, 0x%xu, %s[%u]);", tcond(tm).c_str(), cr, cf, c);
                    break;
                case PC_DIAG_TA:
                    if (tm) E.line("if (%s) pend = c_mul(pend, sang[%u]);", tcond(tm).c_str(), c);
                    else E.line("pend = c_mul(pend, sang[%u]);", c);
                    break;
                case PC_DIAG_MA:
                    E.line("diag_m(a, true, 0x%xu, sang[%u]);", cr, c);
                    break;
                case PC_DIAG_MX:
                case PC_DIAG_TM: {
                    // the entries' thread-conditioned factors folded into f;
                    // MX applies f to its register mask at the end of each run
                    const uint32_t cnt = op.k;
                    bool one = true;  // f is known to be 1
                    E.line("{ T f = make_double2(1.0, 0.0);");
                    for (uint32_t e = 1; e <= cnt; ++e) {
                        const PassOp& r = P.ops[oi + e];
                        const uint32_t rtm = ow[4 * (oi + e) + 2];
                        if (!rtm && one) E.line("f = %s[%u];", cf, (unsigned)r.coef);
                        else if (one) E.line("f = %s ? %s[%u] : make_double2(1.0, 0.0);", tcond(rtm).c_str(), cf, (unsigned)r.coef);
                        else if (!rtm) E.line("f = c_mul(f, %s[%u]);", cf, (unsigned)r.coef);
                        else E.line("if (%s) f = c_mul(f, %s[%u]);", tcond(rtm).c_str(), cf, (unsigned)r.coef);
                        one = false;
                        if (code == PC_DIAG_MX && (e == cnt || ((r.has_tp >> 1) & 1u))) {
                            E.line("diag_m(a, true, 0x%xu, f);", (unsigned)r.cond_reg);
                            if (e != cnt) E.line("f = make_double2(1.0, 0.0);");
                            one = true;
                        }
                    }
                    if (code == PC_DIAG_TM && cnt) E.line("pend = c_mul(pend, f);");
                    E.line("}");
                    oi += cnt;
                    break;
                }
                case PC_DIAG_TAB:
                    // registers whose factor is exactly 1 are left alone
                    for (int v = 0; v < REGS; ++v)
                        if ((tm >> v) & 1) E.line("a[%d] = c_mul(a[%d], %s[%u]);", v, v, cf, c + v);
                    break;
                case PC_FLUSH:
                    for (int v = 0; v < REGS; ++v) E.line("a[%d] = c_mul(a[%d], pend);", v, v);
                    E.line("pend = make_double2(1.0, 0.0);");
                    break;
                case PC_XCHG: {
                    const TileMap& mo = *cur;
                    const TileMap& mn = P.xmap[c];
                    // with the pass's one layout each thread stores where it
                    // last loaded: only the first exchange waits before storing
                    if (!shared_layout || nxchg == 0) E.line("__syncthreads();");
                    ++nxchg;
                    int pos[TILE_BITS];
                    for (int t = 0; t < TILE_BITS; ++t) pos[t] = t;
                    const int so[3] = {mo.lane[0], mo.lane[1], mo.lane[2]};
                    const int sn[3] = {mn.lane[0], mn.lane[1], mn.lane[2]};
                    const Swizzle z = shared_layout ? zp : make_swizzle(so, sn, TILE_BITS);
                    auto off = [&](const TileMap& m, int v) {
                        uint32_t j = 0;
                        for (int k = 0; k < REG_BITS; ++k)
                            if ((v >> k) & 1) j |= 1u << m.reg[k];
                        return z.f(j);
                    };
                    std::vector<uint32_t> ks(REGS);
                    E.line("{ const uint32_t pb = %s;", swz_base(z, mo, pos).c_str());
                    for (int v = 0; v < REGS; ++v) ks[v] = off(mo, v);
                    {
                        const auto acc = swz_access(E, "tile", "ts", swz_base_bits(z, mo, pos), ks);
                        for (int v = 0; v < REGS; ++v) E.line("%s = a[%d];", acc[v].c_str(), v);
                    }
                    E.line("}");
                    // an exchange that keeps the warp bits moves data only within
                    // each warp: with the pass's one layout a warp stores to and
                    // loads from its own part of the tile, so a warp barrier does
                    E.line(shared_layout && same_warps(mo, mn) ? "__syncwarp();" : "__syncthreads();");
                    E.line("{ const uint32_t pb = %s;", swz_base(z, mn, pos).c_str());
                    for (int v = 0; v < REGS; ++v) ks[v] = off(mn, v);
                    {
                        const auto acc = swz_access(E, "tile", "tl", swz_base_bits(z, mn, pos), ks);
                        for (int v = 0; v < REGS; ++v) E.line("a[%d] = %s;", v, acc[v].c_str());
                    }
                    E.line("}");
                    cur = &mn;
                    break;
                }
                default: break;  // PC_NOP
            }
        }
    }

    return cur;
}

// The single-state complex128 pass as a persistent kernel: CTA b runs tiles
// b, b + gridDim.x, ... Each tile arrives by bulk copies into one of two
// shared-memory buffers while the previous tile is computed (that buffer
// then serves the tile's exchanges); the tile's rows are its 64 runs of 32
// consecutive amplitudes (lanes = qubits 0..4), merged into longer runs
// where the lowest high slots are qubits 5, 6, ... The results are stored
// from registers as in k_pass, with the same arithmetic, so a streamed pass
// is bit-identical to k_pass.
std::string jit_pass_body_streamed(const PassParams& P) {
    Emit E;
    const int lt = (int)P.n - TILE_BITS;
    E.line("(double2* __restrict__ amps, const __grid_constant__ qoa::PassParams P,");
    E.line(" const double* __restrict__ norm2_in, double* __restrict__ partials, uint32_t* __restrict__ status) {");
    E.line("%s", kStreamMark);
    E.line("using namespace qoa;");
    E.line("typedef double2 T;");
    E.line("extern __shared__ __align__(128) unsigned char qoa_dsm[];");
    E.line("__shared__ __align__(8) uint64_t mbar[2];");
    E.line("__shared__ double red[PASS_THREADS / 32];");
    if (P.nang) E.line("__shared__ T sang[%u];", P.nang);
    E.line("const int lane = threadIdx.x & 31;");
    E.line("const int wid = threadIdx.x >> 5;");
    E.line("const double nrm = *norm2_in;");
    E.line("const bool valid = nrm > 1e-12;");
    E.line("const uint64_t ntiles = 1ull << %d;", lt);
    // tile origin of tile number b: its bits deposited into the outer qubits
    {
        std::string g = "0ull";
        char b[128];
        for (int k = 0; k < lt;) {
            int len = 1;
            while (k + len < lt && P.outer_qubits[k + len] == P.outer_qubits[k] + len) ++len;
            snprintf(b, sizeof b, " | (((b >> %d) & 0x%llxull) << %d)", k,
                     (unsigned long long)((len >= 64) ? ~0ull : ((1ull << len) - 1)), P.outer_qubits[k]);
            g += b;
            k += len;
        }
        E.line("auto origin = [](uint64_t b) -> uint64_t { return %s; };", g.c_str());
    }
    // rows of a tile: the lowest r high slots on qubits 5 .. 4 + r make runs
    // of 32 << r consecutive amplitudes, 64 >> r runs per tile
    int r = 0;
    while (r < HIGH_SLOTS && P.slot_qubit[r] == LANE_BITS + r) ++r;
    const int nrun = 64 >> r;
    const unsigned run_bytes = (unsigned)(16u * (32u << r));
    {
        std::string off = "0ull";
        char b[96];
        for (int k = r; k < HIGH_SLOTS; ++k) {
            snprintf(b, sizeof b, " + ((c & %uu) ? 0x%llxull : 0ull)", 1u << (k - r),
                     (unsigned long long)(1ull << P.slot_qubit[k]));
            off += b;
        }
        E.line("auto issue = [&](uint64_t b, int buf) {");
        E.line("  uint64_t* mb = &mbar[buf];");
        E.line("  T* dst = reinterpret_cast<T*>(qoa_dsm) + (buf << %d);", TILE_BITS);
        E.line("  const uint64_t gq = origin(b);");
        E.line("  if (lane == 0) mbar_expect_tx(mb, %uu);", 16u << TILE_BITS);
        E.line("  __syncwarp();");
        E.line("  for (uint32_t c = lane; c < %du; c += 32u)", nrun);
        E.line("    bulk_load(dst + (c << %d), amps + (gq + %s), %uu, mb);", 5 + r, off.c_str(), run_bytes);
        E.line("};");
    }
    E.line("if (threadIdx.x == 0) { mbar_init(&mbar[0], 1); mbar_init(&mbar[1], 1); mbar_init_fence(); }");
    E.line("__syncthreads();");
    E.line("if (valid && wid == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);");
    E.line("uint32_t it = 0;");
    E.line("for (uint64_t blk = blockIdx.x; blk < ntiles; blk += gridDim.x, ++it) {");
    E.line("T* const tile = reinterpret_cast<T*>(qoa_dsm) + ((it & 1u) << %d);", TILE_BITS);
    E.line("const uint64_t g0 = origin(blk);");
    E.line("const uint32_t tw = (uint32_t)lane | ((uint32_t)wid << %d) | ((uint32_t)blk << %d);", LANE_BITS,
           LANE_BITS + WARP_BITS);
    if (P.nang) E.line("pass_angles(P, blk, sang);");
    E.line("T pend = valid ? make_double2(P.phase.x / sqrt(nrm), P.phase.y / sqrt(nrm)) : P.phase;");
    E.line("T a[REGS];");
    {
        const TileMap& m = P.map0;
        unsigned joff[REGS];
        for (int v = 0; v < REGS; ++v) {
            joff[v] = 0;
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) joff[v] |= 1u << m.reg[k];
        }
        auto stride = [&](int t) -> unsigned long long {
            return 1ull << (t < LANE_BITS ? t : P.slot_qubit[t - LANE_BITS]);
        };
        E.line("if (valid) {");
        E.line("mbar_wait(&mbar[it & 1u], (it >> 1) & 1u, status);");
        E.line("const uint32_t jb = (uint32_t)lane | ((wid & 1) ? %uu : 0u) | ((wid & 2) ? %uu : 0u);",
               1u << m.warp[0], 1u << m.warp[1]);
        for (int v = 0; v < REGS; ++v) E.line("a[%d] = tile[jb | %uu];", v, joff[v]);
        E.line("} else {");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               stride(m.warp[0]), stride(m.warp[1]));
        for (int v = 0; v < REGS; ++v) {
            unsigned long long off = 0;
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) off += stride(m.reg[k]);
            E.line("a[%d] = make_double2(tb + 0x%llxull == 0 ? 1.0 : 0.0, 0.0);", v, off);
        }
        E.line("}");
    }
    // every thread is done with both buffers' previous contents: the next
    // tile may now arrive in the other one
    E.line("proxy_fence_async();");
    E.line("__syncthreads();");
    E.line("if (valid && wid == 0 && blk + gridDim.x < ntiles) issue(blk + gridDim.x, (int)((it + 1u) & 1u));");

    const TileMap* cur = emit_ops128(E, P, false, "P.coef");

    {
        const TileMap& m = *cur;
        auto ostride = [&](int t) -> unsigned long long { return 1ull << P.out_qubit[t]; };
        E.line("{");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               ostride(m.warp[0]), ostride(m.warp[1]));
        E.line("double ss = 0.0;");
        for (int v = 0; v < REGS; ++v) {
            unsigned long long off = 0;
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) off += ostride(m.reg[k]);
            E.line("{ const T x = c_mul(a[%d], pend); __stcs(amps + (tb + 0x%llxull), x); ss += c_abs2(x); }", v, off);
        }
        E.line("block_norm_partial(ss, red, partials + blk);");
        E.line("}");
    }
    E.line("}");  // tile loop
    E.line("}");
    return E.s;
}

std::string jit_pass_body(const PassParams& P, bool arena) {
    if (!arena && stream_f64()) return jit_pass_body_streamed(P);
    Emit E;
    // complex128 coefficients: the parameter's constant bank, or the staged copy
    const char* cf = arena ? "scoef" : "P.coef";
    emit_head(E, P, false, arena);
    E.line("const bool valid = nrm > 1e-12;");
    E.line("T pend = valid ? make_double2(P.phase.x / sqrt(nrm), P.phase.y / sqrt(nrm)) : P.phase;");
    E.line("T a[REGS];");
    auto stride = [&](int t) -> unsigned long long {
        return 1ull << (t < LANE_BITS ? t : P.slot_qubit[t - LANE_BITS]);
    };
    {
        const TileMap& m = P.map0;
        E.line("{");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               stride(m.warp[0]), stride(m.warp[1]));
        unsigned long long off[REGS];
        for (int v = 0; v < REGS; ++v) {
            off[v] = 0;
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) off[v] += stride(m.reg[k]);
        }
        E.line("if (valid) {");
        for (int v = 0; v < REGS; ++v) E.line("a[%d] = __ldcs(amps + (tb + 0x%llxull));", v, off[v]);
        E.line("} else {");
        for (int v = 0; v < REGS; ++v) E.line("a[%d] = make_double2(tb + 0x%llxull == 0 ? 1.0 : 0.0, 0.0);", v, off[v]);
        E.line("}");
        E.line("}");
    }
    if (P.nang || arena) E.line("__syncthreads();");

    const TileMap* cur = emit_ops128(E, P, arena, cf);

    // store under the final mapping: tile bit t goes to qubit out_qubit[t]
    {
        const TileMap& m = *cur;
        auto ostride = [&](int t) -> unsigned long long { return 1ull << P.out_qubit[t]; };
        E.line("{");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               ostride(m.warp[0]), ostride(m.warp[1]));
        if (!arena) E.line("double ss = 0.0;");
        for (int v = 0; v < REGS; ++v) {
            unsigned long long off = 0;
            for (int k = 0; k < REG_BITS; ++k)
                if ((v >> k) & 1) off += ostride(m.reg[k]);
            E.line("{ const T x = c_mul(a[%d], pend); __stcs(amps + (tb + 0x%llxull), x);%s }", v, off,
                   arena ? "" : " ss += c_abs2(x);");
        }
        if (!arena) E.line("block_norm_partial(ss, red, partials + blk);");
        E.line("}");
    }
    E.line("}");
    return E.s;
}

// The complex64 form: the packed FP32 tile pass of qoa_pass32.cu
// (pass_tile_p32) for the same PassParams. Registers hold re[j] / im[j] =
// packed (amplitude j, amplitude j + 8); coefficients are rounded to float
// once per CTA into shared memory, as the interpreter stages them.
// The op stream of a complex64 pass (packed FP32 registers re[8] / im[8],
// coefficients in scoef, register tables in stab at tab_at[op]); returns
// the mapping in force at its end.
const TileMap* emit_ops64(Emit& E, const PassParams& P, bool arena, const std::vector<uint32_t>& tab_at) {
    // one pair-exchange layout for the whole pass, when every exchange keeps
    // the same pairing bit and one layout serves all of them
    Swizzle zp;
    bool shared_layout = false;
    {
        std::vector<std::array<int, 3>> tr;
        const TileMap* m = &P.map0;
        const int r3 = P.map0.reg[REG_BITS - 1];
        bool all_pair = true;
        for (uint32_t oi = 0; oi < P.nops; ++oi) {
            const PassOp& op = P.ops[oi];
            if (op.code == PC_DIAG_MX || op.code == PC_DIAG_TM) { oi += op.k; continue; }
            if (op.code != PC_XCHG) continue;
            const TileMap& mn = P.xmap[op.coef];
            all_pair = all_pair && m->reg[REG_BITS - 1] == r3 && mn.reg[REG_BITS - 1] == r3;
            tr.push_back({pair_pos(m->lane[0], r3), pair_pos(m->lane[1], r3), pair_pos(m->lane[2], r3)});
            tr.push_back({pair_pos(mn.lane[0], r3), pair_pos(mn.lane[1], r3), pair_pos(mn.lane[2], r3)});
            m = &mn;
        }
        shared_layout = all_pair && !tr.empty() && pass_swizzle(tr, TILE_BITS - 1, zp);
    }
    int nxchg = 0;

    const TileMap* cur = &P.map0;
    const uint32_t* ow = reinterpret_cast<const uint32_t*>(P.ops);
    for (uint32_t oi = 0; oi < P.nops; ++oi) {
        const PassOp& op = P.ops[oi];
        const int code = op.code;
        const uint32_t c = op.coef;
        const uint32_t cr = op.cond_reg;
        const uint32_t tm = ow[4 * oi + 2];
        const bool g1 = (code >= PC_HF && code < PC_XC) || (code >= PC_RXB && code < PC_DIAG_TA);
        if (arena && rotation(code)) {
            const bool x = rot_x(code);
            const char* fb = x ? "G1_RXB" : "G1_RYB";
            const char* fa = x ? "G1_RXA" : "G1_RYA";
            if ((code & 3) == 3)
                E.line("if (P.ops[%u].code >= %d) g1_bit3<%s>(re, im, scoef + %u); else g1_bit3<%s>(re, im, scoef + %u);",
                       oi, x ? PC_RXB : PC_RYB, fb, c, fa, c);
            else
                E.line("if (P.ops[%u].code >= %d) g1p<%s, %d>(re, im, scoef + %u); else g1p<%s, %d>(re, im, scoef + %u);",
                       oi, x ? PC_RXB : PC_RYB, fb, code & 3, c, fa, code & 3, c);
        } else if (g1) {
            if ((code & 3) == 3) E.line("g1_bit3<%s>(re, im, scoef + %u);", g1_name(code), c);
            else E.line("g1p<%s, %d>(re, im, scoef + %u);", g1_name(code), code & 3, c);
        } else if (code >= PC_XC && code < PC_RXB) {
            E.line("g1c<%s, %d>(re, im, %s, 0x%xu);", (code & ~3) == PC_XC ? "G1_X" : "G1_Y", code & 3,
                   tcond(tm).c_str(), cr);
        } else {
            switch (code) {
                case PC_DIAG_T:
                    if (tm) E.line("if (%s) pend = cmulf(pend, scoef[%u]);", tcond(tm).c_str(), c);
                    else E.line("pend = cmulf(pend, scoef[%u]);", c);
                    break;
                case PC_DIAG_M:
                    E.line("diag_p(re, im, %s, 0x%xu, scoef[%u]);", tcond(tm).c_str(), cr, c);
                    break;
                case PC_DIAG_TA:
                    if (tm) E.line("if (%s) pend = cmulf(pend, sang[%u]);", tcond(tm).c_str(), c);
                    else E.line("pend = cmulf(pend, sang[%u]);", c);
                    break;
                case PC_DIAG_MA:
                    E.line("diag_p(re, im, true, 0x%xu, sang[%u]);", cr, c);
                    break;
                case PC_DIAG_MX:
                case PC_DIAG_TM: {
                    const uint32_t cnt = op.k;
                    bool one = true;
                    E.line("{ float2 f = make_float2(1.f, 0.f);");
                    for (uint32_t e = 1; e <= cnt; ++e) {
                        const PassOp& r = P.ops[oi + e];
                        const uint32_t rtm = ow[4 * (oi + e) + 2];
                        if (!rtm && one) E.line("f = scoef[%u];", (unsigned)r.coef);
                        else if (one) E.line("f = %s ? scoef[%u] : make_float2(1.f, 0.f);", tcond(rtm).c_str(), (unsigned)r.coef);
                        else if (!rtm) E.line("f = cmulf(f, scoef[%u]);", (unsigned)r.coef);
                        else E.line("if (%s) f = cmulf(f, scoef[%u]);", tcond(rtm).c_str(), (unsigned)r.coef);
                        one = false;
                        if (code == PC_DIAG_MX && (e == cnt || ((r.has_tp >> 1) & 1u))) {
                            E.line("diag_p(re, im, true, 0x%xu, f);", (unsigned)r.cond_reg);
                            if (e != cnt) E.line("f = make_float2(1.f, 0.f);");
                            one = true;
                        }
                    }
                    if (code == PC_DIAG_TM && cnt) E.line("pend = cmulf(pend, f);");
                    E.line("}");
                    oi += cnt;
                    break;
                }
                case PC_DIAG_TAB:
                    // a pair whose two factors are exactly 1 is left alone
                    for (int j = 0; j < 8; ++j)
                        if (((tm >> j) | (tm >> (j + 8))) & 1)
                            E.line("cmul2(re[%d], im[%d], stab[%u], stab[%u]);", j, j, 16 * tab_at[oi] + j,
                                   16 * tab_at[oi] + 8 + j);
                    break;
                case PC_FLUSH:
                    E.line("{ const u64p cr = bc(pend.x), ci = bc(pend.y);");
                    for (int j = 0; j < 8; ++j) E.line("cmul2(re[%d], im[%d], cr, ci);", j, j);
                    E.line("pend = make_float2(1.f, 0.f); }");
                    break;
                case PC_XCHG: {
                    const TileMap& mo = *cur;
                    const TileMap& mn = P.xmap[c];
                    if (mo.reg[REG_BITS - 1] == mn.reg[REG_BITS - 1]) {
                        // the pairing bit stays on register bit 3: whole
                        // packed pairs (re[j], im[j]) move as 16-byte units,
                        // indexed by the tile index without that bit
                        const int r3 = mo.reg[REG_BITS - 1];
                        int pos[TILE_BITS];
                        for (int t = 0; t < TILE_BITS; ++t) pos[t] = pair_pos(t, r3);
                        const int so[3] = {pos[mo.lane[0]], pos[mo.lane[1]], pos[mo.lane[2]]};
                        const int sn[3] = {pos[mn.lane[0]], pos[mn.lane[1]], pos[mn.lane[2]]};
                        const Swizzle z = shared_layout ? zp : make_swizzle(so, sn, TILE_BITS - 1);
                        auto off = [&](const TileMap& m, int j) {
                            uint32_t q = 0;
                            for (int k = 0; k < REG_BITS - 1; ++k)
                                if ((j >> k) & 1) q |= 1u << pos[m.reg[k]];
                            return z.f(q);
                        };
                        // with the pass's one layout each thread stores where
                        // it last loaded: only the first exchange waits first
                        if (!shared_layout || nxchg == 0) E.line("__syncthreads();");
                        ++nxchg;
                        std::vector<uint32_t> ks(8);
                        E.line("{ ulonglong2* pt = reinterpret_cast<ulonglong2*>(tile); const uint32_t pb = %s;",
                               swz_base(z, mo, pos).c_str());
                        for (int j = 0; j < 8; ++j) ks[j] = off(mo, j);
                        {
                            const auto acc = swz_access(E, "pt", "ts", swz_base_bits(z, mo, pos), ks);
                            for (int j = 0; j < 8; ++j)
                                E.line("%s = make_ulonglong2(re[%d], im[%d]);", acc[j].c_str(), j, j);
                        }
                        E.line("}");
                        E.line(shared_layout && same_warps(mo, mn) ? "__syncwarp();" : "__syncthreads();");
                        E.line("{ const ulonglong2* pt = reinterpret_cast<const ulonglong2*>(tile); const uint32_t pb = %s;",
                               swz_base(z, mn, pos).c_str());
                        for (int j = 0; j < 8; ++j) ks[j] = off(mn, j);
                        {
                            const auto acc = swz_access(E, "pt", "tl", swz_base_bits(z, mn, pos), ks);
                            for (int j = 0; j < 8; ++j)
                                E.line("{ const ulonglong2 u = %s; re[%d] = u.x; im[%d] = u.y; }", acc[j].c_str(), j, j);
                        }
                        E.line("}");
                        cur = &mn;
                        break;
                    }
                    E.line("__syncthreads();");
                    E.line("{ const uint32_t pb = spos(%s);", tile_base(mo).c_str());
                    for (int j = 0; j < 8; ++j)
                        E.line("tile[pb ^ %uu] = make_float2(lo(re[%d]), lo(im[%d])); tile[pb ^ %uu] = make_float2(hi(re[%d]), hi(im[%d]));",
                               reg_part(mo, j), j, j, reg_part(mo, j | 8), j, j);
                    E.line("}");
                    E.line("__syncthreads();");
                    E.line("{ const uint32_t pb = spos(%s);", tile_base(mn).c_str());
                    for (int j = 0; j < 8; ++j)
                        E.line("{ const float2 a = tile[pb ^ %uu], b = tile[pb ^ %uu]; re[%d] = pk(a.x, b.x); im[%d] = pk(a.y, b.y); }",
                               reg_part(mn, j), reg_part(mn, j | 8), j, j);
                    E.line("}");
                    cur = &mn;
                    break;
                }
                default: break;
            }
        }
    }
    return cur;
}

// The single-state complex64 pass as a persistent kernel (the streamed
// form of jit_pass_body_streamed for packed FP32 registers): coefficients
// and register tables are staged once per CTA, tiles stream through two
// 16 KB shared-memory buffers by bulk copies, results are stored from
// registers with the same arithmetic as k_pass_p32.
std::string jit_pass32_body_streamed(const PassParams& P) {
    Emit E;
    const int lt = (int)P.n - TILE_BITS;
    E.line("(float2* __restrict__ amps, const __grid_constant__ qoa::PassParams P,");
    E.line(" const double* __restrict__ norm2_in, double* __restrict__ partials, uint32_t* __restrict__ status) {");
    E.line("%s", kStreamMark);
    E.line("using namespace qoa;");
    E.line("using namespace qoa::p32;");
    E.line("typedef float2 T;");
    E.line("extern __shared__ __align__(128) unsigned char qoa_dsm[];");
    E.line("__shared__ __align__(8) uint64_t mbar[2];");
    E.line("__shared__ double red[PASS_THREADS / 32];");
    E.line("__shared__ __align__(16) T scoef[%u];", P.ncoef ? P.ncoef : 1);
    if (P.nang) E.line("__shared__ T sang[%u];", P.nang);
    E.line("const int lane = threadIdx.x & 31;");
    E.line("const int wid = threadIdx.x >> 5;");
    E.line("const double nrm = *norm2_in;");
    E.line("const bool valid = nrm > 1e-12;");
    E.line("const uint64_t ntiles = 1ull << %d;", lt);
    E.line("for (uint32_t i = threadIdx.x; i < %uu; i += PASS_THREADS) scoef[i] = make_float2((float)P.coef[i].x, (float)P.coef[i].y);",
           P.ncoef);
    std::vector<uint32_t> tab_at(P.nops, 0);
    {
        uint32_t ntab = 0;
        for (uint32_t oi = 0; oi < P.nops; ++oi) {
            const int code = P.ops[oi].code;
            if (code == PC_DIAG_TAB) tab_at[oi] = ntab++;
            if (code == PC_DIAG_MX || code == PC_DIAG_TM) oi += P.ops[oi].k;
        }
        if (ntab) {
            E.line("__shared__ u64p stab[%u];", 16 * ntab);
            for (uint32_t oi = 0; oi < P.nops; ++oi) {
                const PassOp& op = P.ops[oi];
                if (op.code == PC_DIAG_TAB) {
                    const uint32_t t = tab_at[oi], c = op.coef;
                    E.line("if (threadIdx.x < 8) { const int j = threadIdx.x; const double2 x = P.coef[%u + j], y = P.coef[%u + j];", c, c + 8);
                    E.line("  stab[%u + j] = pk((float)x.x, (float)y.x); stab[%u + j] = pk((float)x.y, (float)y.y); }", 16 * t, 16 * t + 8);
                }
                if (op.code == PC_DIAG_MX || op.code == PC_DIAG_TM) oi += op.k;
            }
        }
    }
    {
        std::string g = "0ull";
        char b[128];
        for (int k = 0; k < lt;) {
            int len = 1;
            while (k + len < lt && P.outer_qubits[k + len] == P.outer_qubits[k] + len) ++len;
            snprintf(b, sizeof b, " | (((b >> %d) & 0x%llxull) << %d)", k,
                     (unsigned long long)((len >= 64) ? ~0ull : ((1ull << len) - 1)), P.outer_qubits[k]);
            g += b;
            k += len;
        }
        E.line("auto origin = [](uint64_t b) -> uint64_t { return %s; };", g.c_str());
    }
    int r = 0;
    while (r < HIGH_SLOTS && P.slot_qubit[r] == LANE_BITS + r) ++r;
    const int nrun = 64 >> r;
    const unsigned run_bytes = (unsigned)(8u * (32u << r));
    {
        std::string off = "0ull";
        char b[96];
        for (int k = r; k < HIGH_SLOTS; ++k) {
            snprintf(b, sizeof b, " + ((c & %uu) ? 0x%llxull : 0ull)", 1u << (k - r),
                     (unsigned long long)(1ull << P.slot_qubit[k]));
            off += b;
        }
        E.line("auto issue = [&](uint64_t b, int buf) {");
        E.line("  uint64_t* mb = &mbar[buf];");
        E.line("  T* dst = reinterpret_cast<T*>(qoa_dsm) + (buf << %d);", TILE_BITS);
        E.line("  const uint64_t gq = origin(b);");
        E.line("  if (lane == 0) mbar_expect_tx(mb, %uu);", 8u << TILE_BITS);
        E.line("  __syncwarp();");
        E.line("  for (uint32_t c = lane; c < %du; c += 32u)", nrun);
        E.line("    bulk_load(dst + (c << %d), amps + (gq + %s), %uu, mb);", 5 + r, off.c_str(), run_bytes);
        E.line("};");
    }
    E.line("if (threadIdx.x == 0) { mbar_init(&mbar[0], 1); mbar_init(&mbar[1], 1); mbar_init_fence(); }");
    E.line("__syncthreads();");
    E.line("if (valid && wid == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);");
    E.line("uint32_t it = 0;");
    E.line("for (uint64_t blk = blockIdx.x; blk < ntiles; blk += gridDim.x, ++it) {");
    E.line("T* const tile = reinterpret_cast<T*>(qoa_dsm) + ((it & 1u) << %d);", TILE_BITS);
    E.line("const uint64_t g0 = origin(blk);");
    E.line("const uint32_t tw = (uint32_t)lane | ((uint32_t)wid << %d) | ((uint32_t)blk << %d);", LANE_BITS,
           LANE_BITS + WARP_BITS);
    if (P.nang) E.line("pass_angles(P, blk, sang);");
    E.line("float2 pend = valid ? make_float2((float)(P.phase.x / sqrt(nrm)), (float)(P.phase.y / sqrt(nrm)))");
    E.line("                    : make_float2((float)P.phase.x, (float)P.phase.y);");
    E.line("u64p re[8], im[8];");
    {
        const TileMap& m = P.map0;
        auto stride = [&](int t) -> unsigned long long {
            return 1ull << (t < LANE_BITS ? t : P.slot_qubit[t - LANE_BITS]);
        };
        E.line("if (valid) {");
        E.line("mbar_wait(&mbar[it & 1u], (it >> 1) & 1u, status);");
        E.line("const uint32_t jb = (uint32_t)lane | ((wid & 1) ? %uu : 0u) | ((wid & 2) ? %uu : 0u);",
               1u << m.warp[0], 1u << m.warp[1]);
        const unsigned j3 = 1u << m.reg[3];
        for (int j = 0; j < 8; ++j) {
            unsigned off = 0;
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) off |= 1u << m.reg[k];
            E.line("{ const float2 a = tile[jb | %uu], b = tile[jb | %uu]; re[%d] = pk(a.x, b.x); im[%d] = pk(a.y, b.y); }",
                   off, off | j3, j, j);
        }
        E.line("} else {");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               stride(m.warp[0]), stride(m.warp[1]));
        for (int j = 0; j < 8; ++j) {
            unsigned long long off = 0;
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) off += stride(m.reg[k]);
            E.line("re[%d] = pk(tb + 0x%llxull == 0 ? 1.f : 0.f, 0.f); im[%d] = 0ull;", j, off, j);
        }
        E.line("}");
    }
    E.line("proxy_fence_async();");
    E.line("__syncthreads();");
    E.line("if (valid && wid == 0 && blk + gridDim.x < ntiles) issue(blk + gridDim.x, (int)((it + 1u) & 1u));");

    const TileMap* cur = emit_ops64(E, P, false, tab_at);

    {
        const TileMap& m = *cur;
        auto ostride = [&](int t) -> unsigned long long { return 1ull << P.out_qubit[t]; };
        E.line("{");
        E.line("const u64p cr = bc(pend.x), ci = bc(pend.y);");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               ostride(m.warp[0]), ostride(m.warp[1]));
        const unsigned long long r3 = ostride(m.reg[3]);
        for (int j = 0; j < 8; ++j) {
            unsigned long long off = 0;
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) off += ostride(m.reg[k]);
            E.line("{ cmul2(re[%d], im[%d], cr, ci); const float2 a = make_float2(lo(re[%d]), lo(im[%d])), b = make_float2(hi(re[%d]), hi(im[%d]));",
                   j, j, j, j, j, j);
            E.line("  __stcs(amps + (tb + 0x%llxull), a); __stcs(amps + (tb + 0x%llxull), b); }", off, off + r3);
        }
        E.line("block_norm_partial(norm2_p(re, im), red, partials + blk);");
        E.line("}");
    }
    E.line("}");  // tile loop
    E.line("}");
    return E.s;
}

std::string jit_pass32_body(const PassParams& P, bool arena) {
    if (!arena && stream_f32()) return jit_pass32_body_streamed(P);
    Emit E;
    emit_head(E, P, true, arena);
    // register tables (PC_DIAG_TAB): staged once per CTA already packed as
    // (factor j, factor j + 8) pairs, real parts then imaginary parts
    std::vector<uint32_t> tab_at(P.nops, 0);
    {
        uint32_t ntab = 0;
        for (uint32_t oi = 0; oi < P.nops; ++oi) {
            const int code = P.ops[oi].code;
            if (code == PC_DIAG_TAB) tab_at[oi] = ntab++;
            if (code == PC_DIAG_MX || code == PC_DIAG_TM) oi += P.ops[oi].k;
        }
        if (ntab) {
            E.line("__shared__ u64p stab[%u];", 16 * ntab);
            for (uint32_t oi = 0; oi < P.nops; ++oi) {
                const PassOp& op = P.ops[oi];
                if (op.code == PC_DIAG_TAB) {
                    const uint32_t t = tab_at[oi], c = op.coef;
                    E.line("if (threadIdx.x < 8) { const int j = threadIdx.x; const double2 x = P.coef[%u + j], y = P.coef[%u + j];", c, c + 8);
                    E.line("  stab[%u + j] = pk((float)x.x, (float)y.x); stab[%u + j] = pk((float)x.y, (float)y.y); }", 16 * t, 16 * t + 8);
                }
                if (op.code == PC_DIAG_MX || op.code == PC_DIAG_TM) oi += op.k;
            }
        }
    }
    E.line("const bool valid = nrm > 1e-12;");
    E.line("float2 pend = valid ? make_float2((float)(P.phase.x / sqrt(nrm)), (float)(P.phase.y / sqrt(nrm)))");
    E.line("                    : make_float2((float)P.phase.x, (float)P.phase.y);");
    E.line("u64p re[8], im[8];");
    auto stride = [&](int t) -> unsigned long long {
        return 1ull << (t < LANE_BITS ? t : P.slot_qubit[t - LANE_BITS]);
    };
    {
        const TileMap& m = P.map0;
        E.line("{");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               stride(m.warp[0]), stride(m.warp[1]));
        const unsigned long long r3 = stride(m.reg[3]);
        E.line("if (valid) {");
        for (int j = 0; j < 8; ++j) {
            unsigned long long off = 0;
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) off += stride(m.reg[k]);
            E.line("{ const float2 a = __ldcs(amps + (tb + 0x%llxull)), b = __ldcs(amps + (tb + 0x%llxull)); re[%d] = pk(a.x, b.x); im[%d] = pk(a.y, b.y); }",
                   off, off + r3, j, j);
        }
        E.line("} else {");
        for (int j = 0; j < 8; ++j) {
            unsigned long long off = 0;
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) off += stride(m.reg[k]);
            E.line("re[%d] = pk(tb + 0x%llxull == 0 ? 1.f : 0.f, 0.f); im[%d] = 0ull;", j, off, j);
        }
        E.line("}");
        E.line("}");
    }
    E.line("__syncthreads();");

    const TileMap* cur = emit_ops64(E, P, arena, tab_at);
    {
        const TileMap& m = *cur;
        auto ostride = [&](int t) -> unsigned long long { return 1ull << P.out_qubit[t]; };
        E.line("{");
        E.line("const u64p cr = bc(pend.x), ci = bc(pend.y);");
        E.line("const uint64_t tb = g0 + (uint64_t)lane + ((wid & 1) ? 0x%llxull : 0ull) + ((wid & 2) ? 0x%llxull : 0ull);",
               ostride(m.warp[0]), ostride(m.warp[1]));
        const unsigned long long r3 = ostride(m.reg[3]);
        for (int j = 0; j < 8; ++j) {
            unsigned long long off = 0;
            for (int k = 0; k < 3; ++k)
                if ((j >> k) & 1) off += ostride(m.reg[k]);
            E.line("{ cmul2(re[%d], im[%d], cr, ci); const float2 a = make_float2(lo(re[%d]), lo(im[%d])), b = make_float2(hi(re[%d]), hi(im[%d]));",
                   j, j, j, j, j, j);
            E.line("  __stcs(amps + (tb + 0x%llxull), a); __stcs(amps + (tb + 0x%llxull), b); }", off, off + r3);
        }
        if (!arena) E.line("block_norm_partial(norm2_p(re, im), red, partials + blk);");
        E.line("}");
    }
    E.line("}");
    return E.s;
}

// ------------------------------------------------------------ the cache
struct JitEntry {
    std::atomic<int> state{0};  // 0 compiling, 1 ready, 2 failed
    cudaKernel_t kernel = nullptr;
    std::string name;
    bool streamed = false;  // persistent double-buffered form (jit_pass*_body_streamed)
    unsigned smem = 0;      // its dynamic shared memory (two tile buffers)
    // streamed form, per device: dynamic shared memory allowed and the
    // persistent grid (SMs x resident CTAs), set at the first launch there
    std::mutex setup_mu;
    uint64_t setup_devices = 0;
    unsigned grid[64] = {};
};

namespace {
constexpr unsigned kStreamSmem = 2u * (16u << TILE_BITS);    // two complex128 tiles
constexpr unsigned kStreamSmem32 = 2u * (8u << TILE_BITS);   // two complex64 tiles

// Grid of a streamed kernel on the current device (0: cannot launch).
unsigned streamed_grid(JitEntry& e) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::lock_guard<std::mutex> lk(e.setup_mu);
    if (!((e.setup_devices >> dev) & 1)) {
        const void* f = reinterpret_cast<const void*>(e.kernel);
        int occ = 0, nsm = 0;
        if (cudaKernelSetAttributeForDevice(e.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem,
                                            dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, PASS_THREADS, e.smem) != cudaSuccess ||
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || occ < 1) {
            cudaGetLastError();
            return 0;
        }
        e.grid[dev] = (unsigned)(occ * nsm);
        e.setup_devices |= 1ull << dev;
    }
    return e.grid[dev];
}
}  // namespace

bool JitKernel::ready() const { return e_ && e_->state.load(std::memory_order_acquire) == 1; }
bool JitKernel::failed() const { return !e_ || e_->state.load(std::memory_order_acquire) == 2; }

cudaError_t JitKernel::launch(void* amps, const PassParams& P, const double* norm2_in, double* partials,
                              uint32_t* status, cudaStream_t st) const {
    if (!ready()) return cudaErrorNotReady;
    const unsigned tiles = 1u << (P.n - TILE_BITS);
    if (e_->streamed) {
        unsigned g = streamed_grid(*e_);
        if (!g) return cudaErrorNotSupported;  // the caller runs the pass on k_pass instead
        // QOA_JIT_STREAM_GRID caps the persistent grid (tests: many tiles per CTA)
        if (const char* v = getenv("QOA_JIT_STREAM_GRID")) {
            const int cap = atoi(v);
            if (cap > 0 && (unsigned)cap < g) g = (unsigned)cap;
        }
        void* args[] = {&amps, const_cast<PassParams*>(&P), &norm2_in, &partials, &status};
        return cudaLaunchKernel(reinterpret_cast<const void*>(e_->kernel), dim3(std::min(g, tiles)),
                                dim3(PASS_THREADS), args, e_->smem, st);
    }
    void* args[] = {&amps, const_cast<PassParams*>(&P), &norm2_in, &partials};
    return cudaLaunchKernel(reinterpret_cast<const void*>(e_->kernel), dim3(tiles), dim3(PASS_THREADS), args, 0, st);
}

cudaError_t JitKernel::launch_arena(const ArenaJob* jobs, uint32_t njobs, uint32_t lt, cudaStream_t st) const {
    if (!ready()) return cudaErrorNotReady;
    if (!njobs) return cudaSuccess;
    void* args[] = {&jobs};
    return cudaLaunchKernel(reinterpret_cast<const void*>(e_->kernel), dim3(njobs << lt), dim3(PASS_THREADS), args, 0,
                            st);
}

namespace {

uint64_t fnv64(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char ch : s) {
        h ^= ch;
        h *= 1099511628211ull;
    }
    return h;
}

bool body_is_c64(const std::string& body) {
    return body.find("using namespace qoa::p32;") != std::string::npos;
}

std::string program_text(const std::vector<std::string>& names, const std::vector<std::string>& bodies) {
    std::string src = kPrelude;
    char head[160];
    for (size_t i = 0; i < names.size(); ++i) {
        const bool c64 = body_is_c64(bodies[i]);
        const bool streamed = bodies[i].find(kStreamMark) != std::string::npos;
        snprintf(head, sizeof head, "extern \"C\" __global__ void __launch_bounds__(%d, %d) %s", PASS_THREADS,
                 streamed ? occ_streamed(c64) : occ_target(c64), names[i].c_str());
        src += head;
        src += bodies[i];
    }
    return src;
}

// NVRTC is loaded at first use (dlopen), so that the library loads, and
// runs every pass on the interpreter kernels, where the toolkit's
// libnvrtc is absent.
struct NvrtcApi {
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetErrorString) error_string = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    std::string why;  // set when unavailable
};

void jit_stop_at_exit();

const NvrtcApi& nvrtc() {
    static const NvrtcApi api = [] {
        NvrtcApi a;
        // the toolkit the library was built with first, by full path: a
        // process may already hold another NVRTC under the same soname
        // (PyTorch's wheels bring their own), whose code generation can
        // differ in the last bit from the interpreter kernels'
        const char* paths[] = {
#ifdef QOA_NVRTC_PATH
            QOA_NVRTC_PATH,
#endif
            "libnvrtc.so.12", "libnvrtc.so"};
        void* h = nullptr;
        for (const char* p : paths)
            if ((h = dlopen(p, RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
        if (!h) {
            a.why = "libnvrtc could not be loaded: passes run on the interpreter kernels";
            return a;
        }
        bool ok = true;
        auto sym = [&](auto& f, const char* name) {
            f = reinterpret_cast<std::remove_reference_t<decltype(f)>>(dlsym(h, name));
            ok = ok && f != nullptr;
        };
        sym(a.create, "nvrtcCreateProgram");
        sym(a.compile, "nvrtcCompileProgram");
        sym(a.log_size, "nvrtcGetProgramLogSize");
        sym(a.log, "nvrtcGetProgramLog");
        sym(a.error_string, "nvrtcGetErrorString");
        sym(a.cubin_size, "nvrtcGetCUBINSize");
        sym(a.cubin, "nvrtcGetCUBIN");
        sym(a.destroy, "nvrtcDestroyProgram");
        if (!ok) {
            a = NvrtcApi();
            a.why = "libnvrtc lacks an entry point the engine needs: passes run on the interpreter kernels";
        }
        return a;
    }();
    return api;
}

// NVRTC: the kernels named names[i] with bodies[i], as one sm_100a cubin.
bool build_cubin(const std::vector<std::string>& names, const std::vector<std::string>& bodies,
                 std::vector<char>& cubin, std::string& err) {
    const NvrtcApi& nv = nvrtc();
    if (!nv.create) {
        err = nv.why;
        return false;
    }
    const std::string src = program_text(names, bodies);
    const char* hdrs[] = {kTypesHeader, kDevHeader, kDev32Header};
    const char* hnames[] = {"qoa_kernels.cuh", "qoa_pass_dev.cuh", "qoa_pass32_dev.cuh"};
    nvrtcProgram prog;
    if (nv.create(&prog, src.c_str(), "qoa_jit_pass.cu", 3, hdrs, hnames) != NVRTC_SUCCESS) {
        err = "nvrtcCreateProgram failed";
        return false;
    }
    const char* opts[] = {"-arch=sm_100a", "-std=c++17", "--fmad=true"};
    const nvrtcResult rc = nv.compile(prog, 3, opts);
    // NVRTC registers its own exit-time teardown lazily, inside compiles;
    // exit handlers run last-registered first, so registering the compile
    // threads' shutdown after every compile makes it run before NVRTC's:
    // no compile thread can then still be inside NVRTC when it is torn
    // down (an in-flight compile at exit crashed in nvrtcCompileProgram)
    std::atexit(jit_stop_at_exit);
    if (rc != NVRTC_SUCCESS) {
        size_t n = 0;
        nv.log_size(prog, &n);
        std::string log(n, '\0');
        if (n) nv.log(prog, &log[0]);
        err = std::string("NVRTC: ") + nv.error_string(rc) + ": " + log.substr(0, 2000);
        nv.destroy(&prog);
        return false;
    }
    size_t cs = 0;
    nv.cubin_size(prog, &cs);
    cubin.resize(cs);
    nv.cubin(prog, cubin.data());
    nv.destroy(&prog);
    return true;
}

std::string kernel_name(const std::string& body) {
    char nm[48];
    const bool arena = body.compare(0, 20, "(const qoa::ArenaJob") == 0;
    snprintf(nm, sizeof nm, "qoa_jit_%s%s_%016llx", arena ? "arena" : "pass", body_is_c64(body) ? "32" : "",
             (unsigned long long)fnv64(body));
    return nm;
}

// One kernel per NVRTC program: the kernels of a circuit compile side by
// side on a pool of host threads.
struct JitJob {
    std::shared_ptr<JitEntry> entry;
    std::string body;
};

class JitCompiler {
public:
    ~JitCompiler() { shutdown(); }

    // Stops compiling: queued compiles are dropped (their kernels stay on
    // the interpreter), compiles in flight finish without loading, and the
    // compile threads are joined. Runs at process exit before NVRTC's own
    // teardown (see nvrtc()), so that no thread is inside NVRTC then.
    void shutdown() {
        std::vector<std::thread> ws;
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            for (auto& j : queue_) {
                j.entry->state.store(2, std::memory_order_release);
                --pending_;
                ++failures_;
            }
            queue_.clear();
            ws.swap(workers_);
        }
        cv_.notify_all();
        done_cv_.notify_all();
        for (auto& t : ws)
            if (t.joinable()) t.join();
    }

    std::vector<JitKernel> request(const std::vector<std::string>& bodies, JitWhen when) {
        const bool wait = when == JitWhen::WAIT;
        std::vector<JitKernel> out;
        std::vector<std::shared_ptr<JitEntry>> mine;
        out.reserve(bodies.size());
        bool queued = false;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (stop_) {  // exiting: everything stays on the interpreter
                out.resize(bodies.size());
                return out;
            }
            for (const std::string& b : bodies) {
                const Key key{fnv64(b), std::hash<std::string>()(b)};
                auto it = cache_.find(key);
                if (it != cache_.end()) {
                    ++hits_;
                    out.emplace_back(it->second);
                    mine.push_back(it->second);
                    continue;
                }
                if (when == JitWhen::SECOND_SIGHTING) {
                    // a structure is compiled the second time it is seen:
                    // one-off passes (a noisy trajectory's Pauli draws, a
                    // program run once) never pay for a compile
                    if (seen_.size() > (1u << 20)) seen_.clear();
                    if (++seen_[key.a] < 2) {
                        out.emplace_back();
                        continue;
                    }
                }
                if (cache_.size() >= max_kernels_) {
                    // the cache is full: this structure stays interpreted
                    out.emplace_back();
                    continue;
                }
                ++misses_;
                auto e = std::make_shared<JitEntry>();
                e->name = kernel_name(b);
                e->streamed = b.find(kStreamMark) != std::string::npos;
                e->smem = e->streamed ? (body_is_c64(b) ? kStreamSmem32 : kStreamSmem) : 0;
                cache_.emplace(key, e);
                queue_.push_back(JitJob{e, b});
                ++pending_;
                queued = true;
                out.emplace_back(e);
                mine.push_back(e);
            }
            if (queued && workers_.empty()) {
                const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
                for (unsigned t = 0; t < nt; ++t) workers_.emplace_back([this] { run(); });
            }
        }
        if (queued) cv_.notify_all();
        if (wait) {
            std::unique_lock<std::mutex> lk(mu_);
            done_cv_.wait(lk, [&] {
                for (auto& e : mine)
                    if (e->state.load(std::memory_order_acquire) == 0) return false;
                return true;
            });
        }
        return out;
    }

    void wait_all() {
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }

    JitStats stats() {
        std::lock_guard<std::mutex> lk(mu_);
        return JitStats{ready_, hits_, misses_, failures_, compile_ms_};
    }
    std::string last_error() {
        std::lock_guard<std::mutex> lk(mu_);
        return last_error_;
    }

private:
    void run() {
        // these threads load libraries while other threads may be capturing
        // graphs: they must not join those captures' rules
        cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
        cudaThreadExchangeStreamCaptureMode(&mode);
        for (;;) {
            JitJob job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
                if (stop_) return;
                job = std::move(queue_.front());
                queue_.pop_front();
            }
            const auto t0 = std::chrono::steady_clock::now();
            std::string err;
            const bool ok = compile(job, err);
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            {
                std::lock_guard<std::mutex> lk(mu_);
                compile_ms_ += ms;
                job.entry->state.store(ok ? 1 : 2, std::memory_order_release);
                if (ok) ++ready_;
                else {
                    ++failures_;
                    last_error_ = err;
                }
                --pending_;
            }
            done_cv_.notify_all();
        }
    }

    bool compile(JitJob& job, std::string& err) {
        std::vector<char> cubin;
        if (!build_cubin({job.entry->name}, {job.body}, cubin, err)) return false;
        {
            // at exit the CUDA runtime may already be gone: load nothing
            std::lock_guard<std::mutex> lk(mu_);
            if (stop_) {
                err = "process exiting";
                return false;
            }
        }
        cudaLibrary_t lib = nullptr;
        cudaError_t ce = cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            err = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(ce);
            return false;
        }
        // the library stays loaded for the life of the process (the cache
        // keeps its kernel)
        cudaKernel_t k = nullptr;
        if (cudaLibraryGetKernel(&k, lib, job.entry->name.c_str()) != cudaSuccess) {
            cudaGetLastError();
            err = "kernel missing from the compiled library: " + job.entry->name;
            return false;
        }
        job.entry->kernel = k;
        return true;
    }

    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    // Cache key: two independent 64-bit hashes of the kernel text (the text
    // itself is dropped once compiled).
    struct Key {
        uint64_t a, b;
        bool operator==(const Key& o) const { return a == o.a && b == o.b; }
    };
    struct KeyHash {
        size_t operator()(const Key& k) const { return (size_t)(k.a ^ (k.b * 0x9e3779b97f4a7c15ull)); }
    };
    std::unordered_map<Key, std::shared_ptr<JitEntry>, KeyHash> cache_;
    // At most this many kernels are loaded per process (QOA_JIT_MAX_KERNELS,
    // default 8192): beyond it new structures stay on the interpreter.
    const size_t max_kernels_ = [] {
        const char* v = getenv("QOA_JIT_MAX_KERNELS");
        const long k = v ? atol(v) : 0;
        return k > 0 ? (size_t)k : (size_t)8192;
    }();
    std::unordered_map<uint64_t, uint32_t> seen_;  // sightings of structures not yet compiled
    std::deque<JitJob> queue_;
    std::vector<std::thread> workers_;
    bool stop_ = false;
    uint64_t pending_ = 0;
    uint64_t ready_ = 0, hits_ = 0, misses_ = 0, failures_ = 0;
    double compile_ms_ = 0.0;
    std::string last_error_;
};

JitCompiler& compiler() {
    static JitCompiler c;
    return c;
}

void jit_stop_at_exit() { compiler().shutdown(); }

}  // namespace

std::string jit_program(const std::vector<std::string>& bodies) {
    std::vector<std::string> names;
    for (const std::string& b : bodies) names.push_back(kernel_name(b));
    return program_text(names, bodies);
}

bool jit_compile_only(const std::vector<std::string>& bodies, std::string& err) {
    const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
    std::atomic<size_t> next{0};
    std::mutex emu;
    bool ok = true;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < bodies.size();) {
                std::vector<char> cubin;
                std::string e;
                if (!build_cubin({kernel_name(bodies[i])}, {bodies[i]}, cubin, e)) {
                    std::lock_guard<std::mutex> lk(emu);
                    if (ok) err = e;
                    ok = false;
                }
            }
        });
    for (auto& th : pool) th.join();
    return ok;
}

std::vector<JitKernel> jit_request(const std::vector<std::string>& bodies, JitWhen when) {
    return compiler().request(bodies, when);
}
void jit_wait_all() { compiler().wait_all(); }
JitStats jit_stats() { return compiler().stats(); }
std::string jit_last_error() { return compiler().last_error(); }

}  // namespace qoa
