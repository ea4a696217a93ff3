// qoa_exe.cpp — the bytecode front-end: .qexe / .qx program files executed on
// the engine.
//
// File layout (parse_exe_file, main.rs:1711-1745): 4-byte magic ("QEXE",
// "OEXE", "QOX ", "XEXE", "QEX ", "QX\0\0"), a version byte, a little-endian
// u32 payload length, then the payload of variable-length instructions.
//
// qoa_exe_parse restates the qubit-count scan of `qoa run` (main.rs:3844-4226,
// the same rules as run_exe's first pass, main.rs:1879-2258): the state gets
// (largest qubit byte seen) + 1 qubits.
//
// qoa_exe_run restates run_exe's execution loop (main.rs:2314-3722)
// instruction for instruction, including what that loop leaves out: QINIT,
// RESET, PHASE, APPLYCPHASE, SETPHASE and the ENTANGLE* family advance
// without touching the state, LOOPSTART pushes no loop (so LOOPEND only
// reports a missing LOOPSTART), and SQRT / EXP / LOG leave the registers
// alone. QOA_EXE_LOOPS turns on working loops (LOOPSTART n pushes n
// iterations). Quantum instructions are not applied one by one: they collect
// into an op list that goes to the engine in one qoa_apply (so consecutive
// gates fuse into tile passes) whenever a measurement outcome is needed and
// at the end. Classical control flow never depends on measurement outcomes
// in this instruction set, so the order of effects is unchanged.
//
// Host-side differences, stated: printed text goes to a caller buffer; RAND
// draws from the counter-based generator keyed by the handle seed (SEEDRNG
// re-keys it) instead of an OS-seeded StdRng; INPUT stores 0.0 (a library has
// no console); GETTIME reads the wall clock; DUMPSTATE prints nothing;
// EXITCODE ends the program and returns its code instead of ending the
// process. Measurements draw from the handle's seeded measurement stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qoa_cuda.h"

namespace qoa {
void note_global_error(const char* msg);
}

namespace {

constexpr size_t kRegs = 24;
constexpr size_t kMemBytes = 1 << 20;
constexpr uint32_t kRandStream = 0x72616e64u;  // "rand"

bool magic_kind(const uint8_t* m, char* kind) {
    struct K { const char* magic; const char* name; };
    static const K ks[] = {{"QEXE", "qexe"}, {"OEXE", "oexe"}, {"QOX ", "qox"},
                           {"XEXE", "xexe"}, {"QEX ", "qex"}, {"QX\0\0", "qx"}};
    for (const K& k : ks)
        if (std::memcmp(m, k.magic, 4) == 0) {
            std::snprintf(kind, 8, "%s", k.name);
            return true;
        }
    return false;
}

int parse_header(const uint8_t* file, size_t len, qoa_exe_info* info) {
    std::memset(info, 0, sizeof *info);
    if (!file || len < 9) {
        qoa::note_global_error("exe: file too short to contain a valid header and payload length");
        return QOA_E_ARG;
    }
    if (!magic_kind(file, info->kind)) {
        qoa::note_global_error("exe: unknown or unsupported header");
        return QOA_E_ARG;
    }
    info->version = file[4];
    const uint64_t pl = (uint64_t)file[5] | ((uint64_t)file[6] << 8) | ((uint64_t)file[7] << 16) |
                        ((uint64_t)file[8] << 24);
    if (len < 9 + pl) {
        qoa::note_global_error("exe: file shorter than its header's payload length");
        return QOA_E_ARG;
    }
    info->payload_offset = 9;
    info->payload_len = pl;
    return QOA_OK;
}

// End of a NUL-terminated string starting at `start`: the NUL's index, or
// `start` when there is none (Rust's position(..).unwrap_or(0)).
size_t str_end(const uint8_t* p, size_t len, size_t start) {
    for (size_t k = start; k < len; ++k)
        if (p[k] == 0) return k;
    return start;
}

// The qubit-count scan (main.rs:3855-4225).
uint32_t scan_max_qubit(const uint8_t* p, size_t len, bool* any) {
    size_t i = 0, mq = 0;
    auto q = [&](size_t at) { if (at < len && p[at] > mq) mq = p[at]; };
    auto str_from = [&](size_t start) -> size_t { return str_end(p, len, start) + 1; };
    while (i < len) {
        const uint8_t op = p[i];
        switch (op) {
            case 0x04: case 0x18: case 0x32: case 0x79: case 0x7a:
            case 0x05: case 0x06: case 0x07: case 0x0d: case 0x0e: case 0x0a: case 0x59: case 0x5a:
            case 0x5c: case 0x5d: case 0x61: case 0x62: case 0x6f: case 0x71: case 0x9b: case 0xa0:
            case 0xa1: case 0xac: case 0x50:
                if (i + 1 >= len) return (uint32_t)mq;
                q(i + 1); i += 2; break;
            case 0x1d: case 0x75: case 0x76:
            case 0x08: case 0x22: case 0x23: case 0x0f: case 0x24: case 0x66: case 0x67: case 0x6a:
            case 0x6d: case 0x82: case 0x83: case 0x21: case 0x39: case 0x68: case 0x4e:
                if (i + 9 >= len) return (uint32_t)mq;
                q(i + 1); i += 10; break;
            case 0x74: case 0x77: case 0x37: case 0x6c: case 0x72: case 0x81:
                if (i + 17 >= len) return (uint32_t)mq;
                q(i + 1); i += 18; break;
            case 0xff: case 0x00: case 0x8d: case 0x97:
                i += 1; break;
            case 0x17: case 0x1e: case 0x0b: case 0x1f: case 0x65: case 0x69: case 0x20: case 0xa4:
            case 0x51: case 0x52: case 0x53: case 0x11: case 0x12:
                if (i + 2 >= len) return (uint32_t)mq;
                q(i + 1); q(i + 2); i += 3; break;
            case 0x0c: case 0x54: case 0x55: case 0x56: case 0x57: case 0x58: case 0x63: case 0xa8: case 0x31:
                if (i + 3 >= len) return (uint32_t)mq;
                q(i + 1); i += 4; break;
            case 0x13: case 0x14: {
                if (i + 1 >= len) return (uint32_t)mq;
                const size_t n = p[i + 1];
                if (i + 2 + n > len) return (uint32_t)mq;
                for (size_t j = 0; j < n; ++j) q(i + 2 + j);
                i += 2 + n;
                break;
            }
            case 0x15: case 0x16: {
                if (i + 4 >= len) return (uint32_t)mq;
                // the scan overwrites its running maximum here
                mq = std::max(std::max(p[i + 1], p[i + 2]), std::max(p[i + 3], p[i + 4]));
                if (op == 0x16) {
                    if (i + 5 > len) return (uint32_t)mq;
                    i = str_from(i + 5);
                } else {
                    i += 5;
                }
                break;
            }
            case 0x19: case 0x1a: case 0x1b: case 0x87: case 0x38: case 0x3a: case 0x3b: case 0x3c:
            case 0x5b: case 0x6b: case 0x6e: case 0x73: case 0x7c: case 0x7d: case 0x7f: case 0x85:
            case 0x86:
                if (i + 1 >= len) return (uint32_t)mq;
                q(i + 1); i = str_from(i + 2); break;
            case 0x02: {
                if (i + 9 >= len) return (uint32_t)mq;
                q(i + 1);
                const bool cz = p[i + 2] == 'c' && p[i + 3] == 'z' &&
                                std::all_of(p + i + 4, p + i + 10, [](uint8_t b) { return b == 0; });
                if (cz) {
                    if (i + 10 >= len) return (uint32_t)mq;
                    q(i + 10); i += 11;
                } else {
                    i += 10;
                }
                break;
            }
            case 0x33: i += 11; break;
            case 0x34: {
                if (i + 2 >= len) return (uint32_t)mq;
                const size_t n = p[i + 2];
                for (size_t j = 0; j < n; ++j) q(i + 3 + j);
                i += 3 + n + n * 8;
                break;
            }
            case 0x35: case 0x36:
                if (i + 10 >= len) return (uint32_t)mq;
                q(i + 1); q(i + 2); i += 11; break;
            case 0x3d: case 0x3e: case 0x3f: case 0x40: case 0x4a: case 0x4b: {
                const size_t m = str_from(i + 1);
                i = str_from(m);
                break;
            }
            case 0x41: case 0x42: case 0x43: case 0x44: case 0x45: {
                const size_t a = str_from(i + 1), b = str_from(a);
                i = str_from(b);
                break;
            }
            case 0x46: case 0x47: case 0x4f: case 0x49: case 0x4c: case 0x88:
                i = str_from(i + 1); break;
            case 0x5e: {
                if (i + 2 >= len) return (uint32_t)mq;
                q(i + 1);
                const size_t e = str_from(i + 2);
                if (e + 8 > len) return (uint32_t)mq;
                i = e + 8;
                break;
            }
            case 0x5f: case 0x70:
                if (i + 9 >= len) return (uint32_t)mq;
                q(i + 1); i = str_from(i + 10); break;
            case 0x60: {
                if (i + 1 >= len) return (uint32_t)mq;
                const size_t n = p[i + 1];
                for (size_t j = 0; j < n; ++j) q(i + 2 + j);
                i = str_from(i + 2 + n);
                break;
            }
            case 0x64: case 0x7e: {
                if (i + 1 >= len) return (uint32_t)mq;
                q(i + 1);
                const size_t a = str_from(i + 2);
                i = str_from(a);
                break;
            }
            case 0x80:
                if (i + 2 >= len) return (uint32_t)mq;
                q(i + 1); q(i + 2); i = str_from(i + 3); break;
            case 0x84: {
                if (i + 4 >= len) return (uint32_t)mq;
                const size_t nin = p[i + 1], nout = p[i + 2];
                i = str_from(i + 4) + nin + nout;
                break;
            }
            case 0x90: case 0x91: case 0xa3: case 0xad:
                if (i + 9 >= len) return (uint32_t)mq;
                i += 9; break;
            case 0x92: case 0x93: case 0x94: case 0x95:
                if (i + 11 >= len) return (uint32_t)mq;
                i += 11; break;
            case 0x96: case 0x9e: case 0xa2: case 0x9f:
                if (i + 9 >= len) return (uint32_t)mq;
                i += 10; break;
            case 0x98: {
                if (i + 9 >= len) return (uint32_t)mq;
                uint64_t sl = 0;
                std::memcpy(&sl, p + i + 1, 8);
                if (i + 9 + sl >= len) return (uint32_t)mq;
                i += 1 + 8 + sl + 1 + p[i + 9 + sl];
                break;
            }
            case 0x99: case 0x9a: {
                if (i + 9 >= len) return (uint32_t)mq;
                uint64_t sl = 0;
                std::memcpy(&sl, p + i + 1, 8);
                i += 1 + 8 + sl;
                break;
            }
            case 0xa5: case 0xa6: case 0xa7: case 0xa9: case 0xaa:
                if (i + 3 >= len) return (uint32_t)mq;
                i += 4; break;
            case 0xae:
                if (i + 5 >= len) return (uint32_t)mq;
                i += 5; break;
            case 0x01:
                if (i + 1 >= len) return (uint32_t)mq;
                i += 2; break;
            default:
                i += 1;
        }
        *any = true;
    }
    return (uint32_t)mq;
}

// Rust's `{}` for f64: shortest round-trip digits, never an exponent.
std::string rust_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char b[400];
    auto r = std::to_chars(b, b + sizeof b, v, std::chars_format::fixed);
    return std::string(b, r.ptr);
}

// f64 -> u64 as Rust's `as` (saturating, NaN -> 0)
uint64_t as_u64(double v) {
    if (!(v > 0)) return 0;
    if (v >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)v;
}

struct VM {
    const uint8_t* p = nullptr;
    size_t len = 0;
    uint32_t flags = 0;
    uint64_t max_steps = 0;
    qoa_state_t s = nullptr;          // null: trace only
    std::vector<qoa_op>* trace = nullptr;
    std::vector<qoa_op> pending;
    double regs[kRegs] = {};
    std::vector<uint8_t> mem;
    std::vector<size_t> calls;
    std::vector<std::pair<size_t, uint64_t>> loops;
    std::string out;
    uint64_t rand_seed = 0, rand_ctr = 0;
    qoa_exe_result res{};
    std::string err;

    bool need(size_t i, size_t k) {  // bytes [i, i+k) readable
        if (i + k <= len) return true;
        char b[96];
        std::snprintf(b, sizeof b, "truncated instruction 0x%02X at byte %zu", i < len ? p[i] : 0u, i);
        err = b;
        return false;
    }
    double f64(size_t at) const { double v; std::memcpy(&v, p + at, 8); return v; }
    uint64_t u64(size_t at) const { uint64_t v; std::memcpy(&v, p + at, 8); return v; }
    int64_t i64(size_t at) const { int64_t v; std::memcpy(&v, p + at, 8); return v; }
    size_t after_str(size_t start) const { return str_end(p, len, start) + 1; }

    void gate(uint32_t opc, std::initializer_list<uint32_t> qs, double angle = 0.0) {
        qoa_op o;
        std::memset(&o, 0, sizeof o);
        o.opcode = opc;
        o.nq = (uint32_t)qs.size();
        int k = 0;
        for (uint32_t q : qs) o.q[k++] = q;
        o.angle = angle;
        pending.push_back(o);
        res.gates++;
    }

    int flush() {
        if (pending.empty()) return QOA_OK;
        int rc = QOA_OK;
        if (s) {
            rc = qoa_apply(s, pending.data(), pending.size());
            if (rc == QOA_E_RANGE) {  // skipped out-of-range ops: printed and ignored upstream
                res.range_errors++;
                rc = QOA_OK;
            }
        } else if (trace) {
            trace->insert(trace->end(), pending.begin(), pending.end());
        }
        pending.clear();
        return rc;
    }

    // qs.measure(q): outcome, or 0 in trace mode
    int measure(uint32_t q, uint32_t* outcome) {
        res.measurements++;
        *outcome = 0;
        if (!s) {
            gate(QOA_OP_MEASURE, {q});
            res.gates--;
            return flush();
        }
        int rc = flush();
        if (rc) return rc;
        rc = qoa_measure(s, q, -1.0, outcome);
        if (rc == QOA_E_RANGE) {  // "error measuring qubit": outcome 0, program goes on
            res.range_errors++;
            *outcome = 0;
            return QOA_OK;
        }
        return rc;
    }

    int run() {
        size_t i = 0;
        uint64_t steps = 0;
        while (i < len) {
            if (max_steps && steps >= max_steps) {
                err = "step limit reached (a jump or call loop that does not end?)";
                return QOA_E_STATE;
            }
            ++steps;
            res.instructions++;
            const uint8_t op = p[i];
            const size_t at = i;
            auto rd = [&](size_t k) { return need(at, k); };
            auto jump_to = [&](int64_t target) -> bool {  // false: leaves the program
                if (target < 0 || (uint64_t)target >= len) { i = len; return false; }
                i = (size_t)target;
                return true;
            };
            switch (op) {
                case 0x04: case 0x0a: case 0x79: case 0x7a: case 0x59: case 0x5a: case 0x5c: case 0x5d:
                case 0x61: case 0x62: case 0x6f: case 0xa0: case 0xa1:
                    if (!rd(2)) return QOA_E_ARG;
                    i += 2; break;
                case 0x1d: case 0x75: case 0x76: case 0x24: case 0x39: case 0x4e: case 0x66: case 0x67:
                case 0x68: case 0x6a: case 0x6d:
                    if (!rd(10)) return QOA_E_ARG;
                    i += 10; break;
                case 0x74: case 0x77: case 0x37: case 0x6c: case 0x72: case 0x81:
                    if (!rd(18)) return QOA_E_ARG;
                    i += 18; break;
                case 0x18: {  // charout: measure, print the outcome as a char
                    if (!rd(2)) return QOA_E_ARG;
                    uint32_t v;
                    int rc = measure(p[i + 1], &v);
                    if (rc) return rc;
                    out.push_back((char)(uint8_t)v);
                    res.chars_out++;
                    i += 2;
                    break;
                }
                case 0x32: {
                    if (!rd(2)) return QOA_E_ARG;
                    uint32_t v;
                    int rc = measure(p[i + 1], &v);
                    if (rc) return rc;
                    i += 2;
                    break;
                }
                case 0xff:
                    res.halted = 1;
                    i = len;
                    break;
                case 0x00: case 0x8d: case 0x4d: case 0xab: case 0x9c:
                    i += 1; break;
                case 0x97:
                    if (!calls.empty()) { i = calls.back(); calls.pop_back(); }
                    else i += 1;
                    break;
                case 0x01:
                    if (!rd(2)) return QOA_E_ARG;
                    if (flags & QOA_EXE_LOOPS) loops.push_back({i + 2, p[i + 1]});
                    i += 2;
                    break;
                case 0x10:
                    if (!loops.empty()) {
                        auto [start, left] = loops.back();
                        loops.pop_back();
                        if (left > 1) { loops.push_back({start, left - 1}); i = start; }
                        else i += 1;
                    } else {
                        res.loop_errors++;  // "loopend without matching loopstart"
                        i += 1;
                    }
                    break;
                case 0x02: {  // qgate: 8-byte name, "cz" takes a target byte
                    if (!rd(10)) return QOA_E_ARG;
                    const uint32_t q = p[i + 1];
                    size_t nl = 8;
                    while (nl > 0 && p[i + 2 + nl - 1] == 0) --nl;
                    const std::string name((const char*)p + i + 2, nl);
                    if (name == "h") { gate(QOA_OP_H, {q}); i += 10; }
                    else if (name == "x") { gate(QOA_OP_X, {q}); i += 10; }
                    else if (name == "cz") {
                        if (!rd(11)) return QOA_E_ARG;
                        gate(QOA_OP_CZ, {q, p[i + 10]});
                        i += 11;
                    } else {
                        res.unsupported++;
                        i += 10;
                    }
                    break;
                }
                case 0x05: if (!rd(2)) return QOA_E_ARG; gate(QOA_OP_H, {p[i + 1]}); i += 2; break;
                case 0x06: if (!rd(2)) return QOA_E_ARG; gate(QOA_OP_Z, {p[i + 1]}); i += 2; break;
                case 0x07: if (!rd(2)) return QOA_E_ARG; gate(QOA_OP_X, {p[i + 1]}); i += 2; break;
                case 0x0d: if (!rd(2)) return QOA_E_ARG; gate(QOA_OP_T, {p[i + 1]}); i += 2; break;
                case 0x0e: if (!rd(2)) return QOA_E_ARG; gate(QOA_OP_S, {p[i + 1]}); i += 2; break;
                case 0x08: if (!rd(10)) return QOA_E_ARG; gate(QOA_OP_P, {p[i + 1]}, f64(i + 2)); i += 10; break;
                case 0x0f: if (!rd(10)) return QOA_E_ARG; gate(QOA_OP_RZ, {p[i + 1]}, f64(i + 2)); i += 10; break;
                case 0x22: if (!rd(10)) return QOA_E_ARG; gate(QOA_OP_RX, {p[i + 1]}, f64(i + 2)); i += 10; break;
                case 0x23: if (!rd(10)) return QOA_E_ARG; gate(QOA_OP_RY, {p[i + 1]}, f64(i + 2)); i += 10; break;
                case 0x0b: if (!rd(3)) return QOA_E_ARG; gate(QOA_OP_SWAP, {p[i + 1], p[i + 2]}); i += 3; break;
                case 0x0c:
                    if (!rd(4)) return QOA_E_ARG;
                    gate(QOA_OP_CSWAP, {p[i + 1], p[i + 2], p[i + 3]});
                    i += 4;
                    break;
                case 0x17: if (!rd(3)) return QOA_E_ARG; gate(QOA_OP_CNOT, {p[i + 1], p[i + 2]}); i += 3; break;
                case 0x1e: if (!rd(3)) return QOA_E_ARG; gate(QOA_OP_CZ, {p[i + 1], p[i + 2]}); i += 3; break;
                case 0x1c: gate(QOA_OP_RESETALL, {}); i += 1; break;
                case 0x35:
                    if (!rd(11)) return QOA_E_ARG;
                    gate(QOA_OP_CPHASE, {p[i + 1], p[i + 2]}, f64(i + 3));
                    i += 11;
                    break;
                case 0x36: if (!rd(11)) return QOA_E_ARG; i += 11; break;
                case 0x33: {
                    if (!rd(11)) return QOA_E_ARG;
                    const uint32_t q = p[i + 1];
                    const char axis = (char)p[i + 2];
                    const double a = f64(i + 3);
                    if (axis == 'x') gate(QOA_OP_RX, {q}, a);
                    else if (axis == 'y') gate(QOA_OP_RY, {q}, a);
                    else if (axis == 'z') gate(QOA_OP_RZ, {q}, a);
                    else res.unsupported++;
                    i += 11;
                    break;
                }
                case 0x34: {
                    if (!rd(3)) return QOA_E_ARG;
                    const char axis = (char)p[i + 1];
                    const size_t n = p[i + 2];
                    if (!rd(3 + n + 8)) return QOA_E_ARG;
                    const double a = f64(i + 3 + n);
                    for (size_t j = 0; j < n; ++j) {
                        const uint32_t q = p[i + 3 + j];
                        if (axis == 'x') gate(QOA_OP_RX, {q}, a);
                        else if (axis == 'y') gate(QOA_OP_RY, {q}, a);
                        else if (axis == 'z') gate(QOA_OP_RZ, {q}, a);
                        else res.unsupported++;
                    }
                    i += 3 + n + 8;
                    break;
                }
                case 0x11: case 0x12: case 0x1f: case 0x20: case 0x51: case 0x52: case 0x53: case 0x65:
                case 0x71: case 0x63: case 0xa4:
                    if (!rd(3)) return QOA_E_ARG;
                    i += 3; break;
                case 0x13: case 0x14:
                    if (!rd(2) || !rd(2 + (size_t)p[i + 1])) return QOA_E_ARG;
                    i += 2 + p[i + 1];
                    break;
                case 0x15: if (!rd(5)) return QOA_E_ARG; i += 5; break;
                case 0x16: if (!rd(5)) return QOA_E_ARG; i = after_str(i + 5); break;
                case 0x19: case 0x80: if (!rd(3)) return QOA_E_ARG; i = after_str(i + 3); break;
                case 0x1a: case 0x1b: case 0x38: case 0x3a: case 0x3b: case 0x3c: case 0x5b: case 0x6b:
                case 0x6e: case 0x73:
                    if (!rd(2)) return QOA_E_ARG;
                    i = after_str(i + 2); break;
                case 0x3d: case 0x3e: case 0x3f: case 0x40: case 0x4a: case 0x4b:
                    i = after_str(after_str(i + 1)); break;
                case 0x41: case 0x42: case 0x43: case 0x44: case 0x45:
                    i = after_str(after_str(after_str(i + 1))); break;
                case 0x46: case 0x47: case 0x4f: case 0x49: case 0x4c: case 0x88:
                    i = after_str(i + 1); break;
                case 0x64: case 0x7e: if (!rd(2)) return QOA_E_ARG; i = after_str(after_str(i + 2)); break;
                case 0x5e: {
                    if (!rd(2)) return QOA_E_ARG;
                    const size_t e = str_end(p, len, i + 2);
                    if (e + 9 > len) { need(len, 1); return QOA_E_ARG; }
                    i = e + 9;
                    break;
                }
                case 0x5f: case 0x70: if (!rd(10)) return QOA_E_ARG; i = after_str(i + 10); break;
                case 0x60:
                    if (!rd(2) || !rd(2 + (size_t)p[i + 1])) return QOA_E_ARG;
                    i = after_str(i + 2 + p[i + 1]);
                    break;
                case 0x69: if (!rd(11)) return QOA_E_ARG; i += 11; break;
                case 0x21:  // regset
                    if (!rd(10)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs) regs[p[i + 1]] = f64(i + 2);
                    i += 10;
                    break;
                case 0x31:  // charload
                    if (!rd(4)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs) regs[p[i + 1]] = (double)p[i + 2];
                    i += 4;
                    break;
                case 0x50:  // rand
                    if (!rd(2)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs) regs[p[i + 1]] = qoa_philox_uniform(rand_seed, kRandStream, rand_ctr++, 0);
                    i += 2;
                    break;
                case 0x54: case 0x55: case 0x56: case 0x57: {
                    if (!rd(4)) return QOA_E_ARG;
                    const size_t d = p[i + 1], a = p[i + 2], b = p[i + 3];
                    if (d < kRegs && a < kRegs && b < kRegs) {
                        if (op == 0x54) regs[d] = regs[a] + regs[b];
                        else if (op == 0x55) regs[d] = regs[a] - regs[b];
                        else if (op == 0x56) regs[d] = regs[a] * regs[b];
                        else if (regs[b] != 0.0) regs[d] = regs[a] / regs[b];
                    }
                    i += 4;
                    break;
                }
                case 0x58:
                    if (!rd(3)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs && p[i + 2] < kRegs) regs[p[i + 1]] = regs[p[i + 2]];
                    i += 3;
                    break;
                case 0xa5: case 0xa6: case 0xa7: case 0xa9: case 0xaa: {
                    if (!rd(4)) return QOA_E_ARG;
                    const size_t d = p[i + 1], a = p[i + 2], b = p[i + 3];
                    if (d < kRegs && a < kRegs && b < kRegs) {
                        const uint64_t x = as_u64(regs[a]), y = as_u64(regs[b]);
                        uint64_t r = 0;
                        if (op == 0xa5) r = x & y;
                        else if (op == 0xa6) r = x | y;
                        else if (op == 0xa7) r = x ^ y;
                        else if (op == 0xa9) r = x << (y & 63);
                        else r = x >> (y & 63);
                        regs[d] = (double)r;
                    }
                    i += 4;
                    break;
                }
                case 0xa8:
                    if (!rd(3)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs && p[i + 2] < kRegs) regs[p[i + 1]] = (double)(~as_u64(regs[p[i + 2]]));
                    i += 3;
                    break;
                case 0x90:
                    if (!rd(9)) return QOA_E_ARG;
                    jump_to((int64_t)i + i64(i + 1));
                    break;
                case 0x91:
                    if (!rd(9)) return QOA_E_ARG;
                    if (u64(i + 1) >= len) i = len; else i = (size_t)u64(i + 1);
                    break;
                case 0x92: case 0x93: case 0x94: case 0x95: {
                    if (!rd(11)) return QOA_E_ARG;
                    const size_t a = p[i + 1], b = p[i + 2];
                    bool take = false;
                    if (a < kRegs && b < kRegs) {
                        const double x = regs[a], y = regs[b];
                        const double eps = 2.220446049250313e-16;  // f64::EPSILON
                        if (op == 0x92) take = x > y;
                        else if (op == 0x93) take = x < y;
                        else if (op == 0x94) take = std::fabs(x - y) < eps;
                        else take = std::fabs(x - y) >= eps;
                    }
                    if (take) jump_to((int64_t)i + i64(i + 3));
                    else i += 11;
                    break;
                }
                case 0x96:
                    if (!rd(9)) return QOA_E_ARG;
                    calls.push_back(i + 9);
                    if (u64(i + 1) >= len) i = len; else i = (size_t)u64(i + 1);
                    break;
                case 0x98: {  // printf "%k" -> register k's value
                    if (!rd(9)) return QOA_E_ARG;
                    const uint64_t sl = u64(i + 1);
                    if (sl > len || !rd(9 + sl + 1)) return QOA_E_ARG;
                    const size_t nr = p[i + 9 + sl];
                    if (!rd(9 + sl + 1 + nr)) return QOA_E_ARG;
                    std::string f((const char*)p + i + 9, sl);
                    for (size_t k = 0; k < nr; ++k) {
                        const size_t r = p[i + 10 + sl + k];
                        const std::string val = r < kRegs ? rust_f64(regs[r]) : "NaN";
                        const std::string key = "%" + std::to_string(k);
                        for (size_t pos = 0; (pos = f.find(key, pos)) != std::string::npos; pos += val.size())
                            f.replace(pos, key.size(), val);
                    }
                    out += f;
                    i += 1 + 8 + sl + 1 + nr;
                    break;
                }
                case 0x99: case 0x9a: {
                    if (!rd(9)) return QOA_E_ARG;
                    const uint64_t sl = u64(i + 1);
                    if (sl > len || !rd(9 + sl)) return QOA_E_ARG;
                    out.append((const char*)p + i + 9, sl);
                    if (op == 0x9a) out.push_back('\n');
                    i += 1 + 8 + sl;
                    break;
                }
                case 0x9b:
                    if (!rd(2)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs) regs[p[i + 1]] = 0.0;
                    i += 2;
                    break;
                case 0x9d: {
                    out += "\nclassical registers:\n";
                    char b[64];
                    for (size_t k = 0; k < kRegs; ++k) {
                        std::snprintf(b, sizeof b, "r%zu: %.6f\n", k, regs[k]);
                        out += b;
                    }
                    i += 1;
                    break;
                }
                case 0x9e: {
                    if (!rd(10)) return QOA_E_ARG;
                    const size_t r = p[i + 1];
                    const uint64_t addr = u64(i + 2);
                    if (r < kRegs && addr + 8 <= kMemBytes) {
                        if (mem.empty()) mem.assign(kMemBytes, 0);
                        std::memcpy(&regs[r], mem.data() + addr, 8);
                    }
                    i += 10;
                    break;
                }
                case 0x9f: {
                    if (!rd(10)) return QOA_E_ARG;
                    const uint64_t addr = u64(i + 1);
                    const size_t r = p[i + 9];
                    if (r < kRegs && addr + 8 <= kMemBytes) {
                        if (mem.empty()) mem.assign(kMemBytes, 0);
                        std::memcpy(mem.data() + addr, &regs[r], 8);
                    }
                    i += 10;
                    break;
                }
                case 0xa2: if (!rd(10)) return QOA_E_ARG; i += 10; break;
                case 0xa3: if (!rd(9)) return QOA_E_ARG; i += 9; break;
                case 0xac:
                    if (!rd(2)) return QOA_E_ARG;
                    if (p[i + 1] < kRegs)
                        regs[p[i + 1]] = std::chrono::duration<double>(
                                             std::chrono::system_clock::now().time_since_epoch()).count();
                    i += 2;
                    break;
                case 0xad:
                    if (!rd(9)) return QOA_E_ARG;
                    rand_seed = u64(i + 1);
                    rand_ctr = 0;
                    i += 9;
                    break;
                case 0xae: {
                    if (!rd(5)) return QOA_E_ARG;
                    uint32_t code;
                    std::memcpy(&code, p + i + 1, 4);
                    res.exit_code = (int32_t)code;
                    res.halted = 1;
                    i = len;
                    break;
                }
                default:
                    res.unknown_opcodes++;
                    i += 1;
            }
        }
        return flush();
    }
};

int finish(VM& vm, int rc, qoa_exe_result* res, char* out_text, size_t out_cap, size_t* out_len) {
    std::memcpy(vm.res.registers, vm.regs, sizeof vm.regs);
    if (res) *res = vm.res;
    if (out_len) *out_len = vm.out.size();
    if (out_text && out_cap) {
        const size_t k = std::min(out_cap - 1, vm.out.size());
        std::memcpy(out_text, vm.out.data(), k);
        out_text[k] = 0;
    }
    if (rc != QOA_OK && !vm.err.empty()) qoa::note_global_error(("exe: " + vm.err).c_str());
    return rc;
}

}  // namespace

extern "C" {

int qoa_exe_parse(const uint8_t* file, size_t len, qoa_exe_info* info) {
    if (!info) {
        qoa::note_global_error("qoa_exe_parse: null info");
        return QOA_E_ARG;
    }
    const int rc = parse_header(file, len, info);
    if (rc) return rc;
    bool any = false;
    const uint32_t mq = scan_max_qubit(file + 9, (size_t)info->payload_len, &any);
    info->inferred_qubits = (mq == 0 && info->payload_len == 0) ? 0 : mq + 1;
    return QOA_OK;
}

int qoa_exe_run(qoa_state_t s, const uint8_t* file, size_t len, uint32_t flags, uint64_t max_steps,
                qoa_exe_result* res, char* out_text, size_t out_cap, size_t* out_len) {
    if (!s) {
        qoa::note_global_error("qoa_exe_run: null handle");
        return QOA_E_ARG;
    }
    qoa_exe_info info;
    int rc = parse_header(file, len, &info);
    if (rc) return rc;
    VM vm;
    vm.p = file + 9;
    vm.len = (size_t)info.payload_len;
    vm.flags = flags;
    vm.max_steps = max_steps;
    vm.s = s;
    return finish(vm, vm.run(), res, out_text, out_cap, out_len);
}

int qoa_exe_trace(const uint8_t* file, size_t len, uint32_t flags, uint64_t max_steps, qoa_op* ops, size_t cap,
                  size_t* nops, qoa_exe_result* res, char* out_text, size_t out_cap, size_t* out_len) {
    if (!nops || (!ops && cap)) {
        qoa::note_global_error("qoa_exe_trace: null argument");
        return QOA_E_ARG;
    }
    qoa_exe_info info;
    int rc = parse_header(file, len, &info);
    if (rc) return rc;
    std::vector<qoa_op> trace;
    VM vm;
    vm.p = file + 9;
    vm.len = (size_t)info.payload_len;
    vm.flags = flags;
    vm.max_steps = max_steps;
    vm.trace = &trace;
    rc = finish(vm, vm.run(), res, out_text, out_cap, out_len);
    *nops = trace.size();
    if (ops) std::memcpy(ops, trace.data(), std::min(cap, trace.size()) * sizeof(qoa_op));
    return rc;
}

}  // extern "C"
