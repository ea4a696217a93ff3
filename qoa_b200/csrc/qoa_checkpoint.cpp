// qoa_checkpoint.cpp — `--save-state` / `--load-state` JSON checkpoints.
//
// The file is what serde_json makes of the reference's (QuantumState,
// Vec<f64>) pair (main.rs:3800-3830 loads it, main.rs:4290-4300 saves it):
//
//   [ { "n": N,
//       "amps": [[re, im], ...],            2^N complex amplitudes
//       "regs": [[re, im], ...],            max(N, 10) complex registers
//       "status": {"nan": b, "div_by_zero": b, "overflow": b},
//       "noise_config": null | "Random" | "Ideal" | {"Fixed": p} },
//     [r0, r1, ...] ]                       the executor's f64 registers
//
// (QuantumState's rng field is skipped by serde; Complex64 serialises as a
// two-element array.) Saving writes the normalised amplitudes in the
// shortest round-trip decimal form; loading creates a complex128 handle with
// N qubits, the file's noise configuration, and the amplitudes set through
// qoa_set_state. JSON holds about 45 bytes per amplitude, so it is limited to
// 26 qubits here; qoa_state_save / qoa_state_load dump any size exactly.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qoa_cuda.h"

namespace qoa {
void note_global_error(const char* msg);
}

namespace qoa {
struct JsonExtras {
    bool noise_none;
    bool div_by_zero;
    std::vector<double> regs;
};
JsonExtras json_extras(qoa_state_t s);
int set_json_extras(qoa_state_t s, const JsonExtras& x, bool nan, bool overflow);
}  // namespace qoa

namespace {

constexpr uint32_t kJsonMaxQubits = 26;

int fail(const std::string& m, int code = QOA_E_ARG) {
    qoa::note_global_error(m.c_str());
    return code;
}

// serde_json's number form: shortest round trip, "1.0" for integral values.
void put_f64(std::string& o, double v) {
    if (!std::isfinite(v)) {
        o += "null";
        return;
    }
    char b[64];
    auto r = std::to_chars(b, b + sizeof b, v);
    std::string t(b, r.ptr);
    if (t.find_first_of(".eE") == std::string::npos) t += ".0";
    o += t;
}

// ---- a small JSON reader (enough for the checkpoint layout) --------------
struct J {
    const char* p;
    const char* e;
    std::string err;
    void ws() {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    }
    bool lit(char c) {
        ws();
        if (p < e && *p == c) {
            ++p;
            return true;
        }
        return false;
    }
    bool expect(char c) {
        if (lit(c)) return true;
        err = std::string("expected '") + c + "'";
        return false;
    }
    bool word(const char* w) {
        ws();
        const size_t k = std::strlen(w);
        if ((size_t)(e - p) >= k && std::memcmp(p, w, k) == 0) {
            p += k;
            return true;
        }
        return false;
    }
    bool num(double& v) {
        ws();
        if (word("null")) {  // serde_json writes non-finite floats as null
            v = std::nan("");
            return true;
        }
        const char* s = p;
        while (p < e && (std::strchr("+-0123456789.eE", *p) != nullptr)) ++p;
        if (p == s) {
            err = "expected a number";
            return false;
        }
        auto r = std::from_chars(s, p, v);
        if (r.ec != std::errc() || r.ptr != p) {
            err = "bad number";
            return false;
        }
        return true;
    }
    bool str(std::string& out) {
        ws();
        if (p >= e || *p != '"') {
            err = "expected a string";
            return false;
        }
        ++p;
        out.clear();
        while (p < e && *p != '"') {
            if (*p == '\\' && p + 1 < e) ++p;
            out.push_back(*p++);
        }
        if (p >= e) {
            err = "unterminated string";
            return false;
        }
        ++p;
        return true;
    }
    bool boolean(bool& b) {
        if (word("true")) { b = true; return true; }
        if (word("false")) { b = false; return true; }
        err = "expected true/false";
        return false;
    }
    // [[re, im], ...]
    bool complex_list(std::vector<double>& out) {
        if (!expect('[')) return false;
        out.clear();
        if (lit(']')) return true;
        do {
            double re, im;
            if (!expect('[') || !num(re) || !expect(',') || !num(im) || !expect(']')) return false;
            out.push_back(re);
            out.push_back(im);
        } while (lit(','));
        return expect(']');
    }
    bool real_list(std::vector<double>& out) {
        if (!expect('[')) return false;
        out.clear();
        if (lit(']')) return true;
        do {
            double v;
            if (!num(v)) return false;
            out.push_back(v);
        } while (lit(','));
        return expect(']');
    }
    bool skip_value() {
        ws();
        if (p >= e) return false;
        if (*p == '"') { std::string t; return str(t); }
        if (*p == '[' || *p == '{') {
            const char open = *p, close = open == '[' ? ']' : '}';
            ++p;
            if (lit(close)) return true;
            do {
                if (open == '{') {
                    std::string k;
                    if (!str(k) || !expect(':')) return false;
                }
                if (!skip_value()) return false;
            } while (lit(','));
            return expect(close);
        }
        if (word("true") || word("false") || word("null")) return true;
        double v;
        return num(v);
    }
};

}  // namespace

extern "C" {

int qoa_state_save_json(qoa_state_t s, const double* regs, size_t nregs, const char* path) {
    if (!s || !path || (!regs && nregs)) return fail("qoa_state_save_json: null argument");
    uint32_t n = 0;
    int prec = 0, rc;
    if ((rc = qoa_num_qubits(s, &n)) || (rc = qoa_get_precision(s, &prec))) return rc;
    if (n > kJsonMaxQubits) return fail("qoa_state_save_json: JSON checkpoints are limited to 26 qubits; use qoa_state_save");
    const size_t len = (size_t)1 << n;
    std::vector<double> a(2 * len);
    if (prec == QOA_PREC_F32) {
        std::vector<float> f(2 * len);
        if ((rc = qoa_get_state(s, f.data(), f.size() * sizeof(float)))) return rc;
        for (size_t i = 0; i < f.size(); ++i) a[i] = f[i];
    } else if ((rc = qoa_get_state(s, a.data(), a.size() * sizeof(double)))) {
        return rc;
    }
    qoa_status_t st{};
    if ((rc = qoa_status(s, &st))) return rc;
    int mode = 0;
    double p = 0;
    if ((rc = qoa_get_noise(s, &mode, &p))) return rc;
    std::string o;
    o.reserve(len * 48 + 1024);
    o += "[\n  {\n    \"n\": " + std::to_string(n) + ",\n    \"amps\": [";
    for (size_t i = 0; i < len; ++i) {
        o += i ? ",[" : "[";
        put_f64(o, a[2 * i]);
        o += ',';
        put_f64(o, a[2 * i + 1]);
        o += ']';
    }
    // the state's own registers as loaded (a fresh state: max(n, 10) zeros)
    const qoa::JsonExtras ex = qoa::json_extras(s);
    o += "],\n    \"regs\": [";
    if (!ex.regs.empty()) {
        for (size_t i = 0; i + 1 < ex.regs.size(); i += 2) {
            o += i ? ",[" : "[";
            put_f64(o, ex.regs[i]);
            o += ',';
            put_f64(o, ex.regs[i + 1]);
            o += ']';
        }
    } else {
        const uint32_t nr = n > 10 ? n : 10;
        for (uint32_t i = 0; i < nr; ++i) o += i ? ",[0.0,0.0]" : "[0.0,0.0]";
    }
    o += "],\n    \"status\": {\"nan\": ";
    o += st.nan_seen ? "true" : "false";
    o += ", \"div_by_zero\": ";
    o += ex.div_by_zero ? "true" : "false";
    o += ", \"overflow\": ";
    o += st.inf_seen ? "true" : "false";
    o += "},\n    \"noise_config\": ";
    if (mode == 2) o += "\"Random\"";
    else if (mode == 1) {
        o += "{\"Fixed\": ";
        put_f64(o, p);
        o += "}";
    } else {
        o += ex.noise_none ? "null" : "\"Ideal\"";  // Option::None against Some(Ideal)
    }
    o += "\n  },\n  [";
    for (size_t i = 0; i < nregs; ++i) {
        if (i) o += ',';
        put_f64(o, regs[i]);
    }
    o += "]\n]\n";
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(std::string("qoa_state_save_json: cannot open ") + path);
    const bool ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
    if (std::fclose(f) != 0 || !ok) return fail(std::string("qoa_state_save_json: writing failed: ") + path);
    return QOA_OK;
}

int qoa_state_load_json(const char* path, uint32_t flags, qoa_state_t* out, double* regs, size_t regs_cap,
                        size_t* nregs) {
    if (!path || !out || (!regs && regs_cap)) return fail("qoa_state_load_json: null argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(std::string("qoa_state_load_json: cannot open ") + path);
    std::string text;
    char buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
    std::fclose(f);
    J j{text.data(), text.data() + text.size(), ""};
    double nd = -1;
    std::vector<double> amps, rl, sregs;
    int mode = 0;
    double p = 0;
    bool none = true, nan = false, dbz = false, ovf = false;
    // a JSON boolean
    auto flag = [&](bool& v) {
        if (j.word("true")) v = true;
        else if (j.word("false")) v = false;
        else return false;
        return true;
    };
    bool ok = j.expect('[') && j.expect('{');
    if (ok && !j.lit('}')) {
        do {
            std::string key;
            if (!(ok = j.str(key) && j.expect(':'))) break;
            if (key == "n") ok = j.num(nd);
            else if (key == "amps") ok = j.complex_list(amps);
            else if (key == "noise_config") {
                std::string t;
                none = false;
                if (j.word("null")) {
                    mode = 0;
                    none = true;
                } else if (j.lit('{')) {
                    ok = j.str(t) && j.expect(':') && j.num(p) && j.expect('}');
                    if (ok && t != "Fixed") { ok = false; j.err = "unknown noise_config"; }
                    mode = 1;
                } else {
                    ok = j.str(t);
                    if (t == "Random") mode = 2;
                    else if (t == "Ideal") mode = 0;
                    else if (ok) { ok = false; j.err = "unknown noise_config"; }
                }
            } else if (key == "regs") {
                ok = j.complex_list(sregs);
            } else if (key == "status") {
                // {"nan": b, "div_by_zero": b, "overflow": b}
                ok = j.expect('{');
                if (ok && !j.lit('}')) {
                    do {
                        std::string k2;
                        if (!(ok = j.str(k2) && j.expect(':'))) break;
                        if (k2 == "nan") ok = flag(nan);
                        else if (k2 == "div_by_zero") ok = flag(dbz);
                        else if (k2 == "overflow") ok = flag(ovf);
                        else ok = j.skip_value();
                    } while (ok && j.lit(','));
                    ok = ok && j.expect('}');
                }
            } else {
                ok = j.skip_value();
            }
        } while (ok && j.lit(','));
        ok = ok && j.expect('}');
    }
    ok = ok && j.expect(',') && j.real_list(rl) && j.expect(']');
    if (!ok) return fail("qoa_state_load_json: " + (j.err.empty() ? std::string("malformed file") : j.err));
    if (!(nd >= 1 && nd <= kJsonMaxQubits) || nd != std::floor(nd))
        return fail("qoa_state_load_json: bad or missing qubit count n");
    const uint32_t n = (uint32_t)nd;
    if (amps.size() != ((size_t)2 << n)) return fail("qoa_state_load_json: amps length is not 2^n");
    qoa_state_t s = nullptr;
    int rc = qoa_create(n, QOA_PREC_F64, flags, &s);
    if (rc) return rc;
    if ((rc = qoa_set_noise(s, mode, p)) || (rc = qoa_set_state(s, amps.data(), amps.size() * sizeof(double))) ||
        (rc = qoa::set_json_extras(s, qoa::JsonExtras{none, dbz, sregs}, nan, ovf))) {
        qoa_destroy(s);
        return rc;
    }
    if (nregs) *nregs = rl.size();
    if (regs) std::memcpy(regs, rl.data(), std::min(regs_cap, rl.size()) * sizeof(double));
    *out = s;
    return QOA_OK;
}

}  // extern "C"
