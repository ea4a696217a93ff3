/*
 * qoa_oracle.c — TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * A CPU restatement of the reference's gate-application path, used only as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg.
 * Nothing in qoa_b200/ links or calls it.
 *
 * What it restates (citations are paths inside the planetryan/qoa project):
 *   - the x86-64 gate loops of src/vectorization.rs:915-1260, with the matrix
 *     set-up of the dispatch functions src/vectorization.rs:16-902;
 *   - QuantumState (src/runtime/quantum_state.rs): new 56-90, the gate methods
 *     171-397 (bounds checks that print and no-op), measure 399-458,
 *     execute_arithmetic's instruction dispatch 460-705, apply_noise /
 *     apply_depolarizing_noise / normalize 839-907, measure_all 909-918,
 *     toffoli 960, custom unitaries 1010-1127, controlled-Y 1163.
 *
 * Arithmetic follows num-complex 0.4.6 (Complex64 mul = (ac-bd, ad+bc),
 * from_polar(r,t) = (r cos t, r sin t), Complex/f64 divides both parts) and is
 * compiled with -ffp-contract=off so no FMA is formed, matching rustc. Angles
 * go through the same libm sin/cos that Rust's f64::sin/cos call on Linux.
 *
 * Randomness: the reference draws from StdRng (ChaCha12) seeded from entropy
 * (quantum_state.rs:76), which no run can reproduce. Measurements here take
 * caller-supplied uniforms; noise draws come from Philox4x32-10 (Salmon,
 * Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11),
 * written here from that paper and keyed exactly as the engine keys it, so a
 * trajectory is reproducible on both sides.
 *
 * Two timing profiles:
 *   faithful (default): gate loops single-threaded in index order, as the
 *     x86-64 path runs them; normalize parallel over all cores (rayon in the
 *     reference, OpenMP here). This is the reported CPU baseline.
 *   fast: every loop parallel. Used for parity at large n.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/qoa_cuda.h"

typedef struct { double re, im; } c64;

static int g_fast = 0;

void orc_set_fast(int fast) { g_fast = fast; }
int orc_get_max_threads(void) { return omp_get_max_threads(); }

static inline c64 cx(double re, double im) { c64 z; z.re = re; z.im = im; return z; }
static inline c64 c_mul(c64 a, c64 b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline c64 c_add(c64 a, c64 b) { return cx(a.re + b.re, a.im + b.im); }
static inline c64 c_sub(c64 a, c64 b) { return cx(a.re - b.re, a.im - b.im); }
static inline c64 c_scale(c64 a, double t) { return cx(a.re * t, a.im * t); }
static inline c64 c_from_polar(double r, double t) { return cx(r * cos(t), r * sin(t)); }
static inline double c_norm_sqr(c64 a) { return a.re * a.re + a.im * a.im; }

static inline int bit_ok(size_t b) { return b < 64; }

/* ------------------------------------------------------------------------ */
/* src/vectorization.rs, x86_64_simd module (915-1260) + dispatch set-up     */
/* ------------------------------------------------------------------------ */

/* apply_hadamard_simd 915-939 */
void orc_vec_hadamard(c64* a, size_t len, double nre, double nim, size_t mask_bit) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    c64 nf = cx(nre, nim);
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) == 0) {
            size_t j = i | bit;
            if (j < len) {
                c64 x = a[i], y = a[j];
                a[i] = c_mul(nf, c_add(x, y));
                a[j] = c_mul(nf, c_sub(x, y));
            }
        }
    }
}

/* apply_x_simd 942-961 */
void orc_vec_x(c64* a, size_t len, size_t mask_bit) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) == 0) {
            size_t j = i | bit;
            if (j < len) { c64 t = a[i]; a[i] = a[j]; a[j] = t; }
        }
    }
}

/* apply_y_simd 964-985 */
void orc_vec_y(c64* a, size_t len, size_t mask_bit) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    c64 neg_i = cx(0.0, -1.0), pos_i = cx(0.0, 1.0);
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) == 0) {
            size_t j = i | bit;
            if (j < len) {
                c64 a0 = a[i], a1 = a[j];
                a[i] = c_mul(a1, neg_i);
                a[j] = c_mul(a0, pos_i);
            }
        }
    }
}

/* apply_z_simd 988-999 */
void orc_vec_z(c64* a, size_t len, size_t mask_bit) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) != 0) a[i] = c_scale(a[i], -1.0);
    }
}

/* apply_phaseshift_simd 1002-1017 */
static void vec_phase(c64* a, size_t len, size_t mask_bit, c64 pf) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) != 0) a[i] = c_mul(a[i], pf);
    }
}
/* apply_t_vectorized 217-218: from_polar(1, pi/4) */
void orc_vec_t(c64* a, size_t len, size_t mask_bit) { vec_phase(a, len, mask_bit, c_from_polar(1.0, M_PI / 4.0)); }
/* apply_s_vectorized 262-263: from_polar(1, pi/2) */
void orc_vec_s(c64* a, size_t len, size_t mask_bit) { vec_phase(a, len, mask_bit, c_from_polar(1.0, M_PI / 2.0)); }
/* apply_phaseshift_vectorized 307-308 */
void orc_vec_phaseshift(c64* a, size_t len, size_t mask_bit, double angle) {
    vec_phase(a, len, mask_bit, c_from_polar(1.0, angle));
}

/* apply_reset_simd 1020-1056 */
void orc_vec_reset(c64* a, size_t len, size_t mask_bit) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    double norm_sqr = 0.0;
    for (size_t i = 0; i < len; i++)
        if ((i & bit) == 0) norm_sqr += c_norm_sqr(a[i]);
    if (norm_sqr > 1e-12) {
        double scale = 1.0 / sqrt(norm_sqr);
        long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
        for (long long ii = 0; ii < L; ii++) {
            size_t i = (size_t)ii;
            if ((i & bit) == 0) a[i] = c_scale(a[i], scale);
            else a[i] = cx(0.0, 0.0);
        }
    } else if (len > 0) {
        a[0] = cx(1.0, 0.0);
        for (size_t i = 1; i < len; i++) a[i] = cx(0.0, 0.0);
    }
}

/* apply_rx_simd 1059-1085 (also used for RY, 1088-1100) */
static void vec_mat2(c64* a, size_t len, size_t mask_bit, c64 m00, c64 m01, c64 m10, c64 m11) {
    if (!bit_ok(mask_bit)) return;
    size_t bit = (size_t)1 << mask_bit;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) == 0) {
            size_t j = i | bit;
            if (j < len) {
                c64 x = a[i], y = a[j];
                a[i] = c_add(c_mul(m00, x), c_mul(m01, y));
                a[j] = c_add(c_mul(m10, x), c_mul(m11, y));
            }
        }
    }
}
/* apply_rx_vectorized 528-535 */
void orc_vec_rx(c64* a, size_t len, size_t mask_bit, double angle) {
    double c = cos(angle / 2.0), s = sin(angle / 2.0);
    vec_mat2(a, len, mask_bit, cx(c, 0.0), cx(0.0, -s), cx(0.0, -s), cx(c, 0.0));
}
/* apply_ry_vectorized 588-595 */
void orc_vec_ry(c64* a, size_t len, size_t mask_bit, double angle) {
    double c = cos(angle / 2.0), s = sin(angle / 2.0);
    vec_mat2(a, len, mask_bit, cx(c, 0.0), cx(-s, 0.0), cx(s, 0.0), cx(c, 0.0));
}
/* apply_rz_vectorized 648-651 + apply_rz_simd 1103-1122 */
void orc_vec_rz(c64* a, size_t len, size_t mask_bit, double angle) {
    if (!bit_ok(mask_bit)) return;
    c64 m00 = c_from_polar(1.0, -angle / 2.0);
    c64 m11 = c_from_polar(1.0, angle / 2.0);
    size_t bit = (size_t)1 << mask_bit;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & bit) == 0) a[i] = c_mul(a[i], m00);
        else a[i] = c_mul(a[i], m11);
    }
}

/* apply_cnot_vectorized 699-701 + apply_cnot_simd 1141-1160 */
void orc_vec_cnot(c64* a, size_t len, size_t control, size_t target) {
    if (!bit_ok(control) || !bit_ok(target)) return;
    size_t cm = (size_t)1 << control, tm = (size_t)1 << target;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & cm) == cm && (i & tm) == 0) {
            size_t j = i | tm;
            if (j < len) { c64 t = a[i]; a[i] = a[j]; a[j] = t; }
        }
    }
}

/* apply_cz_simd 1163-1173: takes MASKS */
void orc_vec_cz(c64* a, size_t len, size_t control_mask, size_t target_mask) {
    size_t m = control_mask | target_mask;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & m) == m) a[i] = c_scale(a[i], -1.0);
    }
}

/* apply_controlled_phase_rotation_vectorized 788-794 + simd 1235-1250: MASKS */
void orc_vec_cphase(c64* a, size_t len, size_t control_mask, size_t target_mask, double angle) {
    c64 pf = c_from_polar(1.0, angle);
    size_t m = control_mask | target_mask;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & m) == m) a[i] = c_mul(a[i], pf);
    }
}

/* apply_swap_vectorized 421-423 + apply_swap_simd 1176-1197 */
void orc_vec_swap(c64* a, size_t len, size_t q1, size_t q2) {
    if (!bit_ok(q1) || !bit_ok(q2)) return;
    size_t m1 = (size_t)1 << q1, m2 = (size_t)1 << q2, comb = m1 | m2;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & comb) == 0) {
            size_t x = i | m2, y = i | m1;
            if (x < len && y < len) { c64 t = a[x]; a[x] = a[y]; a[y] = t; }
        }
    }
}

/* apply_controlled_swap_vectorized 469-478 + simd 1200-1232 */
void orc_vec_cswap(c64* a, size_t len, size_t control, size_t t1, size_t t2) {
    if (!bit_ok(control) || !bit_ok(t1) || !bit_ok(t2)) return;
    size_t cm = (size_t)1 << control, m1 = (size_t)1 << t1, m2 = (size_t)1 << t2;
    size_t comb = cm | m1 | m2;
    long long L = (long long)len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & comb) == 0) {
            size_t x = i | cm | m2, y = i | cm | m1;
            if (x < len && y < len) { c64 t = a[x]; a[x] = a[y]; a[y] = t; }
        }
    }
}

/* apply_reset_all_simd 1253-1260 */
void orc_vec_reset_all(c64* a, size_t len) {
    if (len == 0) return;
    a[0] = cx(1.0, 0.0);
    for (size_t i = 1; i < len; i++) a[i] = cx(0.0, 0.0);
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al. SC'11), keyed the way the engine keys it     */
/* ------------------------------------------------------------------------ */
static void philox4x32_10(uint32_t ctr[4], const uint32_t key_in[2]) {
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        uint32_t n3 = lo0;
        ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* Uniform double in [0,1) for draw (stream, event, slot). */
double orc_uniform(uint64_t seed, uint64_t stream, uint64_t event, uint32_t slot) {
    uint32_t ctr[4] = {(uint32_t)event, (uint32_t)(event >> 32), slot, (uint32_t)stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    philox4x32_10(ctr, key);
    uint64_t bits = ((uint64_t)ctr[0] << 32) | ctr[1];
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------------ */
/* QuantumState (src/runtime/quantum_state.rs)                              */
/* ------------------------------------------------------------------------ */
typedef struct orc_state {
    size_t n, len;
    c64* amps;
    uint32_t flags;        /* QOA_FLAG_COMPAT_MASK_QUIRK, QOA_FLAG_NOISE_GATE_QUBITS */
    int noise_mode;        /* 0 ideal, 1 fixed, 2 random */
    double noise_p;
    uint64_t seed, stream; /* Philox key and stream (trajectory) id */
    uint64_t event;        /* apply_noise() call counter */
    uint64_t meas_draws;   /* internal measure draws used (when no uniforms supplied) */
    const double* meas_u;  /* supplied measurement uniforms for orc_apply */
    size_t meas_u_len, meas_u_pos;
    uint32_t zero_resets;
    uint32_t last_touched[4];
    int n_touched;
    int defer_norm;        /* orc_set_defer_norm: skip the per-gate normalize */
} orc_state;

static void st_alloc(orc_state* s, size_t n) {
    if (n < 1) n = 1;
    s->n = n;
    s->len = (size_t)1 << n;
    free(s->amps);
    s->amps = (c64*)calloc(s->len, sizeof(c64));
    s->amps[0] = cx(1.0, 0.0);
}

/* QuantumState::new 56-90 */
orc_state* orc_new(size_t n, uint32_t flags) {
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    s->flags = flags;
    st_alloc(s, n);
    return s;
}
void orc_free(orc_state* s) { if (s) { free(s->amps); free(s); } }
/* Writes every amplitude back in place on all cores, so the pages of a fresh
   allocation are mapped before anything is timed (timing harness only). */
void orc_touch(orc_state* s) {
    long long L = (long long)s->len;
    volatile c64* a = s->amps;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < L; i++) a[i] = a[i];
}
size_t orc_num_qubits(orc_state* s) { return s->n; }
c64* orc_amps(orc_state* s) { return s->amps; }
void orc_set_noise(orc_state* s, int mode, double p, uint64_t seed, uint64_t stream) {
    s->noise_mode = mode; s->noise_p = p; s->seed = seed; s->stream = stream; s->event = 0;
}
uint32_t orc_zero_resets(orc_state* s) { return s->zero_resets; }

/* normalize 888-907 */
void orc_normalize(orc_state* s) {
    double norm_sqr = 0.0;
    long long L = (long long)s->len;
    c64* a = s->amps;
#pragma omp parallel for reduction(+ : norm_sqr) schedule(static)
    for (long long i = 0; i < L; i++) norm_sqr += c_norm_sqr(a[i]);
    if (norm_sqr > 1e-12) {
        double norm = sqrt(norm_sqr);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < L; i++) a[i] = cx(a[i].re / norm, a[i].im / norm);
    } else {
        s->zero_resets++;
        orc_vec_reset_all(a, s->len);
    }
}

/* apply_depolarizing_noise 872-885: per qubit, r < p -> X/Y/Z */
static void depolarize(orc_state* s, double p, uint64_t ev) {
    for (size_t q = 0; q < s->n; q++) {
        if (s->flags & QOA_FLAG_NOISE_GATE_QUBITS) {
            int hit = 0;
            for (int k = 0; k < s->n_touched; k++) hit |= (s->last_touched[k] == q);
            if (!hit) continue;
        }
        double r = orc_uniform(s->seed, s->stream, ev, (uint32_t)(2 * q + 1));
        if (r < p) {
            double u2 = orc_uniform(s->seed, s->stream, ev, (uint32_t)(2 * q + 2));
            int e = (int)(u2 * 3.0);
            if (e > 2) e = 2;
            if (e == 0) orc_vec_x(s->amps, s->len, q);
            else if (e == 1) orc_vec_y(s->amps, s->len, q);
            else orc_vec_z(s->amps, s->len, q);
        }
    }
}

/* apply_noise 839-869 */
static void apply_noise(orc_state* s) {
    uint64_t ev = s->event++;
    if (s->noise_mode == 2) {
        double level = 0.1 + 0.9 * orc_uniform(s->seed, s->stream, ev, 0);
        depolarize(s, level, ev);
    } else if (s->noise_mode == 1 && s->noise_p > 0.0) {
        depolarize(s, s->noise_p, ev);
    }
    if (!s->defer_norm) orc_normalize(s);
}

/* Speed mode for parity runs of large noiseless unitary circuits (test
   harness only): the per-gate normalize of apply_noise is skipped and the
   caller normalizes once at the end. Every gate keeps the norm at 1 to within
   rounding, so the result moves by rounding only (about 1e-16 per gate),
   while each gate costs one sweep of the state instead of three. */
void orc_set_defer_norm(orc_state* s, int on) { s->defer_norm = on; }

static void touched(orc_state* s, int k, uint32_t a, uint32_t b, uint32_t c) {
    s->n_touched = k; s->last_touched[0] = a; s->last_touched[1] = b; s->last_touched[2] = c;
}

/* gate methods 171-397: out-of-range -> no-op, returns 1 */
static int qs_h(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_hadamard(s->amps, s->len, 1.0 / M_SQRT2, 0.0, q);
    touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_x(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_x(s->amps, s->len, q); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_y(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_y(s->amps, s->len, q); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_z(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_z(s->amps, s->len, q); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_t(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_t(s->amps, s->len, q); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_s(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_s(s->amps, s->len, q); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_p(orc_state* s, size_t q, double a) {
    if (q >= s->n) return 1;
    orc_vec_phaseshift(s->amps, s->len, q, a); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_rx(orc_state* s, size_t q, double a) {
    if (q >= s->n) return 1;
    orc_vec_rx(s->amps, s->len, q, a); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_ry(orc_state* s, size_t q, double a) {
    if (q >= s->n) return 1;
    orc_vec_ry(s->amps, s->len, q, a); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_rz(orc_state* s, size_t q, double a) {
    if (q >= s->n) return 1;
    orc_vec_rz(s->amps, s->len, q, a); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
static int qs_cnot(orc_state* s, size_t c, size_t t) {
    if (c >= s->n || t >= s->n || c == t) return 1;
    orc_vec_cnot(s->amps, s->len, c, t); touched(s, 2, (uint32_t)c, (uint32_t)t, 0); apply_noise(s); return 0;
}
/* apply_cz 326-340: the reference passes the qubit INDICES as the masks */
static int qs_cz(orc_state* s, size_t c, size_t t) {
    if (c >= s->n || t >= s->n || c == t) return 1;
    if (s->flags & QOA_FLAG_COMPAT_MASK_QUIRK) orc_vec_cz(s->amps, s->len, c, t);
    else orc_vec_cz(s->amps, s->len, (size_t)1 << c, (size_t)1 << t);
    touched(s, 2, (uint32_t)c, (uint32_t)t, 0); apply_noise(s); return 0;
}
/* apply_controlled_phase 342-363: same index-as-mask call */
static int qs_cphase(orc_state* s, size_t c, size_t t, double a) {
    if (c >= s->n || t >= s->n || c == t) return 1;
    if (s->flags & QOA_FLAG_COMPAT_MASK_QUIRK) orc_vec_cphase(s->amps, s->len, c, t, a);
    else orc_vec_cphase(s->amps, s->len, (size_t)1 << c, (size_t)1 << t, a);
    touched(s, 2, (uint32_t)c, (uint32_t)t, 0); apply_noise(s); return 0;
}
static int qs_swap(orc_state* s, size_t a, size_t b) {
    if (a >= s->n || b >= s->n || a == b) return 1;
    orc_vec_swap(s->amps, s->len, a, b); touched(s, 2, (uint32_t)a, (uint32_t)b, 0); apply_noise(s); return 0;
}
static int qs_cswap(orc_state* s, size_t c, size_t a, size_t b) {
    if (c >= s->n || a >= s->n || b >= s->n || c == a || c == b || a == b) return 1;
    orc_vec_cswap(s->amps, s->len, c, a, b); touched(s, 3, (uint32_t)c, (uint32_t)a, (uint32_t)b); apply_noise(s); return 0;
}
/* reset_qubit 171-181 */
static int qs_reset(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    orc_vec_reset(s->amps, s->len, q); touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
/* apply_reset_all 183-186 */
static int qs_reset_all(orc_state* s) {
    orc_vec_reset_all(s->amps, s->len); touched(s, 0, 0, 0, 0); apply_noise(s); return 0;
}

/* apply_toffoli 960-1008 (clone, then read from the copy) */
static int qs_toffoli(orc_state* s, size_t c1, size_t c2, size_t t) {
    if (c1 >= s->n || c2 >= s->n || t >= s->n || c1 == c2 || c1 == t || c2 == t) return 1;
    size_t m1 = (size_t)1 << c1, m2 = (size_t)1 << c2, mt = (size_t)1 << t;
    c64* old = (c64*)malloc(s->len * sizeof(c64));
    memcpy(old, s->amps, s->len * sizeof(c64));
    long long L = (long long)s->len;
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & m1) && (i & m2)) s->amps[i] = old[i ^ mt];
    }
    free(old);
    touched(s, 3, (uint32_t)c1, (uint32_t)c2, (uint32_t)t); apply_noise(s); return 0;
}
/* apply_custom_unitary 1010-1062 */
static int qs_u1(orc_state* s, size_t q, const double* m) {
    if (q >= s->n || !m) return 1;
    c64 u00 = cx(m[0], m[1]), u01 = cx(m[2], m[3]), u10 = cx(m[4], m[5]), u11 = cx(m[6], m[7]);
    size_t mask = (size_t)1 << q;
    c64* old = (c64*)malloc(s->len * sizeof(c64));
    memcpy(old, s->amps, s->len * sizeof(c64));
    long long L = (long long)s->len;
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if ((i & mask) == 0) s->amps[i] = c_add(c_mul(u00, old[i]), c_mul(u01, old[i | mask]));
        else s->amps[i] = c_add(c_mul(u10, old[i ^ mask]), c_mul(u11, old[i]));
    }
    free(old);
    touched(s, 1, (uint32_t)q, 0, 0); apply_noise(s); return 0;
}
/* apply_two_qubit_unitary 1064-1127: basis index = 2*bit(max(q1,q2)) + bit(min(q1,q2)) */
static int qs_u2(orc_state* s, size_t q1, size_t q2, const double* m) {
    if (q1 >= s->n || q2 >= s->n || q1 == q2 || !m) return 1;
    size_t lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
    size_t ml = (size_t)1 << lo, mh = (size_t)1 << hi;
    c64 u[16];
    for (int k = 0; k < 16; k++) u[k] = cx(m[2 * k], m[2 * k + 1]);
    c64* old = (c64*)malloc(s->len * sizeof(c64));
    memcpy(old, s->amps, s->len * sizeof(c64));
    long long L = (long long)s->len;
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        size_t bl = (i & ml) >> lo, bh = (i & mh) >> hi;
        size_t row = (bh << 1) | bl;
        size_t base = i & ~(ml | mh);
        c64 a00 = old[base], a01 = old[base | ml], a10 = old[base | mh], a11 = old[base | ml | mh];
        c64 r = c_mul(u[4 * row + 0], a00);
        r = c_add(r, c_mul(u[4 * row + 1], a01));
        r = c_add(r, c_mul(u[4 * row + 2], a10));
        r = c_add(r, c_mul(u[4 * row + 3], a11));
        s->amps[i] = r;
    }
    free(old);
    touched(s, 2, (uint32_t)q1, (uint32_t)q2, 0); apply_noise(s); return 0;
}
/* apply_controlled_y 1163-1212 */
static int qs_cy(orc_state* s, size_t c, size_t t) {
    if (c >= s->n || t >= s->n || c == t) return 1;
    size_t cm = (size_t)1 << c, tm = (size_t)1 << t;
    c64 pi = cx(0.0, 1.0), ni = cx(0.0, -1.0);
    c64* old = (c64*)malloc(s->len * sizeof(c64));
    memcpy(old, s->amps, s->len * sizeof(c64));
    long long L = (long long)s->len;
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        if (i & cm) {
            if ((i & tm) == 0) s->amps[i] = c_mul(ni, old[i | tm]);
            else s->amps[i] = c_mul(pi, old[i ^ tm]);
        }
    }
    free(old);
    touched(s, 2, (uint32_t)c, (uint32_t)t, 0); apply_noise(s); return 0;
}

/* measure 399-458 with a supplied uniform u */
int orc_measure(orc_state* s, size_t q, double u, uint32_t* outcome) {
    if (q >= s->n) return 1;
    size_t mask = (size_t)1 << q;
    double p0 = 0.0, p1 = 0.0;
    if (g_fast) {
        long long L = (long long)s->len;
#pragma omp parallel for reduction(+ : p0, p1) schedule(static)
        for (long long ii = 0; ii < L; ii++) {
            double pr = c_norm_sqr(s->amps[ii]);
            if (((size_t)ii & mask) == 0) p0 += pr; else p1 += pr;
        }
    } else {
        for (size_t i = 0; i < s->len; i++) {
            double pr = c_norm_sqr(s->amps[i]);
            if ((i & mask) == 0) p0 += pr; else p1 += pr;
        }
    }
    uint32_t res = (u < p0) ? 0u : 1u;
    double f;
    if (res == 0) f = p0 > 1e-12 ? 1.0 / sqrt(p0) : 0.0;
    else f = p1 > 1e-12 ? 1.0 / sqrt(p1) : 0.0;
    long long L = (long long)s->len;
#pragma omp parallel for schedule(static) if (g_fast)
    for (long long ii = 0; ii < L; ii++) {
        size_t i = (size_t)ii;
        int set = (i & mask) != 0;
        if ((res == 0 && set) || (res == 1 && !set)) s->amps[i] = cx(0.0, 0.0);
        else s->amps[i] = c_scale(s->amps[i], f);
    }
    touched(s, 1, (uint32_t)q, 0, 0);
    apply_noise(s);
    if (outcome) *outcome = res;
    return 0;
}

/* measure_all 909-918: measures a clone, qubits 0..n-1 in order; u[q] per qubit.
 * The clone carries the noise configuration, as self.clone() does. */
uint64_t orc_measure_all(orc_state* s, const double* u) {
    orc_state* c = (orc_state*)calloc(1, sizeof(orc_state));
    *c = *s;
    c->amps = (c64*)malloc(s->len * sizeof(c64));
    memcpy(c->amps, s->amps, s->len * sizeof(c64));
    uint64_t bits = 0;
    for (size_t q = 0; q < s->n; q++) {
        uint32_t r = 0;
        orc_measure(c, q, u[q], &r);
        bits |= (uint64_t)r << q;
    }
    orc_free(c);
    return bits;
}

static double next_meas_u(orc_state* s) {
    if (s->meas_u && s->meas_u_pos < s->meas_u_len) return s->meas_u[s->meas_u_pos++];
    return orc_uniform(s->seed, s->stream ^ 0x6d656173ull, s->meas_draws++, 0);
}

static int qs_measure_op(orc_state* s, size_t q) {
    if (q >= s->n) return 1;
    return orc_measure(s, q, next_meas_u(s), NULL);
}

static int op_qubit(const qoa_op* op, uint32_t k) {
    if (op->nq > 4 && op->qlist) return (int)op->qlist[k];
    return (int)op->q[k];
}

/* execute_arithmetic 460-705 for one op. Returns 0, or 1 when the op (or a
 * part of a macro) was skipped as out of range, 3 for an unsupported op. */
static int exec_one(orc_state* s, const qoa_op* op) {
    uint32_t q0 = op->q[0], q1 = op->q[1], q2 = op->q[2], q3 = op->q[3];
    double a = op->angle;
    int rc = 0;
    switch (op->opcode) {
    case QOA_OP_QINIT: st_alloc(s, q0); return 0;
    case QOA_OP_RESET: return qs_reset(s, q0);
    case QOA_OP_RESETALL: return qs_reset_all(s);
    case QOA_OP_H: return qs_h(s, q0);
    case QOA_OP_X: return qs_x(s, q0);
    case QOA_OP_Y: return qs_y(s, q0);
    case QOA_OP_Z: return qs_z(s, q0);
    case QOA_OP_T: return qs_t(s, q0);
    case QOA_OP_S: return qs_s(s, q0);
    case QOA_OP_P: case QOA_OP_SETPHASE: case QOA_OP_PHASE: return qs_p(s, q0, a);
    case QOA_OP_RX: return qs_rx(s, q0, a);
    case QOA_OP_RY: return qs_ry(s, q0, a);
    case QOA_OP_RZ: return qs_rz(s, q0, a);
    case QOA_OP_CNOT: case QOA_OP_ENTANGLE: case QOA_OP_ECFB: return qs_cnot(s, q0, q1);
    case QOA_OP_CZ: return qs_cz(s, q0, q1);
    case QOA_OP_CPHASE: return qs_cphase(s, q0, q1, a);
    case QOA_OP_EBELL: rc |= qs_h(s, q0); rc |= qs_cnot(s, q0, q1); return rc;
    case QOA_OP_EMULTI: {
        if (op->nq == 0) return 2;
        uint32_t first = (uint32_t)op_qubit(op, 0);
        rc |= qs_h(s, first);
        for (uint32_t k = 1; k < op->nq; k++) rc |= qs_cnot(s, first, (size_t)op_qubit(op, k));
        return rc;
    }
    case QOA_OP_ECLUSTER: {
        for (uint32_t k = 0; k < op->nq; k++) rc |= qs_h(s, (size_t)op_qubit(op, k));
        for (uint32_t k = 0; k + 1 < op->nq; k++) rc |= qs_cz(s, (size_t)op_qubit(op, k), (size_t)op_qubit(op, k + 1));
        return rc;
    }
    case QOA_OP_APPLYGATE:
        switch (q1) {
        case 'H': return qs_h(s, q0);
        case 'X': return qs_x(s, q0);
        case 'Y': return qs_y(s, q0);
        case 'Z': return qs_z(s, q0);
        case 'T': return qs_t(s, q0);
        case 'S': return qs_s(s, q0);
        default: return 3;
        }
    case QOA_OP_ESWAP:
        rc |= qs_cnot(s, q0, q2); rc |= qs_cnot(s, q1, q3); rc |= qs_swap(s, q2, q3); return rc;
    case QOA_OP_ESWAPM:
        rc |= qs_cnot(s, q0, q2); rc |= qs_cnot(s, q1, q3); rc |= qs_swap(s, q2, q3);
        if (qs_measure_op(s, q2)) return 1;
        if (qs_measure_op(s, q3)) return 1;
        return rc;
    case QOA_OP_EDIST: return 0;
    case QOA_OP_MEASB:
        if (q0 >= s->n) return 1;
        if (q1 == 'X') { qs_h(s, q0); qs_measure_op(s, q0); qs_h(s, q0); return 0; }
        if (q1 == 'Y') {
            qs_s(s, q0); qs_h(s, q0); qs_measure_op(s, q0); qs_h(s, q0); qs_s(s, q0); qs_z(s, q0);
            return 0;
        }
        if (q1 == 'Z') { qs_measure_op(s, q0); return 0; }
        return 3;
    case QOA_OP_MEASURE: return qs_measure_op(s, q0);
    case QOA_OP_ROT:
        if (q1 == 'X') return qs_rx(s, q0, a);
        if (q1 == 'Y') return qs_ry(s, q0, a);
        if (q1 == 'Z') return qs_rz(s, q0, a);
        return 3;
    case QOA_OP_SWAP: return qs_swap(s, q0, q1);
    case QOA_OP_CSWAP: return qs_cswap(s, q0, q1, q2);
    case QOA_OP_TOFFOLI: return qs_toffoli(s, q0, q1, q2);
    case QOA_OP_U1: return qs_u1(s, q0, op->matrix);
    case QOA_OP_U2: return qs_u2(s, q0, q1, op->matrix);
    case QOA_OP_CY: return qs_cy(s, q0, q1);
    default: return 3;
    }
}

/* Applies ops in order; returns 0, or the first non-zero status (the op is
 * skipped, later ops still run). meas_u supplies MEASURE uniforms in order. */
int orc_apply(orc_state* s, const qoa_op* ops, size_t nops, const double* meas_u, size_t n_meas_u) {
    s->meas_u = meas_u; s->meas_u_len = n_meas_u; s->meas_u_pos = 0;
    int first = 0;
    for (size_t i = 0; i < nops; i++) {
        int rc = exec_one(s, &ops[i]);
        if (rc && !first) first = rc;
    }
    s->meas_u = NULL;
    return first;
}

/* set_state_vector 1133-1145: copy in, then normalize */
int orc_set_state(orc_state* s, const c64* src, size_t len) {
    if (len != s->len) return 2;
    memcpy(s->amps, src, len * sizeof(c64));
    orc_normalize(s);
    return 0;
}
int orc_get_state(orc_state* s, c64* dst, size_t len) {
    if (len != s->len) return 2;
    memcpy(dst, s->amps, len * sizeof(c64));
    return 0;
}
