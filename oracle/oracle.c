/*
 * oracle.c — CPU restatement of yao-rs's simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only the tests, the smoke check
 * and the CPU-baseline leg of the benchmark call this code; the CUDA library
 * never links or calls it.
 *
 * Every function follows the yao-rs function cited beside it, with the same
 * loop and operation order.  Complex products are num_complex's
 * (ac - bd, ad + bc); sums are left folds from zero like Rust's
 * Iterator::sum; the file is built with -ffp-contract=off so no FMA is
 * formed.  Results are therefore bit-identical to the Rust code's.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double re, im;
} cx;

static inline cx cx_make(double re, double im) {
    cx r;
    r.re = re;
    r.im = im;
    return r;
}
/* num_complex Mul: Complex::new(a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re) */
static inline cx cx_mul(cx a, cx b) {
    return cx_make(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline cx cx_add(cx a, cx b) { return cx_make(a.re + b.re, a.im + b.im); }
static inline cx cx_conj(cx a) { return cx_make(a.re, -a.im); }
static inline double cx_norm_sqr(cx a) { return a.re * a.re + a.im * a.im; }
/* num_complex MulAssign (a *= b): re = re*b.re - im*b.im; im = im*b.re + re_old*b.im */
static inline void cx_mul_assign(cx* a, cx b) {
    double re_old = a->re;
    double re = a->re * b.re;
    re -= a->im * b.im;
    double im = a->im * b.re;
    im += re_old * b.im;
    a->re = re;
    a->im = im;
}
static inline void cx_add_assign(cx* a, cx b) {
    a->re += b.re;
    a->im += b.im;
}
/* Complex<f64> / f64 */
static inline cx cx_div_real(cx a, double d) { return cx_make(a.re / d, a.im / d); }
/* Complex::from_polar(r, theta) = (r cos theta, r sin theta) */
static inline cx cx_from_polar(double r, double theta) { return cx_make(r * cos(theta), r * sin(theta)); }

#define MAXQ 64

/* ============================================================ bitbasis */

/* bit_ops.rs:3-6 */
static inline uint64_t indicator(uint64_t k) { return (uint64_t)1 << k; }

static uint64_t low_mask(uint64_t width) {
    if (width == 0) return 0;
    if (width >= 64) return ~(uint64_t)0;
    return ((uint64_t)1 << width) - 1;
}

/* bit_ops.rs:9-12 */
uint64_t orc_bmask(const uint64_t* positions, uint32_t n) {
    uint64_t acc = 0;
    for (uint32_t i = 0; i < n; i++) acc |= indicator(positions[i]);
    return acc;
}

/* bit_ops.rs:15-23 */
uint64_t orc_bmask_range(uint64_t start, uint64_t stop) {
    if (stop <= start) return 0;
    return low_mask(stop - start) << start;
}

/* bit_ops.rs:62-72 */
uint64_t orc_swapbits(uint64_t b, uint64_t i, uint64_t j) {
    uint64_t mask = indicator(i) | indicator(j);
    uint64_t masked = b & mask;
    if (masked != 0 && masked != mask) return b ^ mask;
    return b;
}

/* bit_ops.rs:75-80 */
uint64_t orc_breflect(uint64_t b, uint64_t nbits) {
    for (uint64_t i = 0; i < nbits / 2; i++) b = orc_swapbits(b, i, nbits - 1 - i);
    return b;
}

/* bit_ops.rs:83-86 */
uint64_t orc_neg(uint64_t b, uint64_t nbits) { return low_mask(nbits) ^ b; }

/* bit_ops.rs:89-92 */
uint64_t orc_btruncate(uint64_t b, uint64_t n) { return b & low_mask(n); }

static void sort_u64(uint64_t* a, uint32_t n) {
    for (uint32_t i = 1; i < n; i++) {
        uint64_t v = a[i];
        uint32_t j = i;
        while (j > 0 && a[j - 1] > v) {
            a[j] = a[j - 1];
            j--;
        }
        a[j] = v;
    }
}

/* iterate_control.rs:108-142 (group_shift). Returns -1 on a duplicate position. */
int orc_group_shift(uint32_t nbits, const uint64_t* positions_in, uint32_t npos, uint64_t* masks,
                    uint64_t* factors, int32_t* nchunks) {
    uint64_t positions[MAXQ];
    if (npos > MAXQ) return -1;
    memcpy(positions, positions_in, sizeof(uint64_t) * npos);
    sort_u64(positions, npos);
    int32_t nc = 0;
    uint64_t previous = 0, free_index = 0;
    for (uint32_t i = 0; i < npos; i++) {
        uint64_t position = positions[i] + 1;
        if (!(position > previous)) return -1; /* "Duplicate position" */
        if (position != previous + 1) {
            factors[nc] = (uint64_t)1 << (previous - free_index);
            uint64_t gap = position - previous - 1;
            masks[nc] = orc_bmask_range(free_index, free_index + gap);
            nc++;
            free_index += gap;
        }
        previous = position;
    }
    uint64_t nfree = nbits - npos;
    if (free_index != nfree) {
        factors[nc] = (uint64_t)1 << (previous - free_index);
        masks[nc] = orc_bmask_range(free_index, nfree);
        nc++;
    }
    *nchunks = nc;
    return 0;
}

/* iterate_control.rs:82-106 (itercontrol) */
int orc_itercontrol(uint32_t nbits, const uint64_t* positions, const uint64_t* configs, uint32_t npos,
                    orc_iterctl* out) {
    uint64_t base = 0;
    for (uint32_t i = 0; i < npos; i++) {
        if (positions[i] >= nbits) return -1;
        if (configs[i] > 1) return -1;
        if (configs[i] == 1) base |= indicator(positions[i]);
    }
    memset(out, 0, sizeof(*out));
    if (orc_group_shift(nbits, positions, npos, out->masks, out->factors, &out->nchunks) != 0) return -1;
    out->n = (uint64_t)1 << (nbits - npos);
    out->base = base;
    return 0;
}

/* iterate_control.rs:32-55 (IterControl::get) */
uint64_t orc_itercontrol_get(const orc_iterctl* ic, uint64_t k) {
    uint64_t out = ic->base;
    for (int32_t j = 0; j < ic->nchunks; j++) out += (k & ic->masks[j]) * ic->factors[j];
    return out;
}

/* iterate_control.rs:144-159 (controller) */
int orc_controller(const uint64_t* cbits, const uint64_t* cvals, uint32_t n, uint64_t basis) {
    uint64_t mask = orc_bmask(cbits, n);
    uint64_t target = 0;
    for (uint32_t i = 0; i < n; i++)
        if (cvals[i] == 1) target |= indicator(cbits[i]);
    return (basis & mask) == target;
}

/* ===================================================== instruct_qubit.rs */

/* instruct_qubit.rs:14-18 */
static inline uint64_t loc_to_bit(uint32_t nbits, uint64_t loc) { return nbits - 1 - loc; }

/* instruct_qubit.rs:23-36 (u1rows) */
static inline void u1rows(cx* st, uint64_t i, uint64_t j, cx a, cx b, cx c, cx d) {
    cx w = st[i];
    cx v = st[j];
    st[i] = cx_add(cx_mul(a, w), cx_mul(b, v));
    st[j] = cx_add(cx_mul(c, w), cx_mul(d, v));
}

static inline void swap_amp(cx* st, uint64_t i, uint64_t j) {
    cx t = st[i];
    st[i] = st[j];
    st[j] = t;
}

/* instruct_qubit.rs:38-79 (for_each_single_control_base), specialised per body */
enum { BODY_SWAP, BODY_U1, BODY_DIAG };
static void single_control_loop(cx* st, uint64_t total, uint64_t target_bit, uint64_t ctrl_bit,
                                uint64_t ctrl_val, int body, const cx* m) {
    uint64_t step = (uint64_t)1 << target_bit;
#define BODY(base)                                                    \
    do {                                                              \
        uint64_t b_ = (base);                                         \
        if (body == BODY_SWAP)                                        \
            swap_amp(st, b_, b_ + step);                              \
        else if (body == BODY_U1)                                     \
            u1rows(st, b_, b_ + step, m[0], m[1], m[2], m[3]);        \
        else {                                                        \
            cx_mul_assign(&st[b_], m[0]);                             \
            cx_mul_assign(&st[b_ + step], m[1]);                      \
        }                                                             \
    } while (0)
    if (target_bit < ctrl_bit) {
        uint64_t low_span = (uint64_t)1 << target_bit;
        uint64_t middle_iters = (uint64_t)1 << (ctrl_bit - target_bit - 1);
        uint64_t outer_step = (uint64_t)1 << (ctrl_bit + 1);
        uint64_t ctrl_offset = ctrl_val << ctrl_bit;
        for (uint64_t outer = 0; outer < total; outer += outer_step) {
            uint64_t ctrl_base = outer + ctrl_offset;
            for (uint64_t mid = 0; mid < middle_iters; mid++) {
                uint64_t mb = ctrl_base + (mid << (target_bit + 1));
                for (uint64_t low = 0; low < low_span; low++) BODY(mb + low);
            }
        }
    } else {
        uint64_t low_span = (uint64_t)1 << ctrl_bit;
        uint64_t middle_iters = (uint64_t)1 << (target_bit - ctrl_bit - 1);
        uint64_t outer_step = (uint64_t)1 << (target_bit + 1);
        uint64_t ctrl_offset = ctrl_val << ctrl_bit;
        for (uint64_t outer = 0; outer < total; outer += outer_step) {
            for (uint64_t mid = 0; mid < middle_iters; mid++) {
                uint64_t mb = outer + (mid << (ctrl_bit + 1)) + ctrl_offset;
                for (uint64_t low = 0; low < low_span; low++) BODY(mb + low);
            }
        }
    }
#undef BODY
}

/* instruct_qubit.rs:82-92 */
void orc_instruct_x(double* s, uint32_t nbits, uint32_t loc) {
    cx* st = (cx*)s;
    uint64_t mask = indicator(loc_to_bit(nbits, loc));
    uint64_t dim = (uint64_t)1 << nbits;
    for (uint64_t basis = 0; basis < dim; basis++)
        if ((basis & mask) == 0) swap_amp(st, basis, basis ^ mask);
}

/* instruct_qubit.rs:95-126 */
void orc_instruct_x_controlled(double* s, uint32_t nbits, uint32_t loc, const uint64_t* ctrl_locs,
                               const uint64_t* ctrl_bits, uint32_t nctrl) {
    cx* st = (cx*)s;
    uint64_t bit = loc_to_bit(nbits, loc);
    uint64_t mask = indicator(bit);
    uint64_t dim = (uint64_t)1 << nbits;
    if (nctrl == 1) {
        single_control_loop(st, dim, bit, loc_to_bit(nbits, ctrl_locs[0]), ctrl_bits[0], BODY_SWAP, NULL);
        return;
    }
    uint64_t cb[MAXQ];
    for (uint32_t i = 0; i < nctrl; i++) cb[i] = loc_to_bit(nbits, ctrl_locs[i]);
    for (uint64_t basis = 0; basis < dim; basis++)
        if ((basis & mask) == 0 && orc_controller(cb, ctrl_bits, nctrl, basis))
            swap_amp(st, basis, basis ^ mask);
}

/* instruct_qubit.rs:138-158 */
void orc_instruct_1q(double* s, uint32_t nbits, uint32_t loc, const double* m) {
    cx* st = (cx*)s;
    const cx* g = (const cx*)m;
    uint64_t bit = loc_to_bit(nbits, loc);
    uint64_t step1 = (uint64_t)1 << bit, step2 = (uint64_t)1 << (bit + 1);
    uint64_t total = (uint64_t)1 << nbits;
    for (uint64_t j = 0; j < total; j += step2)
        for (uint64_t i = j; i < j + step1; i++) u1rows(st, i, i + step1, g[0], g[1], g[2], g[3]);
}

/* instruct_qubit.rs:170-184 */
void orc_instruct_1q_diag(double* s, uint32_t nbits, uint32_t loc, const double* d) {
    cx* st = (cx*)s;
    const cx* dg = (const cx*)d;
    uint64_t bit = loc_to_bit(nbits, loc);
    uint64_t step1 = (uint64_t)1 << bit, step2 = (uint64_t)1 << (bit + 1);
    uint64_t total = (uint64_t)1 << nbits;
    for (uint64_t j = 0; j < total; j += step2)
        for (uint64_t i = j; i < j + step1; i++) {
            cx_mul_assign(&st[i], dg[0]);
            cx_mul_assign(&st[i + step1], dg[1]);
        }
}

/* instruct_qubit.rs:189-206 (unrows) */
static void unrows(cx* st, const uint64_t* inds, uint32_t d, const cx* gate) {
    cx old[4];
    for (uint32_t k = 0; k < d; k++) old[k] = st[inds[k]];
    for (uint32_t i = 0; i < d; i++) {
        cx acc = cx_make(0.0, 0.0);
        for (uint32_t j = 0; j < d; j++) cx_add_assign(&acc, cx_mul(gate[i * d + j], old[j]));
        st[inds[i]] = acc;
    }
}

/* instruct_qubit.rs:215-231 (sort_unitary_2q); returns sorted bits in sorted[] */
static void sort_unitary_2q(const cx* gate, const uint64_t* bits, cx* out, uint64_t* sorted) {
    sorted[0] = bits[0];
    sorted[1] = bits[1];
    if (sorted[0] < sorted[1]) {
        memcpy(out, gate, sizeof(cx) * 16);
        return;
    }
    uint64_t t = sorted[0];
    sorted[0] = sorted[1];
    sorted[1] = t;
    static const int perm[4] = {0, 2, 1, 3};
    for (int i = 0; i < 16; i++) out[i] = cx_make(0.0, 0.0);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[perm[i] * 4 + perm[j]] = gate[i * 4 + j];
}

/* locs_raw of instruct_2q: itercontrol over the non-target bits locked to 0 */
static void locs_raw_2q(uint32_t nbits, const uint64_t* sorted_bits, uint64_t* locs_raw) {
    uint64_t non_target[MAXQ], zeros[MAXQ];
    uint32_t nn = 0;
    for (uint64_t b = 0; b < nbits; b++)
        if (b != sorted_bits[0] && b != sorted_bits[1]) {
            non_target[nn] = b;
            zeros[nn] = 0;
            nn++;
        }
    orc_iterctl ic;
    orc_itercontrol(nbits, non_target, zeros, nn, &ic);
    for (uint64_t k = 0; k < 4; k++) locs_raw[k] = orc_itercontrol_get(&ic, k);
}

/* instruct_qubit.rs:238-265 */
void orc_instruct_2q(double* s, uint32_t nbits, const uint64_t* locs, const double* g) {
    cx* st = (cx*)s;
    uint64_t bits[2] = {loc_to_bit(nbits, locs[0]), loc_to_bit(nbits, locs[1])};
    cx gate[16];
    uint64_t sorted[2];
    sort_unitary_2q((const cx*)g, bits, gate, sorted);
    uint64_t locs_raw[4];
    locs_raw_2q(nbits, sorted, locs_raw);
    uint64_t zeros[2] = {0, 0};
    orc_iterctl ic;
    orc_itercontrol(nbits, sorted, zeros, 2, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        uint64_t inds[4] = {locs_raw[0] + base, locs_raw[1] + base, locs_raw[2] + base, locs_raw[3] + base};
        unrows(st, inds, 4, gate);
    }
}

/* instruct_qubit.rs:270-302 */
void orc_instruct_2q_diag(double* s, uint32_t nbits, const uint64_t* locs, const double* dg) {
    cx* st = (cx*)s;
    const cx* din = (const cx*)dg;
    uint64_t sorted[2] = {loc_to_bit(nbits, locs[0]), loc_to_bit(nbits, locs[1])};
    cx diag[4] = {din[0], din[1], din[2], din[3]};
    if (sorted[0] > sorted[1]) {
        uint64_t t = sorted[0];
        sorted[0] = sorted[1];
        sorted[1] = t;
        diag[1] = din[2];
        diag[2] = din[1];
    }
    uint64_t locs_raw[4];
    locs_raw_2q(nbits, sorted, locs_raw);
    uint64_t zeros[2] = {0, 0};
    orc_iterctl ic;
    orc_itercontrol(nbits, sorted, zeros, 2, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        for (int q = 0; q < 4; q++) cx_mul_assign(&st[locs_raw[q] + base], diag[q]);
    }
}

/* instruct_qubit.rs:305-320 */
void orc_instruct_swap(double* s, uint32_t nbits, const uint64_t* locs) {
    cx* st = (cx*)s;
    uint64_t mask0 = indicator(loc_to_bit(nbits, locs[0]));
    uint64_t mask1 = indicator(loc_to_bit(nbits, locs[1]));
    uint64_t swap_mask = mask0 | mask1;
    uint64_t dim = (uint64_t)1 << nbits;
    for (uint64_t basis = 0; basis < dim; basis++)
        if ((basis & mask0) == 0 && (basis & mask1) == mask1) swap_amp(st, basis, basis ^ swap_mask);
}

/* instruct_qubit.rs:323-372 */
void orc_instruct_nq(double* s, uint32_t nbits, const uint64_t* locs, uint32_t nlocs, const double* g,
                     const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl) {
    cx* st = (cx*)s;
    const cx* gate = (const cx*)g;
    uint64_t gate_dim = (uint64_t)1 << nlocs;
    uint64_t target_bits[MAXQ], locked[MAXQ], vals[MAXQ];
    for (uint32_t i = 0; i < nlocs; i++) target_bits[i] = loc_to_bit(nbits, locs[i]);
    uint32_t nl = 0;
    for (uint32_t i = 0; i < nctrl; i++) {
        locked[nl] = loc_to_bit(nbits, ctrl_locs[i]);
        vals[nl] = ctrl_bits[i];
        nl++;
    }
    for (uint32_t i = 0; i < nlocs; i++) {
        locked[nl] = target_bits[i];
        vals[nl] = 0;
        nl++;
    }
    uint64_t* raw = (uint64_t*)malloc(sizeof(uint64_t) * gate_dim);
    uint64_t* idx = (uint64_t*)malloc(sizeof(uint64_t) * gate_dim);
    cx* temp = (cx*)malloc(sizeof(cx) * gate_dim);
    for (uint64_t config = 0; config < gate_dim; config++) {
        uint64_t acc = 0;
        for (uint32_t k = 0; k < nlocs; k++) acc |= ((config >> k) & 1) << target_bits[k];
        raw[config] = acc;
    }
    orc_iterctl ic;
    orc_itercontrol(nbits, locked, vals, nl, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        for (uint64_t c = 0; c < gate_dim; c++) idx[c] = base + raw[c];
        for (uint64_t row = 0; row < gate_dim; row++) {
            temp[row] = cx_make(0.0, 0.0);
            for (uint64_t col = 0; col < gate_dim; col++)
                cx_add_assign(&temp[row], cx_mul(gate[row * gate_dim + col], st[idx[col]]));
        }
        for (uint64_t c = 0; c < gate_dim; c++) st[idx[c]] = temp[c];
    }
    free(raw);
    free(idx);
    free(temp);
}

/* instruct_qubit.rs:385-423 */
void orc_instruct_1q_controlled(double* s, uint32_t nbits, uint32_t loc, const double* m,
                                const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl) {
    cx* st = (cx*)s;
    const cx* g = (const cx*)m;
    uint64_t target_bit = loc_to_bit(nbits, loc);
    uint64_t step = (uint64_t)1 << target_bit;
    uint64_t total = (uint64_t)1 << nbits;
    if (nctrl == 1) {
        single_control_loop(st, total, target_bit, loc_to_bit(nbits, ctrl_locs[0]), ctrl_bits[0], BODY_U1, g);
        return;
    }
    uint64_t locked[MAXQ], vals[MAXQ];
    for (uint32_t i = 0; i < nctrl; i++) {
        locked[i] = loc_to_bit(nbits, ctrl_locs[i]);
        vals[i] = ctrl_bits[i];
    }
    locked[nctrl] = target_bit;
    vals[nctrl] = 0;
    orc_iterctl ic;
    orc_itercontrol(nbits, locked, vals, nctrl + 1, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        u1rows(st, base, base + step, g[0], g[1], g[2], g[3]);
    }
}

/* instruct_qubit.rs:428-470 */
void orc_instruct_2q_controlled(double* s, uint32_t nbits, const uint64_t* locs, const double* g,
                                const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl) {
    cx* st = (cx*)s;
    uint64_t bits[2] = {loc_to_bit(nbits, locs[0]), loc_to_bit(nbits, locs[1])};
    cx gate[16];
    uint64_t sorted[2];
    sort_unitary_2q((const cx*)g, bits, gate, sorted);
    uint64_t locs_raw[4];
    locs_raw_2q(nbits, sorted, locs_raw);
    uint64_t locked[MAXQ], vals[MAXQ];
    for (uint32_t i = 0; i < nctrl; i++) {
        locked[i] = loc_to_bit(nbits, ctrl_locs[i]);
        vals[i] = ctrl_bits[i];
    }
    locked[nctrl] = sorted[0];
    vals[nctrl] = 0;
    locked[nctrl + 1] = sorted[1];
    vals[nctrl + 1] = 0;
    orc_iterctl ic;
    orc_itercontrol(nbits, locked, vals, nctrl + 2, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        uint64_t inds[4] = {locs_raw[0] + base, locs_raw[1] + base, locs_raw[2] + base, locs_raw[3] + base};
        unrows(st, inds, 4, gate);
    }
}

/* instruct_qubit.rs:475-511 */
void orc_instruct_1q_diag_controlled(double* s, uint32_t nbits, uint32_t loc, const double* d,
                                     const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl) {
    cx* st = (cx*)s;
    const cx* dg = (const cx*)d;
    uint64_t target_bit = loc_to_bit(nbits, loc);
    uint64_t step = (uint64_t)1 << target_bit;
    uint64_t total = (uint64_t)1 << nbits;
    if (nctrl == 1) {
        single_control_loop(st, total, target_bit, loc_to_bit(nbits, ctrl_locs[0]), ctrl_bits[0], BODY_DIAG, dg);
        return;
    }
    uint64_t locked[MAXQ], vals[MAXQ];
    for (uint32_t i = 0; i < nctrl; i++) {
        locked[i] = loc_to_bit(nbits, ctrl_locs[i]);
        vals[i] = ctrl_bits[i];
    }
    locked[nctrl] = target_bit;
    vals[nctrl] = 0;
    orc_iterctl ic;
    orc_itercontrol(nbits, locked, vals, nctrl + 1, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        cx_mul_assign(&st[base], dg[0]);
        cx_mul_assign(&st[base + step], dg[1]);
    }
}

/* instruct_qubit.rs:516-555 */
void orc_instruct_2q_diag_controlled(double* s, uint32_t nbits, const uint64_t* locs, const double* dgin,
                                     const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl) {
    cx* st = (cx*)s;
    const cx* din = (const cx*)dgin;
    uint64_t sorted[2] = {loc_to_bit(nbits, locs[0]), loc_to_bit(nbits, locs[1])};
    cx diag[4] = {din[0], din[1], din[2], din[3]};
    if (sorted[0] > sorted[1]) {
        uint64_t t = sorted[0];
        sorted[0] = sorted[1];
        sorted[1] = t;
        diag[1] = din[2];
        diag[2] = din[1];
    }
    uint64_t locs_raw[4];
    locs_raw_2q(nbits, sorted, locs_raw);
    uint64_t locked[MAXQ], vals[MAXQ];
    for (uint32_t i = 0; i < nctrl; i++) {
        locked[i] = loc_to_bit(nbits, ctrl_locs[i]);
        vals[i] = ctrl_bits[i];
    }
    locked[nctrl] = sorted[0];
    vals[nctrl] = 0;
    locked[nctrl + 1] = sorted[1];
    vals[nctrl + 1] = 0;
    orc_iterctl ic;
    orc_itercontrol(nbits, locked, vals, nctrl + 2, &ic);
    for (uint64_t k = 0; k < ic.n; k++) {
        uint64_t base = orc_itercontrol_get(&ic, k);
        for (int q = 0; q < 4; q++) cx_mul_assign(&st[locs_raw[q] + base], diag[q]);
    }
}

/* ================================================================ gate.rs */

#define FRAC_1_SQRT_2 0.70710678118654752440
#define FRAC_PI_4 0.78539816339744830962
#define FRAC_PI_2 1.57079632679489661923

/* gate.rs:284-393 (qubit_matrix) */
int orc_gate_matrix(int32_t gate, const double* p, double* outd, uint32_t* dim) {
    cx* m = (cx*)outd;
    cx zero = cx_make(0.0, 0.0), one = cx_make(1.0, 0.0), neg_one = cx_make(-1.0, 0.0);
    cx i = cx_make(0.0, 1.0), neg_i = cx_make(0.0, -1.0);
    *dim = 2;
    switch (gate) {
    case YAO_GATE_X: m[0] = zero; m[1] = one; m[2] = one; m[3] = zero; return 0;
    case YAO_GATE_Y: m[0] = zero; m[1] = neg_i; m[2] = i; m[3] = zero; return 0;
    case YAO_GATE_Z: m[0] = one; m[1] = zero; m[2] = zero; m[3] = neg_one; return 0;
    case YAO_GATE_H: {
        cx s = cx_make(FRAC_1_SQRT_2, 0.0), ns = cx_make(-FRAC_1_SQRT_2, 0.0);
        m[0] = s; m[1] = s; m[2] = s; m[3] = ns;
        return 0;
    }
    case YAO_GATE_S: m[0] = one; m[1] = zero; m[2] = zero; m[3] = i; return 0;
    case YAO_GATE_T: m[0] = one; m[1] = zero; m[2] = zero; m[3] = cx_from_polar(1.0, FRAC_PI_4); return 0;
    case YAO_GATE_SWAP:
        *dim = 4;
        for (int k = 0; k < 16; k++) m[k] = zero;
        m[0] = one; m[1 * 4 + 2] = one; m[2 * 4 + 1] = one; m[15] = one;
        return 0;
    case YAO_GATE_PHASE: m[0] = one; m[1] = zero; m[2] = zero; m[3] = cx_from_polar(1.0, p[0]); return 0;
    case YAO_GATE_RX: {
        double t = p[0];
        cx c = cx_make(cos(t / 2.0), 0.0), nis = cx_make(0.0, -sin(t / 2.0));
        m[0] = c; m[1] = nis; m[2] = nis; m[3] = c;
        return 0;
    }
    case YAO_GATE_RY: {
        double t = p[0];
        cx c = cx_make(cos(t / 2.0), 0.0), s = cx_make(sin(t / 2.0), 0.0), ns = cx_make(-sin(t / 2.0), 0.0);
        m[0] = c; m[1] = ns; m[2] = s; m[3] = c;
        return 0;
    }
    case YAO_GATE_RZ: {
        double t = p[0];
        m[0] = cx_from_polar(1.0, -t / 2.0); m[1] = zero; m[2] = zero; m[3] = cx_from_polar(1.0, t / 2.0);
        return 0;
    }
    case YAO_GATE_SQRTX: {
        cx f = cx_make(0.5, 0.5);
        m[0] = cx_mul(f, one); m[1] = cx_mul(f, neg_i); m[2] = cx_mul(f, neg_i); m[3] = cx_mul(f, one);
        return 0;
    }
    case YAO_GATE_SQRTY: {
        cx f = cx_make(0.5, 0.5);
        m[0] = cx_mul(f, one); m[1] = cx_mul(f, neg_one); m[2] = cx_mul(f, one); m[3] = cx_mul(f, one);
        return 0;
    }
    case YAO_GATE_SQRTW: {
        cx cv = cx_make(FRAC_1_SQRT_2, 0.0), nis = cx_make(0.0, -FRAC_1_SQRT_2);
        cx g01 = cx_make(FRAC_1_SQRT_2, -FRAC_1_SQRT_2), g10 = cx_make(FRAC_1_SQRT_2, FRAC_1_SQRT_2);
        m[0] = cv; m[1] = cx_mul(nis, g01); m[2] = cx_mul(nis, g10); m[3] = cv;
        return 0;
    }
    case YAO_GATE_ISWAP:
        *dim = 4;
        for (int k = 0; k < 16; k++) m[k] = zero;
        m[0] = one; m[1 * 4 + 2] = i; m[2 * 4 + 1] = i; m[15] = one;
        return 0;
    case YAO_GATE_FSIM: {
        *dim = 4;
        double th = p[0], ph = p[1];
        cx ct = cx_make(cos(th), 0.0), nist = cx_make(0.0, -sin(th));
        for (int k = 0; k < 16; k++) m[k] = zero;
        m[0] = one; m[5] = ct; m[6] = nist; m[9] = nist; m[10] = ct; m[15] = cx_from_polar(1.0, -ph);
        return 0;
    }
    default:
        return -1;
    }
}

/* gate.rs:98-104 */
int orc_gate_is_diagonal(int32_t gate) {
    return gate == YAO_GATE_Z || gate == YAO_GATE_S || gate == YAO_GATE_T || gate == YAO_GATE_PHASE ||
           gate == YAO_GATE_RZ;
}

/* gate.rs:107-113 */
int orc_gate_num_params(int32_t gate) {
    switch (gate) {
    case YAO_GATE_RX: case YAO_GATE_RY: case YAO_GATE_RZ: case YAO_GATE_PHASE: return 1;
    case YAO_GATE_FSIM: return 2;
    default: return 0;
    }
}

/* gate.rs:153-193 (generator_matrix) */
int orc_gate_generator(int32_t gate, uint32_t idx, double* outd, uint32_t* dim) {
    cx* m = (cx*)outd;
    cx z = cx_make(0.0, 0.0);
    *dim = 2;
    switch (gate) {
    case YAO_GATE_RX: m[0] = z; m[1] = cx_make(0.0, -0.5); m[2] = cx_make(0.0, -0.5); m[3] = z; return 0;
    case YAO_GATE_RY: m[0] = z; m[1] = cx_make(-0.5, 0.0); m[2] = cx_make(0.5, 0.0); m[3] = z; return 0;
    case YAO_GATE_RZ: m[0] = cx_make(0.0, -0.5); m[1] = z; m[2] = z; m[3] = cx_make(0.0, 0.5); return 0;
    case YAO_GATE_PHASE: m[0] = z; m[1] = z; m[2] = z; m[3] = cx_make(0.0, 1.0); return 0;
    case YAO_GATE_FSIM:
        *dim = 4;
        for (int k = 0; k < 16; k++) m[k] = z;
        if (idx == 0) {
            m[1 * 4 + 2] = cx_make(0.0, -1.0);
            m[2 * 4 + 1] = cx_make(0.0, -1.0);
        } else {
            m[15] = cx_make(0.0, -1.0);
        }
        return 0;
    default:
        return -1;
    }
}

/* A gate resolved to its kind, matrix and diagonal flag (the data
 * dispatch_arrayreg_gate reads from a PositionedGate). */
typedef struct {
    int32_t kind;   /* yao_gate_kind; CUSTOM for custom */
    uint32_t dim;   /* matrix rows */
    cx* m;          /* dim*dim */
    int diag;
    uint32_t nt, nc;
    uint64_t t[MAXQ], c[MAXQ], cv[MAXQ];
} rgate;

static int resolve_gate(const yao_element* e, rgate* g) {
    g->kind = e->type;
    g->nt = e->ntargets;
    g->nc = e->nctrl;
    for (uint32_t i = 0; i < e->ntargets; i++) g->t[i] = e->targets[i];
    for (uint32_t i = 0; i < e->nctrl; i++) {
        g->c[i] = e->ctrl_locs[i];
        g->cv[i] = e->ctrl_configs ? (e->ctrl_configs[i] ? 1 : 0) : 1;
    }
    if (e->type == YAO_GATE_CUSTOM) {
        g->dim = e->matrix_dim;
        g->m = (cx*)malloc(sizeof(cx) * g->dim * g->dim);
        memcpy(g->m, e->matrix, sizeof(cx) * g->dim * g->dim);
        g->diag = e->is_diagonal != 0;
    } else {
        g->m = (cx*)malloc(sizeof(cx) * 16);
        if (orc_gate_matrix(e->type, e->params, (double*)g->m, &g->dim) != 0) return -1;
        g->diag = orc_gate_is_diagonal(e->type);
    }
    return 0;
}

static void free_gate(rgate* g) {
    free(g->m);
    g->m = NULL;
}

/* gate.rs:198-281 (dagger): returns the adjoint as a resolved gate. */
static void gate_dagger(const yao_element* e, rgate* out) {
    rgate tmp;
    resolve_gate(e, &tmp);
    *out = tmp;
    double p[4] = {0, 0, 0, 0};
    switch (e->type) {
    case YAO_GATE_H: case YAO_GATE_X: case YAO_GATE_Y: case YAO_GATE_Z: case YAO_GATE_SWAP:
        return;
    case YAO_GATE_S: p[0] = -FRAC_PI_2; out->kind = YAO_GATE_PHASE; break;
    case YAO_GATE_T: p[0] = -FRAC_PI_4; out->kind = YAO_GATE_PHASE; break;
    case YAO_GATE_RX: case YAO_GATE_RY: case YAO_GATE_RZ: case YAO_GATE_PHASE:
        p[0] = -e->params[0];
        break;
    case YAO_GATE_FSIM:
        p[0] = -e->params[0];
        p[1] = -e->params[1];
        break;
    default: {
        /* SqrtX, SqrtY, SqrtW, ISWAP, Custom: conjugate transpose as Custom */
        uint32_t d = tmp.dim;
        cx* ct = (cx*)malloc(sizeof(cx) * d * d);
        for (uint32_t r = 0; r < d; r++)
            for (uint32_t c = 0; c < d; c++) ct[c * d + r] = cx_conj(tmp.m[r * d + c]);
        free(out->m);
        out->m = ct;
        out->kind = YAO_GATE_CUSTOM;
        out->diag = (e->type == YAO_GATE_CUSTOM) ? (e->is_diagonal != 0) : 0;
        return;
    }
    }
    orc_gate_matrix(out->kind, p, (double*)out->m, &out->dim);
    out->diag = orc_gate_is_diagonal(out->kind);
}

/* ============================================================== apply.rs */

/* apply.rs:7-120 (dispatch_arrayreg_gate) */
static void dispatch_gate(uint32_t nbits, cx* st, const rgate* g) {
    int has_c = g->nc > 0;
    double* s = (double*)st;
    const double* m = (const double*)g->m;
    if (g->kind == YAO_GATE_X && !has_c) {
        for (uint32_t i = 0; i < g->nt; i++) orc_instruct_x(s, nbits, (uint32_t)g->t[i]);
    } else if (g->kind == YAO_GATE_X) {
        for (uint32_t i = 0; i < g->nt; i++)
            orc_instruct_x_controlled(s, nbits, (uint32_t)g->t[i], g->c, g->cv, g->nc);
    } else if (g->kind == YAO_GATE_SWAP && !has_c) {
        orc_instruct_swap(s, nbits, g->t);
    } else if (g->kind == YAO_GATE_SWAP) {
        orc_instruct_2q_controlled(s, nbits, g->t, m, g->c, g->cv, g->nc);
    } else if (g->diag && g->nt == 1) {
        cx d[2] = {g->m[0], g->m[3]};
        if (has_c)
            orc_instruct_1q_diag_controlled(s, nbits, (uint32_t)g->t[0], (double*)d, g->c, g->cv, g->nc);
        else
            orc_instruct_1q_diag(s, nbits, (uint32_t)g->t[0], (double*)d);
    } else if (g->diag && g->nt == 2) {
        cx d[4] = {g->m[0], g->m[5], g->m[10], g->m[15]};
        if (has_c)
            orc_instruct_2q_diag_controlled(s, nbits, g->t, (double*)d, g->c, g->cv, g->nc);
        else
            orc_instruct_2q_diag(s, nbits, g->t, (double*)d);
    } else if (g->nt == 1) {
        if (has_c)
            orc_instruct_1q_controlled(s, nbits, (uint32_t)g->t[0], m, g->c, g->cv, g->nc);
        else
            orc_instruct_1q(s, nbits, (uint32_t)g->t[0], m);
    } else if (g->nt == 2) {
        if (has_c)
            orc_instruct_2q_controlled(s, nbits, g->t, m, g->c, g->cv, g->nc);
        else
            orc_instruct_2q(s, nbits, g->t, m);
    } else {
        orc_instruct_nq(s, nbits, g->t, g->nt, m, g->c, g->cv, g->nc);
    }
}

/* apply.rs:123-147 (apply_inplace); channels are skipped, annotations are no-ops */
int orc_apply_inplace(uint32_t nbits, const yao_element* elems, size_t n, double* s) {
    cx* st = (cx*)s;
    for (size_t i = 0; i < n; i++) {
        if (elems[i].kind != YAO_ELEM_GATE) continue;
        rgate g;
        if (resolve_gate(&elems[i], &g) != 0) return -1;
        dispatch_gate(nbits, st, &g);
        free_gate(&g);
    }
    return 0;
}

/* ============================================================ register.rs */

/* register.rs:71-85 */
void orc_deterministic_state(uint32_t nbits, double* s) {
    cx* st = (cx*)s;
    uint64_t dim = (uint64_t)1 << nbits;
    for (uint64_t k = 0; k < dim; k++) {
        double kf = (double)k;
        st[k] = cx_make(cos(0.1 * kf), sin(0.2 * kf));
    }
    double acc = 0.0;
    for (uint64_t k = 0; k < dim; k++) acc += cx_norm_sqr(st[k]);
    double norm = sqrt(acc);
    for (uint64_t k = 0; k < dim; k++) st[k] = cx_div_real(st[k], norm);
}

/* register.rs:98-104 */
double orc_norm(uint32_t nbits, const double* s) {
    const cx* st = (const cx*)s;
    uint64_t dim = (uint64_t)1 << nbits;
    double acc = 0.0;
    for (uint64_t k = 0; k < dim; k++) acc += cx_norm_sqr(st[k]);
    return sqrt(acc);
}

/* register.rs:115-124 */
double orc_fidelity(uint32_t nbits, const double* a, const double* b) {
    const cx* x = (const cx*)a;
    const cx* y = (const cx*)b;
    uint64_t dim = (uint64_t)1 << nbits;
    cx acc = cx_make(0.0, 0.0);
    for (uint64_t k = 0; k < dim; k++) acc = cx_add(acc, cx_mul(cx_conj(x[k]), y[k]));
    return cx_norm_sqr(acc);
}

/* ===================================================== density_matrix.rs */

/* density_matrix.rs:23-35 */
void orc_dm_from_reg(uint32_t nbits, const double* p, double* r) {
    const cx* psi = (const cx*)p;
    cx* rho = (cx*)r;
    uint64_t dim = (uint64_t)1 << nbits;
    for (uint64_t row = 0; row < dim; row++)
        for (uint64_t col = 0; col < dim; col++) rho[row * dim + col] = cx_mul(psi[row], cx_conj(psi[col]));
}

/* density_matrix.rs:63-67 */
void orc_dm_trace(uint32_t nbits, const double* r, double* out) {
    const cx* rho = (const cx*)r;
    uint64_t dim = (uint64_t)1 << nbits;
    cx acc = cx_make(0.0, 0.0);
    for (uint64_t i = 0; i < dim; i++) acc = cx_add(acc, rho[i * dim + i]);
    out[0] = acc.re;
    out[1] = acc.im;
}

/* density_matrix.rs:69-78 */
double orc_dm_purity(uint32_t nbits, const double* r) {
    const cx* rho = (const cx*)r;
    uint64_t dim = (uint64_t)1 << nbits;
    cx acc = cx_make(0.0, 0.0);
    for (uint64_t row = 0; row < dim; row++)
        for (uint64_t in = 0; in < dim; in++) cx_add_assign(&acc, cx_mul(rho[row * dim + in], rho[in * dim + row]));
    return acc.re;
}

/* density_matrix.rs:80-112 (loc is a bit position, least significant first) */
void orc_dm_partial_tr(uint32_t nbits, const double* r, const uint32_t* traced, uint32_t ntraced, double* o) {
    const cx* rho = (const cx*)r;
    cx* out = (cx*)o;
    uint32_t kept[MAXQ], nk = 0;
    for (uint32_t loc = 0; loc < nbits; loc++) {
        int t = 0;
        for (uint32_t j = 0; j < ntraced; j++)
            if (traced[j] == loc) t = 1;
        if (!t) kept[nk++] = loc;
    }
    uint64_t dim = (uint64_t)1 << nbits, dr = (uint64_t)1 << nk;
    for (uint64_t k = 0; k < dr * dr; k++) out[k] = cx_make(0.0, 0.0);
    for (uint64_t row = 0; row < dim; row++)
        for (uint64_t col = 0; col < dim; col++) {
            int ok = 1;
            for (uint32_t j = 0; j < ntraced; j++)
                if (((row >> traced[j]) & 1) != ((col >> traced[j]) & 1)) ok = 0;
            if (!ok) continue;
            uint64_t rr = 0, rc = 0;
            for (uint32_t k = 0; k < nk; k++) {
                rr |= ((row >> kept[k]) & 1) << k;
                rc |= ((col >> kept[k]) & 1) << k;
            }
            cx_add_assign(&out[rr * dr + rc], rho[row * dim + col]);
        }
}

/* density_matrix.rs:123-129 (is_diagonal_matrix) */
static int is_diagonal_matrix(const cx* m, uint32_t d) {
    for (uint32_t r = 0; r < d; r++)
        for (uint32_t c = 0; c < d; c++)
            if (r != c && !(hypot(m[r * d + c].re, m[r * d + c].im) < 1e-15)) return 0;
    return 1;
}

/* density_matrix.rs:131-151 (conjugated_gate + shift_gate) */
static void conj_shift(const rgate* g, uint32_t n, int diag, rgate* out) {
    *out = *g;
    out->m = (cx*)malloc(sizeof(cx) * g->dim * g->dim);
    for (uint32_t k = 0; k < g->dim * g->dim; k++) out->m[k] = cx_conj(g->m[k]);
    out->kind = YAO_GATE_CUSTOM;
    out->diag = diag;
    for (uint32_t i = 0; i < g->nt; i++) out->t[i] = g->t[i] + n;
    for (uint32_t i = 0; i < g->nc; i++) out->c[i] = g->c[i] + n;
}

/* density_matrix.rs:161-178 (apply_gate) */
static void dm_apply_gate(uint32_t n, cx* rho, const rgate* g) {
    dispatch_gate(2 * n, rho, g);
    rgate cg;
    conj_shift(g, n, g->diag, &cg);
    dispatch_gate(2 * n, rho, &cg);
    free_gate(&cg);
}

/* density_matrix.rs:181-224 (apply_channel) */
static int dm_apply_channel(uint32_t n, cx* rho, const yao_element* e) {
    uint32_t nk = 0, d = 0;
    cx* kraus = (cx*)malloc(sizeof(cx) * 16 * 16 * 256);
    if (orc_noise_kraus(e, (double*)kraus, 256, &nk, &d) != 0) {
        free(kraus);
        return -1;
    }
    uint64_t len = (uint64_t)1 << (2 * n);
    cx* original = (cx*)malloc(sizeof(cx) * len);
    cx* acc = (cx*)malloc(sizeof(cx) * len);
    cx* branch = (cx*)malloc(sizeof(cx) * len);
    memcpy(original, rho, sizeof(cx) * len);
    for (uint64_t i = 0; i < len; i++) acc[i] = cx_make(0.0, 0.0);
    for (uint32_t k = 0; k < nk; k++) {
        memcpy(branch, original, sizeof(cx) * len);
        rgate g;
        memset(&g, 0, sizeof(g));
        g.kind = YAO_GATE_CUSTOM;
        g.dim = d;
        g.m = kraus + (size_t)k * d * d;
        g.diag = is_diagonal_matrix(g.m, d);
        g.nt = e->ntargets;
        g.nc = 0;
        for (uint32_t i = 0; i < e->ntargets; i++) g.t[i] = e->targets[i];
        dispatch_gate(2 * n, branch, &g);
        rgate cg;
        conj_shift(&g, n, g.diag, &cg);
        dispatch_gate(2 * n, branch, &cg);
        free_gate(&cg);
        for (uint64_t i = 0; i < len; i++) cx_add_assign(&acc[i], branch[i]);
    }
    memcpy(rho, acc, sizeof(cx) * len);
    free(original);
    free(acc);
    free(branch);
    free(kraus);
    return 0;
}

/* density_matrix.rs:249-259 (Register::apply) */
int orc_dm_apply(uint32_t nbits, const yao_element* elems, size_t n, double* r) {
    cx* rho = (cx*)r;
    for (size_t i = 0; i < n; i++) {
        if (elems[i].kind == YAO_ELEM_GATE) {
            rgate g;
            if (resolve_gate(&elems[i], &g) != 0) return -1;
            dm_apply_gate(nbits, rho, &g);
            free_gate(&g);
        } else if (elems[i].kind == YAO_ELEM_CHANNEL) {
            if (dm_apply_channel(nbits, rho, &elems[i]) != 0) return -1;
        }
    }
    return 0;
}

/* =============================================================== noise.rs */

static void set2(cx* m, cx a, cx b, cx c, cx d) {
    m[0] = a;
    m[1] = b;
    m[2] = c;
    m[3] = d;
}

/* noise.rs:383-458 (phase_amplitude_damping_kraus) */
static uint32_t pad_kraus(double a, double b, double p1, cx* out) {
    cx z = cx_make(0.0, 0.0);
    uint32_t n = 0;
    double rest = sqrt(1.0 - a - b);
    if (fabs(p1 - 1.0) > DBL_EPSILON) {
        double s = sqrt(1.0 - p1);
        set2(out + 4 * n++, cx_make(s, 0.0), z, z, cx_make(s * rest, 0.0));
        if (a > 0.0) {
            double sa = sqrt(a) * s;
            set2(out + 4 * n++, z, cx_make(sa, 0.0), z, z);
        }
        if (b > 0.0) {
            double sb = sqrt(b) * s;
            set2(out + 4 * n++, z, z, z, cx_make(sb, 0.0));
        }
    }
    if (fabs(p1) > DBL_EPSILON) {
        double s = sqrt(p1);
        set2(out + 4 * n++, cx_make(s * rest, 0.0), z, z, cx_make(s, 0.0));
        if (a > 0.0) {
            double sa = sqrt(a) * s;
            set2(out + 4 * n++, z, z, cx_make(sa, 0.0), z);
        }
        if (b > 0.0) {
            double sb = sqrt(b) * s;
            set2(out + 4 * n++, cx_make(sb, 0.0), z, z, z);
        }
    }
    return n;
}

/* noise.rs:513-525 (kron) */
static void kron(const cx* a, uint32_t ad, const cx* b, uint32_t bd, cx* out) {
    uint32_t od = ad * bd;
    for (uint32_t i = 0; i < ad; i++)
        for (uint32_t j = 0; j < ad; j++)
            for (uint32_t k = 0; k < bd; k++)
                for (uint32_t l = 0; l < bd; l++) out[(i * bd + k) * od + j * bd + l] = cx_mul(a[i * ad + j], b[k * bd + l]);
}

static int in01(double v) { return v >= 0.0 && v <= 1.0; }

/* noise.rs:90-176 (validate_params) */
static int validate_noise(const yao_element* e) {
    const double* p = e->params;
    switch (e->type) {
    case YAO_NOISE_BIT_FLIP: case YAO_NOISE_PHASE_FLIP: case YAO_NOISE_DEPOLARIZING:
        return in01(p[0]) ? 0 : -1;
    case YAO_NOISE_PAULI_CHANNEL:
        return (p[0] >= 0.0 && p[1] >= 0.0 && p[2] >= 0.0 && p[0] + p[1] + p[2] <= 1.0) ? 0 : -1;
    case YAO_NOISE_RESET:
        return (p[0] >= 0.0 && p[1] >= 0.0 && p[0] + p[1] <= 1.0) ? 0 : -1;
    case YAO_NOISE_PHASE_AMPLITUDE_DAMPING:
        return (p[0] >= 0.0 && p[1] >= 0.0 && p[0] + p[1] <= 1.0 && in01(p[2])) ? 0 : -1;
    case YAO_NOISE_AMPLITUDE_DAMPING:
        return (in01(p[0]) && in01(p[1])) ? 0 : -1;
    case YAO_NOISE_PHASE_DAMPING:
        return in01(p[0]) ? 0 : -1;
    case YAO_NOISE_THERMAL_RELAXATION:
        return (p[0] > 0.0 && p[1] > 0.0 && p[2] >= 0.0 && p[1] <= 2.0 * p[0] && in01(p[3])) ? 0 : -1;
    case YAO_NOISE_CUSTOM:
        return e->nkraus >= 1 ? 0 : -1;
    case YAO_NOISE_COHERENT:
        return 0;
    default:
        return -1;
    }
}

static uint32_t pauli_kraus(double px, double py, double pz, cx* out) {
    cx z = cx_make(0.0, 0.0);
    double s0 = sqrt(1.0 - px - py - pz), sx = sqrt(px), sy = sqrt(py), sz = sqrt(pz);
    set2(out + 0, cx_make(s0, 0.0), z, z, cx_make(s0, 0.0));
    set2(out + 4, z, cx_make(sx, 0.0), cx_make(sx, 0.0), z);
    set2(out + 8, z, cx_make(0.0, -sy), cx_make(0.0, sy), z);
    set2(out + 12, cx_make(sz, 0.0), z, z, cx_make(-sz, 0.0));
    return 4;
}

/* noise.rs:183-352 (kraus_operators) */
int orc_noise_kraus(const yao_element* e, double* outd, uint32_t max_kraus, uint32_t* nk, uint32_t* dim) {
    cx* out = (cx*)outd;
    cx z = cx_make(0.0, 0.0);
    if (validate_noise(e) != 0) return -1;
    const double* p = e->params;
    *dim = 2;
    switch (e->type) {
    case YAO_NOISE_PHASE_AMPLITUDE_DAMPING: *nk = pad_kraus(p[0], p[1], p[2], out); return 0;
    case YAO_NOISE_AMPLITUDE_DAMPING: *nk = pad_kraus(p[0], 0.0, p[1], out); return 0;
    case YAO_NOISE_PHASE_DAMPING: *nk = pad_kraus(0.0, p[0], 0.0, out); return 0;
    case YAO_NOISE_THERMAL_RELAXATION: {
        double t1 = p[0], t2 = p[1], time = p[2];
        double t_phi = (t1 * t2) / (2.0 * t1 - t2);
        double a = 1.0 - exp(-time / t1);
        double b = 1.0 - exp(-time / t_phi);
        *nk = pad_kraus(a, b, p[3], out);
        return 0;
    }
    case YAO_NOISE_BIT_FLIP: {
        double s0 = sqrt(1.0 - p[0]), s1 = sqrt(p[0]);
        set2(out, cx_make(s0, 0.0), z, z, cx_make(s0, 0.0));
        set2(out + 4, z, cx_make(s1, 0.0), cx_make(s1, 0.0), z);
        *nk = 2;
        return 0;
    }
    case YAO_NOISE_PHASE_FLIP: {
        double s0 = sqrt(1.0 - p[0]), s1 = sqrt(p[0]);
        set2(out, cx_make(s0, 0.0), z, z, cx_make(s0, 0.0));
        set2(out + 4, cx_make(s1, 0.0), z, z, cx_make(-s1, 0.0));
        *nk = 2;
        return 0;
    }
    case YAO_NOISE_PAULI_CHANNEL: *nk = pauli_kraus(p[0], p[1], p[2], out); return 0;
    case YAO_NOISE_DEPOLARIZING: {
        uint32_t n = (uint32_t)e->depol_n;
        if (n == 1) {
            double q = p[0] / 4.0;
            *nk = pauli_kraus(q, q, q, out);
            return 0;
        }
        /* noise.rs:462-508 (depolarizing_multi_qubit_kraus) */
        uint32_t d = 1u << n;
        uint32_t cnt = 1u << (2 * n);
        if (cnt > max_kraus) return -1;
        cx paulis[4][4];
        set2(paulis[0], cx_make(1.0, 0.0), z, z, cx_make(1.0, 0.0));
        set2(paulis[1], z, cx_make(1.0, 0.0), cx_make(1.0, 0.0), z);
        set2(paulis[2], z, cx_make(0.0, -1.0), cx_make(0.0, 1.0), z);
        set2(paulis[3], cx_make(1.0, 0.0), z, z, cx_make(-1.0, 0.0));
        cx* mat = (cx*)malloc(sizeof(cx) * d * d);
        cx* tmp = (cx*)malloc(sizeof(cx) * d * d);
        for (uint32_t idx = 0; idx < cnt; idx++) {
            uint32_t md = 1;
            mat[0] = cx_make(1.0, 0.0);
            uint32_t t = idx;
            for (uint32_t q = 0; q < n; q++) {
                uint32_t pi = t % 4;
                t /= 4;
                kron(mat, md, paulis[pi], 2, tmp);
                md *= 2;
                memcpy(mat, tmp, sizeof(cx) * md * md);
            }
            double weight = (idx == 0) ? (1.0 - p[0] + p[0] / (double)cnt) : p[0] / (double)cnt;
            double s = sqrt(weight);
            for (uint32_t k = 0; k < d * d; k++) out[(size_t)idx * d * d + k] = cx_mul(mat[k], cx_make(s, 0.0));
        }
        free(mat);
        free(tmp);
        *nk = cnt;
        *dim = d;
        return 0;
    }
    case YAO_NOISE_RESET: {
        double s = sqrt(1.0 - p[0] - p[1]);
        uint32_t n = 0;
        set2(out + 4 * n++, cx_make(s, 0.0), z, z, cx_make(s, 0.0));
        if (p[0] > 0.0) {
            double sp0 = sqrt(p[0]);
            set2(out + 4 * n++, cx_make(sp0, 0.0), z, z, z);
            set2(out + 4 * n++, z, cx_make(sp0, 0.0), z, z);
        }
        if (p[1] > 0.0) {
            double sp1 = sqrt(p[1]);
            set2(out + 4 * n++, z, z, z, cx_make(sp1, 0.0));
            set2(out + 4 * n++, z, z, cx_make(sp1, 0.0), z);
        }
        *nk = n;
        return 0;
    }
    case YAO_NOISE_COHERENT: {
        uint32_t d = e->matrix_dim;
        memcpy(out, e->matrix, sizeof(cx) * d * d);
        *nk = 1;
        *dim = d;
        return 0;
    }
    case YAO_NOISE_CUSTOM: {
        uint32_t d = e->matrix_dim;
        if (e->nkraus > max_kraus) return -1;
        memcpy(out, e->matrix, sizeof(cx) * d * d * e->nkraus);
        *nk = e->nkraus;
        *dim = d;
        return 0;
    }
    default:
        return -1;
    }
}

/* noise.rs:359-379 (superop) */
int orc_noise_superop(const yao_element* e, double* outd, uint32_t* dim2) {
    cx* out = (cx*)outd;
    uint32_t nk, d;
    cx* kraus = (cx*)malloc(sizeof(cx) * 16 * 16 * 256);
    if (orc_noise_kraus(e, (double*)kraus, 256, &nk, &d) != 0) {
        free(kraus);
        return -1;
    }
    uint32_t d2 = d * d;
    for (uint32_t k = 0; k < d2 * d2; k++) out[k] = cx_make(0.0, 0.0);
    for (uint32_t q = 0; q < nk; q++) {
        const cx* K = kraus + (size_t)q * d * d;
        for (uint32_t i = 0; i < d; i++)
            for (uint32_t j = 0; j < d; j++)
                for (uint32_t kr = 0; kr < d; kr++)
                    for (uint32_t kc = 0; kc < d; kc++)
                        cx_add_assign(&out[(i * d + kr) * d2 + j * d + kc], cx_mul(cx_conj(K[i * d + j]), K[kr * d + kc]));
    }
    *dim2 = d2;
    free(kraus);
    return 0;
}

/* ============================================================ operator.rs */

/* operator.rs:53-65 (op_matrix) */
static void op_matrix(int32_t op, cx* m) {
    cx z = cx_make(0.0, 0.0), o = cx_make(1.0, 0.0);
    switch (op) {
    case YAO_OP_I: set2(m, o, z, z, o); break;
    case YAO_OP_X: set2(m, z, o, o, z); break;
    case YAO_OP_Y: set2(m, z, cx_make(0.0, -1.0), cx_make(0.0, 1.0), z); break;
    case YAO_OP_Z: set2(m, o, z, z, cx_make(-1.0, 0.0)); break;
    case YAO_OP_P0: set2(m, o, z, z, z); break;
    case YAO_OP_P1: set2(m, z, z, z, o); break;
    case YAO_OP_PU: set2(m, z, o, z, z); break;
    default: set2(m, z, z, o, z); break; /* Pd */
    }
}

/* operator.rs:27-33 (OperatorString::new): stable sort by site, then drop I */
static uint32_t opstring_new(const yao_term* t, uint32_t* sites, int32_t* ops) {
    uint32_t n = t->nops;
    for (uint32_t i = 0; i < n; i++) {
        sites[i] = t->sites[i];
        ops[i] = t->ops[i];
    }
    for (uint32_t i = 1; i < n; i++) {
        uint32_t s = sites[i];
        int32_t o = ops[i];
        uint32_t j = i;
        while (j > 0 && sites[j - 1] > s) {
            sites[j] = sites[j - 1];
            ops[j] = ops[j - 1];
            j--;
        }
        sites[j] = s;
        ops[j] = o;
    }
    uint32_t k = 0;
    for (uint32_t i = 0; i < n; i++)
        if (ops[i] != YAO_OP_I) {
            sites[k] = sites[i];
            ops[k] = ops[i];
            k++;
        }
    return k;
}

/* ============================================================== expect.rs */

/* expect.rs:13-24 (expect_opstring_pure) */
static cx expect_opstring_pure(uint32_t nbits, const cx* psi, const yao_term* t, cx* scratch) {
    uint64_t dim = (uint64_t)1 << nbits;
    uint32_t sites[MAXQ * 4];
    int32_t ops[MAXQ * 4];
    uint32_t n = opstring_new(t, sites, ops);
    memcpy(scratch, psi, sizeof(cx) * dim);
    for (uint32_t i = 0; i < n; i++) {
        cx m[4];
        op_matrix(ops[i], m);
        orc_instruct_1q((double*)scratch, nbits, sites[i], (double*)m);
    }
    cx acc = cx_make(0.0, 0.0);
    for (uint64_t k = 0; k < dim; k++) acc = cx_add(acc, cx_mul(cx_conj(psi[k]), scratch[k]));
    return acc;
}

/* expect.rs:7-11 (expect_arrayreg) */
void orc_expect_arrayreg(uint32_t nbits, const double* p, const yao_term* terms, size_t nterms, double* out) {
    const cx* psi = (const cx*)p;
    cx* scratch = (cx*)malloc(sizeof(cx) * ((size_t)1 << nbits));
    cx acc = cx_make(0.0, 0.0);
    for (size_t i = 0; i < nterms; i++) {
        cx c = cx_make(terms[i].coeff_re, terms[i].coeff_im);
        acc = cx_add(acc, cx_mul(c, expect_opstring_pure(nbits, psi, &terms[i], scratch)));
    }
    free(scratch);
    out[0] = acc.re;
    out[1] = acc.im;
}

/* expect.rs:44-72 (expect_opstring_dm): site s reads bit s (LSB first) */
static cx expect_opstring_dm(uint32_t nbits, const cx* rho, const yao_term* t) {
    uint64_t dim = (uint64_t)1 << nbits;
    uint32_t sites[MAXQ * 4];
    int32_t ops[MAXQ * 4];
    uint32_t n = opstring_new(t, sites, ops);
    cx mats[MAXQ * 4][4];
    for (uint32_t i = 0; i < n; i++) op_matrix(ops[i], mats[i]);
    uint64_t untouched = 0;
    for (uint32_t loc = 0; loc < nbits; loc++) {
        int hit = 0;
        for (uint32_t i = 0; i < n; i++)
            if (sites[i] == loc) hit = 1;
        if (!hit) untouched |= (uint64_t)1 << loc;
    }
    cx trace = cx_make(0.0, 0.0);
    for (uint64_t row = 0; row < dim; row++)
        for (uint64_t col = 0; col < dim; col++) {
            cx entry = cx_make(1.0, 0.0);
            for (uint32_t i = 0; i < n; i++) {
                uint64_t rb = (row >> sites[i]) & 1, cb = (col >> sites[i]) & 1;
                cx_mul_assign(&entry, mats[i][rb * 2 + cb]);
            }
            if (((row ^ col) & untouched) == 0) cx_add_assign(&trace, cx_mul(entry, rho[col * dim + row]));
        }
    return trace;
}

/* expect.rs:38-42 (expect_dm) */
void orc_expect_dm(uint32_t nbits, const double* r, const yao_term* terms, size_t nterms, double* out) {
    const cx* rho = (const cx*)r;
    cx acc = cx_make(0.0, 0.0);
    for (size_t i = 0; i < nterms; i++) {
        cx c = cx_make(terms[i].coeff_re, terms[i].coeff_im);
        acc = cx_add(acc, cx_mul(c, expect_opstring_dm(nbits, rho, &terms[i])));
    }
    out[0] = acc.re;
    out[1] = acc.im;
}

/* ================================================================== ad.rs */

/* ad.rs:19-27 (controls_match) */
static int controls_match(uint64_t basis, uint32_t nbits, const rgate* g) {
    for (uint32_t i = 0; i < g->nc; i++) {
        uint64_t bit = nbits - 1 - g->c[i];
        if (((basis >> bit) & 1) != g->cv[i]) return 0;
    }
    return 1;
}

/* ad.rs:34-65 (apply_generator) */
static void apply_generator(cx* st, uint32_t nbits, const rgate* pg, const cx* gm, uint32_t gdim) {
    rgate tmp = *pg;
    tmp.kind = YAO_GATE_CUSTOM;
    tmp.dim = gdim;
    tmp.m = (cx*)gm;
    tmp.diag = 0;
    if (pg->nc == 0) {
        dispatch_gate(nbits, st, &tmp);
        return;
    }
    uint64_t dim = (uint64_t)1 << nbits;
    cx* tr = (cx*)malloc(sizeof(cx) * dim);
    memcpy(tr, st, sizeof(cx) * dim);
    dispatch_gate(nbits, tr, &tmp);
    for (uint64_t b = 0; b < dim; b++) st[b] = controls_match(b, nbits, pg) ? tr[b] : cx_make(0.0, 0.0);
    free(tr);
}

/* ad.rs:75-156 (expect_grad) */
int orc_expect_grad(uint32_t nbits, const yao_term* terms, size_t nterms, const yao_element* elems,
                    size_t nelems, const double* psi0, double* value, double* grad, size_t ngrad) {
    for (size_t i = 0; i < nelems; i++)
        if (elems[i].kind == YAO_ELEM_CHANNEL) return -1;
    uint64_t dim = (uint64_t)1 << nbits;
    cx* psi = (cx*)malloc(sizeof(cx) * dim);
    memcpy(psi, psi0, sizeof(cx) * dim);
    orc_apply_inplace(nbits, elems, nelems, (double*)psi);
    double ev[2];
    orc_expect_arrayreg(nbits, (double*)psi, terms, nterms, ev);
    *value = ev[0];
    size_t np = 0;
    for (size_t i = 0; i < nelems; i++)
        if (elems[i].kind == YAO_ELEM_GATE) np += (size_t)orc_gate_num_params(elems[i].type);
    if (np != ngrad) {
        free(psi);
        return -2;
    }
    for (size_t i = 0; i < np; i++) grad[i] = 0.0;
    if (np == 0) {
        free(psi);
        return 0;
    }
    cx* lambda = (cx*)malloc(sizeof(cx) * dim);
    cx* tmp = (cx*)malloc(sizeof(cx) * dim);
    for (uint64_t i = 0; i < dim; i++) lambda[i] = cx_make(0.0, 0.0);
    for (size_t t = 0; t < nterms; t++) {
        uint32_t sites[MAXQ * 4];
        int32_t ops[MAXQ * 4];
        uint32_t n = opstring_new(&terms[t], sites, ops);
        memcpy(tmp, psi, sizeof(cx) * dim);
        for (uint32_t i = 0; i < n; i++) {
            cx m[4];
            op_matrix(ops[i], m);
            orc_instruct_1q((double*)tmp, nbits, sites[i], (double*)m);
        }
        cx c = cx_make(terms[t].coeff_re, terms[t].coeff_im);
        for (uint64_t i = 0; i < dim; i++) cx_add_assign(&lambda[i], cx_mul(c, tmp[i]));
    }
    size_t slot = np;
    for (size_t ei = nelems; ei-- > 0;) {
        const yao_element* e = &elems[ei];
        if (e->kind != YAO_ELEM_GATE) continue;
        rgate pg;
        resolve_gate(e, &pg);
        int npar = orc_gate_num_params(e->type);
        for (int i = npar - 1; i >= 0; i--) {
            slot--;
            memcpy(tmp, psi, sizeof(cx) * dim);
            cx gm[16];
            uint32_t gd;
            orc_gate_generator(e->type, (uint32_t)i, (double*)gm, &gd);
            apply_generator(tmp, nbits, &pg, gm, gd);
            cx acc = cx_make(0.0, 0.0);
            for (uint64_t k = 0; k < dim; k++) cx_add_assign(&acc, cx_mul(cx_conj(lambda[k]), tmp[k]));
            grad[slot] = 2.0 * acc.re;
        }
        rgate dg;
        gate_dagger(e, &dg);
        dispatch_gate(nbits, psi, &dg);
        dispatch_gate(nbits, lambda, &dg);
        free_gate(&dg);
        free_gate(&pg);
    }
    free(psi);
    free(lambda);
    free(tmp);
    return 0;
}

/* ============================================================= measure.rs */

/* measure.rs:82-104 (probs for ArrayReg; locs[0] is the outcome MSB) */
void orc_probs(uint32_t nbits, const double* p, const uint32_t* locs, int32_t nlocs, double* out) {
    const cx* psi = (const cx*)p;
    uint64_t dim = (uint64_t)1 << nbits;
    if (nlocs < 0) {
        for (uint64_t b = 0; b < dim; b++) out[b] = cx_norm_sqr(psi[b]);
        return;
    }
    uint64_t np = (uint64_t)1 << nlocs;
    for (uint64_t k = 0; k < np; k++) out[k] = 0.0;
    for (uint64_t b = 0; b < dim; b++) {
        uint64_t idx = 0;
        for (int32_t i = 0; i < nlocs; i++) {
            uint64_t bit = nbits - 1 - locs[i];
            idx |= ((b >> bit) & 1) << (nlocs - 1 - i);
        }
        out[idx] += cx_norm_sqr(psi[b]);
    }
}

/* measure.rs:50-57, 106-122 (probs for DensityMatrix: diagonal, re.max(0)) */
void orc_dm_probs(uint32_t nbits, const double* r, const uint32_t* locs, int32_t nlocs, double* out) {
    const cx* rho = (const cx*)r;
    uint64_t dim = (uint64_t)1 << nbits;
    if (nlocs < 0) {
        for (uint64_t b = 0; b < dim; b++) out[b] = fmax(rho[b * dim + b].re, 0.0);
        return;
    }
    uint64_t np = (uint64_t)1 << nlocs;
    for (uint64_t k = 0; k < np; k++) out[k] = 0.0;
    for (uint64_t b = 0; b < dim; b++) {
        uint64_t idx = 0;
        for (int32_t i = 0; i < nlocs; i++) {
            uint64_t bit = nbits - 1 - locs[i];
            idx |= ((b >> bit) & 1) << (nlocs - 1 - i);
        }
        out[idx] += fmax(rho[b * dim + b].re, 0.0);
    }
}

/* measure.rs:140-150 (sample_from_probs with the uniform draw r given) */
uint64_t orc_sample_from_probs(const double* probs, uint64_t n, double r) {
    double cumsum = 0.0;
    for (uint64_t i = 0; i < n; i++) {
        cumsum += probs[i];
        if (r < cumsum) return i;
    }
    return n - 1;
}

static int matches_values(uint64_t basis, uint32_t nbits, const uint32_t* locs, const uint8_t* vals, uint32_t n) {
    for (uint32_t i = 0; i < n; i++)
        if (((basis >> (nbits - 1 - locs[i])) & 1) != vals[i]) return 0;
    return 1;
}

/* measure.rs:243-274 (measure_with_postprocess) with :152-240 inlined */
int orc_measure_with_postprocess(uint32_t nbits, double* p, const uint32_t* locs, uint32_t nlocs, int32_t post,
                                 uint64_t reset_val, double r, uint8_t* outcome, double* removed_out) {
    cx* st = (cx*)p;
    uint64_t dim = (uint64_t)1 << nbits;
    for (uint32_t i = 0; i < nlocs; i++) {
        if (locs[i] >= nbits) return -1;
        for (uint32_t j = 0; j < i; j++)
            if (locs[j] == locs[i]) return -1;
    }
    uint64_t np = (uint64_t)1 << nlocs;
    double* pr = (double*)malloc(sizeof(double) * np);
    orc_probs(nbits, p, locs, (int32_t)nlocs, pr);
    uint64_t idx = orc_sample_from_probs(pr, np, r);
    free(pr);
    for (uint32_t i = 0; i < nlocs; i++) outcome[i] = (uint8_t)((idx >> (nlocs - 1 - i)) & 1);
    if (post == YAO_POST_NONE) return 0;
    if (post == YAO_POST_RESET_TO && reset_val >= np) return -2;
    /* collapse_qubits_to :158-185 */
    double norm_sq = 0.0;
    for (uint64_t b = 0; b < dim; b++) {
        if (matches_values(b, nbits, locs, outcome, nlocs))
            norm_sq += cx_norm_sqr(st[b]);
        else
            st[b] = cx_make(0.0, 0.0);
    }
    double norm = sqrt(norm_sq);
    if (norm > 1e-15)
        for (uint64_t b = 0; b < dim; b++) st[b] = cx_div_real(st[b], norm);
    if (post == YAO_POST_RESET_TO) {
        /* reset_qubits_to :187-215 */
        uint8_t to_bits[MAXQ];
        int same = 1;
        for (uint32_t i = 0; i < nlocs; i++) {
            to_bits[i] = (uint8_t)((reset_val >> (nlocs - 1 - i)) & 1);
            if (to_bits[i] != outcome[i]) same = 0;
        }
        if (same) return 0;
        uint64_t swap_mask = 0;
        for (uint32_t i = 0; i < nlocs; i++)
            if (outcome[i] != to_bits[i]) swap_mask |= (uint64_t)1 << (nbits - 1 - locs[i]);
        for (uint64_t b = 0; b < dim; b++) {
            if (!matches_values(b, nbits, locs, outcome, nlocs)) continue;
            uint64_t tb = b ^ swap_mask;
            cx amp = st[b];
            st[tb] = amp;
            st[b] = cx_make(0.0, 0.0);
        }
        return 0;
    }
    /* remove_measured_qubits :217-240 */
    uint32_t kept[MAXQ], nk = 0;
    for (uint32_t loc = 0; loc < nbits; loc++) {
        int m = 0;
        for (uint32_t i = 0; i < nlocs; i++)
            if (locs[i] == loc) m = 1;
        if (!m) kept[nk++] = loc;
    }
    cx* ns = (cx*)removed_out;
    uint64_t nd = (uint64_t)1 << nk;
    for (uint64_t k = 0; k < nd; k++) ns[k] = cx_make(0.0, 0.0);
    for (uint64_t b = 0; b < dim; b++) {
        if (cx_norm_sqr(st[b]) < 1e-30) continue;
        uint64_t nb = 0;
        for (uint32_t i = 0; i < nk; i++) nb |= ((b >> (nbits - 1 - kept[i])) & 1) << (nk - 1 - i);
        cx_add_assign(&ns[nb], st[b]);
    }
    double acc = 0.0;
    for (uint64_t k = 0; k < nd; k++) acc += cx_norm_sqr(ns[k]);
    double nn = sqrt(acc);
    if (nn > 0.0)
        for (uint64_t k = 0; k < nd; k++) ns[k] = cx_div_real(ns[k], nn);
    return 0;
}
