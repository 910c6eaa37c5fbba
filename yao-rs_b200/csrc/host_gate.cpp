// host_gate.cpp — host-side gate algebra of the library: gate matrices,
// adjoints and generators (yao-rs src/gate.rs), Kraus operators of the noise
// channels (src/noise.rs) and the lowering of a positioned gate to the kernel
// class that yao-rs's dispatch_arrayreg_gate would pick (src/apply.rs:7-120).
//
// Matrices are built in double precision with the same formulas as gate.rs
// (cos/sin of the same arguments, num_complex's (ac-bd, ad+bc) product), so
// the device kernels receive the same coefficients the CPU path uses.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "yao_internal.h"

namespace yao {

static inline Cx cx(double re, double im) { return Cx{re, im}; }
static inline Cx cmul(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static inline Cx cconj(Cx a) { return Cx{a.re, -a.im}; }
static inline Cx from_polar(double r, double t) { return Cx{r * std::cos(t), r * std::sin(t)}; }

static const double kFrac1Sqrt2 = 0.70710678118654752440;
static const double kFracPi4 = 0.78539816339744830962;
static const double kFracPi2 = 1.57079632679489661923;

uint64_t LGate::cmask() const {
    uint64_t m = 0;
    for (int i = 0; i < nc; i++) m |= (uint64_t)1 << cb[i];
    return m;
}
uint64_t LGate::cval() const {
    uint64_t v = 0;
    for (int i = 0; i < nc; i++)
        if (cv[i]) v |= (uint64_t)1 << cb[i];
    return v;
}

// src/gate.rs:284-393 (qubit_matrix)
int named_gate_matrix(int32_t type, const double* p, std::vector<Cx>& m, uint32_t& dim) {
    const Cx zero = cx(0, 0), one = cx(1, 0), neg_one = cx(-1, 0), I = cx(0, 1), neg_i = cx(0, -1);
    dim = 2;
    m.assign(4, zero);
    switch (type) {
    case YAO_GATE_X: m = {zero, one, one, zero}; return 0;
    case YAO_GATE_Y: m = {zero, neg_i, I, zero}; return 0;
    case YAO_GATE_Z: m = {one, zero, zero, neg_one}; return 0;
    case YAO_GATE_H: {
        Cx s = cx(kFrac1Sqrt2, 0), ns = cx(-kFrac1Sqrt2, 0);
        m = {s, s, s, ns};
        return 0;
    }
    case YAO_GATE_S: m = {one, zero, zero, I}; return 0;
    case YAO_GATE_T: m = {one, zero, zero, from_polar(1.0, kFracPi4)}; return 0;
    case YAO_GATE_SWAP:
        dim = 4;
        m.assign(16, zero);
        m[0] = one; m[1 * 4 + 2] = one; m[2 * 4 + 1] = one; m[15] = one;
        return 0;
    case YAO_GATE_PHASE: m = {one, zero, zero, from_polar(1.0, p[0])}; return 0;
    case YAO_GATE_RX: {
        double t = p[0];
        Cx c = cx(std::cos(t / 2.0), 0), nis = cx(0, -std::sin(t / 2.0));
        m = {c, nis, nis, c};
        return 0;
    }
    case YAO_GATE_RY: {
        double t = p[0];
        Cx c = cx(std::cos(t / 2.0), 0), s = cx(std::sin(t / 2.0), 0), ns = cx(-std::sin(t / 2.0), 0);
        m = {c, ns, s, c};
        return 0;
    }
    case YAO_GATE_RZ: {
        double t = p[0];
        m = {from_polar(1.0, -t / 2.0), zero, zero, from_polar(1.0, t / 2.0)};
        return 0;
    }
    case YAO_GATE_SQRTX: {
        Cx f = cx(0.5, 0.5);
        m = {cmul(f, one), cmul(f, neg_i), cmul(f, neg_i), cmul(f, one)};
        return 0;
    }
    case YAO_GATE_SQRTY: {
        Cx f = cx(0.5, 0.5);
        m = {cmul(f, one), cmul(f, neg_one), cmul(f, one), cmul(f, one)};
        return 0;
    }
    case YAO_GATE_SQRTW: {
        Cx cv = cx(kFrac1Sqrt2, 0), nis = cx(0, -kFrac1Sqrt2);
        Cx g01 = cx(kFrac1Sqrt2, -kFrac1Sqrt2), g10 = cx(kFrac1Sqrt2, kFrac1Sqrt2);
        m = {cv, cmul(nis, g01), cmul(nis, g10), cv};
        return 0;
    }
    case YAO_GATE_ISWAP:
        dim = 4;
        m.assign(16, zero);
        m[0] = one; m[1 * 4 + 2] = I; m[2 * 4 + 1] = I; m[15] = one;
        return 0;
    case YAO_GATE_FSIM: {
        dim = 4;
        double th = p[0], ph = p[1];
        Cx ct = cx(std::cos(th), 0), nist = cx(0, -std::sin(th));
        m.assign(16, zero);
        m[0] = one; m[5] = ct; m[6] = nist; m[9] = nist; m[10] = ct; m[15] = from_polar(1.0, -ph);
        return 0;
    }
    default:
        return -1;
    }
}

// src/gate.rs:98-104
bool named_gate_is_diagonal(int32_t t) {
    return t == YAO_GATE_Z || t == YAO_GATE_S || t == YAO_GATE_T || t == YAO_GATE_PHASE || t == YAO_GATE_RZ;
}

// src/gate.rs:107-113
int gate_num_params(int32_t t) {
    switch (t) {
    case YAO_GATE_RX: case YAO_GATE_RY: case YAO_GATE_RZ: case YAO_GATE_PHASE: return 1;
    case YAO_GATE_FSIM: return 2;
    default: return 0;
    }
}

// src/gate.rs:63-68 (matrix) + :98-104 (is_diagonal)
void gate_matrix(const GateElem& g, std::vector<Cx>& m, uint32_t& dim, bool& diag) {
    if (g.type == YAO_GATE_CUSTOM) {
        m = g.custom;
        dim = g.custom_dim;
        diag = g.custom_diag;
        return;
    }
    named_gate_matrix(g.type, g.params, m, dim);
    diag = named_gate_is_diagonal(g.type);
}

// src/gate.rs:198-281 (dagger)
GateElem gate_dagger(const GateElem& g) {
    GateElem d = g;
    switch (g.type) {
    case YAO_GATE_H: case YAO_GATE_X: case YAO_GATE_Y: case YAO_GATE_Z: case YAO_GATE_SWAP:
        return d;
    case YAO_GATE_S: d.type = YAO_GATE_PHASE; d.params[0] = -kFracPi2; return d;
    case YAO_GATE_T: d.type = YAO_GATE_PHASE; d.params[0] = -kFracPi4; return d;
    case YAO_GATE_RX: case YAO_GATE_RY: case YAO_GATE_RZ: case YAO_GATE_PHASE:
        d.params[0] = -g.params[0];
        return d;
    case YAO_GATE_FSIM:
        d.params[0] = -g.params[0];
        d.params[1] = -g.params[1];
        return d;
    default: {
        // SqrtX, SqrtY, SqrtW, ISWAP and Custom: conjugate transpose as Custom
        std::vector<Cx> m;
        uint32_t dim;
        bool diag;
        gate_matrix(g, m, dim, diag);
        d.type = YAO_GATE_CUSTOM;
        d.custom.assign((size_t)dim * dim, Cx{0, 0});
        for (uint32_t r = 0; r < dim; r++)
            for (uint32_t c = 0; c < dim; c++) d.custom[(size_t)c * dim + r] = cconj(m[(size_t)r * dim + c]);
        d.custom_dim = dim;
        d.custom_diag = (g.type == YAO_GATE_CUSTOM) ? g.custom_diag : false;
        return d;
    }
    }
}

// src/gate.rs:153-193 (generator_matrix)
void gate_generator(const GateElem& g, int i, std::vector<Cx>& m, uint32_t& dim) {
    const Cx z = cx(0, 0);
    dim = 2;
    switch (g.type) {
    case YAO_GATE_RX: m = {z, cx(0, -0.5), cx(0, -0.5), z}; return;
    case YAO_GATE_RY: m = {z, cx(-0.5, 0), cx(0.5, 0), z}; return;
    case YAO_GATE_RZ: m = {cx(0, -0.5), z, z, cx(0, 0.5)}; return;
    case YAO_GATE_PHASE: m = {z, z, z, cx(0, 1)}; return;
    case YAO_GATE_FSIM:
        dim = 4;
        m.assign(16, z);
        if (i == 0) {
            m[1 * 4 + 2] = cx(0, -1);
            m[2 * 4 + 1] = cx(0, -1);
        } else {
            m[15] = cx(0, -1);
        }
        return;
    default:
        m.clear();
        dim = 0;
        return;
    }
}

// src/density_matrix.rs:123-129 (is_diagonal_matrix: off-diagonal norm < 1e-15)
bool matrix_is_diagonal(const Cx* m, uint32_t d) {
    for (uint32_t r = 0; r < d; r++)
        for (uint32_t c = 0; c < d; c++)
            if (r != c && !(std::hypot(m[r * d + c].re, m[r * d + c].im) < 1e-15)) return false;
    return true;
}

// ------------------------------------------------------------- noise.rs

static void push2(std::vector<Cx>& out, Cx a, Cx b, Cx c, Cx d) {
    out.push_back(a);
    out.push_back(b);
    out.push_back(c);
    out.push_back(d);
}

// src/noise.rs:383-458 (phase_amplitude_damping_kraus)
static uint32_t pad_kraus(double a, double b, double p1, std::vector<Cx>& out) {
    const Cx z = cx(0, 0);
    uint32_t n = 0;
    double rest = std::sqrt(1.0 - a - b);
    if (std::fabs(p1 - 1.0) > DBL_EPSILON) {
        double s = std::sqrt(1.0 - p1);
        push2(out, cx(s, 0), z, z, cx(s * rest, 0)), n++;
        if (a > 0.0) push2(out, z, cx(std::sqrt(a) * s, 0), z, z), n++;
        if (b > 0.0) push2(out, z, z, z, cx(std::sqrt(b) * s, 0)), n++;
    }
    if (std::fabs(p1) > DBL_EPSILON) {
        double s = std::sqrt(p1);
        push2(out, cx(s * rest, 0), z, z, cx(s, 0)), n++;
        if (a > 0.0) push2(out, z, z, cx(std::sqrt(a) * s, 0), z), n++;
        if (b > 0.0) push2(out, cx(std::sqrt(b) * s, 0), z, z, z), n++;
    }
    return n;
}

static uint32_t pauli_kraus(double px, double py, double pz, std::vector<Cx>& out) {
    const Cx z = cx(0, 0);
    double s0 = std::sqrt(1.0 - px - py - pz), sx = std::sqrt(px), sy = std::sqrt(py), sz = std::sqrt(pz);
    push2(out, cx(s0, 0), z, z, cx(s0, 0));
    push2(out, z, cx(sx, 0), cx(sx, 0), z);
    push2(out, z, cx(0, -sy), cx(0, sy), z);
    push2(out, cx(sz, 0), z, z, cx(-sz, 0));
    return 4;
}

static bool in01(double v) { return v >= 0.0 && v <= 1.0; }

// src/noise.rs:90-176 (validate_params); message mirrors the panics there
static int validate_channel(const ChannelElem& c) {
    const double* p = c.params;
    char buf[256];
    switch (c.type) {
    case YAO_NOISE_BIT_FLIP: case YAO_NOISE_PHASE_FLIP: case YAO_NOISE_DEPOLARIZING:
        if (!in01(p[0])) {
            snprintf(buf, sizeof buf, "probability p=%g must be in [0, 1]", p[0]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        return 0;
    case YAO_NOISE_PAULI_CHANNEL:
        if (!(p[0] >= 0.0 && p[1] >= 0.0 && p[2] >= 0.0 && p[0] + p[1] + p[2] <= 1.0)) {
            snprintf(buf, sizeof buf, "Pauli probabilities (px=%g, py=%g, pz=%g) must be non-negative and sum <= 1",
                     p[0], p[1], p[2]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        return 0;
    case YAO_NOISE_RESET:
        if (!(p[0] >= 0.0 && p[1] >= 0.0 && p[0] + p[1] <= 1.0)) {
            snprintf(buf, sizeof buf, "Reset probabilities (p0=%g, p1=%g) must be non-negative and sum <= 1", p[0],
                     p[1]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        return 0;
    case YAO_NOISE_PHASE_AMPLITUDE_DAMPING:
        if (!(p[0] >= 0.0 && p[1] >= 0.0 && p[0] + p[1] <= 1.0)) {
            snprintf(buf, sizeof buf, "amplitude=%g and phase=%g must be non-negative and sum <= 1", p[0], p[1]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        if (!in01(p[2])) {
            snprintf(buf, sizeof buf, "excited_population=%g must be in [0, 1]", p[2]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        return 0;
    case YAO_NOISE_AMPLITUDE_DAMPING:
        if (!in01(p[0])) {
            snprintf(buf, sizeof buf, "gamma=%g must be in [0, 1]", p[0]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        if (!in01(p[1])) {
            snprintf(buf, sizeof buf, "excited_population=%g must be in [0, 1]", p[1]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        return 0;
    case YAO_NOISE_PHASE_DAMPING:
        if (!in01(p[0])) {
            snprintf(buf, sizeof buf, "gamma=%g must be in [0, 1]", p[0]);
            return fail(YAO_ERR_NOISE_PARAM, buf);
        }
        return 0;
    case YAO_NOISE_THERMAL_RELAXATION:
        if (!(p[0] > 0.0)) return fail(YAO_ERR_NOISE_PARAM, "t1 must be positive");
        if (!(p[1] > 0.0)) return fail(YAO_ERR_NOISE_PARAM, "t2 must be positive");
        if (!(p[2] >= 0.0)) return fail(YAO_ERR_NOISE_PARAM, "time must be non-negative");
        if (!(p[1] <= 2.0 * p[0])) return fail(YAO_ERR_NOISE_PARAM, "t2 must be <= 2*t1 (physics constraint)");
        if (!in01(p[3])) return fail(YAO_ERR_NOISE_PARAM, "excited_population must be in [0, 1]");
        return 0;
    case YAO_NOISE_CUSTOM:
        if (c.nkraus < 1) return fail(YAO_ERR_NOISE_PARAM, "Custom channel must have at least one Kraus operator");
        return 0;
    case YAO_NOISE_COHERENT:
        return 0;
    default:
        return fail(YAO_ERR_INVALID_ARGUMENT, "unknown noise channel type");
    }
}

// src/noise.rs:462-525 (depolarizing_multi_qubit_kraus + kron)
static void depolarizing_multi(uint32_t n, double p, std::vector<Cx>& out) {
    const Cx z = cx(0, 0);
    Cx paulis[4][4] = {{cx(1, 0), z, z, cx(1, 0)},
                       {z, cx(1, 0), cx(1, 0), z},
                       {z, cx(0, -1), cx(0, 1), z},
                       {cx(1, 0), z, z, cx(-1, 0)}};
    uint32_t cnt = 1u << (2 * n);
    for (uint32_t idx = 0; idx < cnt; idx++) {
        std::vector<Cx> mat(1, cx(1, 0));
        uint32_t md = 1;
        uint32_t t = idx;
        for (uint32_t q = 0; q < n; q++) {
            uint32_t pi = t % 4;
            t /= 4;
            uint32_t od = md * 2;
            std::vector<Cx> k((size_t)od * od);
            for (uint32_t i = 0; i < md; i++)
                for (uint32_t j = 0; j < md; j++)
                    for (uint32_t a = 0; a < 2; a++)
                        for (uint32_t b = 0; b < 2; b++)
                            k[(size_t)(i * 2 + a) * od + j * 2 + b] = cmul(mat[(size_t)i * md + j], paulis[pi][a * 2 + b]);
            mat.swap(k);
            md = od;
        }
        double weight = (idx == 0) ? (1.0 - p + p / (double)cnt) : p / (double)cnt;
        double s = std::sqrt(weight);
        for (auto& v : mat) out.push_back(cmul(v, cx(s, 0)));
    }
}

// src/noise.rs:183-352 (kraus_operators)
int channel_kraus(const ChannelElem& c, std::vector<Cx>& out, uint32_t& nk, uint32_t& dim) {
    int st = validate_channel(c);
    if (st != 0) return st;
    const Cx z = cx(0, 0);
    const double* p = c.params;
    out.clear();
    dim = 2;
    switch (c.type) {
    case YAO_NOISE_PHASE_AMPLITUDE_DAMPING: nk = pad_kraus(p[0], p[1], p[2], out); return 0;
    case YAO_NOISE_AMPLITUDE_DAMPING: nk = pad_kraus(p[0], 0.0, p[1], out); return 0;
    case YAO_NOISE_PHASE_DAMPING: nk = pad_kraus(0.0, p[0], 0.0, out); return 0;
    case YAO_NOISE_THERMAL_RELAXATION: {
        double t1 = p[0], t2 = p[1], time = p[2];
        double t_phi = (t1 * t2) / (2.0 * t1 - t2);
        double a = 1.0 - std::exp(-time / t1);
        double b = 1.0 - std::exp(-time / t_phi);
        nk = pad_kraus(a, b, p[3], out);
        return 0;
    }
    case YAO_NOISE_BIT_FLIP: {
        double s0 = std::sqrt(1.0 - p[0]), s1 = std::sqrt(p[0]);
        push2(out, cx(s0, 0), z, z, cx(s0, 0));
        push2(out, z, cx(s1, 0), cx(s1, 0), z);
        nk = 2;
        return 0;
    }
    case YAO_NOISE_PHASE_FLIP: {
        double s0 = std::sqrt(1.0 - p[0]), s1 = std::sqrt(p[0]);
        push2(out, cx(s0, 0), z, z, cx(s0, 0));
        push2(out, cx(s1, 0), z, z, cx(-s1, 0));
        nk = 2;
        return 0;
    }
    case YAO_NOISE_PAULI_CHANNEL: nk = pauli_kraus(p[0], p[1], p[2], out); return 0;
    case YAO_NOISE_DEPOLARIZING: {
        uint32_t n = (uint32_t)c.depol_n;
        if (n < 1 || n > 4) return fail(YAO_ERR_UNSUPPORTED, "Depolarizing channel supports 1 to 4 qubits");
        if (n == 1) {
            double q = p[0] / 4.0;
            nk = pauli_kraus(q, q, q, out);
            return 0;
        }
        depolarizing_multi(n, p[0], out);
        nk = 1u << (2 * n);
        dim = 1u << n;
        return 0;
    }
    case YAO_NOISE_RESET: {
        double s = std::sqrt(1.0 - p[0] - p[1]);
        nk = 0;
        push2(out, cx(s, 0), z, z, cx(s, 0)), nk++;
        if (p[0] > 0.0) {
            double sp0 = std::sqrt(p[0]);
            push2(out, cx(sp0, 0), z, z, z), nk++;
            push2(out, z, cx(sp0, 0), z, z), nk++;
        }
        if (p[1] > 0.0) {
            double sp1 = std::sqrt(p[1]);
            push2(out, z, z, z, cx(sp1, 0)), nk++;
            push2(out, z, z, cx(sp1, 0), z), nk++;
        }
        return 0;
    }
    case YAO_NOISE_COHERENT:
        out = c.mats;
        nk = 1;
        dim = c.dim;
        return 0;
    case YAO_NOISE_CUSTOM:
        out = c.mats;
        nk = c.nkraus;
        dim = c.dim;
        return 0;
    default:
        return fail(YAO_ERR_INVALID_ARGUMENT, "unknown noise channel type");
    }
}

// ------------------------------------------------------------- lowering

// Fill tb/matrix of an LGate from a matrix placed at `targets`, following the
// branch dispatch_arrayreg_gate takes for a gate that is not a named X/SWAP:
// diagonal 1q/2q, dense 1q, dense 2q (sort_unitary_2q, src/instruct_qubit.rs:
// 215-231), and instruct_nq for more targets (local bit i <-> targets[i]).
static void fill_matrix_gate(LGate& g, const std::vector<Cx>& m, uint32_t dim, bool diag,
                             const std::vector<int32_t>& bits) {
    int k = (int)bits.size();
    g.k = k;
    if (k == 2) {
        int b0 = bits[0], b1 = bits[1];
        bool swap = b0 > b1;
        g.tb[0] = std::min(b0, b1);
        g.tb[1] = std::max(b0, b1);
        if (diag) {
            g.cls = GC_DIAG;
            g.m = {m[0], m[5], m[10], m[15]};
            if (swap) std::swap(g.m[1], g.m[2]);
        } else {
            g.cls = GC_DENSE;
            if (!swap) {
                g.m = m;
            } else {
                static const int perm[4] = {0, 2, 1, 3};
                g.m.assign(16, Cx{0, 0});
                for (int i = 0; i < 4; i++)
                    for (int j = 0; j < 4; j++) g.m[perm[i] * 4 + perm[j]] = m[i * 4 + j];
            }
        }
        return;
    }
    for (int i = 0; i < k; i++) g.tb[i] = bits[i];
    if (diag) {
        // 1 target: instruct_1q_diag.  >=3 targets: instruct_nq multiplies by the
        // diagonal entry plus exact zeros, which gives the same values.
        g.cls = GC_DIAG;
        g.m.resize(dim);
        for (uint32_t i = 0; i < dim; i++) g.m[i] = m[(size_t)i * dim + i];
    } else {
        g.cls = GC_DENSE;
        g.m = m;
    }
}

static void fill_controls(LGate& g, const std::vector<uint32_t>& ctrls, const std::vector<uint8_t>& cfgs,
                          uint32_t nbits, uint32_t shift) {
    g.nc = (int)ctrls.size();
    for (size_t i = 0; i < ctrls.size(); i++) {
        g.cb[i] = (int)(nbits - 1 - (ctrls[i] + shift));
        g.cv[i] = cfgs.empty() ? 1 : (cfgs[i] ? 1 : 0);
    }
}

LGate lower_matrix(const std::vector<Cx>& m, uint32_t dim, bool diag, const std::vector<uint32_t>& targets,
                   const std::vector<uint32_t>& ctrls, const std::vector<uint8_t>& cfgs, uint32_t nbits,
                   uint32_t shift) {
    LGate g;
    std::vector<int32_t> bits;
    for (uint32_t t : targets) bits.push_back((int32_t)(nbits - 1 - (t + shift)));
    fill_matrix_gate(g, m, dim, diag, bits);
    fill_controls(g, ctrls, cfgs, nbits, shift);
    return g;
}

// src/apply.rs:7-120 (dispatch_arrayreg_gate), plus the conjugated and
// shifted copy used for the column index of a density matrix
// (src/density_matrix.rs:131-178).
void lower_gate(const GateElem& ge, uint32_t nbits, uint32_t shift, bool conj, std::vector<LGate>& out) {
    auto bit = [&](uint32_t loc) { return (int32_t)(nbits - 1 - (loc + shift)); };
    if (ge.type == YAO_GATE_X) {
        // instruct_x / instruct_x_controlled on every target; conj(X) = X moves
        // the same amplitudes.
        for (uint32_t t : ge.targets) {
            LGate g;
            g.cls = GC_X;
            g.k = 1;
            g.tb[0] = bit(t);
            fill_controls(g, ge.ctrls, ge.cfgs, nbits, shift);
            out.push_back(g);
        }
        return;
    }
    if (ge.type == YAO_GATE_SWAP) {
        // instruct_swap; with controls yao-rs multiplies by the SWAP matrix,
        // whose entries are exact 0/1, so the moved values are identical.
        LGate g;
        g.cls = GC_SWAP;
        g.k = 2;
        int32_t b0 = bit(ge.targets[0]), b1 = bit(ge.targets[1]);
        g.tb[0] = std::min(b0, b1);
        g.tb[1] = std::max(b0, b1);
        fill_controls(g, ge.ctrls, ge.cfgs, nbits, shift);
        out.push_back(g);
        return;
    }
    std::vector<Cx> m;
    uint32_t dim;
    bool diag;
    gate_matrix(ge, m, dim, diag);
    if (conj)
        for (auto& v : m) v = cconj(v);
    out.push_back(lower_matrix(m, dim, diag, ge.targets, ge.ctrls, ge.cfgs, nbits, shift));
}

}  // namespace yao

namespace yao {

// NoiseChannel::superop (src/noise.rs:359-379): S = sum_K kron(conj(K), K),
// S[(i d + kr), (j d + kc)] += conj(K[i][j]) K[kr][kc], in that loop order.
int channel_superop(const ChannelElem& c, std::vector<Cx>& S, uint32_t& d2) {
    std::vector<Cx> k;
    uint32_t nk, d;
    const int s = channel_kraus(c, k, nk, d);
    if (s) return s;
    d2 = d * d;
    S.assign((size_t)d2 * d2, Cx{0, 0});
    for (uint32_t q = 0; q < nk; q++) {
        const Cx* K = k.data() + (size_t)q * d * d;
        for (uint32_t i = 0; i < d; i++)
            for (uint32_t j = 0; j < d; j++)
                for (uint32_t kr = 0; kr < d; kr++)
                    for (uint32_t kc = 0; kc < d; kc++) {
                        const Cx a{K[i * d + j].re, -K[i * d + j].im}, b = K[kr * d + kc];
                        Cx& t = S[(size_t)(i * d + kr) * d2 + j * d + kc];
                        t.re += a.re * b.re - a.im * b.im;
                        t.im += a.re * b.im + a.im * b.re;
                    }
    }
    return YAO_OK;
}

}  // namespace yao
