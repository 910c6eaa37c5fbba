// tn.cu — tensor networks of circuits and their contraction on the GPU.
//
// The network builders restate yao-rs's einsum export (src/einsum.rs:34-761,
// tensors from src/tensors.rs:26-153): the same labels, leg order, tensor
// data and size dictionary, so a network built here is the one yao-rs
// builds.  yao-rs contracts such a network with omeinsum on the CPU
// (src/contractor.rs) or pairwise with libtorch einsum after omeco's greedy
// order (src/torch_contractor.rs:33-95).  Here the contraction runs on the
// device: a greedy pairwise order on the host (cheapest result first), and
// each pair contracted by one kernel over offset tables (batch, free and
// summed label groups of any order and any leg dimensions), complex128 with
// FMA, deterministic summation order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <tuple>
#include <string>
#include <vector>

#include "device_common.cuh"

namespace yao {

// A tensor network: tensor t has legs ixs[t] (labels; row-major data, the
// first leg slowest), iy the output labels, size[label] the leg dimension.
struct TNet {
    std::vector<std::vector<int64_t>> ixs;
    std::vector<std::vector<Cx>> tensors;
    std::vector<int64_t> iy;
    std::map<int64_t, uint32_t> size;
};

namespace {

Cx conj_c(Cx a) { return Cx{a.re, -a.im}; }

// gate_to_tensor (src/tensors.rs:26-80) with build_controlled_matrix
// (:82-138) and compute_trigger_index (:140-150).  `diag_legs`: the gate is
// diagonal and has no controls (one leg per target, the diagonal entries);
// else legs are (all_locs out..., all_locs in...) with all_locs = controls
// then targets.
int gate_tensor(const GateElem& g, const std::vector<uint32_t>& dims, std::vector<Cx>& data, bool& diag_legs) {
    std::vector<Cx> m;
    uint32_t dim = 0;
    bool diag = false;
    gate_matrix(g, m, dim, diag);
    const bool has_ctrl = !g.ctrls.empty();
    diag_legs = diag && !has_ctrl;
    size_t tgt_dim = 1;
    for (uint32_t t : g.targets) tgt_dim *= dims[t];
    if (tgt_dim != dim)
        return fail(YAO_ERR_INVALID_ARGUMENT,
                    "gate_to_tensor: gate matrix dimension does not match its target sites");
    if (diag_legs) {
        data.resize(dim);
        for (uint32_t i = 0; i < dim; i++) data[i] = m[(size_t)i * dim + i];
        return YAO_OK;
    }
    if (!has_ctrl) {
        data = m;
        return YAO_OK;
    }
    std::vector<size_t> cdims;
    size_t ctrl_dim = 1;
    for (uint32_t c : g.ctrls) {
        cdims.push_back(dims[c]);
        ctrl_dim *= dims[c];
    }
    size_t trigger = 0, stride = 1;
    for (size_t i = g.ctrls.size(); i-- > 0;) {
        const bool on = g.cfgs.empty() ? true : g.cfgs[i] != 0;
        trigger += (on ? 1 : 0) * stride;
        stride *= cdims[i];
    }
    const size_t total = ctrl_dim * tgt_dim;
    data.assign(total * total, Cx{0, 0});
    for (size_t ci = 0; ci < ctrl_dim; ci++)
        for (size_t tr = 0; tr < tgt_dim; tr++) {
            const size_t row = ci * tgt_dim + tr;
            if (ci == trigger)
                for (size_t tc = 0; tc < tgt_dim; tc++) data[row * total + ci * tgt_dim + tc] = m[tr * tgt_dim + tc];
            else
                data[row * total + ci * tgt_dim + tr] = Cx{1, 0};
        }
    return YAO_OK;
}

std::vector<uint32_t> all_locs(const GateElem& g) {
    std::vector<uint32_t> a = g.ctrls;
    a.insert(a.end(), g.targets.begin(), g.targets.end());
    return a;
}

std::vector<Cx> basis0(uint32_t d) {
    std::vector<Cx> v(d, Cx{0, 0});
    v[0] = Cx{1, 0};
    return v;
}

// The gates of a circuit appended to a network whose current leg of site i
// is cur[i] (the loop body shared by circuit_to_einsum,
// circuit_to_einsum_with_boundary and circuit_to_expectation).
int add_gates(const Circuit& c, TNet& tn, std::vector<int64_t>& cur, int64_t& next) {
    for (const Element& el : c.elems) {
        if (el.kind != YAO_ELEM_GATE) continue;
        std::vector<Cx> t;
        bool diag = false;
        int s = gate_tensor(el.g, c.dims, t, diag);
        if (s) return s;
        std::vector<int64_t> ix;
        if (diag) {
            for (uint32_t loc : el.g.targets) ix.push_back(cur[loc]);
        } else {
            const std::vector<uint32_t> locs = all_locs(el.g);
            std::vector<int64_t> fresh;
            for (uint32_t loc : locs) {
                tn.size[next] = c.dims[loc];
                fresh.push_back(next++);
            }
            ix = fresh;
            for (uint32_t loc : locs) ix.push_back(cur[loc]);
            for (size_t i = 0; i < locs.size(); i++) cur[locs[i]] = fresh[i];
        }
        tn.ixs.push_back(ix);
        tn.tensors.push_back(std::move(t));
    }
    return YAO_OK;
}

// op_matrix (src/operator.rs:53-65)
std::vector<Cx> op_matrix(int32_t op) {
    const Cx z{0, 0}, o{1, 0};
    switch (op) {
    case YAO_OP_X: return {z, o, o, z};
    case YAO_OP_Y: return {z, Cx{0, -1}, Cx{0, 1}, z};
    case YAO_OP_Z: return {o, z, z, Cx{-1, 0}};
    case YAO_OP_P0: return {o, z, z, z};
    case YAO_OP_P1: return {z, z, z, o};
    case YAO_OP_PU: return {z, o, z, z};
    case YAO_OP_PD: return {z, z, o, z};
    default: return {o, z, z, o};
    }
}

Cx cmul_c(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

// The single term of an operator as OperatorString::new leaves it
// (src/operator.rs:27-33: sorted by site, stable, Op::I dropped).
int single_term(const yao_term* terms, size_t nterms, uint32_t nsites, const char* who, Cx& coeff,
                std::vector<std::pair<uint32_t, int32_t>>& ops) {
    if (nterms != 1)
        return fail(YAO_ERR_INVALID_ARGUMENT, std::string(who) +
                                                  "() only supports single-term OperatorPolynomial, got " +
                                                  std::to_string(nterms) + " terms");
    const yao_term& t = terms[0];
    coeff = Cx{t.coeff_re, t.coeff_im};
    for (uint32_t i = 0; i < t.nops; i++) {
        if (t.sites[i] >= nsites) return fail(YAO_ERR_INVALID_ARGUMENT, "operator site out of range");
        if (t.ops[i] < YAO_OP_I || t.ops[i] > YAO_OP_PD) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown Op");
        if (t.ops[i] != YAO_OP_I) ops.push_back({t.sites[i], t.ops[i]});
    }
    std::stable_sort(ops.begin(), ops.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    return YAO_OK;
}

}  // namespace

// circuit_to_einsum (src/einsum.rs:34-119), circuit_to_einsum_with_boundary
// (:151-252) and circuit_to_overlap (:127-131).
int tn_from_circuit(const Circuit& c, bool boundary, const std::vector<uint32_t>& pinned, TNet& tn) {
    const uint32_t n = (uint32_t)c.dims.size();
    std::vector<int64_t> cur(n);
    for (uint32_t i = 0; i < n; i++) {
        cur[i] = i;
        tn.size[i] = c.dims[i];
    }
    int64_t next = n;
    if (boundary)
        for (uint32_t i = 0; i < n; i++) {
            tn.ixs.push_back({(int64_t)i});
            tn.tensors.push_back(basis0(c.dims[i]));
        }
    int s = add_gates(c, tn, cur, next);
    if (s) return s;
    std::set<uint32_t> pin(pinned.begin(), pinned.end());
    if (boundary)
        for (uint32_t q : pinned) {
            if (q >= n) return fail(YAO_ERR_INVALID_ARGUMENT, "pinned site out of range");
            tn.ixs.push_back({cur[q]});
            tn.tensors.push_back(basis0(c.dims[q]));
        }
    for (uint32_t i = 0; i < n; i++)
        if (!boundary || !pin.count(i)) tn.iy.push_back(cur[i]);
    return YAO_OK;
}

// circuit_to_expectation (src/einsum.rs:274-500): |0> boundaries, U, the
// operator's single term (the coefficient on the first op's matrix; an
// identity string carries none), U^dagger in reverse (conjugated tensors,
// in and out legs exchanged), <0| boundaries; scalar output.
int tn_expectation(const Circuit& c, const yao_term* terms, size_t nterms, TNet& tn) {
    const uint32_t n = (uint32_t)c.dims.size();
    std::vector<int64_t> cur(n);
    for (uint32_t i = 0; i < n; i++) {
        cur[i] = i;
        tn.size[i] = c.dims[i];
    }
    int64_t next = n;
    for (uint32_t i = 0; i < n; i++) {
        tn.ixs.push_back({(int64_t)i});
        tn.tensors.push_back(basis0(c.dims[i]));
    }
    int s = add_gates(c, tn, cur, next);
    if (s) return s;
    if (nterms == 0) {
        tn.ixs.push_back({});
        tn.tensors.push_back({Cx{0, 0}});
    } else {
        Cx coeff;
        std::vector<std::pair<uint32_t, int32_t>> ops;
        if ((s = single_term(terms, nterms, n, "circuit_to_expectation", coeff, ops))) return s;
        std::vector<int32_t> site_op(n, -1);
        for (const auto& o : ops) site_op[o.first] = o.second;
        for (uint32_t i = 0; i < n; i++) {
            std::vector<Cx> m;
            if (site_op[i] >= 0) {
                m = op_matrix(site_op[i]);
                const uint32_t first = ops.empty() ? i : ops[0].first;
                if (i == first)
                    for (Cx& e : m) e = cmul_c(e, coeff);
            } else {
                m = op_matrix(YAO_OP_I);
            }
            const uint32_t d = c.dims[i];
            if (d != 2) return fail(YAO_ERR_INVALID_ARGUMENT, "circuit_to_expectation: operator sites must be qubits");
            tn.size[next] = d;
            tn.ixs.push_back({next, cur[i]});
            tn.tensors.push_back(m);
            cur[i] = next++;
        }
    }
    for (size_t ei = c.elems.size(); ei-- > 0;) {
        const Element& el = c.elems[ei];
        if (el.kind != YAO_ELEM_GATE) continue;
        std::vector<Cx> t;
        bool diag = false;
        if ((s = gate_tensor(el.g, c.dims, t, diag))) return s;
        for (Cx& e : t) e = conj_c(e);
        if (diag) {
            std::vector<int64_t> ix;
            for (uint32_t loc : el.g.targets) ix.push_back(cur[loc]);
            tn.ixs.push_back(ix);
            tn.tensors.push_back(std::move(t));
            continue;
        }
        const std::vector<uint32_t> locs = all_locs(el.g);
        size_t tot = 1;
        for (uint32_t loc : locs) tot *= c.dims[loc];
        std::vector<Cx> tt(tot * tot);
        for (size_t r = 0; r < tot; r++)
            for (size_t q = 0; q < tot; q++) tt[q * tot + r] = t[r * tot + q];  // legs (in..., out...)
        std::vector<int64_t> fresh, ix;
        for (uint32_t loc : locs) {
            tn.size[next] = c.dims[loc];
            fresh.push_back(next++);
        }
        ix = fresh;
        for (uint32_t loc : locs) ix.push_back(cur[loc]);
        for (size_t i = 0; i < locs.size(); i++) cur[locs[i]] = fresh[i];
        tn.ixs.push_back(ix);
        tn.tensors.push_back(std::move(tt));
    }
    for (uint32_t i = 0; i < n; i++) {
        tn.ixs.push_back({cur[i]});
        tn.tensors.push_back(basis0(c.dims[i]));
    }
    return YAO_OK;
}

// circuit_to_einsum_dm (src/einsum.rs:519-665): ket labels 1..n, bra labels
// their negatives; every gate as a ket tensor and a conjugated bra copy,
// every channel as its superoperator with legs (-out, out, -in, in); output
// (ket slots, bra slots).
int tn_dm(const Circuit& c, TNet& tn) {
    const uint32_t n = (uint32_t)c.dims.size();
    std::vector<int64_t> slot(n);
    for (uint32_t i = 0; i < n; i++) {
        slot[i] = (int64_t)i + 1;
        tn.size[slot[i]] = c.dims[i];
        tn.size[-slot[i]] = c.dims[i];
    }
    int64_t next = (int64_t)n + 1;
    for (uint32_t i = 0; i < n; i++) {
        tn.ixs.push_back({slot[i]});
        tn.tensors.push_back(basis0(c.dims[i]));
        tn.ixs.push_back({-slot[i]});
        tn.tensors.push_back(basis0(c.dims[i]));
    }
    for (const Element& el : c.elems) {
        if (el.kind == YAO_ELEM_GATE) {
            std::vector<Cx> t;
            bool diag = false;
            int s = gate_tensor(el.g, c.dims, t, diag);
            if (s) return s;
            std::vector<Cx> tc = t;
            for (Cx& e : tc) e = conj_c(e);
            if (diag) {
                std::vector<int64_t> ket, bra;
                for (uint32_t loc : el.g.targets) {
                    ket.push_back(slot[loc]);
                    bra.push_back(-slot[loc]);
                }
                tn.ixs.push_back(ket);
                tn.tensors.push_back(std::move(t));
                tn.ixs.push_back(bra);
                tn.tensors.push_back(std::move(tc));
            } else {
                const std::vector<uint32_t> locs = all_locs(el.g);
                std::vector<int64_t> fresh;
                for (uint32_t loc : locs) {
                    tn.size[next] = c.dims[loc];
                    tn.size[-next] = c.dims[loc];
                    fresh.push_back(next++);
                }
                std::vector<int64_t> ket = fresh, bra;
                for (int64_t l : fresh) bra.push_back(-l);
                for (uint32_t loc : locs) {
                    ket.push_back(slot[loc]);
                    bra.push_back(-slot[loc]);
                }
                tn.ixs.push_back(ket);
                tn.tensors.push_back(std::move(t));
                tn.ixs.push_back(bra);
                tn.tensors.push_back(std::move(tc));
                for (size_t i = 0; i < locs.size(); i++) slot[locs[i]] = fresh[i];
            }
        } else if (el.kind == YAO_ELEM_CHANNEL) {
            std::vector<Cx> S;
            uint32_t d2 = 0;
            int s = channel_superop(el.ch, S, d2);
            if (s) return s;
            const std::vector<uint32_t>& locs = el.ch.locs;
            size_t want = 1;
            for (uint32_t loc : locs) want *= (size_t)c.dims[loc] * c.dims[loc];
            if (want != d2) return fail(YAO_ERR_INVALID_ARGUMENT, "channel dimension does not match its sites");
            std::vector<int64_t> fresh;
            for (uint32_t loc : locs) {
                tn.size[next] = c.dims[loc];
                tn.size[-next] = c.dims[loc];
                fresh.push_back(next++);
            }
            std::vector<int64_t> ix;
            for (int64_t l : fresh) ix.push_back(-l);
            for (int64_t l : fresh) ix.push_back(l);
            for (uint32_t loc : locs) ix.push_back(-slot[loc]);
            for (uint32_t loc : locs) ix.push_back(slot[loc]);
            tn.ixs.push_back(ix);
            tn.tensors.push_back(std::move(S));
            for (size_t i = 0; i < locs.size(); i++) slot[locs[i]] = fresh[i];
        }
    }
    for (uint32_t i = 0; i < n; i++) tn.iy.push_back(slot[i]);
    for (uint32_t i = 0; i < n; i++) tn.iy.push_back(-slot[i]);
    return YAO_OK;
}

// circuit_to_expectation_dm (src/einsum.rs:673-761): the DM network with the
// operator's single term on the ket side, each site's matrix (the
// coefficient on site 0's, operator or identity) with legs (bra, ket);
// scalar output (the trace).
int tn_expectation_dm(const Circuit& c, const yao_term* terms, size_t nterms, TNet& tn) {
    int s = tn_dm(c, tn);
    if (s) return s;
    const uint32_t n = (uint32_t)c.dims.size();
    std::vector<int64_t> ket(tn.iy.begin(), tn.iy.begin() + n), bra(tn.iy.begin() + n, tn.iy.end());
    tn.iy.clear();
    if (nterms == 0) {
        tn.ixs.push_back({});
        tn.tensors.push_back({Cx{0, 0}});
        return YAO_OK;
    }
    Cx coeff;
    std::vector<std::pair<uint32_t, int32_t>> ops;
    if ((s = single_term(terms, nterms, n, "circuit_to_expectation_dm", coeff, ops))) return s;
    std::vector<int32_t> site_op(n, -1);
    for (const auto& o : ops) site_op[o.first] = o.second;
    bool first = true;
    for (uint32_t i = 0; i < n; i++) {
        std::vector<Cx> m = op_matrix(site_op[i] >= 0 ? site_op[i] : YAO_OP_I);
        if (first) {
            for (Cx& e : m) e = cmul_c(e, coeff);
            first = false;
        }
        if (c.dims[i] != 2)
            return fail(YAO_ERR_INVALID_ARGUMENT, "circuit_to_expectation_dm: operator sites must be qubits");
        tn.ixs.push_back({bra[i], ket[i]});
        tn.tensors.push_back(m);
    }
    return YAO_OK;
}

// Checks a network: every label has a size, a tensor's data length is the
// product of its legs' sizes, no label twice on one tensor, output labels
// distinct.
int tn_validate(const TNet& tn) {
    if (tn.ixs.size() != tn.tensors.size()) return fail(YAO_ERR_INVALID_ARGUMENT, "tensor count mismatch");
    for (size_t t = 0; t < tn.ixs.size(); t++) {
        size_t len = 1;
        std::set<int64_t> seen;
        for (int64_t l : tn.ixs[t]) {
            auto it = tn.size.find(l);
            if (it == tn.size.end() || it->second == 0)
                return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: a label has no size");
            if (!seen.insert(l).second)
                return fail(YAO_ERR_UNSUPPORTED, "tensor network: a label appears twice on one tensor");
            len *= it->second;
        }
        if (len != tn.tensors[t].size())
            return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: tensor data length does not match its legs");
    }
    std::set<int64_t> out, used;
    for (const auto& ix : tn.ixs) used.insert(ix.begin(), ix.end());
    for (int64_t l : tn.iy) {
        if (!tn.size.count(l)) return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: an output label has no size");
        if (!out.insert(l).second) return fail(YAO_ERR_UNSUPPORTED, "tensor network: an output label appears twice");
        if (!used.count(l)) return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: an output label is on no tensor");
    }
    return YAO_OK;
}

// ------------------------------------------------------------- contraction
//
// One pairwise contraction C = sum_K A * B.  The labels of A and B fall
// into four groups: batch (in A, B and C), M (in A and C), N (in B and C)
// and K (summed: in A and / or B, not kept).  For every group a table maps
// its row-major multi-index to the element offset in A, B and C, so
//   C[cg + cm + cn] = sum_k A[ag + am + ak] * B[bg + bn + bk]
// for any leg order and leg dimensions.  C's legs are (batch, M, N).  One
// thread per output element while K is short; one warp per output element
// (lanes stride K, shuffle sum in fixed order) when K is long.

__global__ void k_tn_pair(const double2* __restrict__ A, const double2* __restrict__ B, double2* __restrict__ C,
                          const int64_t* __restrict__ tg, const int64_t* __restrict__ tm,
                          const int64_t* __restrict__ tn, const int64_t* __restrict__ tk, int64_t G, int64_t M,
                          int64_t N, int64_t K) {
    // tables: tg[3 * g] = {A, B, C} offsets, tm[2 * m] = {A, C}, tn[2 * n] =
    // {B, C}, tk[2 * k] = {A, B}
    const int64_t total = G * M * N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = i % N, q = i / N, m = q % M, g = q / M;
        const int64_t a0 = tg[3 * g] + tm[2 * m], b0 = tg[3 * g + 1] + tn[2 * n];
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t k = 0; k < K; k++) {
            const double2 a = A[a0 + tk[2 * k]], b = B[b0 + tk[2 * k + 1]];
            acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
            acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
        }
        C[tg[3 * g + 2] + tm[2 * m + 1] + tn[2 * n + 1]] = acc;
    }
}

__global__ void k_tn_pair_warp(const double2* __restrict__ A, const double2* __restrict__ B, double2* __restrict__ C,
                               const int64_t* __restrict__ tg, const int64_t* __restrict__ tm,
                               const int64_t* __restrict__ tn, const int64_t* __restrict__ tk, int64_t G, int64_t M,
                               int64_t N, int64_t K) {
    const int64_t total = G * M * N;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const int64_t n = i % N, q = i / N, m = q % M, g = q / M;
        const int64_t a0 = tg[3 * g] + tm[2 * m], b0 = tg[3 * g + 1] + tn[2 * n];
        double re = 0.0, im = 0.0;
        for (int64_t k = lane; k < K; k += 32) {
            const double2 a = A[a0 + tk[2 * k]], b = B[b0 + tk[2 * k + 1]];
            re = fma(a.x, b.x, fma(-a.y, b.y, re));
            im = fma(a.x, b.y, fma(a.y, b.x, im));
        }
        re = warp_sum(re);
        im = warp_sum(im);
        if (lane == 0) C[tg[3 * g + 2] + tm[2 * m + 1] + tn[2 * n + 1]] = make_double2(re, im);
    }
}

namespace {

struct DevTensor {
    std::vector<int64_t> legs;
    double2* d = nullptr;
    size_t len = 1;
};

// Row-major strides of a tensor's legs.
std::map<int64_t, int64_t> strides_of(const std::vector<int64_t>& legs, const std::map<int64_t, uint32_t>& size) {
    std::map<int64_t, int64_t> s;
    int64_t st = 1;
    for (size_t i = legs.size(); i-- > 0;) {
        s[legs[i]] = st;
        st *= size.at(legs[i]);
    }
    return s;
}

// Offset table of a label group: entry v (row-major over `grp`) holds, per
// tensor in `who`, sum_i digit_i * stride_i (0 where the tensor lacks it).
// Built as an odometer: each step adds the strides of the digits it moves.
std::vector<int64_t> group_table(const std::vector<int64_t>& grp, const std::map<int64_t, uint32_t>& size,
                                 const std::vector<const std::map<int64_t, int64_t>*>& who) {
    const size_t ng = grp.size(), w = who.size();
    size_t cnt = 1;
    std::vector<uint32_t> dim(ng);
    std::vector<int64_t> st(ng * w, 0);  // stride of leg i in tensor j
    for (size_t i = 0; i < ng; i++) {
        dim[i] = size.at(grp[i]);
        cnt *= dim[i];
        for (size_t j = 0; j < w; j++) {
            auto it = who[j]->find(grp[i]);
            if (it != who[j]->end()) st[i * w + j] = it->second;
        }
    }
    std::vector<int64_t> t(cnt * w, 0);
    std::vector<uint32_t> dig(ng, 0);
    std::vector<int64_t> cur(w, 0);
    for (size_t v = 0; v < cnt; v++) {
        for (size_t j = 0; j < w; j++) t[v * w + j] = cur[j];
        for (size_t i = ng; i-- > 0;) {  // row-major increment
            if (++dig[i] < dim[i]) {
                for (size_t j = 0; j < w; j++) cur[j] += st[i * w + j];
                break;
            }
            for (size_t j = 0; j < w; j++) cur[j] -= (int64_t)(dim[i] - 1) * st[i * w + j];
            dig[i] = 0;
        }
    }
    return t;
}

double log2_size(const std::vector<int64_t>& legs, const std::map<int64_t, uint32_t>& size) {
    double s = 0.0;
    for (int64_t l : legs) s += std::log2((double)size.at(l));
    return s;
}

}  // namespace

// C = A * B summed over every label of A or B not in `keep`.  C's legs:
// batch, then A's kept-only legs, then B's kept-only legs; or, with
// `order` (B a scalar), exactly `order`.  C's data and the offset tables
// share one stream-ordered allocation (C first), freed with C.
static int contract_pair(Ctx* ctx, const DevTensor& A, const DevTensor& B, const std::set<int64_t>& keep,
                         const std::map<int64_t, uint32_t>& size, DevTensor& Cout, const std::vector<int64_t>* order) {
    std::set<int64_t> inA(A.legs.begin(), A.legs.end()), inB(B.legs.begin(), B.legs.end());
    std::vector<int64_t> g, m, n, k;
    for (int64_t l : A.legs) {
        if (!keep.count(l))
            k.push_back(l);
        else if (inB.count(l))
            g.push_back(l);
        else
            m.push_back(l);
    }
    for (int64_t l : B.legs) {
        if (!keep.count(l)) {
            if (!inA.count(l)) k.push_back(l);
        } else if (!inA.count(l)) {
            n.push_back(l);
        }
    }
    if (order) {
        m = *order;
        g.clear();
        n.clear();
    }
    std::vector<int64_t> cl = g;
    cl.insert(cl.end(), m.begin(), m.end());
    cl.insert(cl.end(), n.begin(), n.end());
    const auto sa = strides_of(A.legs, size), sb = strides_of(B.legs, size), sc = strides_of(cl, size);
    const std::vector<int64_t> tg = group_table(g, size, {&sa, &sb, &sc}), tm = group_table(m, size, {&sa, &sc}),
                               tn = group_table(n, size, {&sb, &sc}), tk = group_table(k, size, {&sa, &sb});
    const int64_t G = (int64_t)(tg.size() / 3), M = (int64_t)(tm.size() / 2), N = (int64_t)(tn.size() / 2),
                  K = (int64_t)(tk.size() / 2);
    size_t clen = 1;
    for (int64_t l : cl) clen *= size.at(l);
    const size_t cbytes = (clen * sizeof(double2) + 255) / 256 * 256;
    const size_t tbytes = (tg.size() + tm.size() + tn.size() + tk.size()) * sizeof(int64_t);
    char* buf = nullptr;
    YAO_CUDA(cudaMallocAsync((void**)&buf, cbytes + tbytes, ctx->stream));
    double2* dc = (double2*)buf;
    int64_t* dtg = (int64_t*)(buf + cbytes);
    int64_t* dtm = dtg + tg.size();
    int64_t* dtn = dtm + tm.size();
    int64_t* dtk = dtn + tn.size();
    YAO_CUDA(cudaMemcpyAsync(dtg, tg.data(), tg.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dtm, tm.data(), tm.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dtn, tn.data(), tn.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dtk, tk.data(), tk.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    const int64_t total = G * M * N;
    {
        ProfScope prof(ctx, "tn_pair", (double)(A.len + B.len + clen) * sizeof(double2));
        if (K >= 64) {
            const int64_t blocks = std::min<int64_t>((total + 7) / 8, (int64_t)ctx->num_sms * 16);
            k_tn_pair_warp<<<(unsigned)std::max<int64_t>(1, blocks), 256, 0, ctx->stream>>>(A.d, B.d, dc, dtg, dtm,
                                                                                             dtn, dtk, G, M, N, K);
        } else {
            k_tn_pair<<<grid_for((uint64_t)total, 256, ctx->num_sms, 16), 256, 0, ctx->stream>>>(A.d, B.d, dc, dtg, dtm,
                                                                                                  dtn, dtk, G, M, N, K);
        }
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    Cout.legs = cl;
    Cout.len = clen;
    Cout.d = dc;
    return YAO_OK;
}

// Checks an explicit contraction order over T tensors: T - 1 pairs (none
// for T <= 1), pair s naming two distinct tensors among the network's
// 0..T-1 and the results T..T+s-1 of the pairs before it, each used once.
static int path_validate(size_t T, const uint32_t* path, size_t npairs) {
    if (npairs != (T > 0 ? T - 1 : 0))
        return fail(YAO_ERR_INVALID_ARGUMENT, "contraction path: a network of T tensors takes exactly T - 1 pairs");
    if (npairs && !path) return fail(YAO_ERR_INVALID_ARGUMENT, "contraction path: null pair list");
    std::vector<bool> used(T + npairs, false);
    for (size_t p = 0; p < npairs; p++) {
        const uint32_t a = path[2 * p], b = path[2 * p + 1];
        if (a == b || a >= T + p || b >= T + p)
            return fail(YAO_ERR_INVALID_ARGUMENT,
                        "contraction path: pair " + std::to_string(p) + " must name two distinct earlier tensors");
        if (used[a] || used[b])
            return fail(YAO_ERR_INVALID_ARGUMENT,
                        "contraction path: pair " + std::to_string(p) + " names a tensor already contracted");
        used[a] = used[b] = true;
    }
    return YAO_OK;
}

// Contracts the whole network on the device and copies the result (legs in
// the order of tn.iy, row-major) to `out` (2 * prod(sizes of iy) doubles).
// Order: `path` when given (pair s contracts path[2s] and path[2s+1], the
// indices counting the network's tensors and then each pair's result, as
// checked by path_validate); otherwise repeatedly the pair of tensors that
// share a label (or, when none do, the two smallest) whose result minus its
// inputs is smallest (sizes as log2 to avoid overflow), ties to the lowest
// indices.  A label is kept in a result while the output or another
// remaining tensor has it.
int tn_contract(Ctx* ctx, const TNet& tn, double* out, const uint32_t* path, size_t npairs, bool by_path) {
    int s = tn_validate(tn);
    if (s) return s;
    if (by_path) {
        s = path_validate(tn.tensors.size(), path, npairs);
        if (s) return s;
    }
    const std::map<int64_t, uint32_t>& size = tn.size;
    std::vector<DevTensor> live;
    std::vector<bool> alive;
    auto release = [&]() {
        for (size_t i = 0; i < live.size(); i++)
            if (alive[i] && live[i].d) cudaFreeAsync(live[i].d, ctx->stream);
    };
    for (size_t t = 0; t < tn.tensors.size(); t++) {
        DevTensor d;
        d.legs = tn.ixs[t];
        d.len = tn.tensors[t].size();
        if (cudaMallocAsync((void**)&d.d, std::max<size_t>(1, d.len) * sizeof(double2), ctx->stream) != cudaSuccess) {
            release();
            return fail(YAO_ERR_OUT_OF_MEMORY, "tensor network: cannot allocate a tensor");
        }
        YAO_CUDA(cudaMemcpyAsync(d.d, tn.tensors[t].data(), d.len * sizeof(double2), cudaMemcpyHostToDevice,
                                 ctx->stream));
        live.push_back(d);
        alive.push_back(true);
    }
    const std::set<int64_t> outset(tn.iy.begin(), tn.iy.end());
    // label -> live tensors holding it
    std::map<int64_t, std::set<size_t>> holders;
    for (size_t t = 0; t < live.size(); t++)
        for (int64_t l : live[t].legs) holders[l].insert(t);
    auto keep_for = [&](size_t a, size_t b) {
        std::set<int64_t> keep;
        for (size_t x : {a, b})
            for (int64_t l : live[x].legs) {
                if (outset.count(l)) {
                    keep.insert(l);
                    continue;
                }
                for (size_t h : holders[l])
                    if (h != a && h != b) {
                        keep.insert(l);
                        break;
                    }
            }
        return keep;
    };
    size_t nlive = live.size();
    if (nlive == 0) {  // the empty product: 1
        out[0] = 1.0;
        out[1] = 0.0;
        return YAO_OK;
    }
    // Candidate pairs (tensors sharing a label) ordered by (growth, a, b):
    // the first is the pair the rule picks.  A pair's growth depends only on
    // which tensors hold its labels, and contracting a and b into c keeps
    // every label another tensor holds (now held by c), so after a step only
    // the pairs with c are new; those with a or b are dropped.
    auto growth = [&](size_t i, size_t j) {
        const std::set<int64_t> keep = keep_for(i, j);
        std::vector<int64_t> ra;
        for (int64_t l : keep)
            if (std::find(live[i].legs.begin(), live[i].legs.end(), l) != live[i].legs.end() ||
                std::find(live[j].legs.begin(), live[j].legs.end(), l) != live[j].legs.end())
                ra.push_back(l);
        return std::exp2(log2_size(ra, size)) - std::exp2(log2_size(live[i].legs, size)) -
               std::exp2(log2_size(live[j].legs, size));
    };
    std::set<std::tuple<double, size_t, size_t>> cand;
    std::map<size_t, std::map<size_t, double>> partner;  // t -> (other, growth of the pair)
    auto add_pairs_of = [&](size_t t) {
        std::set<size_t> nb;
        for (int64_t l : live[t].legs)
            for (size_t h : holders[l])
                if (h != t) nb.insert(h);
        for (size_t h : nb) {
            const size_t i = std::min(t, h), j = std::max(t, h);
            if (partner[i].count(j)) continue;
            const double c = growth(i, j);
            partner[i][j] = c;
            partner[j][i] = c;
            cand.insert(std::make_tuple(c, i, j));
        }
    };
    auto drop_pairs_of = [&](size_t t) {
        for (const auto& kv : partner[t]) {
            const size_t i = std::min(t, kv.first), j = std::max(t, kv.first);
            cand.erase(std::make_tuple(kv.second, i, j));
            partner[kv.first].erase(t);
        }
        partner.erase(t);
    };
    if (!by_path)
        for (size_t t = 0; t < live.size(); t++) add_pairs_of(t);
    for (size_t step = 0; nlive > 1; step++) {
        size_t ba = 0, bb = 0;
        if (by_path) {
            ba = path[2 * step];
            bb = path[2 * step + 1];
        } else if (!cand.empty()) {
            ba = std::get<1>(*cand.begin());
            bb = std::get<2>(*cand.begin());
        } else {  // no shared label: the two smallest (an outer product)
            std::vector<std::pair<double, size_t>> bysize;
            for (size_t t = 0; t < live.size(); t++)
                if (alive[t]) bysize.push_back({log2_size(live[t].legs, size), t});
            std::sort(bysize.begin(), bysize.end());
            ba = std::min(bysize[0].second, bysize[1].second);
            bb = std::max(bysize[0].second, bysize[1].second);
        }
        DevTensor c;
        s = contract_pair(ctx, live[ba], live[bb], keep_for(ba, bb), size, c, nullptr);
        if (s) {
            release();
            return s;
        }
        for (size_t x : {ba, bb}) {
            drop_pairs_of(x);
            for (int64_t l : live[x].legs) {
                holders[l].erase(x);
                if (holders[l].empty()) holders.erase(l);
            }
            YAO_CUDA(cudaFreeAsync(live[x].d, ctx->stream));
            alive[x] = false;
            live[x].d = nullptr;
        }
        live.push_back(c);
        alive.push_back(true);
        for (int64_t l : c.legs) holders[l].insert(live.size() - 1);
        if (!by_path) add_pairs_of(live.size() - 1);
        nlive--;
    }
    size_t last = 0;
    for (size_t t = 0; t < live.size(); t++)
        if (alive[t]) last = t;
    // the result: remaining summed labels traced out, legs in the order of iy
    DevTensor one;
    one.len = 1;
    YAO_CUDA(cudaMallocAsync((void**)&one.d, sizeof(double2), ctx->stream));
    const double2 h1 = make_double2(1.0, 0.0);
    YAO_CUDA(cudaMemcpyAsync(one.d, &h1, sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    DevTensor res;
    s = contract_pair(ctx, live[last], one, outset, size, res, &tn.iy);
    cudaFreeAsync(one.d, ctx->stream);
    cudaFreeAsync(live[last].d, ctx->stream);
    if (s) return s;
    YAO_CUDA(cudaMemcpyAsync(out, res.d, res.len * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaFreeAsync(res.d, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    return YAO_OK;
}

}  // namespace yao

// ------------------------------------------------------------------- C ABI
struct yao_tn : yao::TNet {};

using namespace yao;

extern "C" {

int yao_tn_from_circuit(const yao_circuit* c, int32_t kind, const uint32_t* pinned, uint32_t npinned,
                        const yao_term* terms, size_t nterms, yao_tn** out) {
    if (!c || !out) return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    if (npinned && !pinned) return fail(YAO_ERR_INVALID_ARGUMENT, "null pinned sites");
    if (nterms && !terms) return fail(YAO_ERR_INVALID_ARGUMENT, "null terms");
    std::unique_ptr<yao_tn> tn(new yao_tn());
    int s;
    const uint32_t n = (uint32_t)c->dims.size();
    switch (kind) {
    case YAO_TN_EINSUM: s = tn_from_circuit(*c, false, {}, *tn); break;
    case YAO_TN_BOUNDARY: s = tn_from_circuit(*c, true, std::vector<uint32_t>(pinned, pinned + npinned), *tn); break;
    case YAO_TN_OVERLAP: {
        std::vector<uint32_t> all(n);
        for (uint32_t i = 0; i < n; i++) all[i] = i;
        s = tn_from_circuit(*c, true, all, *tn);
        break;
    }
    case YAO_TN_EXPECTATION: s = tn_expectation(*c, terms, nterms, *tn); break;
    case YAO_TN_DM: s = tn_dm(*c, *tn); break;
    case YAO_TN_EXPECTATION_DM: s = tn_expectation_dm(*c, terms, nterms, *tn); break;
    default: return fail(YAO_ERR_INVALID_ARGUMENT, "unknown tensor-network kind");
    }
    if (s) return s;
    *out = tn.release();
    return YAO_OK;
}

int yao_tn_create(size_t ntensors, const uint32_t* ranks, const int64_t* labels, const double* data, size_t nelems,
                  size_t nlabels, const int64_t* label_ids, const uint32_t* label_dims, uint32_t nout,
                  const int64_t* out_labels, yao_tn** out) {
    if (!out || (ntensors && !ranks) || (nelems && !data) || (nlabels && (!label_ids || !label_dims)) ||
        (nout && !out_labels))
        return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    std::unique_ptr<yao_tn> tn(new yao_tn());
    for (size_t i = 0; i < nlabels; i++) tn->size[label_ids[i]] = label_dims[i];
    size_t lo = 0, dof = 0;
    for (size_t t = 0; t < ntensors; t++) {
        std::vector<int64_t> legs(labels + lo, labels + lo + ranks[t]);
        lo += ranks[t];
        size_t len = 1;
        for (int64_t l : legs) {
            auto it = tn->size.find(l);
            if (it == tn->size.end()) return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: a label has no size");
            len *= it->second;
        }
        if (dof + len > nelems)
            return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: tensor data length does not match its legs");
        std::vector<Cx> v(len);
        if (len) memcpy(v.data(), data + 2 * dof, len * sizeof(Cx));
        dof += len;
        tn->ixs.push_back(legs);
        tn->tensors.push_back(std::move(v));
    }
    if (dof != nelems)
        return fail(YAO_ERR_INVALID_ARGUMENT, "tensor network: tensor data length does not match its legs");
    tn->iy.assign(out_labels, out_labels + nout);
    int s = tn_validate(*tn);
    if (s) return s;
    *out = tn.release();
    return YAO_OK;
}

void yao_tn_free(yao_tn* tn) { delete tn; }

int yao_tn_counts(const yao_tn* tn, size_t* ntensors, size_t* nlegs, size_t* nelems, uint32_t* nout,
                  size_t* nlabels) {
    if (!tn || !ntensors || !nlegs || !nelems || !nout || !nlabels) return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    *ntensors = tn->ixs.size();
    size_t l = 0, e = 0;
    for (size_t t = 0; t < tn->ixs.size(); t++) {
        l += tn->ixs[t].size();
        e += tn->tensors[t].size();
    }
    *nlegs = l;
    *nelems = e;
    *nout = (uint32_t)tn->iy.size();
    *nlabels = tn->size.size();
    return YAO_OK;
}

int yao_tn_export(const yao_tn* tn, uint32_t* ranks, int64_t* labels, double* data, int64_t* out_labels,
                  int64_t* label_ids, uint32_t* label_dims) {
    if (!tn || !ranks || !labels || !data || !out_labels || !label_ids || !label_dims)
        return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    size_t lo = 0, dof = 0;
    for (size_t t = 0; t < tn->ixs.size(); t++) {
        ranks[t] = (uint32_t)tn->ixs[t].size();
        for (int64_t l : tn->ixs[t]) labels[lo++] = l;
        memcpy(data + 2 * dof, tn->tensors[t].data(), tn->tensors[t].size() * sizeof(Cx));
        dof += tn->tensors[t].size();
    }
    for (size_t i = 0; i < tn->iy.size(); i++) out_labels[i] = tn->iy[i];
    size_t i = 0;
    for (const auto& kv : tn->size) {
        label_ids[i] = kv.first;
        label_dims[i++] = kv.second;
    }
    return YAO_OK;
}

int yao_tn_output_len(const yao_tn* tn, size_t* out) {
    if (!tn || !out) return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    size_t n = 1;
    for (int64_t l : tn->iy) {
        auto it = tn->size.find(l);
        if (it == tn->size.end()) return fail(YAO_ERR_INVALID_ARGUMENT, "an output label has no size");
        n *= it->second;
    }
    *out = n;
    return YAO_OK;
}

int yao_tn_contract(yao_ctx* ctx, const yao_tn* tn, double* out, size_t out_len) {
    if (!ctx || !tn || !out) return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    size_t need = 0;
    int s = yao_tn_output_len(tn, &need);
    if (s) return s;
    if (out_len < need) return fail(YAO_ERR_INVALID_ARGUMENT, "output buffer too small for the contraction result");
    YAO_CUDA(cudaSetDevice(ctx->device));
    return tn_contract(ctx, *tn, out, nullptr, 0, false);
}

int yao_tn_contract_path(yao_ctx* ctx, const yao_tn* tn, const uint32_t* path, size_t npairs, double* out,
                         size_t out_len) {
    if (!ctx || !tn || !out) return fail(YAO_ERR_INVALID_ARGUMENT, "null argument");
    clear_error();
    size_t need = 0;
    int s = yao_tn_output_len(tn, &need);
    if (s) return s;
    if (out_len < need) return fail(YAO_ERR_INVALID_ARGUMENT, "output buffer too small for the contraction result");
    s = path_validate(tn->tensors.size(), path, npairs);
    if (s) return s;
    YAO_CUDA(cudaSetDevice(ctx->device));
    return tn_contract(ctx, *tn, out, path, npairs, true);
}

}  // extern "C"
