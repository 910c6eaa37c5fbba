// vqe_batch.cu — energies and adjoint gradients of many parameter sets of
// one circuit (expect_grad, yao-rs src/ad.rs:75-156, for a batch).
//
// The nsets states sit back to back (set s at s * 2^n).  Every gate step is
// one launch over all sets: gates without parameters act on the flattened
// vector (the set index is just higher bits above the n qubit bits, and group
// enumeration by zero-bit insertion skips over them), gates with parameters
// read their per-set coefficients.  Arithmetic per amplitude is the PLAIN
// path's, so each set's forward state equals a single-set run bit for bit.
// Reductions (energies, gradient dots) are per-set deterministic trees.  The
// host synchronises once, at the end.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"

namespace yao {

#define GRID_STRIDE(i, n) \
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

constexpr int kBT = 256;

struct BGate {
    int32_t cls, k, nlocked, pad;
    uint64_t cval;
    int8_t locked[64];
    uint64_t off[4];
};

static BGate make_bgate(const LGate& g) {
    BGate b;
    memset(&b, 0, sizeof(b));
    b.cls = g.cls;
    b.k = g.k;
    std::vector<int> pos;
    for (int i = 0; i < g.k; i++) pos.push_back(g.tb[i]);
    for (int i = 0; i < g.nc; i++) pos.push_back(g.cb[i]);
    std::sort(pos.begin(), pos.end());
    b.nlocked = (int)pos.size();
    for (size_t i = 0; i < pos.size(); i++) b.locked[i] = (int8_t)pos[i];
    b.cval = g.cval();
    for (int l = 0; l < (1 << g.k); l++) {
        uint64_t o = 0;
        for (int i = 0; i < g.k; i++) o |= (uint64_t)((l >> i) & 1) << g.tb[i];
        b.off[l] = o;
    }
    return b;
}

// A diagonal or dense 1-2 qubit gate with per-set coefficients m[set * 16 + i].
template <int CLS, int K>
__global__ void __launch_bounds__(kBT) k_gate_pset(double2* __restrict__ st, uint64_t total_groups, int gshift,
                                                  const BGate op, const double2* __restrict__ m) {
    constexpr int NL = 1 << K;
    GRID_STRIDE(g, total_groups) {
        const double2* c = m + (g >> gshift) * 16;
        const uint64_t base = insert_zeros(g, op.locked, op.nlocked) | op.cval;
        double2 v[NL];
#pragma unroll
        for (int l = 0; l < NL; l++) v[l] = st[base + op.off[l]];
        if (CLS == GC_DIAG) {
#pragma unroll
            for (int l = 0; l < NL; l++) st[base + op.off[l]] = cmulassign_x(v[l], c[l]);
        } else if (K == 1) {
            st[base + op.off[0]] = cadd_x(cmul_x(c[0], v[0]), cmul_x(c[1], v[1]));
            st[base + op.off[1]] = cadd_x(cmul_x(c[2], v[0]), cmul_x(c[3], v[1]));
        } else {
#pragma unroll
            for (int i = 0; i < NL; i++) {
                double2 acc = make_double2(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < NL; j++) acc = cadd_x(acc, cmul_x(c[i * NL + j], v[j]));
                st[base + op.off[i]] = acc;
            }
        }
    }
}

// Adjoint step for all sets: <lambda_s | G_p psi_s> per set (generators are
// the same for every set), then U_s^dagger on psi_s and lambda_s.
// Grid: (blocks per set, nsets); partial[(set * gridDim.x + bx) * 4 + v].
template <int CLS, int K>
__global__ void __launch_bounds__(kBT) k_adjoint_pset(double2* __restrict__ psi, double2* __restrict__ lam,
                                                     uint64_t groups_per_set, int gshift, const BGate op, int ngen,
                                                     const double2* __restrict__ gen, const double2* __restrict__ dag,
                                                     double* __restrict__ partial) {
    constexpr int NL = 1 << K;
    __shared__ double sm[4 * kBT / 32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t set = blockIdx.y;
    const double2* d = dag + set * 16;
    for (uint64_t gl = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gl < groups_per_set;
         gl += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t g = (set << gshift) | gl;
        const uint64_t base = insert_zeros(g, op.locked, op.nlocked) | op.cval;
        double2 x[NL], l[NL];
#pragma unroll
        for (int q = 0; q < NL; q++) {
            x[q] = psi[base + op.off[q]];
            l[q] = lam[base + op.off[q]];
        }
        for (int p = 0; p < ngen; p++) {
            const double2* G = gen + p * 16;
#pragma unroll
            for (int r = 0; r < NL; r++) {
                double2 y;
                if (K == 1) {
                    y = cadd_x(cmul_x(G[r * 2], x[0]), cmul_x(G[r * 2 + 1], x[1]));
                } else {
                    y = make_double2(0.0, 0.0);
#pragma unroll
                    for (int c = 0; c < NL; c++) y = cadd_x(y, cmul_x(G[r * NL + c], x[c]));
                }
                acc[2 * p] += l[r].x * y.x + l[r].y * y.y;
                acc[2 * p + 1] += l[r].x * y.y - l[r].y * y.x;
            }
        }
        if (CLS == GC_DIAG) {
#pragma unroll
            for (int q = 0; q < NL; q++) {
                psi[base + op.off[q]] = cmulassign_x(x[q], d[q]);
                lam[base + op.off[q]] = cmulassign_x(l[q], d[q]);
            }
        } else if (K == 1) {
            psi[base + op.off[0]] = cadd_x(cmul_x(d[0], x[0]), cmul_x(d[1], x[1]));
            psi[base + op.off[1]] = cadd_x(cmul_x(d[2], x[0]), cmul_x(d[3], x[1]));
            lam[base + op.off[0]] = cadd_x(cmul_x(d[0], l[0]), cmul_x(d[1], l[1]));
            lam[base + op.off[1]] = cadd_x(cmul_x(d[2], l[0]), cmul_x(d[3], l[1]));
        } else {
#pragma unroll
            for (int r = 0; r < NL; r++) {
                double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < NL; c++) {
                    a = cadd_x(a, cmul_x(d[r * NL + c], x[c]));
                    b = cadd_x(b, cmul_x(d[r * NL + c], l[c]));
                }
                psi[base + op.off[r]] = a;
                lam[base + op.off[r]] = b;
            }
        }
    }
    block_sum_write(acc, 2 * ngen, sm, partial + ((uint64_t)set * gridDim.x + blockIdx.x) * 4);
}

// grad[set * np + slot + p] = 2 * Re(sum_b partial[set][b][2p])
__global__ void k_grad_final(const double* __restrict__ partial, int nb, int ngen, double* __restrict__ grad, int np,
                             int slot) {
    const uint64_t set = blockIdx.x;
    __shared__ double sm[kBT / 32];
    for (int p = 0; p < ngen; p++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[((uint64_t)set * nb + b) * 4 + 2 * p];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sm[w];
            grad[set * np + slot + p] = 2.0 * t;
        }
        __syncthreads();
    }
}

// <psi_s|P_t|psi_s> for up to 8 monomials sharing an x-mask, every set.
struct BMono {
    uint64_t d1, d2, need1, need0;
    int32_t base, zero;
};
struct BGroup {
    uint64_t xmask;
    int32_t hbit, nt;
    BMono t[8];
};

__device__ __forceinline__ int bphase(const BMono& t, uint64_t i) {
    if (t.zero || (i & t.need1) != t.need1 || (i & t.need0) != 0) return -1;
    return (t.base + __popcll(i & t.d1) + 2 * __popcll(i & t.d2)) & 3;
}
__device__ __forceinline__ double2 bturn(double2 v, int q) {
    switch (q) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
    }
}

__global__ void __launch_bounds__(kBT) k_expect_pset(const double2* __restrict__ st, uint64_t n_amp, const BGroup grp,
                                                    double* __restrict__ partial) {
    __shared__ double sm[16 * kBT / 32];
    double acc[16];
#pragma unroll
    for (int j = 0; j < 16; j++) acc[j] = 0.0;
    const double2* s = st + (uint64_t)blockIdx.y * n_amp;
    const uint64_t nwork = grp.xmask ? n_amp / 2 : n_amp;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nwork; p += (uint64_t)gridDim.x * blockDim.x) {
        if (grp.xmask == 0) {
            double2 v = s[p];
            double pr = v.x * v.x + v.y * v.y;
#pragma unroll
            for (int t = 0; t < 8; t++) {
                if (t >= grp.nt) break;
                int q = bphase(grp.t[t], p);
                if (q < 0) continue;
                double2 c = bturn(make_double2(pr, 0.0), q);
                acc[2 * t] += c.x;
                acc[2 * t + 1] += c.y;
            }
        } else {
            const int h = grp.hbit;
            uint64_t i = ((p >> h) << (h + 1)) | (p & ((1ull << h) - 1));
            uint64_t j = i ^ grp.xmask;
            double2 a = s[i], b = s[j];
            double2 c = make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
            double2 cc = make_double2(c.x, -c.y);
#pragma unroll
            for (int t = 0; t < 8; t++) {
                if (t >= grp.nt) break;
                int qi = bphase(grp.t[t], i), qj = bphase(grp.t[t], j);
                if (qi >= 0) {
                    double2 u = bturn(c, qi);
                    acc[2 * t] += u.x;
                    acc[2 * t + 1] += u.y;
                }
                if (qj >= 0) {
                    double2 u = bturn(cc, qj);
                    acc[2 * t] += u.x;
                    acc[2 * t + 1] += u.y;
                }
            }
        }
    }
    block_sum_write(acc, 2 * grp.nt, sm, partial + ((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * 16);
}

// vals[set * nterms + idx[t]] = sum_b partial[set][b][t]
__global__ void k_expect_final(const double* __restrict__ partial, int nb, int nt, const int* __restrict__ idx,
                               int nterms, double2* __restrict__ vals) {
    const uint64_t set = blockIdx.x;
    __shared__ double sm[kBT / 32];
    for (int v = 0; v < 2 * nt; v++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[((uint64_t)set * nb + b) * 16 + v];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sm[w];
            double* out = (double*)&vals[set * nterms + idx[v / 2]];
            out[v & 1] = t;
        }
        __syncthreads();
    }
}

__global__ void k_broadcast(const double2* __restrict__ src, double2* __restrict__ dst, uint64_t n, uint64_t total) {
    GRID_STRIDE(i, total) dst[i] = src[i % n];
}

// ----------------------------------------------------------------- host

// Coefficients of a parametric gate's lowered matrix for one parameter
// vector: the same steps as lower_gate (2-qubit sort, diagonal extraction).
static void lowered_coefs(const GateElem& g, const double* p, uint32_t nbits, double2* out16) {
    GateElem e = g;
    for (int i = 0; i < gate_num_params(g.type); i++) e.params[i] = p[i];
    std::vector<LGate> lg;
    lower_gate(e, nbits, 0, false, lg);
    for (int i = 0; i < 16; i++) out16[i] = make_double2(0.0, 0.0);
    for (size_t i = 0; i < lg[0].m.size() && i < 16; i++) out16[i] = make_double2(lg[0].m[i].re, lg[0].m[i].im);
}

int expect_grad_batch(Ctx* ctx, const std::vector<MonoTerm>& terms, const Circuit* c, const double* params,
                      size_t nsets, const Reg* psi0, double* values, double* grads) {
    const uint32_t n = psi0->nbits;
    const uint64_t N = (uint64_t)1 << n;
    size_t np = 0;
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_GATE) np += (size_t)gate_num_params(el.g.type);
    // per-gate lowered structure and per-set coefficients of parametric gates
    struct GStep {
        const GateElem* g;
        size_t slot;
        int npar;
        std::vector<LGate> fwd, dag;
        std::vector<LGate> gens;
        size_t coef_off;  // into the per-set coefficient arrays (units of nsets*16)
    };
    std::vector<GStep> steps;
    size_t slot = 0, ncoefgates = 0;
    for (const Element& el : c->elems) {
        if (el.kind != YAO_ELEM_GATE) continue;
        GStep s;
        s.g = &el.g;
        s.slot = slot;
        s.npar = gate_num_params(el.g.type);
        lower_gate(el.g, n, 0, false, s.fwd);
        lower_gate(gate_dagger(el.g), n, 0, false, s.dag);
        for (int i = 0; i < s.npar; i++) {
            std::vector<Cx> gm;
            uint32_t gd;
            gate_generator(el.g, i, gm, gd);
            s.gens.push_back(lower_matrix(gm, gd, false, el.g.targets, el.g.ctrls, el.g.cfgs, n, 0));
        }
        s.coef_off = s.npar ? ncoefgates++ : 0;
        if (s.npar && (s.fwd.size() != 1 || s.fwd[0].k > 2 || s.fwd[0].cls == GC_X || s.fwd[0].cls == GC_SWAP))
            return fail(YAO_ERR_UNSUPPORTED, "batched gradients support 1- and 2-qubit parametric gates");
        slot += (size_t)s.npar;
        steps.push_back(std::move(s));
    }
    // host coefficient tables: [gate][set][16] forward and adjoint
    std::vector<double2> hf(ncoefgates * nsets * 16), hd(ncoefgates * nsets * 16);
    std::vector<double2> hg(std::max<size_t>(1, ncoefgates) * 32, make_double2(0.0, 0.0));
    for (const GStep& s : steps) {
        if (!s.npar) continue;
        for (int p = 0; p < s.npar; p++)
            for (size_t i = 0; i < s.gens[p].m.size() && i < 16; i++)
                hg[s.coef_off * 32 + p * 16 + i] = make_double2(s.gens[p].m[i].re, s.gens[p].m[i].im);
        GateElem dg = gate_dagger(*s.g);
        for (size_t set = 0; set < nsets; set++) {
            const double* p = params + set * np + s.slot;
            double neg[4] = {-p[0], s.npar > 1 ? -p[1] : 0.0, 0.0, 0.0};
            lowered_coefs(*s.g, p, n, &hf[(s.coef_off * nsets + set) * 16]);
            lowered_coefs(dg, neg, n, &hd[(s.coef_off * nsets + set) * 16]);
        }
    }
    // device memory
    const size_t sb = nsets * N * sizeof(double2);
    const int nbx = (int)std::max<uint64_t>(1, std::min<uint64_t>((N / 2 + kBT - 1) / kBT, 64));
    const size_t partial_b = nsets * (size_t)nbx * 16 * sizeof(double);
    const size_t coef_b = std::max<size_t>(1, hf.size()) * sizeof(double2);
    const size_t grad_b = std::max<size_t>(1, nsets * np) * sizeof(double);
    const size_t vals_b = std::max<size_t>(1, nsets * terms.size()) * sizeof(double2);
    // term groups (x-mask, <= 8 terms) of the energy reduction
    std::vector<BGroup> groups;
    std::vector<int> gidx;
    {
        std::vector<bool> done(terms.size(), false);
        for (size_t t0 = 0; t0 < terms.size(); t0++) {
            if (done[t0]) continue;
            BGroup grp;
            memset(&grp, 0, sizeof(grp));
            grp.xmask = terms[t0].xmask;
            grp.hbit = grp.xmask ? 63 - __builtin_clzll(grp.xmask) : 0;
            int cnt = 0;
            for (size_t t = t0; t < terms.size() && cnt < 8; t++)
                if (!done[t] && terms[t].xmask == grp.xmask) {
                    BMono& m = grp.t[cnt];
                    m.d1 = terms[t].d1mask;
                    m.d2 = terms[t].d2mask;
                    m.need1 = terms[t].need1;
                    m.need0 = terms[t].need0;
                    m.base = terms[t].base;
                    m.zero = terms[t].zero;
                    gidx.push_back((int)t);
                    cnt++;
                    done[t] = true;
                }
            for (int q = cnt; q < 8; q++) gidx.push_back(0);
            grp.nt = cnt;
            groups.push_back(grp);
        }
    }
    const size_t gen_b = hg.size() * sizeof(double2), idx_b = std::max<size_t>(1, gidx.size()) * sizeof(int);
    char* buf = nullptr;
    const size_t total = 2 * sb + partial_b + 2 * coef_b + grad_b + vals_b + gen_b + idx_b + 4096;
    if (cudaMallocAsync((void**)&buf, total, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate the batched gradient buffers");
    }
    double2* psi = (double2*)buf;
    double2* lam = (double2*)(buf + sb);
    double* partial = (double*)(buf + 2 * sb);
    double2* dfwd = (double2*)(buf + 2 * sb + partial_b);
    double2* ddag = (double2*)(buf + 2 * sb + partial_b + coef_b);
    double* dgrad = (double*)(buf + 2 * sb + partial_b + 2 * coef_b);
    double2* dvals = (double2*)(buf + 2 * sb + partial_b + 2 * coef_b + grad_b);
    double2* dgen = (double2*)(buf + 2 * sb + partial_b + 2 * coef_b + grad_b + vals_b);
    int* didx = (int*)((char*)dgen + gen_b);
    YAO_CUDA(cudaMemcpyAsync(dfwd, hf.data(), hf.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(ddag, hd.data(), hd.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dgen, hg.data(), gen_b, cudaMemcpyHostToDevice, ctx->stream));
    if (!gidx.empty())
        YAO_CUDA(cudaMemcpyAsync(didx, gidx.data(), gidx.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    const uint64_t tot = nsets * N;
    k_broadcast<<<grid_for(tot, 256, ctx->num_sms), 256, 0, ctx->stream>>>((const double2*)psi0->d, psi, N, tot);
    ctx->launches++;
    // a gate without parameters: one launch over the groups of every set
    auto flat_gate = [&](double2* st, const LGate& g) -> int { return launch_gate_sets(ctx, st, n, g, nsets); };
    auto pset_gate = [&](double2* st, const LGate& g, const double2* m) -> int {
        BGate b = make_bgate(g);
        const int gshift = (int)(n - b.nlocked);
        const uint64_t total_groups = (uint64_t)nsets << gshift;
        const unsigned grid = grid_for(total_groups, kBT, ctx->num_sms, 8);
        ProfScope prof(ctx, "gate_pset", (double)total_groups * (1 << g.k) * 32.0);
        if (g.cls == GC_DIAG && g.k == 1) k_gate_pset<GC_DIAG, 1><<<grid, kBT, 0, ctx->stream>>>(st, total_groups, gshift, b, m);
        else if (g.cls == GC_DIAG) k_gate_pset<GC_DIAG, 2><<<grid, kBT, 0, ctx->stream>>>(st, total_groups, gshift, b, m);
        else if (g.k == 1) k_gate_pset<GC_DENSE, 1><<<grid, kBT, 0, ctx->stream>>>(st, total_groups, gshift, b, m);
        else k_gate_pset<GC_DENSE, 2><<<grid, kBT, 0, ctx->stream>>>(st, total_groups, gshift, b, m);
        ctx->launches++;
        YAO_CUDA(cudaGetLastError());
        return YAO_OK;
    };
    // forward
    for (const GStep& s : steps) {
        int st;
        if (s.npar)
            st = pset_gate(psi, s.fwd[0], dfwd + s.coef_off * nsets * 16);
        else {
            st = YAO_OK;
            for (const LGate& g : s.fwd)
                if ((st = flat_gate(psi, g))) break;
        }
        if (st) {
            cudaFreeAsync(buf, ctx->stream);
            return st;
        }
    }
    // energies: per x-mask group of terms
    for (size_t gi = 0; gi < groups.size(); gi++) {
        dim3 grid(nbx, (unsigned)nsets);
        {
            ProfScope prof(ctx, "expect_pset", (double)nsets * N * 16.0);
            k_expect_pset<<<grid, kBT, 0, ctx->stream>>>(psi, N, groups[gi], partial);
        }
        k_expect_final<<<(unsigned)nsets, kBT, 0, ctx->stream>>>(partial, nbx, groups[gi].nt, didx + 8 * gi,
                                                                 (int)terms.size(), dvals);
        ctx->launches += 2;
        YAO_CUDA(cudaGetLastError());
    }
    // lambda = sum_t c_t P_t psi on the flattened vector (set bits lie above every mask)
    {
        int s = build_lambda_sets(ctx, psi, lam, n, nsets, terms);
        if (s) {
            cudaFreeAsync(buf, ctx->stream);
            return s;
        }
    }
    // reverse sweep
    for (size_t si = steps.size(); si-- > 0;) {
        const GStep& s = steps[si];
        if (!s.npar) {
            for (const LGate& g : s.dag) {
                int st = flat_gate(psi, g);
                if (!st) st = flat_gate(lam, g);
                if (st) {
                    cudaFreeAsync(buf, ctx->stream);
                    return st;
                }
            }
            continue;
        }
        const double2* gens = dgen + s.coef_off * 32;
        const LGate& d = s.dag[0];
        BGate b = make_bgate(d);
        const int gshift = (int)(n - b.nlocked);
        const uint64_t gps = (uint64_t)1 << gshift;
        const int nb = (int)std::max<uint64_t>(1, std::min<uint64_t>((gps + kBT - 1) / kBT, (uint64_t)nbx));
        dim3 grid(nb, (unsigned)nsets);
        const double2* dd = ddag + s.coef_off * nsets * 16;
        {
            ProfScope prof(ctx, "adjoint_pset", (double)nsets * gps * (1 << d.k) * 64.0);
            if (d.cls == GC_DIAG && d.k == 1)
                k_adjoint_pset<GC_DIAG, 1><<<grid, kBT, 0, ctx->stream>>>(psi, lam, gps, gshift, b, s.npar, gens, dd, partial);
            else if (d.cls == GC_DIAG)
                k_adjoint_pset<GC_DIAG, 2><<<grid, kBT, 0, ctx->stream>>>(psi, lam, gps, gshift, b, s.npar, gens, dd, partial);
            else if (d.k == 1)
                k_adjoint_pset<GC_DENSE, 1><<<grid, kBT, 0, ctx->stream>>>(psi, lam, gps, gshift, b, s.npar, gens, dd, partial);
            else
                k_adjoint_pset<GC_DENSE, 2><<<grid, kBT, 0, ctx->stream>>>(psi, lam, gps, gshift, b, s.npar, gens, dd, partial);
        }
        k_grad_final<<<(unsigned)nsets, kBT, 0, ctx->stream>>>(partial, nb, s.npar, dgrad, (int)np, (int)s.slot);
        ctx->launches += 2;
        YAO_CUDA(cudaGetLastError());
    }
    std::vector<double2> hv(nsets * terms.size());
    if (np) YAO_CUDA(cudaMemcpyAsync(grads, dgrad, nsets * np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (!hv.empty())
        YAO_CUDA(cudaMemcpyAsync(hv.data(), dvals, hv.size() * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    YAO_CUDA(cudaFreeAsync(buf, ctx->stream));
    for (size_t set = 0; set < nsets; set++) {
        double re = 0.0;
        for (size_t t = 0; t < terms.size(); t++) {
            Cx cf = terms[t].coeff;
            double2 v = hv[set * terms.size() + t];
            re += cf.re * v.x - cf.im * v.y;
        }
        values[set] = re;
    }
    return YAO_OK;
}

}  // namespace yao
