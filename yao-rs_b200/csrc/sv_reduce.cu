// sv_reduce.cu — state-vector reductions and the kernels built on them:
// norm / fidelity, Pauli-monomial expectation values, the adjoint
// (reverse-sweep) gradient step, probabilities and measurement bookkeeping,
// plus the state initialisers.
//
// Every reduction is deterministic: each block sums its grid-stride slice in
// a fixed order (warp shuffles, then warps in order), block partials go to
// the context scratch, and one block adds the partials in block order.  All
// sums are FP64, also for complex64 registers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "device_common.cuh"

namespace yao {

constexpr int kRT = 256;  // reduction block size

// ------------------------------------------------------------- helpers

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }
template <typename V>
__device__ __forceinline__ V from_d2(double2 v);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 v) {
    return v;
}
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 v) {
    return make_float2((float)v.x, (float)v.y);
}

// Sum partial[b * nv + v] over b for every v (one block, fixed order).
__global__ void k_final_sum(const double* __restrict__ partial, int nblocks, int nv, double* __restrict__ out) {
    __shared__ double sm[kRT / 32];
    for (int v = 0; v < nv; v++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[(size_t)b * nv + v];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sm[w];
            out[v] = t;
        }
        __syncthreads();
    }
}

static int reduce_blocks(Ctx* ctx, uint64_t work) { return (int)grid_for(work, kRT, ctx->num_sms, 4); }

// Scratch layout for one reduction: nblocks * nv partials, then nv results.
static int reduce_scratch(Ctx* ctx, int nblocks, int nv, double** partial) {
    size_t bytes = sizeof(double) * ((size_t)nblocks * nv + nv);
    if (ctx->ensure_scratch(bytes)) return YAO_ERR_OUT_OF_MEMORY;
    *partial = (double*)ctx->scratch;
    return YAO_OK;
}

// Final sum on the device, result copied to host (synchronous).
static int finish_sum(Ctx* ctx, double* partial, int nblocks, int nv, double* host_out) {
    double* dout = partial + (size_t)nblocks * nv;
    k_final_sum<<<1, kRT, 0, ctx->stream>>>(partial, nblocks, nv, dout);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    if (ctx->ensure_host_pinned(sizeof(double) * nv)) return YAO_ERR_OUT_OF_MEMORY;
    YAO_CUDA(cudaMemcpyAsync(ctx->host_pinned, dout, sizeof(double) * nv, cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(host_out, ctx->host_pinned, sizeof(double) * nv);
    return YAO_OK;
}

#define GRID_STRIDE(i, n) \
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

// ------------------------------------------------------------ init states

template <typename V>
__global__ void k_fill(V* st, uint64_t n, double re, double im) {
    V v = from_d2<V>(make_double2(re, im));
    GRID_STRIDE(i, n) st[i] = v;
}
template <typename V>
__global__ void k_set_one(V* st, uint64_t idx, double re, double im) {
    st[idx] = from_d2<V>(make_double2(re, im));
}

static int fill(Ctx* ctx, Reg* r, double re, double im) {
    uint64_t n = (uint64_t)1 << r->nbits;
    unsigned g = grid_for(n, 256, ctx->num_sms);
    if (r->precision == YAO_C128)
        k_fill<double2><<<g, 256, 0, ctx->stream>>>((double2*)r->d, n, re, im);
    else
        k_fill<float2><<<g, 256, 0, ctx->stream>>>((float2*)r->d, n, re, im);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

static int set_one(Ctx* ctx, Reg* r, uint64_t idx, double re, double im) {
    if (r->precision == YAO_C128)
        k_set_one<double2><<<1, 1, 0, ctx->stream>>>((double2*)r->d, idx, re, im);
    else
        k_set_one<float2><<<1, 1, 0, ctx->stream>>>((float2*)r->d, idx, re, im);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// ArrayReg::zero_state / product_state (src/register.rs:21-33)
int launch_fill_zero_state(Ctx* ctx, Reg* r, uint64_t basis) {
    int s = fill(ctx, r, 0.0, 0.0);
    if (s) return s;
    return set_one(ctx, r, basis, 1.0, 0.0);
}

// ArrayReg::uniform_state (src/register.rs:47-54): 1/sqrt(dim) everywhere
int launch_uniform_state(Ctx* ctx, Reg* r) {
    double dim = (double)((uint64_t)1 << r->nbits);
    return fill(ctx, r, 1.0 / std::sqrt(dim), 0.0);
}

// ArrayReg::deterministic_state (src/register.rs:71-85): (cos(0.1k), sin(0.2k)) / norm
template <typename V>
__global__ void k_deterministic(V* st, uint64_t n) {
    GRID_STRIDE(i, n) {
        double kf = (double)i;
        st[i] = from_d2<V>(make_double2(cos(0.1 * kf), sin(0.2 * kf)));
    }
}

int launch_deterministic_state(Ctx* ctx, Reg* r) {
    uint64_t n = (uint64_t)1 << r->nbits;
    unsigned g = grid_for(n, 256, ctx->num_sms);
    if (r->precision == YAO_C128)
        k_deterministic<double2><<<g, 256, 0, ctx->stream>>>((double2*)r->d, n);
    else
        k_deterministic<float2><<<g, 256, 0, ctx->stream>>>((float2*)r->d, n);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    double ns;
    int s = reduce_norm_sqr(ctx, r, &ns);
    if (s) return s;
    return launch_scale(ctx, r, std::sqrt(ns));
}

template <typename A, typename B>
__global__ void k_convert(const A* __restrict__ a, B* __restrict__ b, uint64_t n) {
    GRID_STRIDE(i, n) b[i] = from_d2<B>(to_d2(a[i]));
}

int launch_convert(Ctx* ctx, const Reg* src, Reg* dst) {
    uint64_t n = (uint64_t)1 << src->nbits;
    unsigned g = grid_for(n, 256, ctx->num_sms);
    if (src->precision == YAO_C128 && dst->precision == YAO_C64)
        k_convert<double2, float2><<<g, 256, 0, ctx->stream>>>((const double2*)src->d, (float2*)dst->d, n);
    else if (src->precision == YAO_C64 && dst->precision == YAO_C128)
        k_convert<float2, double2><<<g, 256, 0, ctx->stream>>>((const float2*)src->d, (double2*)dst->d, n);
    else
        YAO_CUDA(cudaMemcpyAsync(dst->d, src->d, src->bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// amp /= norm for every amplitude (ArrayReg::normalize, src/register.rs:106-113)
template <typename V>
__global__ void k_div(V* st, uint64_t n, double d) {
    GRID_STRIDE(i, n) {
        double2 v = to_d2(st[i]);
        st[i] = from_d2<V>(make_double2(__ddiv_rn(v.x, d), __ddiv_rn(v.y, d)));
    }
}

int launch_scale(Ctx* ctx, Reg* r, double norm) {
    uint64_t n = (uint64_t)1 << r->nbits;
    unsigned g = grid_for(n, 256, ctx->num_sms);
    if (r->precision == YAO_C128)
        k_div<double2><<<g, 256, 0, ctx->stream>>>((double2*)r->d, n, norm);
    else
        k_div<float2><<<g, 256, 0, ctx->stream>>>((float2*)r->d, n, norm);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// ------------------------------------------------------ norm / inner product

template <typename V>
__global__ void __launch_bounds__(kRT) k_norm_sqr(const V* __restrict__ st, uint64_t n, double* partial) {
    __shared__ double sm[kRT / 32];
    double acc = 0.0;
    GRID_STRIDE(i, n) {
        double2 v = to_d2(st[i]);
        acc += v.x * v.x + v.y * v.y;
    }
    block_sum_write(&acc, 1, sm, partial + blockIdx.x);
}

int reduce_norm_sqr(Ctx* ctx, const Reg* r, double* out) {
    uint64_t n = (uint64_t)1 << r->nbits;
    int nb = reduce_blocks(ctx, n);
    double* part;
    if (reduce_scratch(ctx, nb, 1, &part)) return YAO_ERR_OUT_OF_MEMORY;
    if (r->precision == YAO_C128)
        k_norm_sqr<double2><<<nb, kRT, 0, ctx->stream>>>((const double2*)r->d, n, part);
    else
        k_norm_sqr<float2><<<nb, kRT, 0, ctx->stream>>>((const float2*)r->d, n, part);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return finish_sum(ctx, part, nb, 1, out);
}

// sum conj(a_i) * b_i (ArrayReg::fidelity, src/register.rs:115-124)
template <typename A, typename B>
__global__ void __launch_bounds__(kRT) k_inner(const A* __restrict__ a, const B* __restrict__ b, uint64_t n,
                                              double* partial) {
    __shared__ double sm[2 * kRT / 32];
    double acc[2] = {0.0, 0.0};
    GRID_STRIDE(i, n) {
        double2 x = to_d2(a[i]), y = to_d2(b[i]);
        acc[0] += x.x * y.x + x.y * y.y;
        acc[1] += x.x * y.y - x.y * y.x;
    }
    block_sum_write(acc, 2, sm, partial + 2 * blockIdx.x);
}

int reduce_inner(Ctx* ctx, const Reg* a, const Reg* b, Cx* out) {
    uint64_t n = (uint64_t)1 << a->nbits;
    int nb = reduce_blocks(ctx, n);
    double* part;
    if (reduce_scratch(ctx, nb, 2, &part)) return YAO_ERR_OUT_OF_MEMORY;
    cudaStream_t s = ctx->stream;
    if (a->precision == YAO_C128 && b->precision == YAO_C128)
        k_inner<double2, double2><<<nb, kRT, 0, s>>>((const double2*)a->d, (const double2*)b->d, n, part);
    else if (a->precision == YAO_C128)
        k_inner<double2, float2><<<nb, kRT, 0, s>>>((const double2*)a->d, (const float2*)b->d, n, part);
    else if (b->precision == YAO_C128)
        k_inner<float2, double2><<<nb, kRT, 0, s>>>((const float2*)a->d, (const double2*)b->d, n, part);
    else
        k_inner<float2, float2><<<nb, kRT, 0, s>>>((const float2*)a->d, (const float2*)b->d, n, part);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    double r[2];
    int st = finish_sum(ctx, part, nb, 2, r);
    out->re = r[0];
    out->im = r[1];
    return st;
}

template <typename A, typename B>
__global__ void __launch_bounds__(kRT) k_maxdiff(const A* __restrict__ a, const B* __restrict__ b, uint64_t n,
                                                double* partial) {
    __shared__ double sm[kRT / 32];
    double m = 0.0;
    GRID_STRIDE(i, n) {
        double2 x = to_d2(a[i]), y = to_d2(b[i]);
        m = fmax(m, fmax(fabs(x.x - y.x), fabs(x.y - y.y)));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmax(t, sm[w]);
        partial[blockIdx.x] = t;
    }
}

__global__ void k_final_max(const double* partial, int nb, double* out) {
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < nb; b++) t = fmax(t, partial[b]);
        out[0] = t;
    }
}

int reduce_max_abs_diff(Ctx* ctx, const Reg* a, const Reg* b, double* out) {
    uint64_t n = (uint64_t)1 << a->nbits;
    int nb = reduce_blocks(ctx, n);
    double* part;
    if (reduce_scratch(ctx, nb, 1, &part)) return YAO_ERR_OUT_OF_MEMORY;
    cudaStream_t s = ctx->stream;
    if (a->precision == YAO_C128 && b->precision == YAO_C128)
        k_maxdiff<double2, double2><<<nb, kRT, 0, s>>>((const double2*)a->d, (const double2*)b->d, n, part);
    else if (a->precision == YAO_C128)
        k_maxdiff<double2, float2><<<nb, kRT, 0, s>>>((const double2*)a->d, (const float2*)b->d, n, part);
    else if (b->precision == YAO_C128)
        k_maxdiff<float2, double2><<<nb, kRT, 0, s>>>((const float2*)a->d, (const double2*)b->d, n, part);
    else
        k_maxdiff<float2, float2><<<nb, kRT, 0, s>>>((const float2*)a->d, (const float2*)b->d, n, part);
    k_final_max<<<1, 32, 0, s>>>(part, nb, part + nb);
    ctx->launches += 2;
    YAO_CUDA(cudaGetLastError());
    if (ctx->ensure_host_pinned(sizeof(double))) return YAO_ERR_OUT_OF_MEMORY;
    YAO_CUDA(cudaMemcpyAsync(ctx->host_pinned, part + nb, sizeof(double), cudaMemcpyDeviceToHost, s));
    YAO_CUDA(cudaStreamSynchronize(s));
    memcpy(out, ctx->host_pinned, sizeof(double));
    return YAO_OK;
}

// ----------------------------------------------------- Pauli monomials

// Every yao-rs Op (I, X, Y, Z, P0, P1, Pu, Pd; src/operator.rs:53-65) has at
// most one non-zero entry per row, and each entry is 0, +-1 or +-i.  A
// product of them maps basis i to phase(i) * |i ^ xmask>, with phase(i) =
// i^(base + popc(i & d1) + 2 popc(i & d2)) when (i & need1) == need1 and
// (i & need0) == 0, else 0.  Applying one such op with instruct_1q (what
// expect.rs:26-36 does) yields exactly phase * psi[i ^ x] for finite inputs.

int build_mono_terms(const yao_term* terms, size_t nterms, uint32_t nbits, bool msb_first,
                     std::vector<MonoTerm>& out) {
    out.clear();
    for (size_t t = 0; t < nterms; t++) {
        const yao_term& tm = terms[t];
        // OperatorString::new: stable sort by site, drop I (src/operator.rs:27-33)
        std::vector<std::pair<uint32_t, int32_t>> ops;
        for (uint32_t i = 0; i < tm.nops; i++) {
            if (tm.ops[i] < YAO_OP_I || tm.ops[i] > YAO_OP_PD) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown Op");
            if (tm.sites[i] >= nbits) return fail(YAO_ERR_INVALID_ARGUMENT, "operator site out of range");
            ops.push_back({tm.sites[i], tm.ops[i]});
        }
        std::stable_sort(ops.begin(), ops.end(),
                         [](const std::pair<uint32_t, int32_t>& a, const std::pair<uint32_t, int32_t>& b) {
                             return a.first < b.first;
                         });
        // Per-site 2x2 matrix, each entry kept as (non-zero?, quarter turns).
        // Pure states (expect.rs:26-36) apply the ops of one site in order, a
        // matrix product with the later op on the left; expect_opstring_dm
        // (expect.rs:55-59) multiplies the ops' entries at the same
        // (row bit, column bit), an elementwise product.
        MonoTerm mt;
        mt.coeff = Cx{tm.coeff_re, tm.coeff_im};
        size_t i = 0;
        while (i < ops.size()) {
            uint32_t site = ops[i].first;
            int nzm[2][2], qm[2][2];
            bool first = true;
            for (; i < ops.size() && ops[i].first == site; i++) {
                int op = ops[i].second;
                if (op == YAO_OP_I) continue;  // dropped by OperatorString::new
                int onz[2][2] = {{0, 0}, {0, 0}}, oq[2][2] = {{0, 0}, {0, 0}};
                switch (op) {
                case YAO_OP_X: onz[0][1] = onz[1][0] = 1; break;
                case YAO_OP_Y: onz[0][1] = onz[1][0] = 1; oq[0][1] = 3; oq[1][0] = 1; break;
                case YAO_OP_Z: onz[0][0] = onz[1][1] = 1; oq[1][1] = 2; break;
                case YAO_OP_P0: onz[0][0] = 1; break;
                case YAO_OP_P1: onz[1][1] = 1; break;
                case YAO_OP_PU: onz[0][1] = 1; break;
                default: onz[1][0] = 1; break;  // Pd
                }
                if (first) {
                    memcpy(nzm, onz, sizeof nzm);
                    memcpy(qm, oq, sizeof qm);
                    first = false;
                } else if (msb_first) {
                    // new = op * old; op has at most one non-zero per row
                    int nn[2][2], nq[2][2];
                    for (int r = 0; r < 2; r++)
                        for (int c = 0; c < 2; c++) {
                            int k = onz[r][0] ? 0 : 1;
                            nn[r][c] = onz[r][k] && nzm[k][c];
                            nq[r][c] = (oq[r][k] + qm[k][c]) & 3;
                        }
                    memcpy(nzm, nn, sizeof nzm);
                    memcpy(qm, nq, sizeof qm);
                } else {
                    for (int r = 0; r < 2; r++)
                        for (int c = 0; c < 2; c++) {
                            nzm[r][c] = nzm[r][c] && onz[r][c];
                            qm[r][c] = (qm[r][c] + oq[r][c]) & 3;
                        }
                }
            }
            if (first) continue;  // only identities on this site
            // row form: row r -> (column, non-zero?, quarter turns)
            int col[2], nz[2], q[2];
            for (int r = 0; r < 2; r++) {
                int c = nzm[r][0] ? 0 : 1;
                col[r] = c;
                nz[r] = nzm[r][c];
                q[r] = qm[r][c];
            }
            uint32_t bit = msb_first ? (nbits - 1 - site) : site;
            uint64_t bm = (uint64_t)1 << bit;
            // the column of a non-zero row tells whether the site bit flips
            if (nz[0] ? (col[0] == 1) : (nz[1] && col[1] == 0)) mt.xmask |= bm;
            if (!nz[0] && !nz[1]) mt.zero = 1;
            if (!nz[0]) mt.need1 |= bm;
            if (!nz[1]) mt.need0 |= bm;
            mt.base = (mt.base + q[0]) & 3;
            int diff = (q[1] - q[0]) & 3;
            if (diff & 1) mt.d1mask |= bm;
            if (diff & 2) mt.d2mask |= bm;
        }
        out.push_back(mt);
    }
    return YAO_OK;
}

struct MonoDev {
    uint64_t d1, d2, need1, need0;
    int32_t base, zero;
};

__device__ __forceinline__ int mono_phase(const MonoDev& t, uint64_t i) {
    if (t.zero || (i & t.need1) != t.need1 || (i & t.need0) != 0) return -1;
    return (t.base + __popcll(i & t.d1) + 2 * __popcll(i & t.d2)) & 3;
}

// multiply by i^q exactly
__device__ __forceinline__ double2 qturn(double2 v, int q) {
    switch (q) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
    }
}

constexpr int kMaxGroupTerms = 8;
struct MonoGroup {
    uint64_t xmask;
    int32_t hbit;  // highest set bit of xmask (pairs are enumerated with it at 0)
    int32_t nt;
    MonoDev t[kMaxGroupTerms];
};

// <psi|O_t|psi> for up to 8 terms sharing one xmask, in one read of psi.
template <typename V>
__global__ void __launch_bounds__(kRT) k_expect_group(const V* __restrict__ st, uint64_t nwork, const MonoGroup grp,
                                                     double* partial) {
    __shared__ double sm[2 * kMaxGroupTerms * kRT / 32];
    double acc[2 * kMaxGroupTerms];
#pragma unroll
    for (int j = 0; j < 2 * kMaxGroupTerms; j++) acc[j] = 0.0;
    if (grp.xmask == 0) {
        GRID_STRIDE(i, nwork) {
            double2 v = to_d2(st[i]);
            double p = v.x * v.x + v.y * v.y;
#pragma unroll
            for (int t = 0; t < kMaxGroupTerms; t++) {
                if (t >= grp.nt) break;
                int q = mono_phase(grp.t[t], i);
                if (q < 0) continue;
                double2 c = qturn(make_double2(p, 0.0), q);
                acc[2 * t] += c.x;
                acc[2 * t + 1] += c.y;
            }
        }
    } else {
        const int h = grp.hbit;
        GRID_STRIDE(p, nwork) {
            uint64_t i = ((p >> h) << (h + 1)) | (p & ((1ull << h) - 1));
            uint64_t j = i ^ grp.xmask;
            double2 a = to_d2(st[i]), b = to_d2(st[j]);
            // c = conj(a) * b; conj(b) * a = conj(c)
            double2 c = make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
            double2 cc = make_double2(c.x, -c.y);
#pragma unroll
            for (int t = 0; t < kMaxGroupTerms; t++) {
                if (t >= grp.nt) break;
                int qi = mono_phase(grp.t[t], i), qj = mono_phase(grp.t[t], j);
                if (qi >= 0) {
                    double2 u = qturn(c, qi);
                    acc[2 * t] += u.x;
                    acc[2 * t + 1] += u.y;
                }
                if (qj >= 0) {
                    double2 u = qturn(cc, qj);
                    acc[2 * t] += u.x;
                    acc[2 * t + 1] += u.y;
                }
            }
        }
    }
    block_sum_write(acc, 2 * grp.nt, sm, partial + (size_t)blockIdx.x * 2 * grp.nt);
}

static MonoDev to_dev(const MonoTerm& m) {
    MonoDev d;
    d.d1 = m.d1mask;
    d.d2 = m.d2mask;
    d.need1 = m.need1;
    d.need0 = m.need0;
    d.base = m.base;
    d.zero = m.zero;
    return d;
}

// values[t] = <psi|O_t|psi> (without the coefficient), in two halves: the
// launch half groups the terms by X mask, runs one reduction per group into
// its own part of the scratch (partials, then the group's sums) and queues
// one copy of every group's sums into pinned host memory; the collect half,
// after the stream has passed that copy, reads them.  Nothing synchronises
// in between, so callers can queue more work before collecting.
int expect_terms_launch(Ctx* ctx, const Reg* r, const std::vector<MonoTerm>& terms, ExpectPending& pend) {
    pend.idx.clear();
    pend.nv.clear();
    pend.nterms = terms.size();
    const uint64_t n = (uint64_t)1 << r->nbits;
    std::vector<bool> done(terms.size(), false);
    std::vector<MonoGroup> groups;
    for (size_t t0 = 0; t0 < terms.size(); t0++) {
        if (done[t0]) continue;
        MonoGroup grp;
        memset(&grp, 0, sizeof(grp));
        grp.xmask = terms[t0].xmask;
        grp.hbit = grp.xmask ? 63 - __builtin_clzll(grp.xmask) : 0;
        for (size_t t = t0; t < terms.size() && grp.nt < kMaxGroupTerms; t++)
            if (!done[t] && terms[t].xmask == grp.xmask) {
                grp.t[grp.nt++] = to_dev(terms[t]);
                pend.idx.push_back(t);
                done[t] = true;
            }
        groups.push_back(grp);
        pend.nv.push_back(2 * grp.nt);
    }
    // scratch: every group's partials, then all groups' sums back to back
    size_t nres = 0, npart = 0;
    std::vector<int> nbs;
    for (const MonoGroup& grp : groups) {
        const int nb = reduce_blocks(ctx, grp.xmask ? n / 2 : n);
        nbs.push_back(nb);
        npart += (size_t)nb * 2 * grp.nt;
        nres += 2 * (size_t)grp.nt;
    }
    if (groups.empty()) return YAO_OK;
    if (ctx->ensure_scratch(sizeof(double) * (npart + nres))) return YAO_ERR_OUT_OF_MEMORY;
    if (ctx->ensure_host_pinned(sizeof(double) * nres)) return YAO_ERR_OUT_OF_MEMORY;
    double* part = (double*)ctx->scratch;
    double* res = part + npart;
    size_t po = 0, ro = 0;
    for (size_t g = 0; g < groups.size(); g++) {
        const MonoGroup& grp = groups[g];
        const uint64_t nwork = grp.xmask ? n / 2 : n;
        {
            ProfScope prof(ctx, "expect_group", (double)n * (r->precision == YAO_C128 ? 16.0 : 8.0));
            if (r->precision == YAO_C128)
                k_expect_group<double2><<<nbs[g], kRT, 0, ctx->stream>>>((const double2*)r->d, nwork, grp, part + po);
            else
                k_expect_group<float2><<<nbs[g], kRT, 0, ctx->stream>>>((const float2*)r->d, nwork, grp, part + po);
        }
        ctx->launches++;
        YAO_CUDA(cudaGetLastError());
        k_final_sum<<<1, kRT, 0, ctx->stream>>>(part + po, nbs[g], 2 * grp.nt, res + ro);
        ctx->launches++;
        YAO_CUDA(cudaGetLastError());
        po += (size_t)nbs[g] * 2 * grp.nt;
        ro += 2 * (size_t)grp.nt;
    }
    YAO_CUDA(cudaMemcpyAsync(ctx->host_pinned, res, sizeof(double) * nres, cudaMemcpyDeviceToHost, ctx->stream));
    return YAO_OK;
}

void expect_terms_collect(Ctx* ctx, const ExpectPending& pend, std::vector<Cx>& values) {
    values.assign(pend.nterms, Cx{0, 0});
    const double* h = (const double*)ctx->host_pinned;
    size_t k = 0, o = 0;
    for (int nv : pend.nv) {
        for (int q = 0; q < nv / 2; q++, k++) values[pend.idx[k]] = Cx{h[o + 2 * q], h[o + 2 * q + 1]};
        o += (size_t)nv;
    }
}

int expect_terms(Ctx* ctx, const Reg* r, const std::vector<MonoTerm>& terms, std::vector<Cx>& values) {
    ExpectPending pend;
    int s = expect_terms_launch(ctx, r, terms, pend);
    if (s) return s;
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    expect_terms_collect(ctx, pend, values);
    return YAO_OK;
}

// lambda = sum_t c_t O_t psi  (ad.rs:98-117), per amplitude in term order:
// acc = 0; acc += c_t * (O_t psi)[i].  (O_t psi)[i] is exact, so lambda is
// bit-identical to the CPU path's.
struct MonoFull {
    MonoDev t;
    uint64_t xmask;
    double2 c;
};

// i^q * v for q in 0..3 without branches (the same values as qturn: every
// step is a swap or a negation, exact)
__device__ __forceinline__ double2 qturn_sel(double2 v, int q) {
    const double2 w = (q & 1) ? make_double2(-v.y, v.x) : v;
    return (q & 2) ? make_double2(-w.x, -w.y) : w;
}

// Each thread builds kLamR amplitudes of lambda (256 apart, coalesced), so a
// term's fields are read once per kLamR amplitudes.  PAULI: every term is a
// Pauli string (factors I, X, Y, Z), whose phase at index i is
// i^(base + 2 popc(i & d2)) (no projector masks, no quarter-turn mask).
// ENERGY: also Re <psi | lambda> = <psi|H|psi>.re (ad.rs:87) per block, in
// the block's fixed order, into partial[blockIdx.x].
constexpr int kLamR = 4;
template <bool PAULI, bool ENERGY>
__global__ void __launch_bounds__(kRT) k_lambda(const double2* __restrict__ psi, double2* __restrict__ lam, uint64_t n,
                                               const MonoFull* __restrict__ terms, int nt,
                                               double* __restrict__ partial) {
    __shared__ double sm[kRT / 32];
    double e = 0.0;
    const uint64_t span = (uint64_t)kRT * kLamR;
    const uint64_t nchunks = (n + span - 1) / span;
    for (uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        uint64_t idx[kLamR];
        double2 acc[kLamR];
#pragma unroll
        for (int k = 0; k < kLamR; k++) {
            idx[k] = ch * span + (uint64_t)k * kRT + threadIdx.x;
            acc[k] = make_double2(0.0, 0.0);
        }
        for (int t = 0; t < nt; t++) {
            const MonoFull m = terms[t];
#pragma unroll
            for (int k = 0; k < kLamR; k++) {
                if (idx[k] >= n) continue;
                const uint64_t i = idx[k];
                double2 v;
                if (PAULI) {
                    v = qturn_sel(psi[i ^ m.xmask], (m.t.base + 2 * __popcll(i & m.t.d2)) & 3);
                } else {
                    const int q = mono_phase(m.t, i);
                    v = q >= 0 ? qturn_sel(psi[i ^ m.xmask], q) : make_double2(0.0, 0.0);
                }
                acc[k] = cadd_x(acc[k], cmul_x(m.c, v));
            }
        }
#pragma unroll
        for (int k = 0; k < kLamR; k++) {
            if (idx[k] >= n) continue;
            lam[idx[k]] = acc[k];
            if (ENERGY) {
                const double2 p = psi[idx[k]];
                e += p.x * acc[k].x + p.y * acc[k].y;
            }
        }
    }
    if (ENERGY) block_sum_write(&e, 1, sm, partial + blockIdx.x);
}

int build_lambda(Ctx* ctx, const Reg* psi, const std::vector<MonoTerm>& terms, Reg* lambda) {
    return build_lambda_sets(ctx, psi->d, lambda->d, psi->nbits, 1, terms);
}

// nsets registers back to back: every mask lies below the register-index
// bits, so one pass over all nsets * 2^nbits amplitudes builds every lambda.
// With `energy`, one register (nsets == 1): Re <psi|lambda> is reduced in the
// same pass, its final sum queued for a copy into ctx->host_pinned[0]
// (read it after the stream has passed the copy: lambda_energy_collect).
static int lambda_launch(Ctx* ctx, const void* psi_d, void* lam_d, uint32_t nbits, uint64_t nsets,
                         const std::vector<MonoTerm>& terms, bool energy) {
    const uint64_t n = nsets << nbits;
    std::vector<MonoFull> h(terms.size());
    bool pauli = true;
    for (size_t t = 0; t < terms.size(); t++) {
        h[t].t = to_dev(terms[t]);
        h[t].xmask = terms[t].xmask;
        h[t].c = make_double2(terms[t].coeff.re, terms[t].coeff.im);
        const MonoDev& d = h[t].t;
        pauli = pauli && d.d1 == 0 && d.need0 == 0 && d.need1 == 0 && d.zero == 0;
    }
    void* d = nullptr;
    size_t bytes = std::max<size_t>(1, h.size()) * sizeof(MonoFull);
    YAO_CUDA(cudaMallocAsync(&d, bytes, ctx->stream));
    if (!h.empty()) YAO_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(MonoFull), cudaMemcpyHostToDevice, ctx->stream));
    const unsigned grid = grid_for((n + kLamR - 1) / kLamR, kRT, ctx->num_sms);
    double* part = nullptr;
    if (energy) {
        if (ctx->ensure_scratch(sizeof(double) * (grid + 1)) || ctx->ensure_host_pinned(sizeof(double))) {
            cudaFreeAsync(d, ctx->stream);
            return YAO_ERR_OUT_OF_MEMORY;
        }
        part = (double*)ctx->scratch;
    }
    {
        // reads psi once per distinct X mask (the low ones hit L2), writes lambda
        ProfScope prof(ctx, "lambda", (double)n * 32.0);
        const double2* ps = (const double2*)psi_d;
        double2* ls = (double2*)lam_d;
        const MonoFull* td = (const MonoFull*)d;
        const int nt = (int)h.size();
        if (pauli && energy)
            k_lambda<true, true><<<grid, kRT, 0, ctx->stream>>>(ps, ls, n, td, nt, part);
        else if (pauli)
            k_lambda<true, false><<<grid, kRT, 0, ctx->stream>>>(ps, ls, n, td, nt, part);
        else if (energy)
            k_lambda<false, true><<<grid, kRT, 0, ctx->stream>>>(ps, ls, n, td, nt, part);
        else
            k_lambda<false, false><<<grid, kRT, 0, ctx->stream>>>(ps, ls, n, td, nt, part);
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaFreeAsync(d, ctx->stream));
    if (energy) {
        k_final_sum<<<1, kRT, 0, ctx->stream>>>(part, (int)grid, 1, part + grid);
        ctx->launches++;
        YAO_CUDA(cudaGetLastError());
        YAO_CUDA(cudaMemcpyAsync(ctx->host_pinned, part + grid, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    return YAO_OK;
}

int build_lambda_sets(Ctx* ctx, const void* psi_d, void* lam_d, uint32_t nbits, uint64_t nsets,
                      const std::vector<MonoTerm>& terms) {
    return lambda_launch(ctx, psi_d, lam_d, nbits, nsets, terms, false);
}

int build_lambda_energy(Ctx* ctx, const Reg* psi, const std::vector<MonoTerm>& terms, Reg* lambda) {
    return lambda_launch(ctx, psi->d, lambda->d, psi->nbits, 1, terms, true);
}

double lambda_energy_collect(Ctx* ctx) { return ((const double*)ctx->host_pinned)[0]; }

// ------------------------------------------------------------- adjoint

// One fused reverse-sweep step for a parametric gate (ad.rs:121-152): for
// every group the gate touches (controls matching, targets at 0) read psi
// and lambda once, accumulate <lambda | G_p psi> for each generator G_p
// (dense product as in apply_generator, which yao-rs restricts to the
// control-matching branch, ad.rs:56-64), then write U^dagger psi and
// U^dagger lambda with the PLAIN arithmetic.
struct AdjOp {
    int32_t k, ngen, dagcls, nlocked;
    uint64_t cval, dag_active;
    int8_t locked[64];
    uint64_t off[4];
    double2 gen[2][16];
    double2 dag[16];
};

template <int K>
__global__ void __launch_bounds__(kRT) k_adjoint(double2* __restrict__ psi, double2* __restrict__ lam, uint64_t ngroups,
                                                const AdjOp op, double* partial) {
    constexpr int NL = 1 << K;
    __shared__ double sm[4 * kRT / 32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    GRID_STRIDE(g, ngroups) {
        uint64_t base = insert_zeros(g, op.locked, op.nlocked) | op.cval;
        double2 x[NL], l[NL];
#pragma unroll
        for (int q = 0; q < NL; q++) {
            x[q] = psi[base + op.off[q]];
            l[q] = lam[base + op.off[q]];
        }
        for (int p = 0; p < op.ngen; p++) {
#pragma unroll
            for (int r = 0; r < NL; r++) {
                double2 y;
                if (K == 1) {
                    y = cadd_x(cmul_x(op.gen[p][r * 2], x[0]), cmul_x(op.gen[p][r * 2 + 1], x[1]));
                } else {
                    y = make_double2(0.0, 0.0);
#pragma unroll
                    for (int c = 0; c < NL; c++) y = cadd_x(y, cmul_x(op.gen[p][r * NL + c], x[c]));
                }
                // conj(lambda) * y
                acc[2 * p] += l[r].x * y.x + l[r].y * y.y;
                acc[2 * p + 1] += l[r].x * y.y - l[r].y * y.x;
            }
        }
        // U^dagger on both states
        if (op.dagcls == GC_DIAG) {
#pragma unroll
            for (int q = 0; q < NL; q++)
                if ((op.dag_active >> q) & 1) {
                    psi[base + op.off[q]] = cmulassign_x(x[q], op.dag[q]);
                    lam[base + op.off[q]] = cmulassign_x(l[q], op.dag[q]);
                }
        } else if (K == 1) {
            psi[base + op.off[0]] = cadd_x(cmul_x(op.dag[0], x[0]), cmul_x(op.dag[1], x[1]));
            psi[base + op.off[1]] = cadd_x(cmul_x(op.dag[2], x[0]), cmul_x(op.dag[3], x[1]));
            lam[base + op.off[0]] = cadd_x(cmul_x(op.dag[0], l[0]), cmul_x(op.dag[1], l[1]));
            lam[base + op.off[1]] = cadd_x(cmul_x(op.dag[2], l[0]), cmul_x(op.dag[3], l[1]));
        } else {
#pragma unroll
            for (int r = 0; r < NL; r++) {
                double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < NL; c++) {
                    a = cadd_x(a, cmul_x(op.dag[r * NL + c], x[c]));
                    b = cadd_x(b, cmul_x(op.dag[r * NL + c], l[c]));
                }
                psi[base + op.off[r]] = a;
                lam[base + op.off[r]] = b;
            }
        }
    }
    block_sum_write(acc, 2 * op.ngen, sm, partial + (size_t)blockIdx.x * 2 * op.ngen);
}

// gen: up to two generator gates (same targets/controls as dag); dag: the
// lowered adjoint (one LGate).  dot_out receives ngen complex dots.
int adjoint_step(Ctx* ctx, Reg* psi, Reg* lambda, const LGate* gen, const std::vector<LGate>& dag, Cx* dot_out) {
    int ngen = 0;
    while (ngen < 2 && gen[ngen].k > 0) ngen++;
    const LGate& d = dag[0];
    if (dag.size() != 1 || d.k > 2 || (d.cls != GC_DIAG && d.cls != GC_DENSE) || gen[0].k != d.k)
        return fail(YAO_ERR_UNSUPPORTED, "adjoint step supports 1- and 2-qubit parametric gates");
    AdjOp op;
    memset(&op, 0, sizeof(op));
    op.k = d.k;
    op.ngen = ngen;
    op.dagcls = d.cls;
    std::vector<int> pos;
    for (int i = 0; i < d.k; i++) pos.push_back(d.tb[i]);
    for (int i = 0; i < d.nc; i++) pos.push_back(d.cb[i]);
    std::sort(pos.begin(), pos.end());
    op.nlocked = (int)pos.size();
    for (size_t i = 0; i < pos.size(); i++) op.locked[i] = (int8_t)pos[i];
    op.cval = d.cval();
    int nl = 1 << d.k;
    for (int l = 0; l < nl; l++) {
        uint64_t off = 0;
        for (int i = 0; i < d.k; i++) off |= (uint64_t)((l >> i) & 1) << d.tb[i];
        op.off[l] = off;
    }
    for (int p = 0; p < ngen; p++)
        for (size_t i = 0; i < gen[p].m.size() && i < 16; i++) op.gen[p][i] = make_double2(gen[p].m[i].re, gen[p].m[i].im);
    for (size_t i = 0; i < d.m.size() && i < 16; i++) op.dag[i] = make_double2(d.m[i].re, d.m[i].im);
    if (d.cls == GC_DIAG)
        for (int l = 0; l < nl; l++)
            if (!(d.m[l].re == 1.0 && d.m[l].im == 0.0)) op.dag_active |= (uint64_t)1 << l;
    uint64_t ngroups = (uint64_t)1 << (psi->nbits - op.nlocked);
    int nb = reduce_blocks(ctx, ngroups);
    double* part;
    if (reduce_scratch(ctx, nb, 2 * ngen, &part)) return YAO_ERR_OUT_OF_MEMORY;
    {
        ProfScope prof(ctx, "adjoint_step", (double)ngroups * nl * 4.0 * 16.0);
        if (d.k == 1)
            k_adjoint<1><<<nb, kRT, 0, ctx->stream>>>((double2*)psi->d, (double2*)lambda->d, ngroups, op, part);
        else
            k_adjoint<2><<<nb, kRT, 0, ctx->stream>>>((double2*)psi->d, (double2*)lambda->d, ngroups, op, part);
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    std::vector<double> res(2 * ngen);
    int s = finish_sum(ctx, part, nb, 2 * ngen, res.data());
    for (int p = 0; p < ngen; p++) dot_out[p] = Cx{res[2 * p], res[2 * p + 1]};
    return s;
}

// ------------------------------------------------------- probabilities

// |amp|^2 = re*re + im*im (norm_sqr), without FMA contraction: bit-identical
// to the CPU path (src/measure.rs:40-42).
template <typename V>
__global__ void k_probs_full(const V* __restrict__ st, double* __restrict__ out, uint64_t n) {
    GRID_STRIDE(i, n) {
        double2 v = to_d2(st[i]);
        out[i] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
    }
}

int launch_probs_full(Ctx* ctx, const Reg* r, double* dprobs) {
    uint64_t n = (uint64_t)1 << r->nbits;
    unsigned g = grid_for(n, 256, ctx->num_sms);
    if (r->precision == YAO_C128)
        k_probs_full<double2><<<g, 256, 0, ctx->stream>>>((const double2*)r->d, dprobs, n);
    else
        k_probs_full<float2><<<g, 256, 0, ctx->stream>>>((const float2*)r->d, dprobs, n);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// Marginal over the bit positions bits[0..nl) (bits[0] is the outcome MSB,
// src/measure.rs:89-104).  Block (o, s) sums split s of outcome o's members.
struct MargSpec {
    int32_t nl, nfree, splits, pad;
    int8_t bits[64];   // outcome bit j (LSB first) -> state bit
    int8_t sorted[64]; // measured bits ascending (for insert_zeros)
};

template <typename V>
__global__ void __launch_bounds__(kRT) k_marginal(const V* __restrict__ st, const MargSpec ms, uint64_t per_split,
                                                 double* partial) {
    __shared__ double sm[kRT / 32];
    const uint64_t o = blockIdx.x / ms.splits, s = blockIdx.x % ms.splits;
    uint64_t obits = 0;
    for (int j = 0; j < ms.nl; j++) obits |= ((o >> j) & 1) << ms.bits[j];
    const uint64_t nfree = 1ull << ms.nfree;
    const uint64_t lo = s * per_split, hi = min(nfree, lo + per_split);
    double acc = 0.0;
    for (uint64_t f = lo + threadIdx.x; f < hi; f += blockDim.x) {
        uint64_t i = insert_zeros(f, ms.sorted, ms.nl) | obits;
        double2 v = to_d2(st[i]);
        acc += v.x * v.x + v.y * v.y;
    }
    block_sum_write(&acc, 1, sm, partial + blockIdx.x);
}

__global__ void k_marginal_final(const double* __restrict__ partial, int splits, uint64_t nout, double* out) {
    GRID_STRIDE(o, nout) {
        double s = 0.0;
        for (int q = 0; q < splits; q++) s += partial[o * splits + q];
        out[o] = s;
    }
}

int reduce_marginal(Ctx* ctx, const Reg* r, const uint32_t* bits, uint32_t nl, double* host_out) {
    MargSpec ms;
    memset(&ms, 0, sizeof(ms));
    ms.nl = (int)nl;
    ms.nfree = (int)(r->nbits - nl);
    std::vector<int> srt;
    for (uint32_t j = 0; j < nl; j++) {
        ms.bits[j] = (int8_t)bits[nl - 1 - j];  // outcome bit j (LSB first) <- locs[nl-1-j]
        srt.push_back((int)bits[j]);
    }
    std::sort(srt.begin(), srt.end());
    for (size_t j = 0; j < srt.size(); j++) ms.sorted[j] = (int8_t)srt[j];
    uint64_t nout = (uint64_t)1 << nl, nfree = (uint64_t)1 << ms.nfree;
    uint64_t target_blocks = (uint64_t)ctx->num_sms * 8;
    uint64_t splits = std::max<uint64_t>(1, std::min<uint64_t>(target_blocks / nout, (nfree + kRT - 1) / kRT));
    ms.splits = (int32_t)splits;
    uint64_t per_split = (nfree + splits - 1) / splits;
    uint64_t nb = nout * splits;
    if (nb > (1ull << 31)) return fail(YAO_ERR_UNSUPPORTED, "too many marginal outcomes");
    size_t bytes = sizeof(double) * (nb + nout);
    if (ctx->ensure_scratch(bytes)) return YAO_ERR_OUT_OF_MEMORY;
    double* part = (double*)ctx->scratch;
    double* dout = part + nb;
    if (r->precision == YAO_C128)
        k_marginal<double2><<<(unsigned)nb, kRT, 0, ctx->stream>>>((const double2*)r->d, ms, per_split, part);
    else
        k_marginal<float2><<<(unsigned)nb, kRT, 0, ctx->stream>>>((const float2*)r->d, ms, per_split, part);
    k_marginal_final<<<grid_for(nout, 256, ctx->num_sms), 256, 0, ctx->stream>>>(part, ms.splits, nout, dout);
    ctx->launches += 2;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaMemcpyAsync(host_out, dout, sizeof(double) * nout, cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    return YAO_OK;
}

// collapse_qubits_to (src/measure.rs:158-185), first half: zero the
// amplitudes that disagree with the outcome, sum |amp|^2 of the others.
template <typename V>
__global__ void __launch_bounds__(kRT) k_collapse(V* __restrict__ st, uint64_t n, uint64_t mask, uint64_t value,
                                                 double* partial) {
    __shared__ double sm[kRT / 32];
    double acc = 0.0;
    GRID_STRIDE(i, n) {
        if ((i & mask) == value) {
            double2 v = to_d2(st[i]);
            acc += v.x * v.x + v.y * v.y;
        } else {
            st[i] = from_d2<V>(make_double2(0.0, 0.0));
        }
    }
    block_sum_write(&acc, 1, sm, partial + blockIdx.x);
}

int launch_collapse(Ctx* ctx, Reg* r, uint64_t mask, uint64_t value, double* norm_sq_out) {
    uint64_t n = (uint64_t)1 << r->nbits;
    int nb = reduce_blocks(ctx, n);
    double* part;
    if (reduce_scratch(ctx, nb, 1, &part)) return YAO_ERR_OUT_OF_MEMORY;
    if (r->precision == YAO_C128)
        k_collapse<double2><<<nb, kRT, 0, ctx->stream>>>((double2*)r->d, n, mask, value, part);
    else
        k_collapse<float2><<<nb, kRT, 0, ctx->stream>>>((float2*)r->d, n, mask, value, part);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return finish_sum(ctx, part, nb, 1, norm_sq_out);
}

// reset_qubits_to (src/measure.rs:187-215): move every amplitude of the
// measured pattern to the reset pattern.
template <typename V>
__global__ void k_reset_move(V* st, uint64_t n, uint64_t mask, uint64_t value, uint64_t swap) {
    GRID_STRIDE(i, n) {
        if ((i & mask) != value) continue;
        st[i ^ swap] = st[i];
        st[i] = from_d2<V>(make_double2(0.0, 0.0));
    }
}

int launch_reset_move(Ctx* ctx, Reg* r, uint64_t mask, uint64_t value, uint64_t swap_mask) {
    uint64_t n = (uint64_t)1 << r->nbits;
    unsigned g = grid_for(n, 256, ctx->num_sms);
    if (r->precision == YAO_C128)
        k_reset_move<double2><<<g, 256, 0, ctx->stream>>>((double2*)r->d, n, mask, value, swap_mask);
    else
        k_reset_move<float2><<<g, 256, 0, ctx->stream>>>((float2*)r->d, n, mask, value, swap_mask);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// remove_measured_qubits (src/measure.rs:217-240): gather the kept bits
// (kept[0] is the MSB of the new index); |amp|^2 < 1e-30 counts as 0.
struct KeepSpec {
    int32_t nk, pad;
    int8_t kept[64];  // new bit j (LSB first) <- old bit
};

template <typename V>
__global__ void k_remove_gather(const V* __restrict__ src, V* __restrict__ dst, uint64_t n_new, uint64_t fixed,
                                const KeepSpec ks) {
    GRID_STRIDE(nb, n_new) {
        uint64_t i = fixed;
        for (int j = 0; j < ks.nk; j++) i |= ((nb >> j) & 1) << ks.kept[j];
        double2 v = to_d2(src[i]);
        if (v.x * v.x + v.y * v.y < 1e-30) v = make_double2(0.0, 0.0);
        dst[nb] = from_d2<V>(v);
    }
}

int launch_remove_gather_fixed(Ctx* ctx, const Reg* src, Reg* dst, const uint32_t* kept_bits, uint32_t nk,
                               uint64_t fixed) {
    KeepSpec ks;
    memset(&ks, 0, sizeof(ks));
    ks.nk = (int)nk;
    for (uint32_t j = 0; j < nk; j++) ks.kept[j] = (int8_t)kept_bits[nk - 1 - j];
    uint64_t n_new = (uint64_t)1 << nk;
    unsigned g = grid_for(n_new, 256, ctx->num_sms);
    if (src->precision == YAO_C128)
        k_remove_gather<double2><<<g, 256, 0, ctx->stream>>>((const double2*)src->d, (double2*)dst->d, n_new, fixed, ks);
    else
        k_remove_gather<float2><<<g, 256, 0, ctx->stream>>>((const float2*)src->d, (float2*)dst->d, n_new, fixed, ks);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// ============================================ expectation without allocation
//
// yao_expect_arrayreg_noalloc computes the same value as yao_expect_arrayreg
// but allocates nothing: no cudaMalloc / cudaMallocHost / cudaFree and no
// heap memory on the normal path.  Its reduction partials live in the
// file-scope device array below (every GPU that loads the library holds it
// until the process exits), the operator terms are converted into fixed-size
// arrays on the stack, and the result is copied straight into the caller's
// host memory.
//
// Limits: at most kNoAllocMaxTerms terms and kNoAllocMaxOps ops per term;
// larger inputs are rejected with YAO_ERR_INVALID_ARGUMENT.  The register
// size is not limited: a reduction uses at most kNoAllocBlocks blocks.
//
// All calls share the array.  Every call writes each partial it reads
// before reading it, so nothing has to start at zero; but two calls that
// overlap on the GPU (different streams or threads at the same time) race
// on the array and must be serialised by the caller.

constexpr int kNoAllocBlocks = 1024;
constexpr int kNoAllocValues = 2 * kMaxGroupTerms;
constexpr size_t kNoAllocDoubles = (size_t)kNoAllocBlocks * kNoAllocValues + kNoAllocValues;  // 131,200 bytes
constexpr int kNoAllocMaxTerms = 64;
constexpr int kNoAllocMaxOps = 64;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Device address of g_noalloc_scratch on each device (host code cannot use
// the symbol itself as a pointer).  The caller makes `device` current before
// the lookup.  Only a successful lookup is kept: a lookup that failed (for
// instance because it was made inside a stream capture) is tried again on
// the next call.
static double* g_noalloc_ptr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(int device, double** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(YAO_ERR_INVALID_ARGUMENT, "device index too large");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        double* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return YAO_OK;
}

// One term to a Pauli monomial (the same rules as build_mono_terms, pure-state
// site order), using only the caller's fixed arrays.
static int noalloc_term(const yao_term& tm, uint32_t nbits, MonoTerm& mt) {
    if (tm.nops > (uint32_t)kNoAllocMaxOps)
        return fail(YAO_ERR_INVALID_ARGUMENT, "noalloc expectation: more than 64 ops in one term");
    uint32_t sites[kNoAllocMaxOps];
    int32_t ops[kNoAllocMaxOps];
    uint32_t n = 0;
    for (uint32_t i = 0; i < tm.nops; i++) {
        if (tm.ops[i] < YAO_OP_I || tm.ops[i] > YAO_OP_PD) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown Op");
        if (tm.sites[i] >= nbits) return fail(YAO_ERR_INVALID_ARGUMENT, "operator site out of range");
        if (tm.ops[i] == YAO_OP_I) continue;  // dropped by OperatorString::new
        // stable insertion by site (OperatorString::new sorts by site)
        uint32_t j = n++;
        while (j > 0 && sites[j - 1] > tm.sites[i]) {
            sites[j] = sites[j - 1];
            ops[j] = ops[j - 1];
            j--;
        }
        sites[j] = tm.sites[i];
        ops[j] = tm.ops[i];
    }
    mt = MonoTerm();
    mt.coeff = Cx{tm.coeff_re, tm.coeff_im};
    uint32_t i = 0;
    while (i < n) {
        uint32_t site = sites[i];
        int nzm[2][2] = {{1, 0}, {0, 1}}, qm[2][2] = {{0, 0}, {0, 0}};
        for (; i < n && sites[i] == site; i++) {
            int onz[2][2] = {{0, 0}, {0, 0}}, oq[2][2] = {{0, 0}, {0, 0}};
            switch (ops[i]) {
            case YAO_OP_X: onz[0][1] = onz[1][0] = 1; break;
            case YAO_OP_Y: onz[0][1] = onz[1][0] = 1; oq[0][1] = 3; oq[1][0] = 1; break;
            case YAO_OP_Z: onz[0][0] = onz[1][1] = 1; oq[1][1] = 2; break;
            case YAO_OP_P0: onz[0][0] = 1; break;
            case YAO_OP_P1: onz[1][1] = 1; break;
            case YAO_OP_PU: onz[0][1] = 1; break;
            default: onz[1][0] = 1; break;
            }
            int nn[2][2], nq[2][2];  // op * accumulated
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 2; c++) {
                    int k = onz[r][0] ? 0 : 1;
                    nn[r][c] = onz[r][k] && nzm[k][c];
                    nq[r][c] = (oq[r][k] + qm[k][c]) & 3;
                }
            memcpy(nzm, nn, sizeof nzm);
            memcpy(qm, nq, sizeof qm);
        }
        int col[2], nz[2], q[2];
        for (int r = 0; r < 2; r++) {
            int c = nzm[r][0] ? 0 : 1;
            col[r] = c;
            nz[r] = nzm[r][c];
            q[r] = qm[r][c];
        }
        uint64_t bm = (uint64_t)1 << (nbits - 1 - site);
        if (nz[0] ? (col[0] == 1) : (nz[1] && col[1] == 0)) mt.xmask |= bm;
        if (!nz[0] && !nz[1]) mt.zero = 1;
        if (!nz[0]) mt.need1 |= bm;
        if (!nz[1]) mt.need0 |= bm;
        mt.base = (mt.base + q[0]) & 3;
        int diff = (q[1] - q[0]) & 3;
        if (diff & 1) mt.d1mask |= bm;
        if (diff & 2) mt.d2mask |= bm;
    }
    return YAO_OK;
}

int expect_noalloc(Ctx* ctx, const Reg* r, const yao_term* terms, size_t nterms, double* out) {
    if (nterms > (size_t)kNoAllocMaxTerms)
        return fail(YAO_ERR_INVALID_ARGUMENT, "noalloc expectation: more than 64 terms");
    if (nterms && !terms) return fail(YAO_ERR_INVALID_ARGUMENT, "null terms");
    double* scratch = nullptr;
    int s = noalloc_scratch(ctx->device, &scratch);
    if (s) return s;
    MonoTerm mt[kNoAllocMaxTerms];
    for (size_t t = 0; t < nterms; t++) {
        s = noalloc_term(terms[t], r->nbits, mt[t]);
        if (s) return s;
    }
    Cx values[kNoAllocMaxTerms];
    bool done[kNoAllocMaxTerms] = {false};
    const uint64_t n = (uint64_t)1 << r->nbits;
    for (size_t t0 = 0; t0 < nterms; t0++) {
        if (done[t0]) continue;
        MonoGroup grp;
        memset(&grp, 0, sizeof(grp));
        grp.xmask = mt[t0].xmask;
        grp.hbit = grp.xmask ? 63 - __builtin_clzll(grp.xmask) : 0;
        size_t idx[kMaxGroupTerms];
        int cnt = 0;
        for (size_t t = t0; t < nterms && cnt < kMaxGroupTerms; t++)
            if (!done[t] && mt[t].xmask == grp.xmask) {
                grp.t[cnt] = to_dev(mt[t]);
                idx[cnt++] = t;
                done[t] = true;
            }
        grp.nt = cnt;
        const int nv = 2 * cnt;
        const uint64_t nwork = grp.xmask ? n / 2 : n;
        const int nb = std::min(reduce_blocks(ctx, nwork), kNoAllocBlocks);
        if (r->precision == YAO_C128)
            k_expect_group<double2><<<nb, kRT, 0, ctx->stream>>>((const double2*)r->d, nwork, grp, scratch);
        else
            k_expect_group<float2><<<nb, kRT, 0, ctx->stream>>>((const float2*)r->d, nwork, grp, scratch);
        double* dres = scratch + (size_t)nb * nv;
        k_final_sum<<<1, kRT, 0, ctx->stream>>>(scratch, nb, nv, dres);
        ctx->launches += 2;
        YAO_CUDA(cudaGetLastError());
        double res[kNoAllocValues];
        YAO_CUDA(cudaMemcpyAsync(res, dres, sizeof(double) * nv, cudaMemcpyDeviceToHost, ctx->stream));
        YAO_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int q = 0; q < cnt; q++) values[idx[q]] = Cx{res[2 * q], res[2 * q + 1]};
    }
    // sum_t coeff_t * value_t in term order (src/expect.rs:7-11)
    double re = 0.0, im = 0.0;
    for (size_t t = 0; t < nterms; t++) {
        Cx c = mt[t].coeff, v = values[t];
        re += c.re * v.re - c.im * v.im;
        im += c.re * v.im + c.im * v.re;
    }
    out[0] = re;
    out[1] = im;
    return YAO_OK;
}

// ------------------------------------------------ batched norm restore
// FUSED complex64 batches: every register's squared norm in two launches
// (chunk partials, then each register's partials in chunk order), and one
// launch that divides each register by sqrt(n1 / n0).  Deterministic like the
// single-register reductions; nothing returns to the host.

constexpr uint32_t kNormChunk = 1u << 16;  // amplitudes per chunk

struct NormChunk {
    uint64_t p;     // first amplitude of the chunk
    uint32_t len;   // amplitudes in the chunk
    uint32_t slot;  // index of the register's norm
};

template <typename V>
__global__ void __launch_bounds__(kRT) k_chunk_norm_sqr(const NormChunk* __restrict__ ch, double* __restrict__ part) {
    __shared__ double sm[kRT / 32];
    const NormChunk c = ch[blockIdx.x];
    const V* st = (const V*)(uintptr_t)c.p;
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < c.len; i += blockDim.x) {
        double2 v = to_d2(st[i]);
        acc += v.x * v.x + v.y * v.y;
    }
    block_sum_write(&acc, 1, sm, part + blockIdx.x);
}

__global__ void __launch_bounds__(kRT) k_slot_sums(const uint32_t* __restrict__ first, uint32_t nslots,
                                                   const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sm[kRT / 32];
    for (uint32_t r = blockIdx.x; r < nslots; r += gridDim.x) {
        double acc = 0.0;
        for (uint32_t i = first[r] + threadIdx.x; i < first[r + 1]; i += blockDim.x) acc += part[i];
        block_sum_write(&acc, 1, sm, out + r);
    }
}

template <typename V>
__global__ void __launch_bounds__(kRT) k_chunk_rescale(const NormChunk* __restrict__ ch, const double* __restrict__ n0,
                                                       const double* __restrict__ n1) {
    const NormChunk c = ch[blockIdx.x];
    const double a = n0[c.slot], b = n1[c.slot];
    if (!(a > 0.0 && b > 0.0)) return;
    const double d = sqrt(b / a);
    V* st = (V*)(uintptr_t)c.p;
    for (uint32_t i = threadIdx.x; i < c.len; i += blockDim.x) {
        double2 v = to_d2(st[i]);
        st[i] = from_d2<V>(make_double2(__ddiv_rn(v.x, d), __ddiv_rn(v.y, d)));
    }
}

static void norm_chunks(const std::vector<Reg*>& regs, std::vector<NormChunk>& ch, std::vector<uint32_t>& first) {
    first.assign(1, 0);
    for (size_t s = 0; s < regs.size(); s++) {
        const uint64_t n = (uint64_t)1 << regs[s]->nbits, es = regs[s]->precision == YAO_C128 ? 16 : 8;
        for (uint64_t o = 0; o < n; o += kNormChunk)
            ch.push_back(NormChunk{(uint64_t)(uintptr_t)regs[s]->d + o * es, (uint32_t)std::min<uint64_t>(kNormChunk, n - o),
                                   (uint32_t)s});
        first.push_back((uint32_t)ch.size());
    }
}

// out[s] (device) = squared norm of regs[s]; all registers share one precision
int launch_batch_norm_sqr(Ctx* ctx, const std::vector<Reg*>& regs, double* out) {
    if (regs.empty()) return YAO_OK;
    std::vector<NormChunk> ch;
    std::vector<uint32_t> first;
    norm_chunks(regs, ch, first);
    const size_t b_ch = (ch.size() * sizeof(NormChunk) + 255) / 256 * 256,
                 b_first = (first.size() * sizeof(uint32_t) + 255) / 256 * 256;
    char* buf = nullptr;
    YAO_CUDA(cudaMallocAsync((void**)&buf, b_ch + b_first + ch.size() * sizeof(double), ctx->stream));
    NormChunk* d_ch = (NormChunk*)buf;
    uint32_t* d_first = (uint32_t*)(buf + b_ch);
    double* d_part = (double*)(buf + b_ch + b_first);
    YAO_CUDA(cudaMemcpyAsync(d_ch, ch.data(), ch.size() * sizeof(NormChunk), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(d_first, first.data(), first.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    if (regs[0]->precision == YAO_C128)
        k_chunk_norm_sqr<double2><<<(unsigned)ch.size(), kRT, 0, ctx->stream>>>(d_ch, d_part);
    else
        k_chunk_norm_sqr<float2><<<(unsigned)ch.size(), kRT, 0, ctx->stream>>>(d_ch, d_part);
    const unsigned g = (unsigned)std::min<size_t>(regs.size(), (size_t)ctx->num_sms * 8);
    k_slot_sums<<<g, kRT, 0, ctx->stream>>>(d_first, (uint32_t)regs.size(), d_part, out);
    ctx->launches += 2;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaFreeAsync(buf, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    return YAO_OK;
}

// regs[s] /= sqrt(n1[s] / n0[s]) where both are positive (device arrays)
int launch_batch_rescale(Ctx* ctx, const std::vector<Reg*>& regs, const double* n0, const double* n1) {
    if (regs.empty()) return YAO_OK;
    std::vector<NormChunk> ch;
    std::vector<uint32_t> first;
    norm_chunks(regs, ch, first);
    NormChunk* d_ch = nullptr;
    YAO_CUDA(cudaMallocAsync((void**)&d_ch, ch.size() * sizeof(NormChunk), ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(d_ch, ch.data(), ch.size() * sizeof(NormChunk), cudaMemcpyHostToDevice, ctx->stream));
    if (regs[0]->precision == YAO_C128)
        k_chunk_rescale<double2><<<(unsigned)ch.size(), kRT, 0, ctx->stream>>>(d_ch, n0, n1);
    else
        k_chunk_rescale<float2><<<(unsigned)ch.size(), kRT, 0, ctx->stream>>>(d_ch, n0, n1);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaFreeAsync(d_ch, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    return YAO_OK;
}

}  // namespace yao
