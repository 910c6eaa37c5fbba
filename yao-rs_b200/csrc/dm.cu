// dm.cu — density-matrix kernels.
//
// rho is stored row-major (rho[row * dim + col], yao-rs
// src/density_matrix.rs:7-12) and treated as a 2n-qubit vector whose high n
// bits are the row index.  yao-rs applies a gate as two full passes (U on
// the row bits, then conj(U) on the column bits, :161-178) and a channel as
// about eight passes per Kraus operator (:181-224).  Here:
//
//  - a gate is ONE pass: each group of 4^k entries (k row targets x k column
//    targets) is loaded once, U is applied along the row bits and then
//    conj(U) along the column bits, with the PLAIN arithmetic.  Every entry
//    sees the same operation sequence as in the two-pass CPU code, so the
//    result is bit-identical.
//  - a channel is ONE pass: for each group, branch = original, K_i on the
//    rows, conj(K_i) on the columns, acc += branch, for every Kraus operator
//    in order: the CPU path's accumulation, per entry, in one HBM round trip.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"

namespace yao {

#define GRID_STRIDE(i, n) \
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

constexpr int kDT = 256;

// ------------------------------------------------------------- from_reg

// rho[r, c] = psi[r] * conj(psi[c]) (src/density_matrix.rs:23-35)
__global__ void k_dm_from_reg(const double2* __restrict__ psi, double2* __restrict__ rho, uint32_t n) {
    const uint64_t dim = 1ull << n;
    GRID_STRIDE(i, dim * dim) {
        uint64_t r = i >> n, c = i & (dim - 1);
        double2 a = psi[r], b = psi[c];
        rho[i] = cmul_x(a, make_double2(b.x, -b.y));
    }
}

int launch_dm_from_reg(Ctx* ctx, const Reg* r, DM* d) {
    uint64_t tot = (uint64_t)1 << (2 * r->nbits);
    k_dm_from_reg<<<grid_for(tot, 256, ctx->num_sms), 256, 0, ctx->stream>>>((const double2*)r->d, (double2*)d->d,
                                                                             r->nbits);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// rho[r, c] += (w * psi[r]) * conj(psi[c]) (DensityMatrix::mixed, :37-57)
__global__ void k_dm_mixed(const double2* __restrict__ psi, double2* __restrict__ rho, uint32_t n, double w) {
    const uint64_t dim = 1ull << n;
    GRID_STRIDE(i, dim * dim) {
        uint64_t r = i >> n, c = i & (dim - 1);
        double2 a = cmul_x(make_double2(w, 0.0), psi[r]);
        double2 b = psi[c];
        rho[i] = cadd_x(rho[i], cmul_x(a, make_double2(b.x, -b.y)));
    }
}

int launch_dm_mixed_accum(Ctx* ctx, const Reg* r, double w, DM* d) {
    uint64_t tot = (uint64_t)1 << (2 * r->nbits);
    k_dm_mixed<<<grid_for(tot, 256, ctx->num_sms), 256, 0, ctx->stream>>>((const double2*)r->d, (double2*)d->d,
                                                                          r->nbits, w);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// ------------------------------------------------------------- gate pass

struct DMGate {
    int32_t cls, k, nlocked, pad;
    int8_t locked[32];
    uint64_t roff[4], coff[4];
    uint64_t rcmask, rcval, ccmask, ccval;
    uint32_t ractive, cactive;
    double2 mr[16], mc[16];
};

// apply a k<=2 gate (class CLS) along one axis of a 2^k x 2^k block v[a][b]
template <int CLS, int K>
__device__ __forceinline__ void axis_apply(double2 (&v)[1 << K][1 << K], const double2* m, uint32_t active, bool rows) {
    constexpr int NL = 1 << K;
#pragma unroll
    for (int o = 0; o < NL; o++) {
        double2 x[NL];
#pragma unroll
        for (int i = 0; i < NL; i++) x[i] = rows ? v[i][o] : v[o][i];
        double2 y[NL];
#pragma unroll
        for (int i = 0; i < NL; i++) y[i] = x[i];
        if (CLS == GC_X) {
            y[0] = x[1];
            y[1] = x[0];
        } else if (CLS == GC_SWAP) {
            y[1] = x[2];
            y[2] = x[1];
        } else if (CLS == GC_DIAG) {
#pragma unroll
            for (int i = 0; i < NL; i++)
                if ((active >> i) & 1) y[i] = cmulassign_x(x[i], m[i]);
        } else if (K == 1) {
            y[0] = cadd_x(cmul_x(m[0], x[0]), cmul_x(m[1], x[1]));
            y[1] = cadd_x(cmul_x(m[2], x[0]), cmul_x(m[3], x[1]));
        } else {
#pragma unroll
            for (int i = 0; i < NL; i++) {
                double2 acc = make_double2(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < NL; j++) acc = cadd_x(acc, cmul_x(m[i * NL + j], x[j]));
                y[i] = acc;
            }
        }
#pragma unroll
        for (int i = 0; i < NL; i++) {
            if (rows)
                v[i][o] = y[i];
            else
                v[o][i] = y[i];
        }
    }
}

template <int CLS, int K>
__global__ void __launch_bounds__(kDT) k_dm_gate(double2* __restrict__ rho, uint64_t ngroups, const DMGate op) {
    constexpr int NL = 1 << K;
    GRID_STRIDE(g, ngroups) {
        uint64_t base = insert_zeros(g, op.locked, op.nlocked);
        bool rok = (base & op.rcmask) == op.rcval, cok = (base & op.ccmask) == op.ccval;
        if (!rok && !cok) continue;
        double2 v[NL][NL];
#pragma unroll
        for (int a = 0; a < NL; a++)
#pragma unroll
            for (int b = 0; b < NL; b++) v[a][b] = rho[base + op.roff[a] + op.coff[b]];
        if (rok) axis_apply<CLS, K>(v, op.mr, op.ractive, true);
        if (cok) axis_apply<CLS, K>(v, op.mc, op.cactive, false);
#pragma unroll
        for (int a = 0; a < NL; a++)
#pragma unroll
            for (int b = 0; b < NL; b++) rho[base + op.roff[a] + op.coff[b]] = v[a][b];
    }
}

static uint32_t active_mask(const LGate& g) {
    uint32_t a = 0;
    if (g.cls != GC_DIAG) return 0;
    for (size_t i = 0; i < g.m.size(); i++)
        if (!(g.m[i].re == 1.0 && g.m[i].im == 0.0)) a |= 1u << i;
    return a;
}

static void offsets(const LGate& g, uint64_t* off) {
    for (int l = 0; l < (1 << g.k); l++) {
        uint64_t o = 0;
        for (int i = 0; i < g.k; i++) o |= (uint64_t)((l >> i) & 1) << g.tb[i];
        off[l] = o;
    }
}

int launch_dm_gate(Ctx* ctx, DM* d, const LGate& row, const LGate& col) {
    uint32_t nb = 2 * d->nbits;
    if (row.k > 2 || row.cls != col.cls) {
        int s = launch_gate(ctx, d->d, YAO_C128, nb, row);
        if (s) return s;
        return launch_gate(ctx, d->d, YAO_C128, nb, col);
    }
    DMGate op;
    memset(&op, 0, sizeof(op));
    op.cls = row.cls;
    op.k = row.k;
    std::vector<int> pos;
    for (int i = 0; i < row.k; i++) pos.push_back(row.tb[i]);
    for (int i = 0; i < col.k; i++) pos.push_back(col.tb[i]);
    std::sort(pos.begin(), pos.end());
    op.nlocked = (int)pos.size();
    for (size_t i = 0; i < pos.size(); i++) op.locked[i] = (int8_t)pos[i];
    offsets(row, op.roff);
    offsets(col, op.coff);
    op.rcmask = row.cmask();
    op.rcval = row.cval();
    op.ccmask = col.cmask();
    op.ccval = col.cval();
    op.ractive = active_mask(row);
    op.cactive = active_mask(col);
    for (size_t i = 0; i < row.m.size() && i < 16; i++) op.mr[i] = make_double2(row.m[i].re, row.m[i].im);
    for (size_t i = 0; i < col.m.size() && i < 16; i++) op.mc[i] = make_double2(col.m[i].re, col.m[i].im);
    if (op.cls == GC_DIAG && op.ractive == 0 && op.cactive == 0) return YAO_OK;
    uint64_t ngroups = (uint64_t)1 << (nb - op.nlocked);
    unsigned grid = grid_for(ngroups, kDT, ctx->num_sms);
    cudaStream_t s = ctx->stream;
    ProfScope prof(ctx, "dm_gate", (double)ngroups * (double)(1 << (2 * op.k)) * 32.0);
    switch (op.cls * 4 + op.k) {
    case GC_X * 4 + 1: k_dm_gate<GC_X, 1><<<grid, kDT, 0, s>>>((double2*)d->d, ngroups, op); break;
    case GC_SWAP * 4 + 2: k_dm_gate<GC_SWAP, 2><<<grid, kDT, 0, s>>>((double2*)d->d, ngroups, op); break;
    case GC_DIAG * 4 + 1: k_dm_gate<GC_DIAG, 1><<<grid, kDT, 0, s>>>((double2*)d->d, ngroups, op); break;
    case GC_DIAG * 4 + 2: k_dm_gate<GC_DIAG, 2><<<grid, kDT, 0, s>>>((double2*)d->d, ngroups, op); break;
    case GC_DENSE * 4 + 1: k_dm_gate<GC_DENSE, 1><<<grid, kDT, 0, s>>>((double2*)d->d, ngroups, op); break;
    case GC_DENSE * 4 + 2: k_dm_gate<GC_DENSE, 2><<<grid, kDT, 0, s>>>((double2*)d->d, ngroups, op); break;
    default: return fail(YAO_ERR_INVALID_ARGUMENT, "unsupported density-matrix gate class");
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

// ---------------------------------------------------------- channel pass

constexpr int kMaxKraus = 16;
constexpr int kDCT = 128;  // channel kernel block size
// A channel pass's description travels in the kernel parameters (about
// 8.7 KB: no allocation and no copy per launch).  `mono[q]`: Kraus operator q
// and its conjugate have at most one non-zero entry per row (Pauli products,
// amplitude-damping jumps); perm[q][axis][i] is that entry's column (-1: the
// row is zero).
struct DMChan {
    int32_t k, nk, nlocked, pad;
    int8_t locked[32];
    uint64_t roff[4], coff[4];
    int32_t cls[kMaxKraus];       // GC_DIAG or GC_DENSE per Kraus operator
    uint32_t active[kMaxKraus];
    int32_t mono[kMaxKraus];
    int8_t perm[kMaxKraus][2][4];
    int32_t xmask[kMaxKraus][2];  // XOR channels: row / column permutation a -> a ^ xmask
    int8_t ckind[kMaxKraus][2];   // XOR channels: 0 every non-zero row / column coefficient real, 1 imaginary, 2 neither
    double2 kr[kMaxKraus * 16], kc[kMaxKraus * 16];  // row / column matrices, 2^k x 2^k each
};

// c * x with the operation structure of num_complex, for a coefficient that
// is real (c.y == 0) or imaginary (c.x == 0) by two products: the omitted
// terms are products with an exact zero, so the result is the same number
// (at most the sign of a zero differs).
__device__ __forceinline__ double2 cmul_sparse(double2 c, double2 x) {
    if (c.y == 0.0) return make_double2(__dmul_rn(c.x, x.x), __dmul_rn(c.x, x.y));
    if (c.x == 0.0) return make_double2(-__dmul_rn(c.y, x.y), __dmul_rn(c.y, x.x));
    return cmul_x(c, x);
}
// x *= c (MulAssign) for a diagonal entry, same shortcut
__device__ __forceinline__ double2 cmulassign_sparse(double2 x, double2 c) {
    if (c.y == 0.0) return make_double2(__dmul_rn(x.x, c.x), __dmul_rn(x.y, c.x));
    return cmulassign_x(x, c);
}

// The untouched original group is kept in shared memory (one column per
// thread) and the accumulator in registers.  For each Kraus operator in
// order: branch = original, K on the row bits, conj(K) on the column bits,
// acc += branch (src/density_matrix.rs:181-224, per entry).  For a diagonal
// or monomial operator, branch entry (a, b) depends on one original entry:
// (K conj(K) applied per axis) it is
//     cmul(kc[b], cmul(kr[a], orig[pr[a]][pc[b]]))
// (monomial: kr[a] = K[a][pr[a]], kc[b] = conj(K)[b][pc[b]]; a zero row
// contributes exact zeros, which leave the accumulator as it is) or
//     (orig[a][b] *= kr[a]) *= kc[b]
// (diagonal), the same operations on the same values as the row pass
// followed by the column pass.  DENSE instantiation: channels with some
// operator that is neither (the whole branch block in registers).
template <int K, bool DENSE>
__global__ void __launch_bounds__(kDCT, DENSE ? 1 : 4) k_dm_channel(double2* __restrict__ rho, uint64_t ngroups,
                                                    const __grid_constant__ DMChan op) {
    constexpr int NL = 1 << K, MS = NL * NL;
    __shared__ double2 smr[kMaxKraus * MS], smc[kMaxKraus * MS];
    __shared__ double2 sorig[MS * kDCT];
    __shared__ int8_t sperm[kMaxKraus][2][4];
    for (int i = threadIdx.x; i < op.nk * MS; i += blockDim.x) {
        smr[i] = op.kr[i];
        smc[i] = op.kc[i];
    }
    for (int i = threadIdx.x; i < op.nk * 8; i += blockDim.x) (&sperm[0][0][0])[i] = (&op.perm[0][0][0])[i];
    __syncthreads();
    double2* orig = sorig + threadIdx.x;  // orig[(a*NL+b) * kDCT]
    GRID_STRIDE(g, ngroups) {
        uint64_t base = insert_zeros(g, op.locked, op.nlocked);
        double2 acc[NL][NL];
#pragma unroll
        for (int a = 0; a < NL; a++)
#pragma unroll
            for (int b = 0; b < NL; b++) {
                orig[(a * NL + b) * kDCT] = rho[base + op.roff[a] + op.coff[b]];
                acc[a][b] = make_double2(0.0, 0.0);
            }
        for (int q = 0; q < op.nk; q++) {
            const double2* mr = smr + q * MS;
            const double2* mc = smc + q * MS;
            if (op.cls[q] == GC_DIAG) {
#pragma unroll
                for (int a = 0; a < NL; a++) {
                    const double2 dr = mr[a * (NL + 1)];
#pragma unroll
                    for (int b = 0; b < NL; b++) {
                        const double2 y = cmulassign_sparse(cmulassign_sparse(orig[(a * NL + b) * kDCT], dr),
                                                            mc[b * (NL + 1)]);
                        acc[a][b] = cadd_x(acc[a][b], y);
                    }
                }
            } else if (!DENSE || op.mono[q]) {
                const int8_t* pr = sperm[q][0];
                const int8_t* pc = sperm[q][1];
#pragma unroll
                for (int a = 0; a < NL; a++) {
                    const int ra = pr[a];
                    if (ra < 0) continue;
                    const double2 cr = mr[a * NL + ra];
#pragma unroll
                    for (int b = 0; b < NL; b++) {
                        const int cb = pc[b];
                        if (cb < 0) continue;
                        const double2 y = cmul_sparse(mc[b * NL + cb], cmul_sparse(cr, orig[(ra * NL + cb) * kDCT]));
                        acc[a][b] = cadd_x(acc[a][b], y);
                    }
                }
            } else if constexpr (DENSE) {
                double2 br[NL][NL];
#pragma unroll
                for (int a = 0; a < NL; a++)
#pragma unroll
                    for (int b = 0; b < NL; b++) br[a][b] = orig[(a * NL + b) * kDCT];
                axis_apply<GC_DENSE, K>(br, mr, 0, true);
                axis_apply<GC_DENSE, K>(br, mc, 0, false);
#pragma unroll
                for (int a = 0; a < NL; a++)
#pragma unroll
                    for (int b = 0; b < NL; b++) acc[a][b] = cadd_x(acc[a][b], br[a][b]);
            }
        }
#pragma unroll
        for (int a = 0; a < NL; a++)
#pragma unroll
            for (int b = 0; b < NL; b++) rho[base + op.roff[a] + op.coff[b]] = acc[a][b];
    }
}

// Channels whose every Kraus operator (and its conjugate) is a permutation
// a -> a ^ x times one coefficient per row (the Pauli products of the
// depolarizing and Pauli channels, bit and phase flips; diagonal operators
// with x = 0): the group stays in registers, and each operator is one of
// NL^2 code paths with compile-time source indices (no shared-memory reads
// of the group).  Operation per entry and operator as in k_dm_channel's
// monomial path: acc += cmul(kc[b], cmul(kr[a], orig[a ^ xr][b ^ xc])).
// cmul_sparse for a coefficient known to be real (KIND 0) or imaginary
// (KIND 1): the same two products, without the tests
template <int KIND>
__device__ __forceinline__ double2 cmul_kind(double2 c, double2 x) {
    if (KIND == 0) return make_double2(__dmul_rn(c.x, x.x), __dmul_rn(c.x, x.y));
    return make_double2(-__dmul_rn(c.y, x.y), __dmul_rn(c.y, x.x));
}

// xor_op for an operator whose row and column permutations are both
// a -> a ^ X and whose coefficients are all real / all imaginary per axis
template <int K, int X, int RK, int CK>
__device__ __forceinline__ void xor_op_kind(const double2 (&x)[1 << K][1 << K], double2 (&acc)[1 << K][1 << K],
                                            const double2* mr, const double2* mc) {
    constexpr int NL = 1 << K;
#pragma unroll
    for (int a = 0; a < NL; a++) {
        const double2 cr = mr[a * NL + (a ^ X)];
#pragma unroll
        for (int b = 0; b < NL; b++) {
            const double2 y = cmul_kind<CK>(mc[b * NL + (b ^ X)], cmul_kind<RK>(cr, x[a ^ X][b ^ X]));
            acc[a][b] = cadd_x(acc[a][b], y);
        }
    }
}

template <int K, int XR, int XC>
__device__ __forceinline__ void xor_op(const double2 (&x)[1 << K][1 << K], double2 (&acc)[1 << K][1 << K],
                                       const double2* mr, const double2* mc) {
    constexpr int NL = 1 << K;
#pragma unroll
    for (int a = 0; a < NL; a++) {
        const double2 cr = mr[a * NL + (a ^ XR)];
#pragma unroll
        for (int b = 0; b < NL; b++) {
            const double2 y = cmul_sparse(mc[b * NL + (b ^ XC)], cmul_sparse(cr, x[a ^ XR][b ^ XC]));
            acc[a][b] = cadd_x(acc[a][b], y);
        }
    }
}

template <int K, int XR>
__device__ __forceinline__ void xor_op_c(int xc, const double2 (&x)[1 << K][1 << K], double2 (&acc)[1 << K][1 << K],
                                         const double2* mr, const double2* mc) {
    if constexpr (K == 1) {
        if (xc == 0) xor_op<K, XR, 0>(x, acc, mr, mc); else xor_op<K, XR, 1>(x, acc, mr, mc);
    } else {
        switch (xc) {
        case 0: xor_op<K, XR, 0>(x, acc, mr, mc); break;
        case 1: xor_op<K, XR, 1>(x, acc, mr, mc); break;
        case 2: xor_op<K, XR, 2>(x, acc, mr, mc); break;
        default: xor_op<K, XR, 3>(x, acc, mr, mc); break;
        }
    }
}

template <int K>
__global__ void __launch_bounds__(kDCT, 2) k_dm_channel_xor(double2* __restrict__ rho, uint64_t ngroups,
                                                            const __grid_constant__ DMChan op) {
    constexpr int NL = 1 << K, MS = NL * NL;
    __shared__ double2 smr[kMaxKraus * MS], smc[kMaxKraus * MS];
    __shared__ int sx[kMaxKraus][2];
    __shared__ int sk[kMaxKraus];  // 1-qubit: x * 4 + row kind * 2 + column kind, or -1
    for (int i = threadIdx.x; i < op.nk * MS; i += blockDim.x) {
        smr[i] = op.kr[i];
        smc[i] = op.kc[i];
    }
    for (int i = threadIdx.x; i < op.nk * 2; i += blockDim.x) (&sx[0][0])[i] = (&op.xmask[0][0])[i];
    for (int q = threadIdx.x; q < op.nk; q += blockDim.x)
        sk[q] = K == 1 && op.xmask[q][0] == op.xmask[q][1] && op.ckind[q][0] < 2 && op.ckind[q][1] < 2
                    ? op.xmask[q][0] * 4 + op.ckind[q][0] * 2 + op.ckind[q][1]
                    : -1;
    __syncthreads();
    GRID_STRIDE(g, ngroups) {
        const uint64_t base = insert_zeros(g, op.locked, op.nlocked);
        double2 x[NL][NL], acc[NL][NL];
#pragma unroll
        for (int a = 0; a < NL; a++)
#pragma unroll
            for (int b = 0; b < NL; b++) {
                x[a][b] = rho[base + op.roff[a] + op.coff[b]];
                acc[a][b] = make_double2(0.0, 0.0);
            }
        for (int q = 0; q < op.nk; q++) {
            const double2* mr = smr + q * MS;
            const double2* mc = smc + q * MS;
            const int xr = sx[q][0], xc = sx[q][1];
            if constexpr (K == 1) {
                switch (sk[q]) {
                case 0: xor_op_kind<1, 0, 0, 0>(x, acc, mr, mc); break;
                case 1: xor_op_kind<1, 0, 0, 1>(x, acc, mr, mc); break;
                case 2: xor_op_kind<1, 0, 1, 0>(x, acc, mr, mc); break;
                case 3: xor_op_kind<1, 0, 1, 1>(x, acc, mr, mc); break;
                case 4: xor_op_kind<1, 1, 0, 0>(x, acc, mr, mc); break;
                case 5: xor_op_kind<1, 1, 0, 1>(x, acc, mr, mc); break;
                case 6: xor_op_kind<1, 1, 1, 0>(x, acc, mr, mc); break;
                case 7: xor_op_kind<1, 1, 1, 1>(x, acc, mr, mc); break;
                default:
                    if (xr == 0) xor_op_c<K, 0>(xc, x, acc, mr, mc); else xor_op_c<K, 1>(xc, x, acc, mr, mc);
                }
            } else {
                switch (xr) {
                case 0: xor_op_c<K, 0>(xc, x, acc, mr, mc); break;
                case 1: xor_op_c<K, 1>(xc, x, acc, mr, mc); break;
                case 2: xor_op_c<K, 2>(xc, x, acc, mr, mc); break;
                default: xor_op_c<K, 3>(xc, x, acc, mr, mc); break;
                }
            }
        }
#pragma unroll
        for (int a = 0; a < NL; a++)
#pragma unroll
            for (int b = 0; b < NL; b++) rho[base + op.roff[a] + op.coff[b]] = acc[a][b];
    }
}

// 2-qubit XOR channels with two threads per 4 x 4 group: thread h of a
// pair owns output rows 2h and 2h + 1.  It loads the group with its rows
// relabelled by a ^ 2h, y[r][b] = rho[row r ^ 2h][b], so that the source
// y[a' ^ xr][b ^ xc] of its local row a' (output row a = a' ^ 2h) has a
// compile-time register index; coefficients are read at the output row.
// Every output entry gets the operations of k_dm_channel_xor in the same
// order, and a thread needs 16 + 8 entries instead of 16 + 16 registers.
template <int XR, int XC>
__device__ __forceinline__ void xor_half(int h2, const double2 (&y)[4][4], double2 (&acc)[2][4], const double2* mr,
                                         const double2* mc) {
#pragma unroll
    for (int ap = 0; ap < 2; ap++) {
        const int a = ap ^ h2;
        const double2 cr = mr[a * 4 + (a ^ XR)];
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const double2 v = cmul_sparse(mc[b * 4 + (b ^ XC)], cmul_sparse(cr, y[ap ^ XR][b ^ XC]));
            acc[ap][b] = cadd_x(acc[ap][b], v);
        }
    }
}

template <int XR>
__device__ __forceinline__ void xor_half_c(int xc, int h2, const double2 (&y)[4][4], double2 (&acc)[2][4],
                                           const double2* mr, const double2* mc) {
    switch (xc) {
    case 0: xor_half<XR, 0>(h2, y, acc, mr, mc); break;
    case 1: xor_half<XR, 1>(h2, y, acc, mr, mc); break;
    case 2: xor_half<XR, 2>(h2, y, acc, mr, mc); break;
    default: xor_half<XR, 3>(h2, y, acc, mr, mc); break;
    }
}

template <int XR, int RK, int CK>
__device__ __forceinline__ void xor_half_kind(int h2, const double2 (&y)[4][4], double2 (&acc)[2][4],
                                              const double2* mr, const double2* mc) {
#pragma unroll
    for (int ap = 0; ap < 2; ap++) {
        const int a = ap ^ h2;
        const double2 cr = mr[a * 4 + (a ^ XR)];
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const double2 v = cmul_kind<CK>(mc[b * 4 + (b ^ XR)], cmul_kind<RK>(cr, y[ap ^ XR][b ^ XR]));
            acc[ap][b] = cadd_x(acc[ap][b], v);
        }
    }
}

__global__ void __launch_bounds__(kDCT, 3) k_dm_channel_xor2h(double2* __restrict__ rho, uint64_t ngroups,
                                                              const __grid_constant__ DMChan op) {
    __shared__ double2 smr[kMaxKraus * 16], smc[kMaxKraus * 16];
    __shared__ int sx[kMaxKraus][2];
    __shared__ int sk[kMaxKraus];  // xr * 4 + row kind * 2 + column kind, or -1
    for (int i = threadIdx.x; i < op.nk * 16; i += blockDim.x) {
        smr[i] = op.kr[i];
        smc[i] = op.kc[i];
    }
    for (int i = threadIdx.x; i < op.nk * 2; i += blockDim.x) (&sx[0][0])[i] = (&op.xmask[0][0])[i];
    for (int q = threadIdx.x; q < op.nk; q += blockDim.x)
        sk[q] = op.xmask[q][0] == op.xmask[q][1] && op.ckind[q][0] < 2 && op.ckind[q][1] < 2
                    ? op.xmask[q][0] * 4 + op.ckind[q][0] * 2 + op.ckind[q][1]
                    : -1;
    __syncthreads();
    GRID_STRIDE(t, 2 * ngroups) {
        const uint64_t base = insert_zeros(t >> 1, op.locked, op.nlocked);
        const int h2 = (int)(t & 1) << 1;
        double2 y[4][4], acc[2][4];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int b = 0; b < 4; b++) y[r][b] = rho[base + op.roff[r ^ h2] + op.coff[b]];
#pragma unroll
        for (int ap = 0; ap < 2; ap++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[ap][b] = make_double2(0.0, 0.0);
        for (int q = 0; q < op.nk; q++) {
            const double2* mr = smr + q * 16;
            const double2* mc = smc + q * 16;
            const int xr = sx[q][0], xc = sx[q][1];
            // same permutation on rows and columns (K and conj(K)) and
            // coefficients of one kind per axis: a branch-free variant
            const int code = sk[q];
            if (code >= 0) {
                switch (code) {
#define XOR_KIND_CASE(X, R, C) \
    case X * 4 + R * 2 + C: xor_half_kind<X, R, C>(h2, y, acc, mr, mc); break;
                XOR_KIND_CASE(0, 0, 0) XOR_KIND_CASE(0, 0, 1) XOR_KIND_CASE(0, 1, 0) XOR_KIND_CASE(0, 1, 1)
                XOR_KIND_CASE(1, 0, 0) XOR_KIND_CASE(1, 0, 1) XOR_KIND_CASE(1, 1, 0) XOR_KIND_CASE(1, 1, 1)
                XOR_KIND_CASE(2, 0, 0) XOR_KIND_CASE(2, 0, 1) XOR_KIND_CASE(2, 1, 0) XOR_KIND_CASE(2, 1, 1)
                XOR_KIND_CASE(3, 0, 0) XOR_KIND_CASE(3, 0, 1) XOR_KIND_CASE(3, 1, 0) XOR_KIND_CASE(3, 1, 1)
#undef XOR_KIND_CASE
                default: break;
                }
                continue;
            }
            switch (xr) {
            case 0: xor_half_c<0>(xc, h2, y, acc, mr, mc); break;
            case 1: xor_half_c<1>(xc, h2, y, acc, mr, mc); break;
            case 2: xor_half_c<2>(xc, h2, y, acc, mr, mc); break;
            default: xor_half_c<3>(xc, h2, y, acc, mr, mc); break;
            }
        }
        // both threads of the pair (adjacent lanes, always both in the loop:
        // 2 ngroups is even) read the whole group before either writes
        __syncwarp(3u << (threadIdx.x & 30));
#pragma unroll
        for (int ap = 0; ap < 2; ap++)
#pragma unroll
            for (int b = 0; b < 4; b++) rho[base + op.roff[ap ^ h2] + op.coff[b]] = acc[ap][b];
    }
}

// 1-qubit channels whose every Kraus operator has at most one non-zero
// entry per row (and so its conjugate: amplitude and phase damping, resets,
// and the Pauli channels): the 2 x 2 group stays in registers and each
// branch entry (a, b) is the one original entry it depends on, chosen by a
// select, times the two coefficients — k_dm_channel's monomial path with
// the same operations on the same values, a zero row contributing nothing.
__device__ __forceinline__ double2 pick2(const double2 (&x)[2][2], int r, int c) {
    const double2 a = c ? x[0][1] : x[0][0];
    const double2 b = c ? x[1][1] : x[1][0];
    return r ? b : a;
}

__global__ void __launch_bounds__(kDCT, 2) k_dm_channel_mono1(double2* __restrict__ rho, uint64_t ngroups,
                                                              const __grid_constant__ DMChan op) {
    __shared__ double2 smr[kMaxKraus * 4], smc[kMaxKraus * 4];
    __shared__ int8_t sp[kMaxKraus][4];  // row sources of rows 0, 1, column sources of columns 0, 1
    for (int i = threadIdx.x; i < op.nk * 4; i += blockDim.x) {
        smr[i] = op.kr[i];
        smc[i] = op.kc[i];
    }
    for (int q = threadIdx.x; q < op.nk; q += blockDim.x) {
        const bool diag = op.cls[q] == GC_DIAG;
        sp[q][0] = diag ? 0 : op.perm[q][0][0];
        sp[q][1] = diag ? 1 : op.perm[q][0][1];
        sp[q][2] = diag ? 0 : op.perm[q][1][0];
        sp[q][3] = diag ? 1 : op.perm[q][1][1];
    }
    __syncthreads();
    GRID_STRIDE(g, ngroups) {
        const uint64_t base = insert_zeros(g, op.locked, op.nlocked);
        double2 x[2][2], acc[2][2];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                x[a][b] = rho[base + op.roff[a] + op.coff[b]];
                acc[a][b] = make_double2(0.0, 0.0);
            }
        for (int q = 0; q < op.nk; q++) {
            const double2* mr = smr + q * 4;
            const double2* mc = smc + q * 4;
#pragma unroll
            for (int a = 0; a < 2; a++) {
                const int ra = sp[q][a];
                if (ra < 0) continue;
                const double2 cr = mr[a * 2 + ra];
#pragma unroll
                for (int b = 0; b < 2; b++) {
                    const int cb = sp[q][2 + b];
                    if (cb < 0) continue;
                    const double2 y = cmul_sparse(mc[b * 2 + cb], cmul_sparse(cr, pick2(x, ra, cb)));
                    acc[a][b] = cadd_x(acc[a][b], y);
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) rho[base + op.roff[a] + op.coff[b]] = acc[a][b];
    }
}

// Column of the single non-zero entry of each row of a d x d matrix (-1 for
// a zero row); false when some row has two or more.
static bool monomial_rows(const std::vector<Cx>& m, int d, int8_t* perm) {
    for (int i = 0; i < d; i++) {
        perm[i] = -1;
        for (int j = 0; j < d; j++) {
            const Cx c = m[(size_t)i * d + j];
            if (c.re == 0.0 && c.im == 0.0) continue;
            if (perm[i] >= 0) return false;
            perm[i] = (int8_t)j;
        }
    }
    return true;
}

int launch_dm_channel(Ctx* ctx, DM* d, const std::vector<LGate>& rows, const std::vector<LGate>& cols,
                      const std::vector<uint32_t>& row_bits, const std::vector<uint32_t>& col_bits) {
    const int k = rows.empty() ? 0 : rows[0].k;
    const int nk = (int)rows.size();
    if (k < 1 || k > 2 || nk > kMaxKraus) return fail(YAO_ERR_UNSUPPORTED, "channel pass supports 1- and 2-qubit channels with <= 16 Kraus operators");
    DMChan op;
    memset(&op, 0, sizeof(op));
    op.k = k;
    op.nk = nk;
    std::vector<int> pos;
    for (int i = 0; i < k; i++) pos.push_back(rows[0].tb[i]);
    for (int i = 0; i < k; i++) pos.push_back(cols[0].tb[i]);
    std::sort(pos.begin(), pos.end());
    op.nlocked = (int)pos.size();
    for (size_t i = 0; i < pos.size(); i++) op.locked[i] = (int8_t)pos[i];
    offsets(rows[0], op.roff);
    offsets(cols[0], op.coff);
    const int NL = 1 << k, MS = NL * NL;
    for (int q = 0; q < nk; q++) {
        // the 2q lowering sorts each Kraus operator's bits identically
        op.cls[q] = rows[q].cls;
        op.active[q] = active_mask(rows[q]) | active_mask(cols[q]);
        if (rows[q].cls == GC_DIAG) {
            // a diagonal operator's entries, on the diagonal of the block
            for (int i = 0; i < NL; i++) {
                op.kr[q * MS + i * (NL + 1)] = make_double2(rows[q].m[i].re, rows[q].m[i].im);
                op.kc[q * MS + i * (NL + 1)] = make_double2(cols[q].m[i].re, cols[q].m[i].im);
            }
            op.active[q] = (1u << NL) - 1;  // multiply every entry, as the CPU path does
            continue;
        }
        for (int i = 0; i < MS; i++) {
            op.kr[q * MS + i] = make_double2(rows[q].m[i].re, rows[q].m[i].im);
            op.kc[q * MS + i] = make_double2(cols[q].m[i].re, cols[q].m[i].im);
        }
        op.mono[q] = monomial_rows(rows[q].m, NL, op.perm[q][0]) && monomial_rows(cols[q].m, NL, op.perm[q][1]);
    }
    // XOR channels: every operator a monomial whose permutation is a ^ x on
    // rows and columns (diagonal operators: x = 0); their diagonal entries
    // sit at m[a * NL + a] already
    bool xr_ok = true;
    for (int q = 0; q < nk && xr_ok; q++) {
        if (rows[q].cls == GC_DIAG) {
            op.xmask[q][0] = op.xmask[q][1] = 0;
            continue;
        }
        if (!op.mono[q]) {
            xr_ok = false;
            break;
        }
        for (int ax = 0; ax < 2 && xr_ok; ax++) {
            const int x0 = op.perm[q][ax][0];
            if (x0 < 0) {
                xr_ok = false;
                break;
            }
            for (int a = 0; a < NL; a++)
                if (op.perm[q][ax][a] != (a ^ x0)) xr_ok = false;
            op.xmask[q][ax] = x0;
        }
    }
    // coefficient kinds of each operator's non-zero entries (rows: K, columns:
    // conj(K)): all real, all imaginary, or mixed
    for (int q = 0; q < nk; q++)
        for (int ax = 0; ax < 2; ax++) {
            const double2* m = ax == 0 ? op.kr + q * MS : op.kc + q * MS;
            bool re = true, im = true;
            for (int i = 0; i < MS; i++) {
                if (m[i].x == 0.0 && m[i].y == 0.0) continue;
                re &= m[i].y == 0.0;
                im &= m[i].x == 0.0;
            }
            op.ckind[q][ax] = (int8_t)(re ? 0 : (im ? 1 : 2));
        }
    uint64_t ngroups = (uint64_t)1 << (2 * d->nbits - op.nlocked);
    unsigned grid = grid_for(ngroups, kDT, ctx->num_sms);
    const double bytes = (double)ngroups * (double)(1 << (2 * k)) * 32.0;
    auto off = [](const char* name) {
        const char* e = getenv(name);
        return e && e[0] == '0';
    };
    bool dense = false;
    for (int q = 0; q < nk; q++) dense |= op.cls[q] != GC_DIAG && !op.mono[q];
    if (xr_ok && !off("YAO_DM_XOR")) {
        // Pauli-type channels: the group in registers
        if (k == 1) {
            ProfScope prof(ctx, "dm_channel_xor1", bytes);
            k_dm_channel_xor<1><<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op);
        } else if (off("YAO_DM_XOR2H")) {
            ProfScope prof(ctx, "dm_channel_xor2", bytes);
            k_dm_channel_xor<2><<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op);
        } else {  // two threads per group
            ProfScope prof(ctx, "dm_channel_xor2", bytes);
            k_dm_channel_xor2h<<<grid_for(2 * ngroups, kDT, ctx->num_sms), kDCT, 0, ctx->stream>>>((double2*)d->d,
                                                                                                ngroups, op);
        }
    } else if (k == 1 && !dense && !off("YAO_DM_MONO")) {
        // 1-qubit channels of diagonal and row-monomial operators: registers
        ProfScope prof(ctx, "dm_channel_mono1", bytes);
        k_dm_channel_mono1<<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op);
    } else {
        ProfScope prof(ctx, "dm_channel", bytes);
        if (k == 1)
            dense ? k_dm_channel<1, true><<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op)
                  : k_dm_channel<1, false><<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op);
        else
            dense ? k_dm_channel<2, true><<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op)
                  : k_dm_channel<2, false><<<grid, kDCT, 0, ctx->stream>>>((double2*)d->d, ngroups, op);
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    (void)row_bits;
    (void)col_bits;
    return YAO_OK;
}

// ------------------------------------------------------------ reductions

static int dm_finish(Ctx* ctx, double* part, int nb, int nv, double* host_out);

__global__ void k_dm_final(const double* __restrict__ partial, int nblocks, int nv, double* __restrict__ out) {
    __shared__ double sm[kDT / 32];
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

static int dm_finish(Ctx* ctx, double* part, int nb, int nv, double* host_out) {
    double* dout = part + (size_t)nb * nv;
    k_dm_final<<<1, kDT, 0, ctx->stream>>>(part, nb, nv, dout);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    if (ctx->ensure_host_pinned(sizeof(double) * nv)) return YAO_ERR_OUT_OF_MEMORY;
    YAO_CUDA(cudaMemcpyAsync(ctx->host_pinned, dout, sizeof(double) * nv, cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(host_out, ctx->host_pinned, sizeof(double) * nv);
    return YAO_OK;
}

static int dm_scratch(Ctx* ctx, int nb, int nv, double** part) {
    if (ctx->ensure_scratch(sizeof(double) * ((size_t)nb * nv + nv))) return YAO_ERR_OUT_OF_MEMORY;
    *part = (double*)ctx->scratch;
    return YAO_OK;
}

// trace (src/density_matrix.rs:63-67)
__global__ void __launch_bounds__(kDT) k_dm_trace(const double2* __restrict__ rho, uint64_t dim, double* partial) {
    __shared__ double sm[2 * kDT / 32];
    double acc[2] = {0.0, 0.0};
    GRID_STRIDE(i, dim) {
        double2 v = rho[i * dim + i];
        acc[0] += v.x;
        acc[1] += v.y;
    }
    block_sum_write(acc, 2, sm, partial + 2 * blockIdx.x);
}

int reduce_dm_trace(Ctx* ctx, const DM* d, Cx* out) {
    uint64_t dim = (uint64_t)1 << d->nbits;
    int nb = (int)grid_for(dim, kDT, ctx->num_sms, 2);
    double* part;
    if (dm_scratch(ctx, nb, 2, &part)) return YAO_ERR_OUT_OF_MEMORY;
    k_dm_trace<<<nb, kDT, 0, ctx->stream>>>((const double2*)d->d, dim, part);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    double r[2];
    int s = dm_finish(ctx, part, nb, 2, r);
    *out = Cx{r[0], r[1]};
    return s;
}

// purity = Re sum_{r,i} rho[r,i] rho[i,r] (src/density_matrix.rs:69-78).
// A block takes a 32x32 tile pair (R, C), R <= C, reading rho[R, C] and
// rho[C, R] with coalesced rows; an off-diagonal pair counts twice.
__global__ void __launch_bounds__(kDT) k_dm_purity(const double2* __restrict__ rho, uint64_t dim, uint64_t nt,
                                                  uint64_t npairs, double* partial) {
    __shared__ double2 A[32][33], B[32][33];
    __shared__ double sm[kDT / 32];
    double acc = 0.0;
    for (uint64_t p = blockIdx.x; p < npairs; p += gridDim.x) {
        // p -> (R, C) with R <= C, row-major over the upper triangle
        double est = (2.0 * nt + 1.0 - sqrt((2.0 * nt + 1.0) * (2.0 * nt + 1.0) - 8.0 * (double)p)) / 2.0;
        uint64_t R = est <= 0.0 ? 0 : (uint64_t)est;
        if (R > nt - 1) R = nt - 1;
        // row R starts at pair R*nt - R(R-1)/2; fix a rounding error of the estimate
        while (R > 0 && R * nt - R * (R - 1) / 2 > p) R--;
        while (R + 1 < nt && (R + 1) * nt - (R + 1) * R / 2 <= p) R++;
        uint64_t C = R + (p - (R * nt - R * (R - 1) / 2));
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
        for (int r = ty; r < 32; r += kDT / 32) {
            A[r][tx] = rho[(R * 32 + r) * dim + C * 32 + tx];
            B[r][tx] = rho[(C * 32 + r) * dim + R * 32 + tx];
        }
        __syncthreads();
        double w = (R == C) ? 1.0 : 2.0;
        for (int r = ty; r < 32; r += kDT / 32) {
            double2 a = A[r][tx], b = B[tx][r];
            acc += w * (a.x * b.x - a.y * b.y);
        }
        __syncthreads();
    }
    block_sum_write(&acc, 1, sm, partial + blockIdx.x);
}

__global__ void __launch_bounds__(kDT) k_dm_purity_small(const double2* __restrict__ rho, uint64_t dim,
                                                        double* partial) {
    __shared__ double sm[kDT / 32];
    double acc = 0.0;
    GRID_STRIDE(i, dim * dim) {
        uint64_t r = i / dim, c = i % dim;
        double2 a = rho[r * dim + c], b = rho[c * dim + r];
        acc += a.x * b.x - a.y * b.y;
    }
    block_sum_write(&acc, 1, sm, partial + blockIdx.x);
}

int reduce_dm_purity(Ctx* ctx, const DM* d, double* out) {
    uint64_t dim = (uint64_t)1 << d->nbits;
    int nb;
    double* part;
    if (dim < 64) {
        nb = 1;
        if (dm_scratch(ctx, nb, 1, &part)) return YAO_ERR_OUT_OF_MEMORY;
        k_dm_purity_small<<<1, kDT, 0, ctx->stream>>>((const double2*)d->d, dim, part);
    } else {
        uint64_t nt = dim / 32, npairs = nt * (nt + 1) / 2;
        nb = (int)std::min<uint64_t>(npairs, (uint64_t)ctx->num_sms * 8);
        if (dm_scratch(ctx, nb, 1, &part)) return YAO_ERR_OUT_OF_MEMORY;
        k_dm_purity<<<nb, kDT, 0, ctx->stream>>>((const double2*)d->d, dim, nt, npairs, part);
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return dm_finish(ctx, part, nb, 1, out);
}

// Tr(O rho) for monomial terms (src/expect.rs:44-72): for each row r the
// only non-zero entry of O is at column c = r ^ xmask with value phase(r),
// and yao-rs reads rho[c * dim + r].
struct DMTerm {
    uint64_t xmask, d1, d2, need1, need0;
    int32_t base, zero;
};

__global__ void __launch_bounds__(kDT) k_dm_expect(const double2* __restrict__ rho, uint64_t dim, const DMTerm t,
                                                  double* partial) {
    __shared__ double sm[2 * kDT / 32];
    double acc[2] = {0.0, 0.0};
    if (!t.zero) {
        GRID_STRIDE(r, dim) {
            if ((r & t.need1) != t.need1 || (r & t.need0) != 0) continue;
            int q = (t.base + __popcll(r & t.d1) + 2 * __popcll(r & t.d2)) & 3;
            uint64_t c = r ^ t.xmask;
            double2 v = rho[c * dim + r];
            double2 u;
            switch (q) {
            case 0: u = v; break;
            case 1: u = make_double2(-v.y, v.x); break;
            case 2: u = make_double2(-v.x, -v.y); break;
            default: u = make_double2(v.y, -v.x); break;
            }
            acc[0] += u.x;
            acc[1] += u.y;
        }
    }
    block_sum_write(acc, 2, sm, partial + 2 * blockIdx.x);
}

int reduce_dm_expect(Ctx* ctx, const DM* d, const std::vector<MonoTerm>& terms, std::vector<Cx>& values) {
    uint64_t dim = (uint64_t)1 << d->nbits;
    values.assign(terms.size(), Cx{0, 0});
    for (size_t i = 0; i < terms.size(); i++) {
        DMTerm t;
        t.xmask = terms[i].xmask;
        t.d1 = terms[i].d1mask;
        t.d2 = terms[i].d2mask;
        t.need1 = terms[i].need1;
        t.need0 = terms[i].need0;
        t.base = terms[i].base;
        t.zero = terms[i].zero;
        int nb = (int)grid_for(dim, kDT, ctx->num_sms, 2);
        double* part;
        if (dm_scratch(ctx, nb, 2, &part)) return YAO_ERR_OUT_OF_MEMORY;
        k_dm_expect<<<nb, kDT, 0, ctx->stream>>>((const double2*)d->d, dim, t, part);
        ctx->launches++;
        YAO_CUDA(cudaGetLastError());
        double r[2];
        int s = dm_finish(ctx, part, nb, 2, r);
        if (s) return s;
        values[i] = Cx{r[0], r[1]};
    }
    return YAO_OK;
}

// probabilities of a density matrix: diagonal, re.max(0) (src/measure.rs:50-57, 106-122)
__global__ void k_dm_diag_probs(const double2* __restrict__ rho, uint64_t dim, double* out) {
    GRID_STRIDE(i, dim) out[i] = fmax(rho[i * dim + i].x, 0.0);
}

int reduce_dm_marginal(Ctx* ctx, const DM* d, const uint32_t* bits, int32_t nl, double* host_out) {
    uint64_t dim = (uint64_t)1 << d->nbits;
    if (ctx->ensure_scratch(sizeof(double) * dim)) return YAO_ERR_OUT_OF_MEMORY;
    double* dp = (double*)ctx->scratch;
    k_dm_diag_probs<<<grid_for(dim, 256, ctx->num_sms), 256, 0, ctx->stream>>>((const double2*)d->d, dim, dp);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    std::vector<double> diag(dim);
    YAO_CUDA(cudaMemcpyAsync(diag.data(), dp, sizeof(double) * dim, cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    if (nl < 0) {
        memcpy(host_out, diag.data(), sizeof(double) * dim);
        return YAO_OK;
    }
    // the diagonal has only 2^n entries: bin it on the host in basis order,
    // exactly as the CPU loop does
    uint64_t nout = (uint64_t)1 << nl;
    for (uint64_t o = 0; o < nout; o++) host_out[o] = 0.0;
    for (uint64_t b = 0; b < dim; b++) {
        uint64_t idx = 0;
        for (int32_t i = 0; i < nl; i++) idx |= ((b >> bits[i]) & 1) << (nl - 1 - i);
        host_out[idx] += diag[b];
    }
    return YAO_OK;
}

// partial_tr (src/density_matrix.rs:80-112; loc = bit position, LSB first).
// One thread per reduced entry sums its 2^nt contributions in increasing
// (row, col) order, which is the CPU loop's order: bit-identical.
struct PTSpec {
    int32_t nk, nt;
    int8_t kept[64];
    int8_t traced[64];
};

__global__ void k_dm_partial_tr(const double2* __restrict__ rho, double2* __restrict__ out, uint32_t n,
                                const PTSpec sp) {
    const uint64_t dr = 1ull << sp.nk, dim = 1ull << n, ntr = 1ull << sp.nt;
    GRID_STRIDE(o, dr * dr) {
        uint64_t rr = o / dr, rc = o % dr;
        uint64_t row0 = 0, col0 = 0;
        for (int k = 0; k < sp.nk; k++) {
            row0 |= ((rr >> k) & 1) << sp.kept[k];
            col0 |= ((rc >> k) & 1) << sp.kept[k];
        }
        double2 acc = make_double2(0.0, 0.0);
        for (uint64_t t = 0; t < ntr; t++) {
            uint64_t tb = 0;
            for (int j = 0; j < sp.nt; j++) tb |= ((t >> j) & 1) << sp.traced[j];
            acc = cadd_x(acc, rho[(row0 | tb) * dim + (col0 | tb)]);
        }
        out[o] = acc;
    }
}

int launch_dm_partial_tr(Ctx* ctx, const DM* d, const uint32_t* traced, uint32_t nt, DM* out) {
    PTSpec sp;
    memset(&sp, 0, sizeof(sp));
    std::vector<int> tr(traced, traced + nt);
    std::sort(tr.begin(), tr.end());
    tr.erase(std::unique(tr.begin(), tr.end()), tr.end());
    sp.nt = (int)tr.size();
    for (int j = 0; j < sp.nt; j++) sp.traced[j] = (int8_t)tr[j];
    int nk = 0;
    for (uint32_t loc = 0; loc < d->nbits; loc++)
        if (!std::binary_search(tr.begin(), tr.end(), (int)loc)) sp.kept[nk++] = (int8_t)loc;
    sp.nk = nk;
    uint64_t tot = (uint64_t)1 << (2 * nk);
    k_dm_partial_tr<<<grid_for(tot, 256, ctx->num_sms), 256, 0, ctx->stream>>>((const double2*)d->d, (double2*)out->d,
                                                                               d->nbits, sp);
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

}  // namespace yao
