// ad_tiles.cu — the adjoint (reverse-sweep) gradient of expect_grad
// (yao-rs src/ad.rs:75-156) over shared-memory tiles.
//
// The per-gate form reads and writes psi and lambda once per gate of the
// reverse sweep.  Here a pass takes reverse-sweep steps whose targets all lie
// in one tile (the low 4 bits plus up to 7 scattered bits), loads psi's and
// lambda's tile into shared memory, and for every step
//   - accumulates Re <lambda | G psi> over the tile's groups for each
//     generator G of a parametric gate (only the control-matching branch,
//     ad.rs:56-64), and
//   - applies U^dagger to both tiles,
// then writes both tiles back.  A pass is list-scheduled over the sweep: it
// takes every step that no skipped earlier step shares a qubit with (steps
// on disjoint qubits commute, and a generator dot does not change under
// steps on other qubits), and within the pass consecutive 1-qubit steps on
// at most two target bits form a register segment: each thread keeps its
// 4-amplitude group of both tiles in registers across the segment.  On the
// host, runs of uncontrolled 1-qubit steps on one target fold into one op,
// and an X step (a CNOT) in a segment merges into the run on its target,
// which then carries a coefficient set per pair or per group.  Dots are
// reduced over the warp down to four partial sums, added per warp in shared
// memory (tiles of a CTA in a fixed order), summed over warps per CTA and
// over CTAs in block order: deterministic for a given launch shape.
// Arithmetic is FP64 with FMA; the result is the reverse sweep of the
// per-gate form up to rounding (~1e-15 relative).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>
#include <vector>

#include "device_common.cuh"
#include "tc_sm100.cuh"
#include "tma_sm100.cuh"

namespace yao {

constexpr int kAdjThreads = 512;
constexpr int kAdjLowBits = 4;      // contiguous low bits of every tile (256-byte runs)
constexpr int kAdjScatter = 7;      // scattered tile bits at most
constexpr int kAdjMaxOps = 64;      // reverse-sweep ops per pass
constexpr int kAdjMaxSlots = 48;    // generator dots per pass

// A run of uncontrolled 1-qubit reverse-sweep steps on one target bit,
// folded on the host into one op (cls kAdjFused): with A the product of the
// run's U^dagger matrices so far, the dot of a generator G taken after them
// is Re <A lambda | G A psi> = Re <lambda | (A^dagger G A) psi>, so every dot
// of the run is taken against the run's input amplitudes with G' = A^dagger
// G A, and the run's U^dagger steps are one 2 x 2 product A at the end.
// m[0..3] = A, m[4 + 4 j ..] = G'_j, gslot[j] its dot slot (ngen <= 3).
constexpr int32_t kAdjFused = 16;
constexpr int kAdjFusedGens = 3;

// A folded run (at most 2 dots) merged inside a register segment with an X
// step whose only control is the segment's other bit (a CNOT between the
// segment's two qubits): the X acts on one of the group's two pairs, so the
// op carries one coefficient set per pair q (the value of the other bit):
// m[8 q .. 8 q + 3] = A_q, m[8 q + 4 + 2 j] = (-Im G'_q,j[0][0],
// -Im G'_q,j[1][1]), m[8 q + 5 + 2 j] = G'_q,j[0][1].  X before the run:
// A_q = A X, G'_q = X G' X on the X's pair; X after it: A_q = X A.
constexpr int32_t kAdjFusedPair = 17;
constexpr int kAdjPairGens = 2;
// The same with an X step whose controls are off the segment (in-tile bits
// xmask / xval, out-of-tile bits xgmask / xgval): the X acts on both pairs of
// a group or on neither, so set 1 (m[8 ..]) serves the groups whose bits
// match and set 0 the others.
constexpr int32_t kAdjFusedCtl = 18;

// The control fields of an op: 64 bytes, 16-byte aligned, so the register
// segments copy them into registers with four 16-byte loads per op.
struct __align__(16) AdjOpCtl {
    int32_t gen;     // 1: accumulate Re <lambda | G psi> into `slot`; 0: U^dagger on psi and lambda
    int32_t cls;     // GC_X / GC_SWAP / GC_DIAG / GC_DENSE (generators: GC_DENSE), or kAdjFused
    int32_t k;       // 1 or 2 targets
    int32_t slot;
    int8_t tl[2];    // local target positions; tl[0] is bit 0 of the gate-local index
    int8_t sync;     // barrier after this op (the next op moves amplitudes along other bits)
    int8_t ngen;     // kAdjFused: generator dots of the run
    int8_t seg[2];   // 1-qubit ops: the segment's two local positions (seg[0] < seg[1])
    int8_t upair;    // segment op whose only in-tile control is the other segment bit: 1 + that bit's value
    int8_t pad[1];
    int32_t gslot[kAdjFusedGens];
    int32_t a_id;    // kAdjFused: A is the identity (no U^dagger in the run)
    uint32_t lcmask, lcval;  // in-tile controls (local positions)
    uint64_t gcmask, gcval;  // out-of-tile controls (global bits)
};
static_assert(sizeof(AdjOpCtl) == 64, "the control fields are four 16-byte words");

struct AdjTileOp : AdjOpCtl {
    uint64_t active;         // DIAG: entries different from 1
    uint32_t xmask, xval;    // kAdjFusedCtl: in-tile controls of the merged X step
    uint64_t xgmask, xgval;  // kAdjFusedCtl: its out-of-tile controls
    double2 m[16];           // dense 2^k x 2^k row-major, or the 2^k diagonal entries
};
static_assert(sizeof(AdjTileOp) % 16 == 0, "AdjTileOp is staged as 64-bit words, 16-byte aligned");

struct AdjTileHdr {
    int32_t tbits, nops, nslots, nouts;
    int8_t hb[kAdjScatter];  // global bits of local positions kAdjLowBits ..
    int8_t pad[1];
    int8_t outb[64];         // global bits outside the tile, ascending
    uint64_t ntiles;
    int32_t use_tma;         // psi's and lambda's tiles move by TMA (maps of the same plan)
    int32_t nstage;          // tile buffers (psi + lambda each) in flight
    TmaPlan tma;
};

__device__ __forceinline__ uint32_t adj_ins0(uint32_t v, int p) {
    return ((v >> p) << (p + 1)) | (v & ((1u << p) - 1));
}
// XOR swizzle of the double2 tile against bank conflicts
__device__ __forceinline__ uint32_t adj_swz(uint32_t l) { return l ^ ((l >> 3) & 7); }

__device__ __forceinline__ double2 cfma2(double2 acc, double2 a, double2 x) {
    acc.x = fma(a.x, x.x, acc.x);
    acc.x = fma(-a.y, x.y, acc.x);
    acc.y = fma(a.x, x.y, acc.y);
    acc.y = fma(a.y, x.x, acc.y);
    return acc;
}
__device__ __forceinline__ double2 cmul2(double2 a, double2 x) {
    return make_double2(fma(a.x, x.x, -a.y * x.y), fma(a.x, x.y, a.y * x.x));
}
// Re(conj(l) * y)
__device__ __forceinline__ double redot(double2 l, double2 y) { return fma(l.x, y.x, l.y * y.y); }

// Dot accumulators: kAdjSub per warp and slot, acc[(slot * nw + warp) *
// kAdjSub + sub].  A dot is summed over the warp only down to kAdjSub
// partial sums (three shuffle rounds instead of five); the CTA adds them up
// once, in a fixed order, after its last tile.
constexpr int kAdjSub = 4;

// Lanes 0..3 return the sums over lanes {i, i + 4, ..., i + 28}.
__device__ __forceinline__ double warp_part(double v) {
#pragma unroll
    for (int o = 16; o >= kAdjSub; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Two values in three rounds: after the exchange across the half warps,
// lanes 0..15 carry partial sums of a and lanes 16..31 of b; lanes 0..3
// return the partial sums of a, lanes 16..19 those of b.
__device__ __forceinline__ double warp_part_pair(double a, double b) {
    const bool hi = (threadIdx.x & 16) != 0;
    double v = hi ? b : a;
    v += __shfl_xor_sync(0xffffffffu, hi ? a : b, 16);
#pragma unroll
    for (int o = 8; o >= kAdjSub; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The warp's partial sums of one dot into its accumulators (lanes 0..3).
__device__ __forceinline__ void acc_part(double* __restrict__ acc, int slot, uint32_t nw, double d) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane < (uint32_t)kAdjSub) acc[((uint32_t)slot * nw + warp) * kAdjSub + lane] += d;
}

// One reverse-sweep op on the groups of the tile owned by this thread.
// A run of up to kAdjRun consecutive ops on the same target positions (in
// the same order): each group the thread owns is loaded once, every op of
// the run is applied (or its dot accumulated) in registers, and the group is
// stored once.  Ops whose controls do not match a group skip it.
constexpr int kAdjRun = 8;

template <int K>
__device__ __forceinline__ void adj_run(const AdjTileOp* __restrict__ rops, int nr, uint64_t base,
                                        double2* __restrict__ sp, double2* __restrict__ sl, uint32_t T,
                                        double* __restrict__ acc, uint32_t nw) {
    constexpr int NL = 1 << K;
    const uint32_t ngroups = T >> K;
    const int p0 = rops[0].tl[0], p1 = K == 2 ? rops[0].tl[1] : 0;
    const int lo = K == 2 ? min(p0, p1) : p0, hi = K == 2 ? max(p0, p1) : p0;
    bool on[kAdjRun];
    double dot[kAdjRun];
#pragma unroll
    for (int j = 0; j < kAdjRun; j++) {
        on[j] = j < nr && (base & rops[j].gcmask) == rops[j].gcval;  // uniform over the tile
        dot[j] = 0.0;
    }
    for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
        uint32_t b = adj_ins0(g, lo);
        if (K == 2) b = adj_ins0(b, hi);
        uint32_t idx[NL];
        double2 x[NL], l[NL];
#pragma unroll
        for (int q = 0; q < NL; q++) {
            uint32_t li = b;
            if (q & 1) li |= 1u << p0;
            if (K == 2 && (q & 2)) li |= 1u << p1;
            idx[q] = adj_swz(li);
            x[q] = sp[idx[q]];
            l[q] = sl[idx[q]];
        }
#pragma unroll
        for (int j = 0; j < kAdjRun; j++) {
            if (!on[j]) continue;
            const AdjTileOp& op = rops[j];
            if ((b & op.lcmask) != op.lcval) continue;
            if (op.gen) {
#pragma unroll
                for (int r = 0; r < NL; r++) {
                    double2 y = make_double2(0.0, 0.0);
#pragma unroll
                    for (int c = 0; c < NL; c++) y = cfma2(y, op.m[r * NL + c], x[c]);
                    dot[j] += redot(l[r], y);
                }
            } else if (op.cls == GC_X) {
                double2 t = x[0];
                x[0] = x[1];
                x[1] = t;
                t = l[0];
                l[0] = l[1];
                l[1] = t;
            } else if (op.cls == GC_SWAP) {
                double2 t = x[1];
                x[1] = x[NL / 2];
                x[NL / 2] = t;
                t = l[1];
                l[1] = l[NL / 2];
                l[NL / 2] = t;
            } else if (op.cls == GC_DIAG) {
#pragma unroll
                for (int q = 0; q < NL; q++)
                    if ((op.active >> q) & 1) {
                        x[q] = cmul2(op.m[q], x[q]);
                        l[q] = cmul2(op.m[q], l[q]);
                    }
            } else {
                double2 nx[NL], nl[NL];
#pragma unroll
                for (int r = 0; r < NL; r++) {
                    double2 a = make_double2(0.0, 0.0), c2 = make_double2(0.0, 0.0);
#pragma unroll
                    for (int c = 0; c < NL; c++) {
                        const double2 mm = op.m[r * NL + c];
                        a = cfma2(a, mm, x[c]);
                        c2 = cfma2(c2, mm, l[c]);
                    }
                    nx[r] = a;
                    nl[r] = c2;
                }
#pragma unroll
                for (int q = 0; q < NL; q++) {
                    x[q] = nx[q];
                    l[q] = nl[q];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NL; q++) {
            sp[idx[q]] = x[q];
            sl[idx[q]] = l[q];
        }
    }
#pragma unroll
    for (int j = 0; j < kAdjRun; j++)
        if (on[j] && rops[j].gen) acc_part(acc, rops[j].slot, nw, warp_part(dot[j]));
}

// A run of one X step (the CNOTs of the sweep: X on one target under
// controls): the pairs whose controls match swap in psi and lambda.
__device__ __forceinline__ void adj_x1(const AdjTileOp& op, uint64_t base, double2* __restrict__ sp,
                                       double2* __restrict__ sl, uint32_t T) {
    if ((base & op.gcmask) != op.gcval) return;  // uniform over the tile
    const int p = op.tl[0];
    const uint32_t cm = op.lcmask, cv = op.lcval;
    const uint32_t ngroups = T >> 1;
    for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
        const uint32_t b = adj_ins0(g, p);
        if ((b & cm) != cv) continue;
        const uint32_t i0 = adj_swz(b), i1 = adj_swz(b | (1u << p));
        const double2 x0 = sp[i0], x1 = sp[i1], l0 = sl[i0], l1 = sl[i1];
        sp[i0] = x1;
        sp[i1] = x0;
        sl[i0] = l1;
        sl[i1] = l0;
    }
}

// A fused run (kAdjFused) on the groups of the tile owned by this thread:
// coefficients in registers, every group read once, P = conj(lambda_r) psi_c
// formed once for all the run's dots, A applied once.
__device__ __forceinline__ void adj_fused1(const AdjTileOp& op, double2* __restrict__ sp, double2* __restrict__ sl,
                                           uint32_t T, double* __restrict__ acc, uint32_t nw) {
    const uint32_t ngroups = T >> 1;
    const int p = op.tl[0];
    const int ng = op.ngen;
    const bool apply = !op.a_id;
    const double2 a0 = op.m[0], a1 = op.m[1], a2 = op.m[2], a3 = op.m[3];
    double2 G[kAdjFusedGens][4];
    double dot[kAdjFusedGens];
#pragma unroll
    for (int j = 0; j < kAdjFusedGens; j++) {
        dot[j] = 0.0;
#pragma unroll
        for (int q = 0; q < 4; q++) G[j][q] = j < ng ? op.m[4 + 4 * j + q] : make_double2(0.0, 0.0);
    }
    for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
        const uint32_t b = adj_ins0(g, p);
        const uint32_t i0 = adj_swz(b), i1 = adj_swz(b | (1u << p));
        const double2 x0 = sp[i0], x1 = sp[i1], l0 = sl[i0], l1 = sl[i1];
        // P[r][c] = conj(l_r) * x_c
        const double2 p00 = make_double2(fma(l0.x, x0.x, l0.y * x0.y), fma(l0.x, x0.y, -l0.y * x0.x));
        const double2 p01 = make_double2(fma(l0.x, x1.x, l0.y * x1.y), fma(l0.x, x1.y, -l0.y * x1.x));
        const double2 p10 = make_double2(fma(l1.x, x0.x, l1.y * x0.y), fma(l1.x, x0.y, -l1.y * x0.x));
        const double2 p11 = make_double2(fma(l1.x, x1.x, l1.y * x1.y), fma(l1.x, x1.y, -l1.y * x1.x));
#pragma unroll
        for (int j = 0; j < kAdjFusedGens; j++) {
            if (j < ng) {
                // Re sum_rc G'[r][c] P[r][c]
                double d = fma(G[j][0].x, p00.x, -G[j][0].y * p00.y);
                d = fma(G[j][1].x, p01.x, fma(-G[j][1].y, p01.y, d));
                d = fma(G[j][2].x, p10.x, fma(-G[j][2].y, p10.y, d));
                d = fma(G[j][3].x, p11.x, fma(-G[j][3].y, p11.y, d));
                dot[j] += d;
            }
        }
        if (apply) {
            sp[i0] = cfma2(cmul2(a0, x0), a1, x1);
            sp[i1] = cfma2(cmul2(a2, x0), a3, x1);
            sl[i0] = cfma2(cmul2(a0, l0), a1, l1);
            sl[i1] = cfma2(cmul2(a2, l0), a3, l1);
        }
    }
#pragma unroll
    for (int j = 0; j < kAdjFusedGens; j++)
        if (j < ng) acc_part(acc, op.gslot[j], nw, warp_part(dot[j]));
}

// A segment: consecutive 1-qubit ops of a pass whose targets lie on two
// local positions p0 < p1.  Thread g owns group g (the 4 amplitudes of psi
// and lambda at local indices b, b + 2^p0, b + 2^p1, b + 2^p0 + 2^p1, b with
// zeros at p0 and p1), loads it once, applies every op of the segment in
// registers in order (pairs along the op's position; in-tile controls
// checked per pair, out-of-tile controls per tile) and stores it once.
// Each generator dot is reduced over the warp right after its op and added
// to the warp's slot (lane 0), as in the one-op forms.
template <int S>
__device__ __forceinline__ void seg_pair_idx(int q, int& a, int& b) {
    // q-th pair (q = 0, 1) along segment bit S of the group's index 0..3
    if (S == 0) {
        a = 2 * q;
        b = 2 * q + 1;
    } else {
        a = q;
        b = q + 2;
    }
}

// A non-folded segment op on pair Q of the group (its controls checked by
// the caller): a generator dot, or U^dagger on psi and lambda.
template <int S, int Q>
__device__ __forceinline__ void seg_pair(const AdjOpCtl& c, const AdjTileOp& op, double2 (&x)[4], double2 (&l)[4],
                                         bool valid, double& dot) {
    int ia, ib;
    seg_pair_idx<S>(Q, ia, ib);
    if (c.gen) {
        if (!valid) return;
        const double2 y0 = cfma2(cmul2(op.m[0], x[ia]), op.m[1], x[ib]);
        const double2 y1 = cfma2(cmul2(op.m[2], x[ia]), op.m[3], x[ib]);
        dot += redot(l[ia], y0) + redot(l[ib], y1);
    } else if (c.cls == GC_X) {
        double2 t = x[ia];
        x[ia] = x[ib];
        x[ib] = t;
        t = l[ia];
        l[ia] = l[ib];
        l[ib] = t;
    } else if (c.cls == GC_DIAG) {
        if (op.active & 1) {
            x[ia] = cmul2(op.m[0], x[ia]);
            l[ia] = cmul2(op.m[0], l[ia]);
        }
        if (op.active & 2) {
            x[ib] = cmul2(op.m[1], x[ib]);
            l[ib] = cmul2(op.m[1], l[ib]);
        }
    } else {
        const double2 x0 = x[ia], x1 = x[ib], l0 = l[ia], l1 = l[ib];
        x[ia] = cfma2(cmul2(op.m[0], x0), op.m[1], x1);
        x[ib] = cfma2(cmul2(op.m[2], x0), op.m[3], x1);
        l[ia] = cfma2(cmul2(op.m[0], l0), op.m[1], l1);
        l[ib] = cfma2(cmul2(op.m[2], l0), op.m[3], l1);
    }
}

// One op of a segment on the thread's group (base gb, segment bit masks m0,
// m1).  Dots are summed over the group's two pairs, then over the warp, and
// added to the warp's slot.
template <int S>
__device__ __forceinline__ void seg_op(const AdjOpCtl& c, const AdjTileOp& op, double2 (&x)[4], double2 (&l)[4],
                                       uint32_t gb, uint32_t m0, uint32_t m1, bool valid, uint64_t base,
                                       double* __restrict__ acc, uint32_t nw) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (c.cls == kAdjFusedPair || c.cls == kAdjFusedCtl) {
        const int ng = c.ngen;
        double dot[kAdjPairGens] = {0.0, 0.0};
        // coefficient set of each pair: by pair, or by the group's bits
        const int sel = (gb & op.xmask) == op.xval && (base & op.xgmask) == op.xgval ? 1 : 0;
        const int s0 = c.cls == kAdjFusedPair ? 0 : sel, s1 = c.cls == kAdjFusedPair ? 1 : sel;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            int ia, ib;
            seg_pair_idx<S>(q, ia, ib);
            const double2* mq = op.m + 8 * (q ? s1 : s0);
            const double2 x0 = x[ia], x1 = x[ib], l0 = l[ia], l1 = l[ib];
            if (valid && ng > 0) {
                const double i00 = fma(l0.x, x0.y, -l0.y * x0.x);  // Im P00
                const double i11 = fma(l1.x, x1.y, -l1.y * x1.x);  // Im P11
                const double qx = fma(l0.x, x1.x, fma(l0.y, x1.y, fma(-l1.x, x0.x, -l1.y * x0.y)));
                const double qy = fma(l0.x, x1.y, fma(-l0.y, x1.x, fma(-l1.y, x0.x, l1.x * x0.y)));
#pragma unroll
                for (int j = 0; j < kAdjPairGens; j++)
                    if (j < ng) {
                        const double2 gd = mq[4 + 2 * j], g01 = mq[5 + 2 * j];
                        dot[j] += fma(gd.x, i00, fma(gd.y, i11, fma(g01.x, qx, -g01.y * qy)));
                    }
            }
            const double2 a0 = mq[0], a1 = mq[1], a2 = mq[2], a3 = mq[3];
            x[ia] = cfma2(cmul2(a0, x0), a1, x1);
            x[ib] = cfma2(cmul2(a2, x0), a3, x1);
            l[ia] = cfma2(cmul2(a0, l0), a1, l1);
            l[ib] = cfma2(cmul2(a2, l0), a3, l1);
        }
        if (ng == 2) {
            const double d = warp_part_pair(dot[0], dot[1]);
            acc_part(acc, c.gslot[0], nw, d);
            __syncwarp();  // (the two slots may coincide)
            if ((lane & 16) && (lane & 15) < (uint32_t)kAdjSub)
                acc[((uint32_t)c.gslot[1] * nw + warp) * kAdjSub + (lane & 15)] += d;
        } else if (ng == 1) {
            acc_part(acc, c.gslot[0], nw, warp_part(dot[0]));
        }
        return;
    }
    if (c.cls == kAdjFused) {
        // G'_j = A^dagger G_j A is anti-Hermitian like the generators
        // (G = -i times a Hermitian matrix; the host folds only such runs):
        // Re sum_rc G'[r][c] P[r][c] = -Im G'00 Im P00 - Im G'11 Im P11
        //                              + Re(G'01 (P01 - conj(P10))),
        // P[r][c] = conj(l_r) x_c
        const int ng = c.ngen;
        double dot[kAdjFusedGens] = {0.0, 0.0, 0.0};
        const bool apply = !c.a_id;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            int ia, ib;
            seg_pair_idx<S>(q, ia, ib);
            const double2 x0 = x[ia], x1 = x[ib], l0 = l[ia], l1 = l[ib];
            if (valid && ng > 0) {
                const double i00 = fma(l0.x, x0.y, -l0.y * x0.x);  // Im P00
                const double i11 = fma(l1.x, x1.y, -l1.y * x1.x);  // Im P11
                const double qx = fma(l0.x, x1.x, fma(l0.y, x1.y, fma(-l1.x, x0.x, -l1.y * x0.y)));
                const double qy = fma(l0.x, x1.y, fma(-l0.y, x1.x, fma(-l1.y, x0.x, l1.x * x0.y)));
#pragma unroll
                for (int j = 0; j < kAdjFusedGens; j++)
                    if (j < ng) {
                        const double2 g01 = op.m[5 + 4 * j];
                        dot[j] += fma(-op.m[4 + 4 * j].y, i00,
                                      fma(-op.m[7 + 4 * j].y, i11, fma(g01.x, qx, -g01.y * qy)));
                    }
            }
            if (apply) {
                const double2 a0 = op.m[0], a1 = op.m[1], a2 = op.m[2], a3 = op.m[3];
                x[ia] = cfma2(cmul2(a0, x0), a1, x1);
                x[ib] = cfma2(cmul2(a2, x0), a3, x1);
                l[ia] = cfma2(cmul2(a0, l0), a1, l1);
                l[ib] = cfma2(cmul2(a2, l0), a3, l1);
            }
        }
        if (ng >= 2) {
            const double d = warp_part_pair(dot[0], dot[1]);
            acc_part(acc, c.gslot[0], nw, d);
            __syncwarp();  // (the two slots may coincide)
            if ((lane & 16) && (lane & 15) < (uint32_t)kAdjSub)
                acc[((uint32_t)c.gslot[1] * nw + warp) * kAdjSub + (lane & 15)] += d;
            if (ng == 3) acc_part(acc, c.gslot[2], nw, warp_part(dot[2]));
        } else if (ng == 1) {
            acc_part(acc, c.gslot[0], nw, warp_part(dot[0]));
        }
        return;
    }
    double dot = 0.0;
    if (c.upair) {
        // the only in-tile control is the other segment bit: one pair, the
        // same in every lane
        if (c.upair == 1)
            seg_pair<S, 0>(c, op, x, l, valid, dot);
        else
            seg_pair<S, 1>(c, op, x, l, valid, dot);
    } else {
        // local index of a pair's first amplitude: the group base with the
        // other segment bit q
        if ((gb & c.lcmask) == c.lcval) seg_pair<S, 0>(c, op, x, l, valid, dot);
        if (((gb | (S == 0 ? m1 : m0)) & c.lcmask) == c.lcval) seg_pair<S, 1>(c, op, x, l, valid, dot);
    }
    if (c.gen) acc_part(acc, c.slot, nw, warp_part(dot));
}

__device__ __forceinline__ void adj_seg(const AdjTileOp* __restrict__ sops, int nr, uint64_t base,
                                        double2* __restrict__ sp, double2* __restrict__ sl, uint32_t T,
                                        double* __restrict__ acc, uint32_t nw) {
    const int p0 = sops[0].seg[0], p1 = sops[0].seg[1];
    const uint32_t m0 = 1u << p0, m1 = 1u << p1;
    const uint32_t g = threadIdx.x;
    const bool valid = g < (T >> 2);
    const uint32_t gb = valid ? adj_ins0(adj_ins0(g, p0), p1) : 0u;
    double2 x[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint32_t li = gb | ((q & 1) ? m0 : 0u) | ((q & 2) ? m1 : 0u);
        if (valid) {
            x[q] = sp[adj_swz(li)];
            l[q] = sl[adj_swz(li)];
        } else {
            x[q] = l[q] = make_double2(0.0, 0.0);
        }
    }
    for (int j = 0; j < nr; j++) {
        const AdjTileOp& op = sops[j];
        const AdjOpCtl c = static_cast<const AdjOpCtl&>(op);  // four 16-byte loads
        if ((base & c.gcmask) != c.gcval) continue;  // uniform over the tile
        if (c.tl[0] == p0)
            seg_op<0>(c, op, x, l, gb, m0, m1, valid, base, acc, nw);
        else
            seg_op<1>(c, op, x, l, gb, m0, m1, valid, base, acc, nw);
    }
    if (valid)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t li = gb | ((q & 1) ? m0 : 0u) | ((q & 2) ? m1 : 0u);
            sp[adj_swz(li)] = x[q];
            sl[adj_swz(li)] = l[q];
        }
}

constexpr uint64_t kAdjWaitNs = 1000000000ull;  // 1 s
constexpr int kAdjMaxStages = 3;

__device__ __forceinline__ uint64_t adj_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One pass of the reverse sweep over every tile of psi and lambda.
// TMA form (hdr.use_tma): `nstage` buffers, each psi's and lambda's tile;
// one thread issues the next tile's box copies (tensor maps mpsi, mlam)
// while the current tile is computed, every thread waits for its tile on
// the buffer's mbarrier (bounded: 1 s, then `*err` is set and the pass's
// results are void), and the same thread stores both tiles back with bulk
// tensor stores.  Plain form (tiny states): cp.async in, plain stores out.
__global__ void __launch_bounds__(kAdjThreads, 1)
    k_adjoint_tiles(double2* __restrict__ psi, double2* __restrict__ lam, const AdjTileHdr phdr,
                    const AdjTileOp* __restrict__ gops, double* __restrict__ partial, int* __restrict__ err,
                    const __grid_constant__ CUtensorMap mpsi, const __grid_constant__ CUtensorMap mlam) {
    extern __shared__ __align__(1024) unsigned char adj_smem[];
    __shared__ AdjTileHdr hdr;
    __shared__ uint64_t hoff[1 << kAdjScatter];
    __shared__ uint64_t full_bar[kAdjMaxStages];
    if (threadIdx.x == 0) hdr = phdr;
    __syncthreads();
    const uint32_t T = 1u << hdr.tbits;
    const uint32_t nw = blockDim.x >> 5;
    const bool use_tma = hdr.use_tma != 0;
    const int nbuf = use_tma ? hdr.nstage : 1;
    unsigned char* smem = adj_smem + ((1024u - (tc::smem_u32(adj_smem) & 1023u)) & 1023u);
    const uint32_t tile_bytes = T * (uint32_t)sizeof(double2);  // one array's tile
    AdjTileOp* ops = (AdjTileOp*)(smem + (size_t)nbuf * 2 * tile_bytes);
    double* acc = (double*)(ops + hdr.nops);  // [slot][warp][kAdjSub]
    const int nlow = min(kAdjLowBits, hdr.tbits), nh = hdr.tbits - nlow;
    {
        const uint64_t* src = (const uint64_t*)gops;
        uint64_t* dst = (uint64_t*)ops;
        for (int i = threadIdx.x; i < hdr.nops * (int)(sizeof(AdjTileOp) / 8); i += blockDim.x) dst[i] = src[i];
        for (int i = threadIdx.x; i < hdr.nslots * (int)nw * kAdjSub; i += blockDim.x) acc[i] = 0.0;
        for (uint32_t h = threadIdx.x; h < (1u << nh); h += blockDim.x) {
            uint64_t o = 0;
            for (int j = 0; j < nh; j++) o |= (uint64_t)((h >> j) & 1) << hdr.hb[j];
            hoff[h] = o;
        }
    }
    auto tile_base = [&](uint64_t t) {
        uint64_t base = 0;
        for (int i = 0; i < hdr.nouts; i++) base |= ((t >> i) & 1) << hdr.outb[i];
        return base;
    };
    const uint32_t sbase = tc::smem_u32(smem);
    auto issue = [&](uint64_t t, int b) {  // thread 0: both tiles of tile t into buffer b
        tc::mbar_arrive_expect_tx(&full_bar[b], 2 * tile_bytes);
        const uint64_t base = tile_base(t);
        const uint32_t dst = sbase + (uint32_t)b * 2 * tile_bytes;
        tma::load_boxes(&mpsi, hdr.tma, base, dst, tc::smem_u32(&full_bar[b]));
        tma::load_boxes(&mlam, hdr.tma, base, dst + tile_bytes, tc::smem_u32(&full_bar[b]));
    };
    uint32_t pending = 0;
    if (use_tma && threadIdx.x == 0) {
        tma::prefetch_map(&mpsi);
        tma::prefetch_map(&mlam);
        for (int q = 0; q < nbuf; q++) tc::mbar_init(&full_bar[q], 1);
        for (int q = 0; q < (nbuf > 2 ? nbuf - 1 : 1); q++)
            if (blockIdx.x + (uint64_t)q * gridDim.x < hdr.ntiles) {
                issue(blockIdx.x + (uint64_t)q * gridDim.x, q);
                pending |= 1u << q;
            }
    }
    __syncthreads();
    const uint32_t lmask = (1u << nlow) - 1;
    bool dead = false;
    uint32_t it = 0;
    // buffer of this tile (it % nbuf) and the parity of its use (it / nbuf),
    // carried from tile to tile instead of divided out
    uint32_t bcur = 0, bpar = 0;
    for (uint64_t t = blockIdx.x; t < hdr.ntiles;
         t += gridDim.x, it++, bcur = bcur + 1 == (uint32_t)nbuf ? 0u : bcur + 1, bpar ^= bcur == 0 ? 1u : 0u) {
        const uint64_t base = tile_base(t);
        const int b = use_tma ? (int)bcur : 0;
        double2* sp = (double2*)(smem + (size_t)b * 2 * tile_bytes);
        double2* sl = sp + T;
        if (use_tma) {
            if (threadIdx.x == 0 && nbuf == 2 && t + gridDim.x < hdr.ntiles) {
                const int bn = (int)((it + 1) & 1u);
                tma::wait_group_read<0>();  // the previous tile's stores have read buffer bn
                issue(t + gridDim.x, bn);
                pending |= 1u << bn;
            }
            if (!dead) {
                const uint32_t parity = bpar;
                const uint64_t t0 = adj_ns();
                while (!tc::mbar_try_wait(&full_bar[b], parity)) {
                    if (adj_ns() - t0 > kAdjWaitNs) {
                        dead = true;
                        atomicExch(err, 1);
                        break;
                    }
                }
                if (!dead && threadIdx.x == 0) pending &= ~(1u << b);
            }
        } else {
            // the tile's copies are issued back to back (cp.async), then waited for
            for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) {
                const uint64_t gi = base | (l & lmask) | hoff[l >> nlow];
                const uint32_t s = adj_swz(l);
                const uint32_t dp = (uint32_t)__cvta_generic_to_shared(&sp[s]);
                const uint32_t dl = (uint32_t)__cvta_generic_to_shared(&sl[s]);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dp), "l"(&psi[gi]) : "memory");
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dl), "l"(&lam[gi]) : "memory");
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            __syncthreads();
        }
        for (int oi = 0; oi < hdr.nops;) {
            // the run ends at the first op followed by a barrier
            int e = oi;
            while (!ops[e].sync) e++;
            e++;
            if (ops[oi].k == 1 && ops[oi].seg[0] != ops[oi].seg[1])
                adj_seg(ops + oi, e - oi, base, sp, sl, T, acc, nw);
            else if (ops[oi].cls == kAdjFused)
                adj_fused1(ops[oi], sp, sl, T, acc, nw);
            else if (e - oi == 1 && ops[oi].k == 1 && ops[oi].cls == GC_X && !ops[oi].gen)
                adj_x1(ops[oi], base, sp, sl, T);
            else if (ops[oi].k == 1)
                adj_run<1>(ops + oi, e - oi, base, sp, sl, T, acc, nw);
            else
                adj_run<2>(ops + oi, e - oi, base, sp, sl, T, acc, nw);
            __syncthreads();
            oi = e;
        }
        if (use_tma) {
            tc::fence_proxy_async();  // the tiles' writes are visible to the bulk stores
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint32_t src = sbase + (uint32_t)b * 2 * tile_bytes;
                tma::store_boxes(&mpsi, hdr.tma, base, src);
                tma::store_boxes(&mlam, hdr.tma, base, src + tile_bytes);
                tma::commit_group();
                if (nbuf == 1 && t + gridDim.x < hdr.ntiles) {
                    tma::wait_group_read<0>();
                    issue(t + gridDim.x, 0);
                    pending |= 1u;
                }
                // three buffers: the tile nbuf - 1 ahead into the buffer of
                // the previous tile, whose stores have had this tile's
                // compute to read it
                const uint64_t tn = t + (uint64_t)(nbuf - 1) * gridDim.x;
                if (nbuf > 2 && tn < hdr.ntiles) {
                    const int bn = (int)(bcur == 0 ? (uint32_t)nbuf - 1 : bcur - 1);
                    tma::wait_group_read<1>();
                    issue(tn, bn);
                    pending |= 1u << bn;
                }
            }
        } else {
            for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) {
                const uint64_t gi = base | (l & lmask) | hoff[l >> nlow];
                const uint32_t s = adj_swz(l);
                psi[gi] = sp[s];
                lam[gi] = sl[s];
            }
            __syncthreads();
        }
    }
    if (use_tma && threadIdx.x == 0) {
        tma::wait_group<0>();  // stores complete before the shared memory goes away
        const uint64_t t0 = adj_ns();
        for (int q = 0; q < nbuf; q++)
            if (pending & (1u << q))
                for (uint32_t ph = 0; ph < 2; ph++)
                    while (!tc::mbar_try_wait(&full_bar[q], ph) && adj_ns() - t0 < kAdjWaitNs) {
                    }
    }
    __syncthreads();
    // per CTA: slot sums over the warps' partial sums in order
    for (int sidx = threadIdx.x; sidx < hdr.nslots; sidx += blockDim.x) {
        double s = 0.0;
        for (uint32_t w = 0; w < nw * kAdjSub; w++) s += acc[sidx * nw * kAdjSub + w];
        partial[(size_t)blockIdx.x * hdr.nslots + sidx] = s;
    }
}

// dots[s] = sum over blocks of partial[b][s] (one block per slot, fixed order)
__global__ void k_adj_slot_sums(const double* __restrict__ partial, int nblocks, int nslots, double* __restrict__ dots) {
    __shared__ double sm[kAdjThreads / 32];
    const int s = blockIdx.x;
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partial[(size_t)b * nslots + s];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sm[w];
        dots[s] = t;
    }
}

// ------------------------------------------------------------------ host

namespace {

struct HostOp {
    AdjTileOp op;   // tl / lcmask / gcmask filled per pass
    int tb[2];      // global target bits
    std::vector<int> cb, cv;
    int grad = -1;  // generator: gradient index
};

struct AdjPass {
    AdjTileHdr hdr;
    std::vector<AdjTileOp> ops;
    std::vector<int> slot_grad;  // gradient index of each slot
};

bool to_host_op(const LGate& g, bool gen, int grad, HostOp& h) {
    if (g.k < 1 || g.k > 2 || g.nc > 62) return false;
    memset(&h.op, 0, sizeof(h.op));
    h.op.gen = gen ? 1 : 0;
    h.op.cls = gen ? GC_DENSE : g.cls;
    h.op.k = g.k;
    const size_t nl = (size_t)1 << g.k;
    if (h.op.cls == GC_DENSE) {
        if (g.m.size() != nl * nl) return false;
    } else if (h.op.cls == GC_DIAG) {
        if (g.m.size() != nl) return false;
        for (size_t q = 0; q < nl; q++)
            if (!(g.m[q].re == 1.0 && g.m[q].im == 0.0)) h.op.active |= (uint64_t)1 << q;
    } else if (h.op.cls == GC_X) {
        if (g.k != 1) return false;
    } else if (h.op.cls == GC_SWAP) {
        if (g.k != 2) return false;
    } else {
        return false;
    }
    for (size_t i = 0; i < g.m.size() && i < 16; i++) h.op.m[i] = make_double2(g.m[i].re, g.m[i].im);
    h.tb[0] = g.tb[0];
    h.tb[1] = g.k == 2 ? g.tb[1] : -1;
    h.cb.assign(g.cb, g.cb + g.nc);
    h.cv.assign(g.cv, g.cv + g.nc);
    h.grad = grad;
    return true;
}

// 2 x 2 complex helpers (host, FP64)
struct M2 {
    double2 e[4];
};
static M2 m2_mul(const M2& a, const M2& b) {
    M2 r;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            double re = 0, im = 0;
            for (int k = 0; k < 2; k++) {
                const double2 x = a.e[i * 2 + k], y = b.e[k * 2 + j];
                re += x.x * y.x - x.y * y.y;
                im += x.x * y.y + x.y * y.x;
            }
            r.e[i * 2 + j] = make_double2(re, im);
        }
    return r;
}
static M2 m2_adj(const M2& a) {
    M2 r;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) r.e[i * 2 + j] = make_double2(a.e[j * 2 + i].x, -a.e[j * 2 + i].y);
    return r;
}
static bool m2_of(const AdjTileOp& op, M2& m) {
    const double2 z = make_double2(0, 0), one = make_double2(1, 0);
    if (op.cls == GC_DENSE)
        for (int q = 0; q < 4; q++) m.e[q] = op.m[q];
    else if (op.cls == GC_DIAG)
        m = M2{{op.m[0], z, z, op.m[1]}};
    else if (op.cls == GC_X)
        m = M2{{z, one, one, z}};
    else
        return false;
    return true;
}

// G' anti-Hermitian to 1e-12 of its largest entry (the generators of
// parametric gates are -i times a Hermitian matrix, src/gate.rs, and so is
// A^dagger G A): real parts of the diagonal zero, G'10 = -conj(G'01)
static bool m2_antihermitian(const M2& g) {
    double mx = 0.0;
    for (int q = 0; q < 4; q++) mx = std::max(mx, std::hypot(g.e[q].x, g.e[q].y));
    const double tol = 1e-12 * std::max(mx, 1e-300);
    return std::fabs(g.e[0].x) <= tol && std::fabs(g.e[3].x) <= tol && std::fabs(g.e[1].x + g.e[2].x) <= tol &&
           std::fabs(g.e[1].y - g.e[2].y) <= tol;
}

// Fold runs of uncontrolled 1-qubit steps on one target into kAdjFused ops
// (at most kAdjFusedGens generator dots each).
static void fuse_runs(std::vector<AdjTileOp>& ops) {
    const char* env = getenv("YAO_ADJ_FUSE");
    if (env && env[0] == '0') return;  // YAO_ADJ_FUSE=0: every step its own op
    auto plain = [](const AdjTileOp& o) { return o.k == 1 && o.lcmask == 0 && o.gcmask == 0; };
    std::vector<AdjTileOp> out;
    size_t i = 0;
    while (i < ops.size()) {
        if (!plain(ops[i])) {
            out.push_back(ops[i++]);
            continue;
        }
        AdjTileOp f;
        memset(&f, 0, sizeof(f));
        f.cls = kAdjFused;
        f.k = 1;
        f.tl[0] = ops[i].tl[0];
        f.slot = -1;
        M2 A{{make_double2(1, 0), make_double2(0, 0), make_double2(0, 0), make_double2(1, 0)}};
        bool any_u = false;
        size_t j = i;
        for (; j < ops.size() && plain(ops[j]) && ops[j].tl[0] == f.tl[0]; j++) {
            const AdjTileOp& o = ops[j];
            M2 m;
            if (!m2_of(o, m)) break;
            if (o.gen) {
                if (f.ngen == kAdjFusedGens) break;
                const M2 g = m2_mul(m2_adj(A), m2_mul(m, A));
                if (!m2_antihermitian(g)) break;  // the register segments' dot formula needs G'^dagger = -G'
                for (int q = 0; q < 4; q++) f.m[4 + 4 * f.ngen + q] = g.e[q];
                f.gslot[f.ngen++] = o.slot;
            } else {
                A = m2_mul(m, A);
                any_u = true;
            }
        }
        if (j == i) {  // not foldable after all
            out.push_back(ops[i++]);
            continue;
        }
        for (int q = 0; q < 4; q++) f.m[q] = A.e[q];
        f.a_id = any_u ? 0 : 1;
        out.push_back(f);
        i = j;
    }
    ops.swap(out);
}

// YAO_ADJ_SEGMENTS=0: one-op forms only (no register segments)
static bool segments_on() {
    const char* e = getenv("YAO_ADJ_SEGMENTS");
    return !(e && e[0] == '0');
}

// YAO_ADJ_XFOLD=0: keep segment X steps as ops of their own
static bool xfold_on() {
    const char* e = getenv("YAO_ADJ_XFOLD");
    return !(e && e[0] == '0');
}

// The steps of a pass re-sequenced for register segments: a scan in sweep
// order emits every ready 1-qubit step whose target is one of the current
// segment's two bits (or becomes its second; a step with one control that
// opens a segment brings its control as the second bit, when steps of the
// pass act on that qubit); when a scan emits nothing the
// segment closes and the next one starts at the first remaining step (a
// 2-qubit step is emitted alone).  A step is ready when no earlier
// remaining step of the pass shares a qubit with it, so the dependencies of
// the sweep hold.
static std::vector<size_t> segment_order(const std::vector<HostOp>& hops, const std::vector<uint64_t>& qm,
                                         const std::vector<size_t>& take) {
    std::vector<size_t> order;
    order.reserve(take.size());
    std::vector<char> done(take.size(), 0);
    size_t left = take.size();
    int sb[2] = {-1, -1}, nsb = 0;
    // remaining 1-qubit steps per target qubit
    std::vector<int> on_target(64, 0);
    for (size_t i = 0; i < take.size(); i++)
        if (hops[take[i]].op.k == 1) on_target[hops[take[i]].tb[0]]++;
    while (left) {
        bool emitted = false;
        uint64_t blocked = 0;
        for (size_t i = 0; i < take.size(); i++) {
            if (done[i]) continue;
            const HostOp& h = hops[take[i]];
            const uint64_t m = qm[take[i]];
            if (m & blocked) {
                blocked |= m;
                continue;
            }
            bool fit = false;
            if (h.op.k == 1) {
                const int t = h.tb[0];
                if (t == sb[0] || t == sb[1]) {
                    fit = true;
                } else if (nsb < 2) {
                    sb[nsb++] = t;
                    fit = true;
                    // a step with one control (a CNOT) opens the segment: its
                    // control becomes the second bit when steps of the pass act
                    // on it, so the step can merge into a folded run
                    if (nsb == 1 && xfold_on() && h.cb.size() == 1 && h.cb[0] != t && on_target[h.cb[0]] > 0)
                        sb[nsb++] = h.cb[0];
                }
            }
            if (!fit) {
                blocked |= m;
                continue;
            }
            order.push_back(take[i]);
            if (h.op.k == 1) on_target[h.tb[0]]--;
            done[i] = 1;
            left--;
            emitted = true;
        }
        if (emitted) continue;
        sb[0] = sb[1] = -1;
        nsb = 0;
        for (size_t i = 0; i < take.size(); i++)
            if (!done[i]) {
                if (hops[take[i]].op.k == 2) {
                    order.push_back(take[i]);
                    done[i] = 1;
                    left--;
                }
                break;
            }
    }
    return order;
}

// Barriers and segments of a pass's ops.  Segments (on): maximal runs of
// 1-qubit ops on at most two local positions, seg[] = those positions (a
// second one added when the run uses one), a barrier after the last.  Runs
// of 2-qubit ops (and, segments off, of 1-qubit ops) on the same positions
// share a barrier up to kAdjRun ops; fused ops stand alone.
static bool upair_on() {
    const char* e = getenv("YAO_ADJ_UPAIR");
    return !(e && e[0] == '0');
}

// One segment's ops [i, j) (seg[], upair set) with every X step that acts on
// one pair of every group (upair, no out-of-tile controls) merged into an
// adjacent folded run on its target (kAdjFusedPair); returns the new ops.
static std::vector<AdjTileOp> fold_segment_x(const std::vector<AdjTileOp>& ops, size_t i, size_t j) {
    struct Pair {
        M2 a[2], g[2][kAdjPairGens];
    };
    std::vector<AdjTileOp> out;
    std::vector<Pair> pp;        // per-pair coefficients of out[k] (when its cls is kAdjFusedPair)
    const uint32_t segbits = (1u << ops[i].seg[0]) | (1u << ops[i].seg[1]);
    // the merged kind of an X step: per pair (its only control is the other
    // segment bit), per group (in-tile controls off the segment), or none
    auto x_kind = [&](const AdjTileOp& o) -> int32_t {
        if (o.cls != GC_X || o.gen || o.k != 1) return 0;
        if (o.upair && o.gcmask == 0) return kAdjFusedPair;
        if ((o.lcmask || o.gcmask) && !(o.lcmask & segbits)) return kAdjFusedCtl;
        return 0;
    };
    // out[k] becomes a merged run of `kind` (with the X's controls) when it can
    auto to_pair = [&](size_t k, int32_t kind, const AdjTileOp& x) -> bool {
        AdjTileOp& f = out[k];
        if (f.cls == kind)
            return kind == kAdjFusedPair || (f.xmask == x.lcmask && f.xval == x.lcval && f.xgmask == x.gcmask &&
                                             f.xgval == x.gcval);
        if (f.cls != kAdjFused || f.ngen > kAdjPairGens) return false;
        Pair p;
        for (int q = 0; q < 2; q++) {
            for (int e = 0; e < 4; e++) p.a[q].e[e] = f.m[e];
            for (int g = 0; g < f.ngen; g++)
                for (int e = 0; e < 4; e++) p.g[q][g].e[e] = f.m[4 + 4 * g + e];
        }
        pp[k] = p;
        f.cls = kind;
        f.a_id = 0;
        if (kind == kAdjFusedCtl) {
            f.xmask = x.lcmask;
            f.xval = x.lcval;
            f.xgmask = x.gcmask;
            f.xgval = x.gcval;
        }
        return true;
    };
    std::vector<bool> used(j, false);  // runs already moved back and merged
    for (size_t q = i; q < j; q++) {
        if (used[q]) continue;
        const AdjTileOp& o = ops[q];
        const int32_t kind = x_kind(o);
        if (kind) {
            // coefficient set the X acts on: its pair, or set 1
            const int cv = kind == kAdjFusedPair ? o.upair - 1 : 1;
            // after the previous run on the same target: A_cv = X A
            if (!out.empty() && out.back().tl[0] == o.tl[0] && to_pair(out.size() - 1, kind, o)) {
                M2& a = pp.back().a[cv];
                a = M2{{a.e[2], a.e[3], a.e[0], a.e[1]}};
                continue;
            }
            // before the next run on the same target, which moves back to the
            // X past the steps in between (they neither act on nor are
            // controlled by its bit, so they commute with it and their dots
            // do not change): A_cv = A X, G'_cv = X G' X
            const uint32_t tbit = 1u << o.tl[0];
            size_t k = q + 1;
            // (runs already moved back sit before this X: passed over)
            while (k < j && (used[k] || (ops[k].tl[0] != o.tl[0] && !(ops[k].lcmask & tbit)))) k++;
            if (k < j && !used[k] && ops[k].tl[0] == o.tl[0] && ops[k].cls == kAdjFused &&
                ops[k].ngen <= kAdjPairGens) {
                out.push_back(ops[k]);
                pp.emplace_back();
                to_pair(out.size() - 1, kind, o);
                Pair& p = pp.back();
                M2& a = p.a[cv];
                a = M2{{a.e[1], a.e[0], a.e[3], a.e[2]}};
                for (int g = 0; g < out.back().ngen; g++) {
                    M2& m = p.g[cv][g];
                    m = M2{{m.e[3], m.e[2], m.e[1], m.e[0]}};
                }
                used[k] = true;
                continue;
            }
        }
        out.push_back(o);
        pp.emplace_back();
    }
    for (size_t k = 0; k < out.size(); k++) {
        AdjTileOp& f = out[k];
        if (f.cls != kAdjFusedPair && f.cls != kAdjFusedCtl) continue;
        const Pair& p = pp[k];
        for (int q = 0; q < 2; q++) {
            for (int e = 0; e < 4; e++) f.m[8 * q + e] = p.a[q].e[e];
            for (int g = 0; g < kAdjPairGens; g++) {
                const M2& m = p.g[q][g];
                f.m[8 * q + 4 + 2 * g] = g < f.ngen ? make_double2(-m.e[0].y, -m.e[3].y) : make_double2(0, 0);
                f.m[8 * q + 5 + 2 * g] = g < f.ngen ? m.e[1] : make_double2(0, 0);
            }
        }
    }
    return out;
}

static void mark_barriers(std::vector<AdjTileOp>& ops, bool seg) {
    size_t i = 0;
    while (i < ops.size()) {
        if (seg && ops[i].k == 1) {
            int P[2] = {ops[i].tl[0], -1};
            size_t j = i + 1;
            for (; j < ops.size() && ops[j].k == 1; j++) {
                const int t = ops[j].tl[0];
                if (t == P[0] || t == P[1]) continue;
                if (P[1] >= 0) break;
                P[1] = t;
            }
            if (P[1] < 0) P[1] = P[0] == 0 ? 1 : 0;
            const int lo = std::min(P[0], P[1]), hi = std::max(P[0], P[1]);
            for (size_t q = i; q < j; q++) {
                ops[q].seg[0] = (int8_t)lo;
                ops[q].seg[1] = (int8_t)hi;
                ops[q].sync = (int8_t)(q + 1 == j ? 1 : 0);
                const uint32_t other = 1u << (ops[q].tl[0] == lo ? hi : lo);
                ops[q].upair = (int8_t)(upair_on() && ops[q].cls != kAdjFused && ops[q].lcmask == other
                                            ? 1 + (ops[q].lcval != 0)
                                            : 0);
            }
            if (xfold_on()) {
                std::vector<AdjTileOp> f = fold_segment_x(ops, i, j);
                if (f.size() < j - i) {
                    for (AdjTileOp& o : f) o.sync = 0;
                    f.back().sync = 1;
                    ops.erase(ops.begin() + (std::ptrdiff_t)i, ops.begin() + (std::ptrdiff_t)j);
                    ops.insert(ops.begin() + (std::ptrdiff_t)i, f.begin(), f.end());
                    j = i + f.size();
                }
            }
            i = j;
            continue;
        }
        ops[i].seg[0] = ops[i].seg[1] = 0;
        size_t j = i + 1;
        if (ops[i].cls != kAdjFused)
            while (j < ops.size() && (int)(j - i) < kAdjRun && ops[j].cls != kAdjFused && ops[j].k == ops[i].k &&
                   ops[j].tl[0] == ops[i].tl[0] && (ops[i].k == 1 || ops[j].tl[1] == ops[i].tl[1]) &&
                   !(seg && ops[j].k == 1)) {
                ops[j].seg[0] = ops[j].seg[1] = 0;
                ops[j - 1].sync = 0;
                j++;
            }
        ops[j - 1].sync = 1;
        i = j;
    }
}

// Passes by list scheduling over the reverse sweep's dependencies.  Steps
// on disjoint qubits (targets and controls) commute exactly (in
// arithmetic they differ by rounding only), and a generator dot taken
// before or after a step on other qubits is the same number
// (<l| h G h^dagger |p> = <l|G|p> when h and G act on different qubits).
// So a pass scans the remaining steps in sweep order and takes every step
// that no skipped earlier step shares a qubit with, while the targets above
// the low bits fit the tile's scattered bits and the op / slot limits hold;
// a skipped step blocks its qubits for the rest of the scan.  The steps of
// a pass keep their sweep order.
void plan_adj(const std::vector<HostOp>& hops, uint32_t nbits, std::vector<AdjPass>& out) {
    const int tbits = (int)std::min<uint32_t>(nbits, kAdjLowBits + kAdjScatter);
    const int nlow = std::min(kAdjLowBits, tbits), S = tbits - nlow;
    const uint64_t all = nbits >= 64 ? ~0ull : ((1ull << nbits) - 1);
    std::vector<uint64_t> qm(hops.size(), 0);
    for (size_t j = 0; j < hops.size(); j++) {
        for (int q = 0; q < hops[j].op.k; q++) qm[j] |= 1ull << hops[j].tb[q];
        for (int b : hops[j].cb) qm[j] |= 1ull << b;
    }
    std::vector<char> used(hops.size(), 0);
    const char* env = getenv("YAO_ADJ_REORDER");
    const bool reorder = !(env && env[0] == '0');  // YAO_ADJ_REORDER=0: consecutive steps only
    size_t first = 0;
    while (first < hops.size()) {
        std::set<int> H;
        std::vector<size_t> take;
        uint64_t blocked = 0;
        int nslots = 0;
        for (size_t j = first; j < hops.size(); j++) {
            if (used[j]) continue;
            if (qm[j] & blocked) {
                blocked |= qm[j];
                if ((blocked & all) == all) break;
                continue;
            }
            std::set<int> need;
            for (int q = 0; q < hops[j].op.k; q++)
                if (hops[j].tb[q] >= nlow && !H.count(hops[j].tb[q])) need.insert(hops[j].tb[q]);
            const bool fits = (int)(H.size() + need.size()) <= S && (int)take.size() < kAdjMaxOps &&
                              !(hops[j].op.gen && nslots >= kAdjMaxSlots);
            if (!fits) {
                if (!reorder) break;
                blocked |= qm[j];
                if ((blocked & all) == all) break;
                continue;
            }
            H.insert(need.begin(), need.end());
            if (hops[j].op.gen) nslots++;
            take.push_back(j);
        }
        for (size_t j : take) used[j] = 1;
        while (first < hops.size() && used[first]) first++;
        if (segments_on()) take = segment_order(hops, qm, take);
        // the tile's scattered bits: the targets', then the lowest free bits
        for (int b = nlow; (int)H.size() < S && b < (int)nbits; b++) H.insert(b);
        AdjPass pass;
        memset(&pass.hdr, 0, sizeof(pass.hdr));
        pass.hdr.tbits = tbits;
        int local[64];
        for (int b = 0; b < 64; b++) local[b] = -1;
        for (int b = 0; b < nlow; b++) local[b] = b;
        int pos = nlow;
        for (int b : H) {
            pass.hdr.hb[pos - nlow] = (int8_t)b;
            local[b] = pos++;
        }
        int no = 0;
        for (int b = 0; b < (int)nbits; b++)
            if (local[b] < 0) pass.hdr.outb[no++] = (int8_t)b;
        pass.hdr.nouts = no;
        pass.hdr.ntiles = (uint64_t)1 << (nbits - tbits);
        for (size_t q : take) {
            AdjTileOp op = hops[q].op;
            op.tl[0] = (int8_t)local[hops[q].tb[0]];
            if (op.k == 2) op.tl[1] = (int8_t)local[hops[q].tb[1]];
            for (size_t c = 0; c < hops[q].cb.size(); c++) {
                const int b = hops[q].cb[c];
                if (local[b] >= 0) {
                    op.lcmask |= 1u << local[b];
                    if (hops[q].cv[c]) op.lcval |= 1u << local[b];
                } else {
                    op.gcmask |= (uint64_t)1 << b;
                    if (hops[q].cv[c]) op.gcval |= (uint64_t)1 << b;
                }
            }
            if (op.gen) {
                op.slot = (int32_t)pass.slot_grad.size();
                pass.slot_grad.push_back(hops[q].grad);
            }
            pass.ops.push_back(op);
        }
        fuse_runs(pass.ops);
        mark_barriers(pass.ops, segments_on());
        pass.hdr.nops = (int32_t)pass.ops.size();
        pass.hdr.nslots = (int32_t)pass.slot_grad.size();
        out.push_back(std::move(pass));
    }
}

}  // namespace

// The host plan of a reverse sweep: its passes, their op and dot counts.
struct AdjPlan {
    std::vector<AdjPass> passes;
    size_t nops = 0, ndots = 0;
};

// The plan of expect_grad's reverse sweep over tiles (host only).  *status
// is YAO_ERR_UNSUPPORTED, and the result null, when some step is not a 1- or
// 2-qubit gate (the caller then runs the per-gate form).
AdjPlan* adjoint_plan_new(const Circuit* c, uint32_t n, int32_t precision, size_t np, int* status) {
    *status = YAO_ERR_UNSUPPORTED;
    if (n < 3 || n > 62 || precision != YAO_C128) return nullptr;
    std::vector<HostOp> hops;
    size_t slot = np;
    for (size_t ei = c->elems.size(); ei-- > 0;) {
        const Element& el = c->elems[ei];
        if (el.kind != YAO_ELEM_GATE) continue;
        const GateElem& g = el.g;
        std::vector<LGate> dag;
        lower_gate(gate_dagger(g), n, 0, false, dag);
        const int npar = gate_num_params(g.type);
        if (npar > 0) {
            if (slot < (size_t)npar) return nullptr;
            for (int i = 0; i < npar; i++) {
                std::vector<Cx> gm;
                uint32_t gd;
                gate_generator(g, i, gm, gd);
                HostOp h;
                if (!to_host_op(lower_matrix(gm, gd, false, g.targets, g.ctrls, g.cfgs, n, 0), true,
                                (int)(slot - npar + i), h))
                    return nullptr;
                hops.push_back(h);
            }
            slot -= npar;
        }
        for (const LGate& d : dag) {
            HostOp h;
            if (!to_host_op(d, false, -1, h)) return nullptr;
            hops.push_back(h);
        }
    }
    AdjPlan* plan = new AdjPlan();
    plan_adj(hops, n, plan->passes);
    for (const AdjPass& p : plan->passes) {
        plan->nops += p.ops.size();
        plan->ndots += p.slot_grad.size();
    }
    *status = YAO_OK;
    return plan;
}

void adjoint_plan_free(AdjPlan* p) { delete p; }

void adjoint_plan_counts(const AdjPlan* p, int64_t out[3]) {
    out[0] = (int64_t)p->passes.size();
    out[1] = (int64_t)p->nops;
    out[2] = (int64_t)p->ndots;
}

// The reverse sweep of a plan; psi holds the forward state and lambda =
// H psi on entry.  grad receives 2 Re <lambda | G psi> per parameter.
// Synchronises at the end; a set error word (from this sweep's bounded
// waits or from work queued before it) is reported as YAO_ERR_TIMEOUT.
int adjoint_run(Ctx* ctx, Reg* psi, Reg* lam, const AdjPlan* plan, double* grad) {
    const uint32_t n = psi->nbits;
    const std::vector<AdjPass>& passes = plan->passes;
    const size_t nops = plan->nops, ndots = plan->ndots;
    if (passes.empty()) return read_device_err(ctx, "expect_grad");
    const int tbits = passes[0].hdr.tbits;
    const size_t tile_bytes = (size_t)2 * ((size_t)1 << tbits) * sizeof(double2);  // psi's and lambda's tile
    // shared memory: the tile buffers (three when they fit), the ops and
    // slot accumulators of the largest pass, 1 KiB for aligning the tiles
    static int optin = 0;
    if (!optin) YAO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    size_t max_ops = 0, max_slots = 0;
    for (const AdjPass& p : passes) {
        max_ops = std::max(max_ops, p.ops.size());
        max_slots = std::max(max_slots, p.slot_grad.size());
    }
    const size_t slot_bytes = (size_t)(kAdjThreads / 32) * kAdjSub * sizeof(double);
    const size_t rest = max_ops * sizeof(AdjTileOp) + max_slots * slot_bytes + 1024;
    const size_t budget = (size_t)optin - 4096;  // static shared memory of the kernel
    const int nstage = 3 * tile_bytes + rest <= budget ? 3 : (2 * tile_bytes + rest <= budget ? 2 : 1);
    const size_t smem_max = (size_t)nstage * tile_bytes + rest;
    static bool attr = false;
    if (!attr) {
        YAO_CUDA(cudaFuncSetAttribute(k_adjoint_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
        attr = true;
    }
    int per_sm = 0;
    YAO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjoint_tiles, kAdjThreads, smem_max));
    const uint64_t ntiles = (uint64_t)1 << (n - tbits);
    const int grid = (int)std::min<uint64_t>(ntiles, (uint64_t)std::max(1, per_sm) * (uint64_t)ctx->num_sms);
    // device buffers: every pass's ops, the CTA partials, every pass's dots
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t b_ops = al(std::max<size_t>(1, nops) * sizeof(AdjTileOp)),
                 b_part = al((size_t)grid * kAdjMaxSlots * sizeof(double)), b_dots = al(std::max<size_t>(1, ndots) * 8);
    char* buf = nullptr;
    YAO_CUDA(cudaMallocAsync((void**)&buf, b_ops + b_part + b_dots, ctx->stream));
    AdjTileOp* d_ops = (AdjTileOp*)buf;
    double* d_part = (double*)(buf + b_ops);
    double* d_dots = (double*)(buf + b_ops + b_part);
    {
        std::vector<AdjTileOp> all;
        all.reserve(nops);
        for (const AdjPass& p : passes) all.insert(all.end(), p.ops.begin(), p.ops.end());
        YAO_CUDA(cudaMemcpyAsync(d_ops, all.data(), all.size() * sizeof(AdjTileOp), cudaMemcpyHostToDevice,
                                 ctx->stream));
    }
    if (!ctx->d_err) {
        YAO_CUDA(cudaMalloc((void**)&ctx->d_err, sizeof(int)));
        YAO_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    }
    size_t ooff = 0, doff = 0;
    for (const AdjPass& p : passes) {
        AdjTileHdr hdr = p.hdr;
        CUtensorMap mpsi, mlam;
        memset(&mpsi, 0, sizeof(mpsi));
        memset(&mlam, 0, sizeof(mlam));
        int8_t tb[kAdjLowBits + kAdjScatter];
        const int nlow = std::min(kAdjLowBits, hdr.tbits);
        for (int q = 0; q < hdr.tbits; q++) tb[q] = (int8_t)(q < nlow ? q : hdr.hb[q - nlow]);
        hdr.use_tma = tma_enabled() && tma_make_plan(tb, hdr.tbits, n, sizeof(double2), psi->d, hdr.tma, &mpsi) &&
                              tma_make_plan(tb, hdr.tbits, n, sizeof(double2), lam->d, hdr.tma, &mlam)
                          ? 1
                          : 0;
        hdr.nstage = hdr.use_tma ? nstage : 1;
        const size_t smem = 1024 + (size_t)(hdr.use_tma ? nstage : 1) * tile_bytes + p.ops.size() * sizeof(AdjTileOp) +
                            p.slot_grad.size() * slot_bytes;
        {
            ProfScope prof(ctx, "adjoint_tiles", (double)((uint64_t)1 << n) * 4.0 * sizeof(double2));
            k_adjoint_tiles<<<grid, kAdjThreads, smem, ctx->stream>>>((double2*)psi->d, (double2*)lam->d, hdr,
                                                                       d_ops + ooff, d_part, ctx->d_err, mpsi, mlam);
        }
        ctx->launches++;
        YAO_CUDA(cudaGetLastError());
        if (!p.slot_grad.empty()) {
            k_adj_slot_sums<<<(unsigned)p.slot_grad.size(), kAdjThreads, 0, ctx->stream>>>(
                d_part, grid, (int)p.slot_grad.size(), d_dots + doff);
            ctx->launches++;
            YAO_CUDA(cudaGetLastError());
        }
        ooff += p.ops.size();
        doff += p.slot_grad.size();
    }
    std::vector<double> dots(std::max<size_t>(1, ndots));
    if (ndots)
        YAO_CUDA(cudaMemcpyAsync(dots.data(), d_dots, ndots * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaFreeAsync(buf, ctx->stream));
    int herr = 0;
    YAO_CUDA(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    if (herr) {
        YAO_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        return fail(YAO_ERR_TIMEOUT, "expect_grad: a bounded wait of a kernel (tile copy) gave up");
    }
    doff = 0;
    for (const AdjPass& p : passes)
        for (size_t s = 0; s < p.slot_grad.size(); s++) grad[p.slot_grad[s]] = 2.0 * dots[doff++];
    return YAO_OK;
}

int adjoint_tiles(Ctx* ctx, Reg* psi, Reg* lam, const Circuit* c, double* grad, size_t np) {
    int st = YAO_OK;
    AdjPlan* plan = adjoint_plan_new(c, psi->nbits, psi->precision, np, &st);
    if (!plan) return st;
    st = adjoint_run(ctx, psi, lam, plan, grad);
    adjoint_plan_free(plan);
    return st;
}

}  // namespace yao
