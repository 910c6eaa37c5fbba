// sv_tiles.cu — multi-gate passes over shared-memory tiles, and the planner
// that builds them.
//
// A tile is the set of 2^tbits amplitudes that agree on every bit outside
// the tile bit set TB (ascending; it always starts with the contiguous low
// bits 0..m-1, so a tile is 2^(tbits-m) runs of 2^m consecutive amplitudes).
// One pass loads each tile into shared memory once, applies a run of gates
// whose moving targets lie in TB, and writes the tile back: many gates per
// HBM round trip.
//
//  - TILED form: a pass holds a contiguous run of the circuit's gates, in
//    order, with the PLAIN kernels' arithmetic, so the result is bit-identical
//    to gate-by-gate application.  Diagonal gates and all controls may sit on
//    any bit: a diagonal entry and a control test only read the amplitude's
//    global index.
//  - FUSED form: gates are first multiplied into dense blocks of at most k
//    qubits (host, FP64); each block is one op of a pass, and a pass may take
//    blocks out of order past blocks on disjoint qubits.  On complex64
//    registers the block coefficients are split into an FP32 high part and
//    an FP32 low part (c = hi + lo), and both products are accumulated in
//    FP32 (a two-term compensated product).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <atomic>
#include <chrono>
#include <vector>

#include <cudaTypedefs.h>

#include "device_common.cuh"
#include "tc_sm100.cuh"
#include "tma_sm100.cuh"

namespace yao {

struct TileHdr {
    int32_t tbits;
    int32_t m;
    int32_t nops;
    int32_t nsegs;
    int8_t tb[16];
    uint64_t ntiles;
    int32_t ncoef;
    int32_t staged;  // op table, segments and coefficients are copied to shared memory
    int32_t mma;     // some wide op of the pass runs on the tensor cores
    int32_t dmma;    // complex128 FUSED: some dense 3..5-qubit block runs on the FP64 tensor cores
    int32_t tc_test; // failure-path test: tensor-core ops issue no copy and no MMA, waits give up after 0.1 s
    int32_t use_tma; // tiles move by TMA (tma, nstage); else by cp.async
    int32_t nstage;  // TMA tile buffers in flight (2..4)
    int32_t tc_variant;  // tensor-core block variant bits (kTcVar*)
    int32_t tc_resident; // tensor-core ops whose B operands stay in shared memory for the pass (0: one slot, reloaded)
    int32_t pad2_;
    TmaPlan tma;
};

struct TOp {
    int32_t cls;
    int32_t k;
    int8_t tl[kMaxTargets];  // local target positions (-1 = outside the tile, DIAG only)
    int8_t tg[kMaxTargets];  // global target positions
    int8_t rp[kMaxTargets];  // register segments: target positions among the segment's register bits
    int8_t ts[kMaxTargets];  // wide ops: local target positions, ascending
    uint32_t lcmask, lcval;  // in-tile controls (local bit positions)
    uint64_t gcmask, gcval;  // out-of-tile controls (global bit positions)
    uint64_t active;         // DIAG: non-unit entries
    int32_t moff;            // first coefficient in the pass's coefficient array
    int32_t all_local;
    int32_t mma;             // tensor-core op: offset of its operand matrices (floats), else -1
    int32_t mpad;
};
static_assert(sizeof(TOp) % 8 == 0, "TOp is copied as 32-bit words and read as 64-bit fields");

// Coefficient types: double2 for C128, float4 {hi.re, hi.im, lo.re, lo.im}
// for C64 (split coefficient).
template <typename V>
struct CoefT;
template <>
struct CoefT<double2> {
    typedef double2 C;
};
template <>
struct CoefT<float2> {
    typedef float4 C;
};

template <bool EXACT>
__device__ __forceinline__ double2 cmul_c(double2 c, double2 x) {
    if (EXACT) return cmul_x(c, x);
    return make_double2(fma(c.x, x.x, -c.y * x.y), fma(c.x, x.y, c.y * x.x));
}
template <bool EXACT>
__device__ __forceinline__ double2 cfma_c(double2 acc, double2 c, double2 x) {
    if (EXACT) return cadd_x(acc, cmul_x(c, x));
    return make_double2(fma(c.x, x.x, fma(-c.y, x.y, acc.x)), fma(c.x, x.y, fma(c.y, x.x, acc.y)));
}
template <bool EXACT>
__device__ __forceinline__ double2 cmulassign_c(double2 x, double2 c) {
    if (EXACT) return cmulassign_x(x, c);
    return cmul_c<false>(c, x);
}
// split-coefficient products for complex64 data: (hi + lo) * x as one FMA
// chain per component, the small lo terms first, FP32 accumulate
template <bool EXACT>
__device__ __forceinline__ float2 cmul_c(float4 c, float2 x) {
    const float re = fmaf(c.x, x.x, fmaf(-c.y, x.y, fmaf(c.z, x.x, -c.w * x.y)));
    const float im = fmaf(c.x, x.y, fmaf(c.y, x.x, fmaf(c.z, x.y, c.w * x.x)));
    return make_float2(re, im);
}
template <bool EXACT>
__device__ __forceinline__ float2 cfma_c(float2 acc, float4 c, float2 x) {
    const float re = fmaf(c.x, x.x, fmaf(-c.y, x.y, fmaf(c.z, x.x, fmaf(-c.w, x.y, acc.x))));
    const float im = fmaf(c.x, x.y, fmaf(c.y, x.x, fmaf(c.z, x.y, fmaf(c.w, x.x, acc.y))));
    return make_float2(re, im);
}
template <bool EXACT>
__device__ __forceinline__ float2 cmulassign_c(float2 x, float4 c) {
    return cmul_c<EXACT>(c, x);
}

__device__ __forceinline__ uint32_t ins0(uint32_t v, int p) {
    return ((v >> p) << (p + 1)) | (v & ((1u << p) - 1));
}

template <typename V, typename C>
__device__ __forceinline__ bool coef_is_one(C c);
template <>
__device__ __forceinline__ bool coef_is_one<double2, double2>(double2 c) {
    return c.x == 1.0 && c.y == 0.0;
}
template <>
__device__ __forceinline__ bool coef_is_one<float2, float4>(float4 c) {
    return c.x == 1.f && c.y == 0.f && c.z == 0.f && c.w == 0.f;
}

constexpr int kTileThreads = 512;
constexpr size_t kMaxStagedBytes = 48 * 1024;  // pass description staged in shared memory

// A pass is cut into segments.  In a register segment every thread owns
// 2^RB amplitudes that differ only in the segment's register bits `rbs` (tile
// positions, ascending); the segment's ops move amplitudes only along those
// bits, so the thread applies all of them in registers and touches shared
// memory once on entry and once on exit.  A wide segment is one dense op on
// more than two targets, computed through shared memory.
struct TSeg {
    int32_t wide;
    int32_t op_begin, op_end;
    int8_t rbs[4];
};

// XOR swizzle of the shared-memory tile against bank conflicts when the
// lanes of a warp step through higher tile bits.
// It is the 128-byte swizzle of the TMA unit: in every 1024-byte block,
// 16-byte chunk q of 128-byte row r sits at chunk q ^ (r % 8), i.e. bits
// 4..6 of the byte offset are XORed with bits 7..9.  In amplitude units:
// complex128 (16 B) XORs position bits 0..2 with bits 3..5, complex64 (8 B)
// bits 1..3 with bits 4..6 (bit 0 stays: the two halves of a 16-byte chunk
// stay together, and swz(l | 1) = swz(l) | 1).
__device__ __forceinline__ uint32_t swz(uint32_t l, double2*) { return l ^ ((l >> 3) & 7); }
__device__ __forceinline__ uint32_t swz(uint32_t l, float2*) { return l ^ (((l >> 4) & 7) << 1); }

// Global index of tile position l: the low m positions are the low bits
// themselves; the rest scatter to the tile's higher bits through a table of
// 2^(tbits - m) offsets built once per pass in shared memory.
constexpr int kMaxScatterBits = 9;

__device__ __forceinline__ void tile_offsets(const TileHdr& hdr, uint64_t* hoff) {
    const uint32_t nh = 1u << (hdr.tbits - hdr.m);
    for (uint32_t h = threadIdx.x; h < nh; h += blockDim.x) {
        uint64_t o = 0;
        for (int j = hdr.m; j < hdr.tbits; j++) o |= (uint64_t)((h >> (j - hdr.m)) & 1) << hdr.tb[j];
        hoff[h] = o;
    }
    __syncthreads();
}

// Base index of tile t (t's bits deposited on the positions outside the
// tile): the deposit is linear over disjoint bit fields, so four 256-entry
// tables of 8-bit chunks of t, built once per CTA, replace the loop.
__device__ __forceinline__ void tile_base_tables(const TileHdr& hdr, uint64_t* bt) {
    for (uint32_t e = threadIdx.x; e < 4 * 256; e += blockDim.x)
        bt[e] = insert_zeros((uint64_t)(e & 255) << (8 * (e >> 8)), hdr.tb, hdr.tbits);
    __syncthreads();
}
__device__ __forceinline__ uint64_t tile_base(uint64_t t, const uint64_t* bt) {
    return bt[t & 255] | bt[256 + ((t >> 8) & 255)] | bt[512 + ((t >> 16) & 255)] | bt[768 + ((t >> 24) & 255)];
}

__device__ __forceinline__ uint64_t tile_global(uint64_t base, uint32_t l, int m, const uint64_t* hoff) {
    return base | (l & ((1u << m) - 1)) | hoff[l >> m];
}

// 1-qubit op (X or dense) on register bit P
template <typename V, bool EXACT, int RB, int P>
__device__ __forceinline__ void reg1(V (&v)[1 << RB], const uint32_t lbase, const uint32_t (&roff)[1 << RB],
                                     const TOp& op, const typename CoefT<V>::C* m) {
    typedef typename CoefT<V>::C C;
    const bool isx = op.cls == GC_X;
    C a, b, c, d;
    if (!isx) {
        a = m[0];
        b = m[1];
        c = m[2];
        d = m[3];
    }
    const bool ctl = op.lcmask != 0;  // in-tile controls: test every pair
#pragma unroll
    for (int j = 0; j < (1 << RB); j++) {
        if (j & (1 << P)) continue;
        const int j1 = j | (1 << P);
        if (ctl && ((lbase | roff[j]) & op.lcmask) != op.lcval) continue;
        V w = v[j], x = v[j1];
        if (isx) {
            v[j] = x;
            v[j1] = w;
        } else {
            v[j] = cfma_c<EXACT>(cmul_c<EXACT>(a, w), b, x);
            v[j1] = cfma_c<EXACT>(cmul_c<EXACT>(c, w), d, x);
        }
    }
}

template <typename V, bool EXACT, int RB, int P>
__device__ __forceinline__ void reg1_at(int p, V (&v)[1 << RB], const uint32_t lbase,
                                        const uint32_t (&roff)[1 << RB], const TOp& op,
                                        const typename CoefT<V>::C* m) {
    if constexpr (P < RB) {
        if (p == P)
            reg1<V, EXACT, RB, P>(v, lbase, roff, op, m);
        else
            reg1_at<V, EXACT, RB, P + 1>(p, v, lbase, roff, op, m);
    }
}

// 2-qubit op (SWAP or dense, bits sorted) on register bits P0 < P1
template <typename V, bool EXACT, int RB, int P0, int P1>
__device__ __forceinline__ void reg2(V (&v)[1 << RB], const uint32_t lbase, const uint32_t (&roff)[1 << RB],
                                     const TOp& op, const typename CoefT<V>::C* m) {
    typedef typename CoefT<V>::C C;
#pragma unroll
    for (int j = 0; j < (1 << RB); j++) {
        if (j & ((1 << P0) | (1 << P1))) continue;
        if (((lbase | roff[j]) & op.lcmask) != op.lcval) continue;
        const int i1 = j | (1 << P0), i2 = j | (1 << P1), i3 = j | (1 << P0) | (1 << P1);
        if (op.cls == GC_SWAP) {
            V t = v[i1];
            v[i1] = v[i2];
            v[i2] = t;
        } else {
            V old[4] = {v[j], v[i1], v[i2], v[i3]};
            V out[4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                V acc = VecT<V>::zero();
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    C cc = m[r * 4 + q];
                    acc = cfma_c<EXACT>(acc, cc, old[q]);
                }
                out[r] = acc;
            }
            v[j] = out[0];
            v[i1] = out[1];
            v[i2] = out[2];
            v[i3] = out[3];
        }
    }
}

template <typename V, bool EXACT, int RB, int P0, int P1>
__device__ __forceinline__ void reg2_at(int p0, int p1, V (&v)[1 << RB], const uint32_t lbase,
                                        const uint32_t (&roff)[1 << RB], const TOp& op,
                                        const typename CoefT<V>::C* m) {
    if constexpr (P0 < RB - 1) {
        if constexpr (P1 < RB) {
            if (p0 == P0 && p1 == P1)
                reg2<V, EXACT, RB, P0, P1>(v, lbase, roff, op, m);
            else
                reg2_at<V, EXACT, RB, P0, P1 + 1>(p0, p1, v, lbase, roff, op, m);
        } else {
            reg2_at<V, EXACT, RB, P0 + 1, P0 + 2>(p0, p1, v, lbase, roff, op, m);
        }
    }
}

__device__ __forceinline__ double2 ld_l2(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ float2 ld_l2(const float2* p) { return __ldcg(p); }

// ------------------------------------------------------- tensor-core ops
//
// A dense 5-qubit block on complex64 data in a 4096-amplitude tile runs on
// the tensor cores as one real GEMM: the tile's G = 128 groups are the rows
// of X (K = 64 reals per group: re, im of local index 0, 1, ...), the block's
// real form B (64 x 64: rows 2i, 2i+1 = re, im of output i) is the second
// operand, D = X B^T (128 x 64, FP32) accumulates in tensor memory.  FP32
// accuracy comes from three TF32 products, D = Xh Bh + Xh Bl + Xl Bh, where
// Xh = tf32(X), Xl = X - Xh (and Bh / Bl likewise, prepared on the host).
// Operands are K-major in the no-swizzle canonical layout: element (r, k) at
// byte (r / 8) * 2048 + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4.
constexpr int kTcK = 5;                 // qubits of a tensor-core block
constexpr int kTcTileBits = 12;         // tile of a tensor-core pass (2^12 complex64)
constexpr int kTcRows = 128;            // groups per tile = MMA M
constexpr int kTcN = 64;                // real outputs = MMA N
constexpr int kTcKr = 64;               // real inputs = reduction length
// One op's operand slot (floats): Bh, Bl, Bll (B - Bh - Bl rounded to TF32),
// then the five int8 digit arrays of the integer form (kTc8Off on)
constexpr int kTc8Off = 3 * kTcN * kTcKr;
constexpr int kTcOpFloats = kTc8Off + 5 * kTcN * kTcKr / 4;
constexpr uint32_t kTcSbo = (kTcKr / 4) * 128;  // bytes between 8-row groups
constexpr size_t kTcXBytes = 2 * (size_t)kTcRows * kTcKr * 4;  // Xh, Xl
constexpr size_t kTcBPart = (size_t)kTcN * kTcKr * 4;            // one of Bh, Bl, Bll
constexpr int kTcCols = 128;  // tensor-memory columns: the main accumulator, then the correction accumulator
// Variants of the tensor-core block (hdr.tc_variant bits, from YAO_TC_VARIANT):
//   1: X's low part rounded to TF32 (round to nearest) before the MMAs read it
//   2: the correction products (Xh Bl + Xl Bh [+ Xh Bll]) accumulate apart from
//      Xh Bh, and the two are added in FP32 (round to nearest) on read-back
//   4: B in three TF32 parts, a fourth product Xh Bll
//   8: the integer form (wide_tc8): exact int8 products, int32 accumulation
constexpr int kTcVarXlRound = 1, kTcVarSplitAcc = 2, kTcVarB3 = 4, kTcVarInt8 = 8;

// Integer form of the tensor-core block.  The tensor cores' FP32
// accumulation truncates (every accumulation step biases the sum toward
// zero, so the norm shrinks block by block); integer MMAs accumulate
// exactly.  X (the tile's amplitudes) is scaled by a power of two 2^(27 - e)
// with 2^e above the tile's largest |x| and rounded to the nearest integer
// (|q| < 2^27; exact for every amplitude within 2^3 of the largest, since
// an FP32 value has 24 significant bits), then written as four balanced
// base-2^7 digits q = d0 2^21 + d1 2^14 + d2 2^7 + d3 (|d| <= 64, int8).  B
// (|b| <= 1) is rounded to 2^-34 on the host, five digits b 2^34 = e0 2^28 +
// ... + e4.  The products d_i e_j are summed exactly in int32 per level
// L = i + j <= 3 (accumulator L, TMEM columns 64 L; 10 products), and
// y = 2^(e - 12) (A0 + A1 2^-7 + A2 2^-14 + A3 2^-21) is formed exactly in
// 64-bit integers and rounded to FP32 once (to nearest).  Levels 4 and above
// weigh below 2^-30 of the block's largest output and are left out: a
// level's K = 64 sum of digit products reaches 2^15 and more, so every
// level up to 3 is kept whole.
constexpr int kTc8XDigits = 4, kTc8BDigits = 5;
constexpr uint32_t kTc8Sbo = (kTcKr / 16) * 128;       // bytes between 8-row groups (64 int8 a row)
constexpr uint32_t kTc8XDigit = kTcRows * kTcKr;       // bytes of one X digit array
constexpr uint32_t kTc8BDigit = kTcN * kTcKr;          // bytes of one B digit array
constexpr uint32_t kTc8BBytes = kTc8BDigits * kTc8BDigit;
constexpr uint64_t kTcWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ uint64_t global_ns_tc() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct TcCtx {
    uint32_t tmem;       // accumulator (64 columns)
    uint64_t* bar;       // MMA completion barrier
    uint32_t phase;      // parity of the next completion
    uint64_t* bbar;      // B operand copy barrier
    uint32_t bphase;
    float* xh;           // operands in shared memory (1 KiB aligned)
    float* xl;
    float* bh;
    float* bl;
    float* bll;
    int variant;         // kTcVar* bits
    int resident;        // B operands of every op resident (slot = op.mma / kTcOpFloats)
    uint32_t bfloats;    // floats of one op's B operands in shared memory
    const float* mmat;   // every tensor-core op's Bh, Bl, Bll of the pass (global)
    int loaded;          // op offset whose B operands are in shared memory
    int failed;          // a completion wait ran out (results of the pass are void)
    int* err;
    uint64_t wait_ns;    // limit of every wait
    int stall;           // failure-path test: nothing is issued, so every wait runs out
};

__device__ __forceinline__ uint32_t tc_off(uint32_t r, uint32_t k) {
    return (r >> 3) * kTcSbo + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

template <typename V>
__device__ __noinline__ void wide_tc(const TOp& op, V* s, TcCtx& tc) {
    if constexpr (sizeof(V) == 8) {
        float2* t = (float2*)s;
        const uint32_t nt = blockDim.x, tid = threadIdx.x;
        __shared__ uint32_t co[1 << kTcK];  // tile offset of local index c
        // B operands of this op (Bh, Bl[, Bll]: 32 or 48 KiB contiguous): one
        // bulk copy started now, waited for by the MMA-issuing thread
        const bool split = tc.variant & kTcVarSplitAcc, b3 = tc.variant & kTcVarB3;
        const uint32_t bbytes = tc.bfloats * 4;
        float* bslot = tc.resident ? tc.bh + (size_t)(op.mma / kTcOpFloats) * tc.bfloats : tc.bh;
        const bool need_b = !tc.resident && tc.loaded != op.mma;
        if (need_b && tid == 0 && !tc.stall) {
            tc::mbar_arrive_expect_tx(tc.bbar, bbytes);
            tc::bulk_g2s(bslot, tc.mmat + op.mma, bbytes, tc.bbar);
        }
        if (tid < (1u << kTcK)) {
            uint32_t o = 0;
#pragma unroll
            for (int q = 0; q < kTcK; q++) o |= (uint32_t)((tid >> q) & 1) << op.tl[q];
            co[tid] = o;
        }
        __syncthreads();
        // 1. X: row g = tid % 128 (one group per thread), 16-byte chunks jp,
        // in two halves of K: the MMAs on columns 0..31 run while the
        // threads build columns 32..63
        const uint32_t g = tid & (kTcRows - 1);
        uint32_t gb = g;
#pragma unroll
        for (int q = 0; q < kTcK; q++) gb = ins0(gb, op.ts[q]);
        auto build_x = [&](uint32_t jp0) {
            for (uint32_t jp = jp0 + (tid >> 7); jp < jp0 + 8; jp += nt >> 7) {
                const float2 v0 = t[swz(gb | co[2 * jp], (float2*)nullptr)];
                const float2 v1 = t[swz(gb | co[2 * jp + 1], (float2*)nullptr)];
                const float4 h = make_float4(tc::to_tf32(v0.x), tc::to_tf32(v0.y), tc::to_tf32(v1.x), tc::to_tf32(v1.y));
                float4 l = make_float4(v0.x - h.x, v0.y - h.y, v1.x - h.z, v1.y - h.w);
                if (tc.variant & kTcVarXlRound)
                    l = make_float4(tc::to_tf32(l.x), tc::to_tf32(l.y), tc::to_tf32(l.z), tc::to_tf32(l.w));
                const uint32_t off = tc_off(g, 4 * jp);
                *(float4*)((char*)tc.xh + off) = h;
                *(float4*)((char*)tc.xl + off) = l;
            }
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
        };
        // 2. one thread issues the MMAs: 8 K-steps x 3 products, 4 K-steps
        // per half; the B operands are waited for before the first
        bool b_ok = true;
        constexpr uint32_t idesc = tc::idesc_tf32(kTcRows, kTcN);
        const uint32_t xh = tc::smem_u32(tc.xh), xl = tc::smem_u32(tc.xl);
        const uint32_t bh = tc::smem_u32(bslot), bl = bh + (uint32_t)kTcBPart, bll = bl + (uint32_t)kTcBPart;
        const uint32_t acc_c = tc.tmem + (split ? (uint32_t)kTcN : 0u);  // correction accumulator
        auto issue = [&](int k0) {
            tc::fence_after_sync();
#pragma unroll
            for (int k8 = k0; k8 < k0 + kTcKr / 16; k8++) {
                const uint32_t o = (uint32_t)k8 * 256;
                tc::mma_tf32(tc.tmem, tc::smem_desc(xh + o, 128, kTcSbo), tc::smem_desc(bh + o, 128, kTcSbo), idesc,
                             k8 > 0);
                tc::mma_tf32(acc_c, tc::smem_desc(xh + o, 128, kTcSbo), tc::smem_desc(bl + o, 128, kTcSbo), idesc,
                             split ? k8 > 0 : 1);
                tc::mma_tf32(acc_c, tc::smem_desc(xl + o, 128, kTcSbo), tc::smem_desc(bh + o, 128, kTcSbo), idesc, 1);
                if (b3)
                    tc::mma_tf32(acc_c, tc::smem_desc(xh + o, 128, kTcSbo), tc::smem_desc(bll + o, 128, kTcSbo), idesc,
                                 1);
            }
        };
        build_x(0);
        if (need_b) {
            tc.loaded = op.mma;
            if (tid == 0) {
                const uint64_t tb = global_ns_tc();
                while (!(b_ok = tc::mbar_try_wait(tc.bbar, tc.bphase)))
                    if (global_ns_tc() - tb > tc.wait_ns) break;
            }
            tc.bphase ^= 1u;
        }
        if (tid == 0 && b_ok) issue(0);
        build_x(8);
        if (tid == 0 && !b_ok) {
            tc.failed = 1;
            atomicExch(tc.err, 1);
            if (!tc.stall) tc::commit(tc.bar);  // no MMA: the barrier completes right away
        } else if (tid == 0) {
            issue(kTcKr / 16);
            tc::commit(tc.bar);
        }
        // 3. every thread waits for completion (bounded)
        bool done = false;
        const uint64_t t0 = global_ns_tc();
        while (!(done = tc::mbar_try_wait(tc.bar, tc.phase))) {
            if (global_ns_tc() - t0 > tc.wait_ns) break;
        }
        tc.phase ^= 1u;
        if (!done) {
            tc.failed = 1;
            if (tid == 0) atomicExch(tc.err, 1);
        }
        tc::fence_after_sync();
        // 4. warp w reads accumulator lanes 32 (w % 4) .. + 31 (lane = group)
        // and a quarter (16 warps) or half (8 warps) of the 64 columns, and
        // writes those outputs of its group into the tile
        const uint32_t warp = tid >> 5, nwarp = nt >> 5;
        const uint32_t cpw = 64 / (nwarp >> 2);  // columns per warp (16 or 32)
        if (done) {
            const uint32_t g = ((warp & 3) << 5) | (tid & 31);
            uint32_t b = g;
#pragma unroll
            for (int q = 0; q < kTcK; q++) b = ins0(b, op.ts[q]);
            const uint32_t c0 = (warp >> 2) * cpw;
            for (uint32_t c = c0; c < c0 + cpw; c += 16) {
                uint32_t r[16], rc[16];
                tc::tmem_ld16(tc.tmem + (((warp & 3) << 5) << 16) + c, r);
                if (split) tc::tmem_ld16(tc.tmem + (((warp & 3) << 5) << 16) + kTcN + c, rc);
                tc::tmem_wait_ld();
                if (split)
#pragma unroll
                    for (int i = 0; i < 16; i++) r[i] = __float_as_uint(__uint_as_float(r[i]) + __uint_as_float(rc[i]));
#pragma unroll
                for (int i = 0; i < 8; i++)
                    t[swz(b | co[(c >> 1) + i], (float2*)nullptr)] =
                        make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
            }
        }
        tc::fence_before_sync();
    }
}

__device__ __forceinline__ uint32_t tc8_off(uint32_t r, uint32_t k) {
    return (r >> 3) * kTc8Sbo + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

__device__ __forceinline__ void tc8_digits(int q, int c, uint32_t (&w)[kTc8XDigits]) {
    const int d0 = (q + (1 << 20)) >> 21;
    const int r0 = q - (d0 << 21);
    const int d1 = (r0 + (1 << 13)) >> 14;
    const int r1 = r0 - (d1 << 14);
    const int d2 = (r1 + 64) >> 7;
    const int d3 = r1 - (d2 << 7);
    w[0] |= (uint32_t)(uint8_t)(int8_t)d0 << (8 * c);
    w[1] |= (uint32_t)(uint8_t)(int8_t)d1 << (8 * c);
    w[2] |= (uint32_t)(uint8_t)(int8_t)d2 << (8 * c);
    w[3] |= (uint32_t)(uint8_t)(int8_t)d3 << (8 * c);
}

template <typename V>
__device__ __noinline__ void wide_tc8(const TOp& op, V* s, TcCtx& tc) {
    if constexpr (sizeof(V) == 8) {
        float2* t = (float2*)s;
        const uint32_t nt = blockDim.x, tid = threadIdx.x;
        __shared__ uint32_t co[1 << kTcK];
        __shared__ float wmax[32];
        __shared__ int sexp;
        const uint32_t bbytes = tc.bfloats * 4;
        float* bslot = tc.resident ? tc.bh + (size_t)(op.mma / kTcOpFloats) * tc.bfloats : tc.bh;
        const bool need_b = !tc.resident && tc.loaded != op.mma;
        if (need_b && tid == 0 && !tc.stall) {
            tc::mbar_arrive_expect_tx(tc.bbar, bbytes);
            tc::bulk_g2s(bslot, tc.mmat + op.mma + kTc8Off, bbytes, tc.bbar);
        }
        if (tid < (1u << kTcK)) {
            uint32_t o = 0;
#pragma unroll
            for (int q = 0; q < kTcK; q++) o |= (uint32_t)((tid >> q) & 1) << op.tl[q];
            co[tid] = o;
        }
        // 1. the scale: 2^e above the largest |x| of the tile
        float mx = 0.f;
        for (uint32_t l = tid; l < (1u << kTcTileBits); l += nt) {
            const float2 v = t[l];
            mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((tid & 31) == 0) wmax[tid >> 5] = mx;
        __syncthreads();
        if (tid == 0) {
            float m = 0.f;
            for (uint32_t w = 0; w < (nt >> 5); w++) m = fmaxf(m, wmax[w]);
            int e = 0;
            frexpf(m, &e);  // m < 2^e
            sexp = e;
        }
        __syncthreads();
        const int e = sexp;
        const float f = ldexpf(1.f, 27 - e);
        // 2. X as four int8 digit arrays (row g = group, 64 bytes a row)
        unsigned char* xd = (unsigned char*)tc.xh;
        const uint32_t g = tid & (kTcRows - 1);
        uint32_t gb = g;
#pragma unroll
        for (int q = 0; q < kTcK; q++) gb = ins0(gb, op.ts[q]);
        for (uint32_t jp = tid >> 7; jp < 16; jp += nt >> 7) {
            const float2 v0 = t[swz(gb | co[2 * jp], (float2*)nullptr)];
            const float2 v1 = t[swz(gb | co[2 * jp + 1], (float2*)nullptr)];
            uint32_t w[kTc8XDigits] = {0, 0, 0, 0};
            tc8_digits(__float2int_rn(v0.x * f), 0, w);
            tc8_digits(__float2int_rn(v0.y * f), 1, w);
            tc8_digits(__float2int_rn(v1.x * f), 2, w);
            tc8_digits(__float2int_rn(v1.y * f), 3, w);
            const uint32_t off = tc8_off(g, 4 * jp);
#pragma unroll
            for (int d = 0; d < kTc8XDigits; d++) *(uint32_t*)(xd + d * kTc8XDigit + off) = w[d];
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        // 3. one thread issues the MMAs: 10 digit products x 2 K-steps
        bool b_ok = true;
        if (need_b) {
            tc.loaded = op.mma;
            if (tid == 0) {
                const uint64_t tb = global_ns_tc();
                while (!(b_ok = tc::mbar_try_wait(tc.bbar, tc.bphase)))
                    if (global_ns_tc() - tb > tc.wait_ns) break;
            }
            tc.bphase ^= 1u;
        }
        if (tid == 0) {
            if (!b_ok) {
                tc.failed = 1;
                atomicExch(tc.err, 1);
                if (!tc.stall) tc::commit(tc.bar);
            } else {
                tc::fence_after_sync();
                constexpr uint32_t idesc = tc::idesc_i8(kTcRows, kTcN);
                const uint32_t xa = tc::smem_u32(xd), ba = tc::smem_u32(bslot);
                // (X digit, B digit, level): first product of each level initialises it
                const int prod[10][3] = {{0, 0, 0}, {0, 1, 1}, {1, 0, 1}, {0, 2, 2}, {1, 1, 2},
                                         {2, 0, 2}, {0, 3, 3}, {1, 2, 3}, {2, 1, 3}, {3, 0, 3}};
#pragma unroll
                for (int p = 0; p < 10; p++) {
                    const int i = prod[p][0], j = prod[p][1], L = prod[p][2];
                    const bool first = p == 0 || prod[p - 1][2] != L;
#pragma unroll
                    for (int ks = 0; ks < 2; ks++) {
                        const uint32_t o = (uint32_t)ks * 256;
                        tc::mma_i8(tc.tmem + (uint32_t)(64 * L),
                                   tc::smem_desc(xa + (uint32_t)i * kTc8XDigit + o, 128, kTc8Sbo),
                                   tc::smem_desc(ba + (uint32_t)j * kTc8BDigit + o, 128, kTc8Sbo), idesc,
                                   (first && ks == 0) ? 0u : 1u);
                    }
                }
                tc::commit(tc.bar);
            }
        }
        // 4. every thread waits for completion (bounded)
        bool done = false;
        const uint64_t t0 = global_ns_tc();
        while (!(done = tc::mbar_try_wait(tc.bar, tc.phase))) {
            if (global_ns_tc() - t0 > tc.wait_ns) break;
        }
        tc.phase ^= 1u;
        if (!done) {
            tc.failed = 1;
            if (tid == 0) atomicExch(tc.err, 1);
        }
        tc::fence_after_sync();
        // 5. read-back: warp w reads accumulator lanes 32 (w % 4) .. + 31
        // (lane = group) of its share of the 64 columns of every level
        const uint32_t warp = tid >> 5, nwarp = nt >> 5;
        const uint32_t cpw = 64 / (nwarp >> 2);
        if (done) {
            const uint32_t g2 = ((warp & 3) << 5) | (tid & 31);
            uint32_t b = g2;
#pragma unroll
            for (int q = 0; q < kTcK; q++) b = ins0(b, op.ts[q]);
            const uint32_t c0 = (warp >> 2) * cpw;
            const uint32_t lane_base = tc.tmem + ((((warp & 3) << 5)) << 16);
            for (uint32_t c = c0; c < c0 + cpw; c += 16) {
                uint32_t r0[16], r1[16], r2[16], r3[16];
                tc::tmem_ld16(lane_base + c, r0);
                tc::tmem_ld16(lane_base + 64 + c, r1);
                tc::tmem_ld16(lane_base + 128 + c, r2);
                tc::tmem_ld16(lane_base + 192 + c, r3);
                tc::tmem_wait_ld();
                float y[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    // 2^(e-33) (H 2^14 + Lo), H = A0 2^7 + A1, Lo = A2 2^7 + A3:
                    // exact in 64 bits (|.| < 2^41), one rounding to FP32
                    const long long H = (long long)(int)r0[i] * 128 + (int)r1[i];
                    const long long Lo = (long long)(int)r2[i] * 128 + (int)r3[i];
                    y[i] = (float)ldexp((double)(H * 16384 + Lo), e - 33);
                }
#pragma unroll
                for (int i = 0; i < 8; i++)
                    t[swz(b | co[(c >> 1) + i], (float2*)nullptr)] = make_float2(y[2 * i], y[2 * i + 1]);
            }
        }
        tc::fence_before_sync();
    }
}

// ------------------------------------------------- FP64 tensor-core ops
//
// A dense K-qubit block (K = 3..5) of a complex128 FUSED pass as one real
// FP64 GEMM on the tensor cores (`mma.sync` m8n8k4 f64; tcgen05 has no FP64
// kind): Y = A X, where column g of X holds the 2^K amplitudes of group g as
// 2^(K+1) reals (re, im of local index 0, 1, ...) and A is the block's real
// form (row 2r + o, column 2c + i: Re U[r][c] where o = i, -Im U[r][c] for
// o = 0, i = 1, Im U[r][c] for o = 1, i = 0), read straight from the complex
// coefficients, stored by the host with a row stride of 2^K + 2.  Warp w owns the 8-group column blocks w NB .. w NB + NB - 1
// and every row block, so it reads and writes only its own groups'
// amplitudes: 2^(RB+1) FP64 accumulators per thread.  Fragments (m8n8k4,
// lane l): A (8 x 4) element (l / 4, l % 4); B (4 x 8) element (l % 4, l / 4);
// D (8 x 8) elements (l / 4, 2 (l % 4) + j), j = 0, 1.  `wsw[c]`: swizzled
// tile offset of local index c.
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

template <int K, int RB>
__device__ __forceinline__ void wide_dmma(const TOp& op, const double2* __restrict__ m, double2* s,
                                          const uint32_t* wsw) {
    constexpr int NL = 1 << K, KS = NL / 2, MB = NL / 4;  // k-steps of 4 reals, 8-row blocks
    constexpr int NB = (1 << (RB + 2)) >> K;                // 8-group column blocks per warp
    static_assert(NB >= 1, "a warp needs at least one column block");
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t ri = lane & 1, ro = (lane >> 2) & 1, cb = (lane & 3) >> 1;
    double* sd = (double*)s;
    double2* tag = nullptr;
    uint32_t sb[NB];  // swizzled base of the input group of B column l / 4
#pragma unroll
    for (int j = 0; j < NB; j++) {
        uint32_t b = (warp * NB + j) * 8 + (lane >> 2);
#pragma unroll
        for (int q = 0; q < K; q++) b = ins0(b, op.ts[q]);
        sb[j] = swz(b, tag);
    }
    double acc[NB][MB][2];
#pragma unroll
    for (int j = 0; j < NB; j++)
#pragma unroll
        for (int mb = 0; mb < MB; mb++) acc[j][mb][0] = acc[j][mb][1] = 0.0;
    constexpr int RS = NL + 2;  // padded row stride: the A fragment's 8 coefficients sit in 8 bank groups
    const double2* mr = m + (size_t)(lane >> 3) * RS + cb;  // row r = 4 mb + l / 8
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        const uint32_t wc = wsw[2 * ks + cb];
        double bf[NB];
#pragma unroll
        for (int j = 0; j < NB; j++) bf[j] = sd[2 * (sb[j] ^ wc) + ri];
#pragma unroll
        for (int mb = 0; mb < MB; mb++) {
            const double2 u = mr[(size_t)mb * 4 * RS + 2 * ks];
            const double a = ro == ri ? u.x : (ro ? u.y : -u.y);
#pragma unroll
            for (int j = 0; j < NB; j++) dmma884(acc[j][mb][0], acc[j][mb][1], a, bf[j]);
        }
    }
    __syncwarp();
    // output group 8 (w NB + j) + 2 (l % 4) + i, row r = 4 mb + l / 8,
    // component o; groups outside the in-tile controls keep their amplitudes
#pragma unroll
    for (int j = 0; j < NB; j++)
#pragma unroll
        for (int i = 0; i < 2; i++) {
            uint32_t b = (warp * NB + j) * 8 + 2 * (lane & 3) + i;
#pragma unroll
            for (int q = 0; q < K; q++) b = ins0(b, op.ts[q]);
            if ((b & op.lcmask) != op.lcval) continue;
            const uint32_t so = swz(b, tag);
#pragma unroll
            for (int mb = 0; mb < MB; mb++) sd[2 * (so ^ wsw[4 * mb + (lane >> 3)]) + ro] = acc[j][mb][i];
        }
}

// Whether a wide op runs on the FP64 tensor cores: dense 3..RB+2 qubits (at
// most 5), every thread of the tile present (T = threads << RB) in whole warps.
__host__ __device__ inline bool dmma_op(int k, int rb, uint32_t tbits, uint32_t threads) {
    return k >= 3 && k <= rb + 2 && k <= 5 && rb >= 2 && ((1u << tbits) >> rb) == threads && threads >= 32;
}

// The segments of one pass on one tile held in shared memory `s` (the tile
// at `base`).  Ends with the tile updated in `s` and a __syncthreads().
template <typename V, bool EXACT, int RB, bool TC = false, bool DM = false>
__device__ __forceinline__ void tile_compute(const TileHdr& hdr, uint64_t base, const TOp* __restrict__ ops,
                                             const TSeg* __restrict__ segs,
                                             const typename CoefT<V>::C* __restrict__ coef, V* s,
                                             TcCtx* tcx = nullptr, bool last_sync = true) {
    typedef typename CoefT<V>::C C;
    constexpr int NA = 1 << RB;
    V* tag = nullptr;  // selects the swizzle overload
    const uint32_t T = 1u << hdr.tbits;
    const uint32_t nt = blockDim.x;
    for (int si = 0; si < hdr.nsegs; si++) {
        const TSeg sg = segs[si];
        if (!sg.wide) {
            if (threadIdx.x < (T >> RB)) {
                uint32_t lbase = threadIdx.x;
#pragma unroll
                for (int i = 0; i < RB; i++) lbase = ins0(lbase, sg.rbs[i]);
                uint32_t roff[NA];
                V v[NA];
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    uint32_t o = 0;
#pragma unroll
                    for (int i = 0; i < RB; i++) o |= (uint32_t)((j >> i) & 1) << sg.rbs[i];
                    roff[j] = o;
                }
                // complex64 with tile bit 0 among the register bits: the
                // pairs (l, l | 1) are one 16-byte chunk each
                const bool pair = sizeof(V) == 8 && sg.rbs[0] == 0;
                if constexpr (sizeof(V) == 8) {
                    if (pair) {
#pragma unroll
                        for (int j = 0; j < NA; j += 2) {
                            const float4 q = *(const float4*)&s[swz(lbase | roff[j], tag)];
                            v[j] = make_float2(q.x, q.y);
                            v[j + 1] = make_float2(q.z, q.w);
                        }
                    }
                }
                if (!pair) {
#pragma unroll
                    for (int j = 0; j < NA; j++) v[j] = s[swz(lbase | roff[j], tag)];
                }
                for (int oi = sg.op_begin; oi < sg.op_end; oi++) {
                    const TOp& op = ops[oi];
                    if ((base & op.gcmask) != op.gcval) continue;  // uniform over the tile
                    const C* m = coef + op.moff;
                    if (op.cls == GC_DIAG) {
                        // entry index: out-of-tile target bits come from the
                        // tile base, in-tile ones from the amplitude's position
                        uint32_t dl0 = 0;
                        if (!op.all_local)
                            for (int i = 0; i < op.k; i++)
                                if (op.tl[i] < 0) dl0 |= (uint32_t)((base >> op.tg[i]) & 1) << i;
#pragma unroll
                        for (int j = 0; j < NA; j++) {
                            const uint32_t l = lbase | roff[j];
                            if ((l & op.lcmask) != op.lcval) continue;
                            uint32_t dl = dl0;
                            for (int i = 0; i < op.k; i++)
                                if (op.tl[i] >= 0) dl |= ((l >> op.tl[i]) & 1) << i;
                            if ((op.active >> dl) & 1) v[j] = cmulassign_c<EXACT>(v[j], m[dl]);
                        }
                    } else if (op.k == 1) {
                        reg1_at<V, EXACT, RB, 0>(op.rp[0], v, lbase, roff, op, m);
                    } else {
                        reg2_at<V, EXACT, RB, 0, 1>(op.rp[0], op.rp[1], v, lbase, roff, op, m);
                    }
                }
                if constexpr (sizeof(V) == 8) {
                    if (pair) {
#pragma unroll
                        for (int j = 0; j < NA; j += 2) {
                            const float2 a = v[j], b = v[j + 1];
                            *(float4*)&s[swz(lbase | roff[j], tag)] = make_float4(a.x, a.y, b.x, b.y);
                        }
                    }
                }
                if (!pair) {
#pragma unroll
                    for (int j = 0; j < NA; j++) s[swz(lbase | roff[j], tag)] = v[j];
                }
            }
        } else {
            // one dense op on k >= 3 targets (a 2^k x 2^k matrix times the
            // G = T / 2^k groups of the tile).  Item it = (row, group) with
            // the group index fastest, so a warp reads one matrix row
            // (broadcast) against 32 groups.  When G divides the thread
            // count, a thread's NA items share one group and every amplitude
            // it loads serves NA rows.  Outputs stay in registers until
            // every thread has read its inputs.
            __shared__ uint32_t wco[1 << kMaxTargets];  // local offset of column / row c
            const TOp& op = ops[sg.op_begin];
            const bool on = (base & op.gcmask) == op.gcval;
            if constexpr (TC) {
                if (op.mma >= 0) {  // no controls, 5 targets, 2^12 tile (host-checked)
                    if (tcx->variant & kTcVarInt8)
                        wide_tc8<V>(op, s, *tcx);
                    else
                        wide_tc<V>(op, s, *tcx);
                    if (si + 1 < hdr.nsegs || last_sync) __syncthreads();
                    continue;
                }
            }
            if constexpr (DM && sizeof(V) == 16 && !EXACT && RB >= 2) {
                if (dmma_op(op.k, RB, hdr.tbits, nt)) {
                    __shared__ uint32_t wsw[32];
                    if (threadIdx.x < (1u << op.k)) {
                        uint32_t co = 0;
                        for (int q = 0; q < op.k; q++) co |= (uint32_t)((threadIdx.x >> q) & 1) << op.tl[q];
                        wsw[threadIdx.x] = swz(co, tag);
                    }
                    __syncthreads();
                    if (on) {
                        const double2* md = (const double2*)(coef + op.moff);
                        if (op.k == 3)
                            wide_dmma<3, RB>(op, md, (double2*)s, wsw);
                        else if (op.k == 4)
                            wide_dmma<4, RB>(op, md, (double2*)s, wsw);
                        else if constexpr (RB >= 3)
                            wide_dmma<5, RB>(op, md, (double2*)s, wsw);
                    }
                    __syncthreads();
                    continue;
                }
            }
            const C* m = coef + op.moff;
            const int k = op.k, nl = 1 << k;
            const uint32_t G = T >> k;
            for (int c = threadIdx.x; c < nl; c += nt) {
                uint32_t co = 0;
                for (int q = 0; q < k; q++) co |= (uint32_t)((c >> q) & 1) << op.tl[q];
                wco[c] = co;
            }
            __syncthreads();
            V outv[NA];
            uint32_t outi[NA];
#pragma unroll
            for (int i = 0; i < NA; i++) {
                outi[i] = 0xffffffffu;
                outv[i] = VecT<V>::zero();
            }
            if (on && G <= nt) {
                const uint32_t g = threadIdx.x & (G - 1);
                uint32_t b = g;
                for (int q = 0; q < k; q++) b = ins0(b, op.ts[q]);
                const uint32_t row0 = threadIdx.x / G, rstep = nt / G;
                if ((b & op.lcmask) == op.lcval) {
                    for (int c = 0; c < nl; c++) {
                        const V x = s[swz(b | wco[c], tag)];
#pragma unroll
                        for (int i = 0; i < NA; i++) {
                            const uint32_t row = row0 + (uint32_t)i * rstep;
                            if (row < (uint32_t)nl) outv[i] = cfma_c<EXACT>(outv[i], m[(size_t)row * nl + c], x);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < NA; i++) {
                        const uint32_t row = row0 + (uint32_t)i * rstep;
                        if (row < (uint32_t)nl) outi[i] = b | wco[row];
                    }
                }
            } else if (on) {
#pragma unroll
                for (int i = 0; i < NA; i++) {
                    const uint32_t it = threadIdx.x + (uint32_t)i * nt;
                    if (it >= T) continue;
                    const uint32_t g = it & (G - 1), row = it / G;
                    uint32_t b = g;
                    for (int q = 0; q < k; q++) b = ins0(b, op.ts[q]);
                    if ((b & op.lcmask) != op.lcval) continue;
                    V acc = VecT<V>::zero();
                    const C* mr = m + (size_t)row * nl;
                    for (int c = 0; c < nl; c++) acc = cfma_c<EXACT>(acc, mr[c], s[swz(b | wco[c], tag)]);
                    outv[i] = acc;
                    outi[i] = b | wco[row];
                }
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NA; i++)
                if (outi[i] != 0xffffffffu) s[swz(outi[i], tag)] = outv[i];
        }
        // the next segment moves amplitudes along other bits; after the last
        // one the caller synchronises itself when last_sync is false
        if (si + 1 < hdr.nsegs || last_sync) __syncthreads();
    }
}

// Plain (synchronous) tile load and store.  COHERENT loads bypass L1 (the
// tile may have been written by another SM during the same launch).
template <typename V, bool COHERENT>
__device__ __forceinline__ void tile_load(const V* __restrict__ st, const TileHdr& hdr, const uint64_t* hoff,
                                          uint64_t base, V* s) {
    V* tag = nullptr;
    const uint32_t T = 1u << hdr.tbits;
    const int m = hdr.m;
    for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) {
        const V* src = &st[tile_global(base, l, m, hoff)];
        s[swz(l, tag)] = COHERENT ? ld_l2(src) : *src;
    }
    __syncthreads();
}

template <typename V>
__device__ __forceinline__ void tile_store(V* __restrict__ st, const TileHdr& hdr, const uint64_t* hoff,
                                           uint64_t base, const V* s) {
    const V* tag = nullptr;
    const uint32_t T = 1u << hdr.tbits;
    const int m = hdr.m;
    for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) st[tile_global(base, l, m, hoff)] = s[swz(l, (V*)tag)];
}

// Bytes of shared memory that hold a staged pass description.
__host__ __device__ inline size_t staged_bytes(int nops, int nsegs, int ncoef, size_t coef_size) {
    auto a16 = [](size_t x) { return (x + 15) / 16 * 16; };
    return a16((size_t)nops * sizeof(TOp)) + a16((size_t)nsegs * sizeof(TSeg)) + a16((size_t)ncoef * coef_size);
}

// Copy a pass description (ops, segments, coefficients) after the tile in
// shared memory when the host marked it `staged`; returns the pointers the
// tile body reads.
template <typename V>
__device__ __forceinline__ void staged_ptrs(const TileHdr& hdr, unsigned char* smem, int nbuf, TOp*& so, TSeg*& ss,
                                            typename CoefT<V>::C*& sc) {
    typedef typename CoefT<V>::C C;
    auto a16 = [](size_t x) { return (x + 15) / 16 * 16; };
    unsigned char* p = smem + (size_t)nbuf * ((size_t)1 << hdr.tbits) * sizeof(V);
    so = (TOp*)p;
    p += a16((size_t)hdr.nops * sizeof(TOp));
    ss = (TSeg*)p;
    p += a16((size_t)hdr.nsegs * sizeof(TSeg));
    sc = (C*)p;
}

template <typename V>
__device__ __forceinline__ void stage_pass(const TileHdr& hdr, unsigned char* smem, int nbuf, const TOp*& ops,
                                           const TSeg*& segs, const typename CoefT<V>::C*& coef) {
    typedef typename CoefT<V>::C C;
    TOp* so;
    TSeg* ss;
    C* sc;
    staged_ptrs<V>(hdr, smem, nbuf, so, ss, sc);
    {
        const int* src = (const int*)ops;
        int* dst = (int*)so;
        for (int i = threadIdx.x; i < hdr.nops * (int)(sizeof(TOp) / 4); i += blockDim.x) dst[i] = src[i];
        src = (const int*)segs;
        dst = (int*)ss;
        for (int i = threadIdx.x; i < hdr.nsegs * (int)(sizeof(TSeg) / 4); i += blockDim.x) dst[i] = src[i];
    }
    for (int i = threadIdx.x; i < hdr.ncoef; i += blockDim.x) sc[i] = coef[i];
    __syncthreads();
    ops = so;
    segs = ss;
    coef = sc;
}

// One thread: every box of the tile at `base` into shared memory at `dst`,
// all counted on `bar` (armed here with the tile's bytes).
__device__ __forceinline__ void tma_load_tile(const CUtensorMap* map, const TileHdr& hdr, uint64_t base,
                                              uint32_t dst, uint64_t* bar, uint32_t tile_bytes) {
    tc::mbar_arrive_expect_tx(bar, tile_bytes);
    tma::load_boxes(map, hdr.tma, base, dst, tc::smem_u32(bar));
}

// One thread: every box of the tile at `base` from shared memory at `src`
// back to the state, as one bulk async-group.
__device__ __forceinline__ void tma_store_tile(const CUtensorMap* map, const TileHdr& hdr, uint64_t base,
                                               uint32_t src) {
    tma::store_boxes(map, hdr.tma, base, src);
    tma::commit_group();
}

constexpr uint64_t kTileWaitNs = 1000000000ull;  // 1 s
constexpr int kMaxStages = 4;

// One pass over every tile.  Persistent: each CTA loops over the tiles t =
// blockIdx.x, blockIdx.x + gridDim.x, ...
//  - TMA form (hdr.use_tma): `nstage` tile buffers; one thread issues the
//    tile's box copies (tensor map `tmap`) nstage - 1 tiles ahead, every
//    thread waits for its tile on the buffer's mbarrier (bounded: 1 s, then
//    the error word is set and the pass's results are void), the tile is
//    computed, and the same thread stores it back with bulk tensor stores
//    while the next tiles compute.  No thread computes an address.
//  - plain form (tiles of less than 2 KiB, and passes without a TMA
//    plan): each tile is loaded, computed and stored in turn.
// TCK: the pass holds tensor-core ops (complex64 FUSED only); a separate
// instantiation, so passes without them carry none of its state.
// DM: the pass holds dense blocks for the FP64 tensor cores (complex128
// FUSED only); a separate instantiation like TCK.
// STG: the pass description is copied to shared memory, unconditionally, so
// every read of it compiles to a shared-memory load (a pointer chosen at run
// time between global and shared memory would make them generic loads).
template <typename V, bool EXACT, int RB, bool TCK, bool STG, bool DM = false>
__global__ void __launch_bounds__(kTileThreads, RB <= 2 ? 2 : 1)
    k_tile_pass(V* __restrict__ st, const TileHdr phdr, const TOp* __restrict__ gops, const TSeg* __restrict__ gsegs,
                const typename CoefT<V>::C* __restrict__ gcoef, const float* __restrict__ mmat, int* __restrict__ err,
                const __grid_constant__ CUtensorMap tmap) {
    constexpr bool TC = TCK && sizeof(V) == 8 && !EXACT;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ TileHdr hdr;  // indexed with run-time subscripts: keep it out of the parameter space
    __shared__ uint64_t hoff[1 << kMaxScatterBits];
    __shared__ uint64_t tc_bar, tc_bbar;
    __shared__ uint64_t full_bar[kMaxStages];
    __shared__ uint32_t tc_tmem;
    __shared__ uint64_t bt[4 * 256];  // tile base tables
    if (threadIdx.x == 0) hdr = phdr;
    __syncthreads();
    // tile buffers from the first 1024-byte boundary (the TMA swizzle
    // pattern is a function of the shared-memory address)
    unsigned char* smem =
        smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    const bool use_tma = hdr.use_tma != 0;
    const int nbuf = use_tma ? hdr.nstage : 1;
    const TOp* ops = gops;
    const TSeg* segs = gsegs;
    const typename CoefT<V>::C* coef = gcoef;
    if constexpr (STG) stage_pass<V>(hdr, smem, nbuf, ops, segs, coef);
    if (!use_tma) tile_offsets(hdr, hoff);
    tile_base_tables(hdr, bt);
    TcCtx tcx;
    constexpr bool use_tc = TC;
    if constexpr (use_tc) {
        // operands after the tiles and the staged pass description (1 KiB aligned)
        size_t off = (size_t)nbuf * ((size_t)1 << hdr.tbits) * sizeof(V);
        if (STG) off += staged_bytes(hdr.nops, hdr.nsegs, hdr.ncoef, sizeof(typename CoefT<V>::C));
        off = (off + 1023) & ~(size_t)1023;
        tcx.xh = (float*)(smem + off);
        tcx.xl = tcx.xh + kTcRows * kTcKr;
        tcx.bh = tcx.xl + kTcRows * kTcKr;
        tcx.bl = tcx.bh + kTcN * kTcKr;
        tcx.bll = tcx.bl + kTcN * kTcKr;
        tcx.variant = hdr.tc_variant;
        tcx.resident = hdr.tc_resident > 0;
        tcx.bfloats = hdr.tc_variant & kTcVarInt8 ? kTc8BBytes / 4 : (hdr.tc_variant & kTcVarB3 ? 3u : 2u) * kTcN * kTcKr;
        tcx.mmat = mmat;
        tcx.loaded = -1;
        tcx.failed = 0;
        tcx.err = err;
        tcx.wait_ns = hdr.tc_test ? 100000000ull : kTcWaitNs;
        tcx.stall = hdr.tc_test;
        tcx.phase = 0;
        tcx.bar = &tc_bar;
        tcx.bphase = 0;
        tcx.bbar = &tc_bbar;
        if (threadIdx.x == 0) {
            tc::mbar_init(&tc_bar, 1);
            tc::mbar_init(&tc_bbar, 1);
        }
        if (threadIdx.x < 32) {
            tc::tmem_alloc(&tc_tmem, hdr.tc_variant & kTcVarInt8 ? 256u : (uint32_t)kTcCols);
            tc::tmem_relinquish();
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        tcx.tmem = tc_tmem;
        if (tcx.resident) {
            // every op's B operands in their slots, once for the whole pass
            // (thread 0 issues the MMAs: it alone waits, bounded)
            if (threadIdx.x == 0) {
                tc::mbar_arrive_expect_tx(tcx.bbar, (uint32_t)hdr.tc_resident * tcx.bfloats * 4);
                const size_t src0 = hdr.tc_variant & kTcVarInt8 ? (size_t)kTc8Off : 0;
                for (int j = 0; j < hdr.tc_resident; j++)
                    tc::bulk_g2s(tcx.bh + (size_t)j * tcx.bfloats, mmat + (size_t)j * kTcOpFloats + src0,
                                 tcx.bfloats * 4, tcx.bbar);
                const uint64_t t0 = global_ns_tc();
                bool ok;
                while (!(ok = tc::mbar_try_wait(tcx.bbar, 0)))
                    if (global_ns_tc() - t0 > tcx.wait_ns) break;
                if (!ok) {
                    tcx.failed = 1;
                    atomicExch(err, 1);
                }
            }
            tcx.loaded = -2;
        }
    }
    const uint32_t T = 1u << hdr.tbits;
    const uint32_t tile_bytes = T * (uint32_t)sizeof(V);
    const uint32_t sbase = tc::smem_u32(smem);
    const uint64_t grid = gridDim.x;
    uint64_t t = blockIdx.x;
    // loads in flight per buffer (thread 0's view): a wait that gave up
    // leaves one, waited for again before the CTA exits
    uint32_t pending = 0;
    if (use_tma) {
        if (threadIdx.x == 0) {
            tma::prefetch_map(&tmap);
            for (int q = 0; q < nbuf; q++) tc::mbar_init(&full_bar[q], 1);
            for (int q = 0; q < nbuf - 1; q++) {
                const uint64_t tq = t + (uint64_t)q * grid;
                if (tq < hdr.ntiles) {
                    tma_load_tile(&tmap, hdr, tile_base(tq, bt), sbase + q * tile_bytes, &full_bar[q], tile_bytes);
                    pending |= 1u << q;
                }
            }
        }
        __syncthreads();
    }
    bool dead = false;  // a wait gave up: skip the remaining waits
    // buffer of this tile (it % nbuf) and the parity of its use (it / nbuf),
    // carried from tile to tile instead of divided out
    uint32_t bcur = 0, bpar = 0;
    for (uint32_t it = 0; t < hdr.ntiles;
         t += grid, it++, bcur = bcur + 1 == (uint32_t)nbuf ? 0u : bcur + 1, bpar ^= bcur == 0 ? 1u : 0u) {
        const uint32_t b = use_tma ? bcur : 0;
        V* cur = (V*)(smem + (size_t)b * tile_bytes);
        const uint64_t base = tile_base(t, bt);
        if (use_tma) {
            // two buffers: the next tile's load goes out now, once the
            // previous tile's store has read the buffer it needs
            if (threadIdx.x == 0 && nbuf == 2) {
                const uint64_t tn = t + grid;
                if (tn < hdr.ntiles) {
                    const uint32_t bn = (it + 1) & 1u;
                    tma::wait_group_read<0>();
                    tma_load_tile(&tmap, hdr, tile_base(tn, bt), sbase + bn * tile_bytes, &full_bar[bn], tile_bytes);
                    pending |= 1u << bn;
                }
            }
            if (!dead) {
                const uint32_t parity = bpar;
                const uint64_t t0 = global_ns_tc();
                while (!tc::mbar_try_wait(&full_bar[b], parity)) {
                    if (global_ns_tc() - t0 > kTileWaitNs) {
                        dead = true;
                        atomicExch(err, 1);
                        break;
                    }
                }
                if (!dead && threadIdx.x == 0) pending &= ~(1u << b);
            }
        } else {
            tile_load<V, false>(st, hdr, hoff, base, cur);  // ends with __syncthreads
        }
        // TMA form: the tile's last barrier is the one before its store below
        if constexpr (use_tc)
            tile_compute<V, EXACT, RB, true>(hdr, base, ops, segs, coef, cur, &tcx, !use_tma);
        else
            tile_compute<V, EXACT, RB, false, DM>(hdr, base, ops, segs, coef, cur, nullptr, !use_tma);
        if (use_tma) {
            tc::fence_proxy_async();  // this thread's tile writes are visible to the bulk store
            __syncthreads();
            if (threadIdx.x == 0) {
                tma_store_tile(&tmap, hdr, base, sbase + b * tile_bytes);
                // three or more buffers: the load of tile it + nbuf - 1 goes
                // into the buffer of tile it - 1, whose store has had this
                // whole tile's compute to read it (at most this tile's store
                // may still be reading), so no thread waits before computing
                const uint64_t tn = t + (uint64_t)(nbuf - 1) * grid;
                if (nbuf > 2 && tn < hdr.ntiles) {
                    const uint32_t bn = bcur == 0 ? (uint32_t)nbuf - 1 : bcur - 1;
                    tma::wait_group_read<1>();
                    tma_load_tile(&tmap, hdr, tile_base(tn, bt), sbase + bn * tile_bytes, &full_bar[bn], tile_bytes);
                    pending |= 1u << bn;
                }
            }
        } else {
            tile_store<V>(st, hdr, hoff, base, cur);
            __syncthreads();  // `cur` is read out before it receives the next tile
        }
    }
    if (use_tma && threadIdx.x == 0) {
        tma::wait_group<0>();  // stores complete before the shared memory goes away
        const uint64_t t0 = global_ns_tc();
        for (int q = 0; q < nbuf; q++)
            if (pending & (1u << q))
                for (uint32_t ph = 0; ph < 2; ph++)
                    while (!tc::mbar_try_wait(&full_bar[q], ph) && global_ns_tc() - t0 < kTileWaitNs) {
                    }
    }
    if constexpr (use_tc) {
        // an MMA still in flight after a wait that gave up: wait for it
        // again (bounded) before the accumulator is freed
        if (tcx.failed) {
            const uint64_t t0 = global_ns_tc();
            while (!tc::mbar_try_wait(tcx.bar, tcx.phase ^ 1u) && global_ns_tc() - t0 < tcx.wait_ns) {
            }
            while (tcx.loaded >= 0 && !tc::mbar_try_wait(tcx.bbar, tcx.bphase ^ 1u) &&
                   global_ns_tc() - t0 < 2 * tcx.wait_ns) {
            }
            while (tcx.resident && !tc::mbar_try_wait(tcx.bbar, 0) && global_ns_tc() - t0 < 3 * tcx.wait_ns) {
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        if (threadIdx.x < 32) {
            tc::fence_after_sync();
            tc::tmem_dealloc(tcx.tmem, tcx.variant & kTcVarInt8 ? 256u : (uint32_t)kTcCols);
        }
    }
}

// ------------------------------------------------------------- batches
//
// Many circuits (uneven sizes) in one persistent launch.  Every (circuit,
// pass) is an entry; its tiles are cut into chunks of consecutive tiles.
// Entries are ordered level-major (every circuit's pass 0, then every
// circuit's pass 1, ...), chunks are taken from a global counter in that
// order, and a chunk first waits until all tiles of its circuit's previous
// passes are done (`done[circuit]` counts finished tiles).  A chunk only
// waits on chunks taken before it, by CTAs that are running, so the waits
// end; each wait is still bounded in time, and a wait that gives up sets
// `*err` (the host reports the batch as failed).
struct BatchEntry {
    TileHdr hdr;
    uint64_t state;  // device address of the circuit's state
    uint32_t circuit, pass;
    int32_t ops_off, segs_off, coef_off, pad;
};

struct BatchChunk {
    uint32_t entry, tile0, ntile, pad;
};

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint64_t kBatchWaitNs = 2000000000ull;  // 2 s

// STG: every entry's pass description is staged (shared-memory loads only);
// DM: entries may hold dense blocks for the FP64 tensor cores (complex128
// FUSED), as in k_tile_pass.
template <typename V, bool EXACT, int RB, bool STG = false, bool DM = false>
__global__ void __launch_bounds__(kTileThreads, 1)
    k_batch_tiles(const BatchEntry* __restrict__ entries, const BatchChunk* __restrict__ chunks, uint64_t nchunks,
                  unsigned long long* __restrict__ next, unsigned int* __restrict__ done, int* __restrict__ err,
                  const TOp* __restrict__ ops, const TSeg* __restrict__ segs,
                  const typename CoefT<V>::C* __restrict__ coef, uint64_t wait_ns) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ unsigned long long sj;
    __shared__ int sskip;
    __shared__ uint64_t hoff[1 << kMaxScatterBits];
    int staged = -1;  // entry whose pass description and offsets are in shared memory
    const TOp* o = ops;
    const TSeg* sgs = segs;
    const typename CoefT<V>::C* cf = coef;
    for (;;) {
        if (threadIdx.x == 0) sj = atomicAdd(next, 1ull);
        __syncthreads();
        const uint64_t c = sj;
        if (c >= nchunks) break;
        const BatchChunk ch = chunks[c];
        const BatchEntry& e = entries[ch.entry];
        if (threadIdx.x == 0) {
            const unsigned int need = (unsigned int)(e.pass * e.hdr.ntiles);
            int skip = 0;
            if (need > 0) {
                const uint64_t t0 = global_ns();
                while (*((volatile unsigned int*)&done[e.circuit]) < need) {
                    if (global_ns() - t0 > wait_ns) {
                        atomicExch(err, 1);
                        skip = 1;
                        break;
                    }
                    __nanosleep(256);
                }
                __threadfence();
            }
            sskip = skip;
        }
        __syncthreads();
        if (!sskip) {
            if ((int)ch.entry != staged) {
                o = ops + e.ops_off;
                sgs = segs + e.segs_off;
                cf = coef + e.coef_off;
                if (e.hdr.staged) stage_pass<V>(e.hdr, smem_raw, 1, o, sgs, cf);
                tile_offsets(e.hdr, hoff);
                staged = (int)ch.entry;
            }
            const TOp* po = o;
            const TSeg* ps = sgs;
            const typename CoefT<V>::C* pc = cf;
            if constexpr (STG) {
                // the staged copy, addressed from the shared-memory base
                TOp* so;
                TSeg* ss;
                typename CoefT<V>::C* sc;
                staged_ptrs<V>(e.hdr, smem_raw, 1, so, ss, sc);
                po = so;
                ps = ss;
                pc = sc;
            }
            for (uint32_t t = ch.tile0; t < ch.tile0 + ch.ntile; t++) {
                const uint64_t base = insert_zeros(t, e.hdr.tb, e.hdr.tbits);
                tile_load<V, true>((V*)e.state, e.hdr, hoff, base, (V*)smem_raw);
                tile_compute<V, EXACT, RB, false, DM>(e.hdr, base, po, ps, pc, (V*)smem_raw);
                tile_store<V>((V*)e.state, e.hdr, hoff, base, (V*)smem_raw);
                __syncthreads();
            }
            __threadfence();  // the stores are visible device-wide before the tiles are counted done
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&done[e.circuit], ch.ntile);
        }
        __syncthreads();
    }
}

// ================================================================ planner

struct PassPlan {
    bool single = false;  // true: one gate through the PLAIN kernels
    LGate gate;
    TileHdr hdr;
    std::vector<TOp> ops;
    std::vector<TSeg> segs;
    std::vector<Cx> coef;
    int rb = 0;           // register bits per thread in register segments
    std::vector<float> mmat;  // tensor-core operands (Bh, Bl per op, canonical layout)
};

// Largest number of register bits per thread (512 threads own a 2^12
// complex128 or 2^13 complex64 tile).
template <typename V>
constexpr int max_reg_bits() {
    return sizeof(V) == 16 ? 3 : 4;
}

// Cut a pass's ops into segments (see TSeg): consecutive ops whose moving
// tile bits fit in rb register bits share a register segment; a dense op on
// three or more targets is a wide segment of its own.
// pair0 (complex64 tiles): tile bit 0 is the first padding bit of a
// register segment, so each thread's amplitudes come in 16-byte pairs.
static void plan_segments(PassPlan& pp, int rb, bool pair0 = false) {
    // every non-wide op must fit one register segment
    for (const TOp& op : pp.ops)
        if (op.cls != GC_DIAG && !(op.cls == GC_DENSE && op.k >= 3)) rb = std::max(rb, (int)op.k);
    pp.rb = rb;
    pp.segs.clear();
    const int tbits = pp.hdr.tbits;
    size_t i = 0;
    while (i < pp.ops.size()) {
        TOp& op0 = pp.ops[i];
        TSeg sg;
        memset(&sg, 0, sizeof(sg));
        sg.op_begin = (int32_t)i;
        if (op0.cls == GC_DENSE && op0.k >= 3) {
            sg.wide = 1;
            sg.op_end = (int32_t)i + 1;
            pp.segs.push_back(sg);
            i++;
            continue;
        }
        std::set<int> bits;
        size_t j = i;
        for (; j < pp.ops.size(); j++) {
            const TOp& op = pp.ops[j];
            if (op.cls == GC_DENSE && op.k >= 3) break;
            std::set<int> nb = bits;
            if (op.cls != GC_DIAG)
                for (int q = 0; q < op.k; q++) nb.insert(op.tl[q]);
            if ((int)nb.size() > rb) break;
            bits = nb;
        }
        // pad with the highest unused tile bits: lanes of a warp then step
        // through the low bits, which are contiguous in shared memory
        if (pair0 && (int)bits.size() < rb) bits.insert(0);
        for (int b = tbits - 1; (int)bits.size() < rb && b >= 0; b--) bits.insert(b);
        std::vector<int> rbs(bits.begin(), bits.end());
        for (int q = 0; q < rb; q++) sg.rbs[q] = (int8_t)rbs[q];
        for (size_t q = i; q < j; q++) {
            TOp& op = pp.ops[q];
            if (op.cls == GC_DIAG) continue;
            for (int t = 0; t < op.k; t++)
                op.rp[t] = (int8_t)(std::find(rbs.begin(), rbs.end(), (int)op.tl[t]) - rbs.begin());
        }
        sg.op_end = (int32_t)j;
        pp.segs.push_back(sg);
        i = j;
    }
    pp.hdr.nsegs = (int32_t)pp.segs.size();
}

// Bits a gate moves amplitudes along (DIAG moves none).
// YAO_PASS_REORDER=0: FUSED passes keep program order too
static bool pass_reorder() {
    const char* e = getenv("YAO_PASS_REORDER");
    return !(e && e[0] == '0');
}

static uint64_t moving_mask(const LGate& g) {
    uint64_t m = 0;
    if (g.cls == GC_DIAG) return 0;
    for (int i = 0; i < g.k; i++) m |= (uint64_t)1 << g.tb[i];
    return m;
}

// Split a gate list into passes: each pass is a maximal contiguous run whose
// moving bits fit in `tbits` tile bits together with the low bits.  With
// `reorder` (FUSED runs) a pass is list-scheduled instead: the scan takes
// every gate that no skipped earlier gate shares a qubit with (targets or
// controls), so gates on disjoint qubits may run before gates they commute
// with; the arithmetic then differs from program order by rounding only.
// TILED runs keep program order (bit-identical to PLAIN).
static void plan_passes(const std::vector<LGate>& prog, uint32_t nbits, int tbits_max, std::vector<PassPlan>& out,
                        bool reorder = false) {
    int tbits = std::min<int>((int)nbits, tbits_max);
    const uint64_t all = nbits >= 64 ? ~0ull : ((1ull << nbits) - 1);
    std::vector<char> used(prog.size(), 0);
    size_t i = 0;
    while (i < prog.size()) {
        uint64_t hi = 0;  // moving bits of the run
        PassPlan pp;
        std::vector<const LGate*> run;
        // The tile is bits 0..3 (runs of >= 16 consecutive amplitudes per
        // load), the moving bits and the lowest other bits, tbits in total:
        // at most tbits - 4 moving bits outside bits 0..3.
        const bool whole = (int)nbits <= tbits;
        uint64_t blocked = 0;
        for (size_t j = i; j < prog.size(); j++) {
            if (used[j]) continue;
            uint64_t qm = moving_mask(prog[j]);
            for (int q = 0; q < prog[j].k; q++) qm |= (uint64_t)1 << prog[j].tb[q];
            for (int c = 0; c < prog[j].nc; c++) qm |= (uint64_t)1 << prog[j].cb[c];
            if (qm & blocked) {
                blocked |= qm;
                if ((blocked & all) == all) break;
                continue;
            }
            const uint64_t mb = moving_mask(prog[j]);
            const uint64_t nh = hi | mb;
            const int nused = whole ? __builtin_popcountll(nh) : __builtin_popcountll(nh & ~(uint64_t)0xF);
            if (nused > (whole ? (int)nbits : tbits - 4) || __builtin_popcountll(mb) > kMaxTargets) {
                if (!reorder) break;
                blocked |= qm;
                if ((blocked & all) == all) break;
                continue;
            }
            hi = nh;
            run.push_back(&prog[j]);
            used[j] = 1;
        }
        if (run.empty()) {
            PassPlan sp;
            sp.single = true;
            sp.gate = prog[i];
            out.push_back(sp);
            used[i] = 1;
            while (i < prog.size() && used[i]) i++;
            continue;
        }
        while (i < prog.size() && used[i]) i++;
        uint64_t tile = whole ? hi : (hi | (uint64_t)0xF);
        for (int b = 0; __builtin_popcountll(tile) < tbits && b < (int)nbits; b++) tile |= (uint64_t)1 << b;
        std::vector<int> TB;
        int local_tab[64];
        for (int b = 0; b < 64; b++) {
            local_tab[b] = -1;
            if ((tile >> b) & 1) {
                local_tab[b] = (int)TB.size();
                TB.push_back(b);
            }
        }
        memset(&pp.hdr, 0, sizeof(pp.hdr));
        pp.hdr.tbits = (int32_t)TB.size();
        int m = 0;
        while (m < (int)TB.size() && TB[m] == m) m++;
        pp.hdr.m = m;
        for (size_t q = 0; q < TB.size(); q++) pp.hdr.tb[q] = (int8_t)TB[q];
        pp.hdr.ntiles = (uint64_t)1 << (nbits - TB.size());
        auto local_of = [&](int gbit) -> int { return local_tab[gbit]; };
        for (const LGate* g : run) {
            TOp op;
            memset(&op, 0, sizeof(op));
            op.cls = g->cls;
            op.k = g->k;
            op.all_local = 1;
            op.mma = -1;
            for (int q = 0; q < g->k; q++) {
                op.tg[q] = (int8_t)g->tb[q];
                op.tl[q] = (int8_t)local_of(g->tb[q]);
                if (op.tl[q] < 0) op.all_local = 0;
                op.ts[q] = op.tl[q];
            }
            std::sort(op.ts, op.ts + g->k);
            for (int c = 0; c < g->nc; c++) {
                int lb = local_of(g->cb[c]);
                if (lb >= 0) {
                    op.lcmask |= 1u << lb;
                    if (g->cv[c]) op.lcval |= 1u << lb;
                } else {
                    op.gcmask |= (uint64_t)1 << g->cb[c];
                    if (g->cv[c]) op.gcval |= (uint64_t)1 << g->cb[c];
                }
            }
            op.moff = (int32_t)pp.coef.size();
            if (g->cls == GC_DIAG) {
                op.active = 0;
                for (size_t q = 0; q < g->m.size(); q++)
                    if (!(g->m[q].re == 1.0 && g->m[q].im == 0.0)) op.active |= (uint64_t)1 << q;
                if (op.active == 0) continue;
            }
            for (const Cx& c : g->m) pp.coef.push_back(c);
            if (pp.coef.empty()) pp.coef.push_back(Cx{0, 0});
            pp.ops.push_back(op);
        }
        pp.hdr.nops = (int32_t)pp.ops.size();
        out.push_back(pp);
    }
}

// ------------------------------------------------------------- fusion

// Left-multiply a block matrix (d x d over the block's local bits, row
// index = local output index) by an LGate whose bits are all block bits:
// M <- G M, column by column (host, FP64).
static void apply_gate_to_block(const LGate& g, const int* local_of_bit, size_t d, Cx* M) {
    uint64_t cm = 0, cvv = 0;
    for (int c = 0; c < g.nc; c++) {
        cm |= (uint64_t)1 << local_of_bit[g.cb[c]];
        if (g.cv[c]) cvv |= (uint64_t)1 << local_of_bit[g.cb[c]];
    }
    const int nl = 1 << g.k;
    uint64_t tmask = 0;
    size_t sc[1 << kMaxTargets];
    for (int l = 0; l < nl; l++) {
        size_t o = 0;
        for (int q = 0; q < g.k; q++)
            if ((l >> q) & 1) o |= (size_t)1 << local_of_bit[g.tb[q]];
        sc[l] = o;
    }
    for (int q = 0; q < g.k; q++) tmask |= (uint64_t)1 << local_of_bit[g.tb[q]];
    Cx old[1 << kMaxTargets];
    for (size_t b = 0; b < d; b++) {
        if (b & tmask) continue;
        if ((b & cm) != cvv) continue;
        for (size_t col = 0; col < d; col++) {
            for (int l = 0; l < nl; l++) old[l] = M[(b | sc[l]) * d + col];
            if (g.cls == GC_X) {
                M[(b | sc[0]) * d + col] = old[1];
                M[(b | sc[1]) * d + col] = old[0];
            } else if (g.cls == GC_SWAP) {
                M[(b | sc[1]) * d + col] = old[2];
                M[(b | sc[2]) * d + col] = old[1];
            } else if (g.cls == GC_DIAG) {
                for (int l = 0; l < nl; l++) {
                    const Cx a = old[l], e = g.m[l];
                    M[(b | sc[l]) * d + col] = Cx{a.re * e.re - a.im * e.im, a.re * e.im + a.im * e.re};
                }
            } else {
                for (int r = 0; r < nl; r++) {
                    Cx acc{0, 0};
                    for (int c = 0; c < nl; c++) {
                        const Cx m = g.m[(size_t)r * nl + c], x = old[c];
                        acc.re += m.re * x.re - m.im * x.im;
                        acc.im += m.re * x.im + m.im * x.re;
                    }
                    M[(b | sc[r]) * d + col] = acc;
                }
            }
        }
    }
}

struct Block {
    std::vector<int> bits;  // ascending global bit positions
    std::vector<Cx> m;      // 2^|bits| x 2^|bits|
    bool passthrough = false;  // a gate on more than kMaxTargets qubits, kept as is
    LGate gate;
};

static void block_extend(Block& b, const std::vector<int>& add) {
    std::vector<int> nb = b.bits;
    for (int x : add)
        if (std::find(nb.begin(), nb.end(), x) == nb.end()) nb.push_back(x);
    std::sort(nb.begin(), nb.end());
    if (nb.size() == b.bits.size()) return;
    size_t od = (size_t)1 << b.bits.size(), nd = (size_t)1 << nb.size();
    std::vector<int> pos_old(b.bits.size());  // old local bit i -> new local position
    for (size_t i = 0; i < b.bits.size(); i++)
        pos_old[i] = (int)(std::find(nb.begin(), nb.end(), b.bits[i]) - nb.begin());
    uint64_t oldmask_new = 0;
    for (int p : pos_old) oldmask_new |= (uint64_t)1 << p;
    std::vector<Cx> nm(nd * nd, Cx{0, 0});
    for (size_t r = 0; r < nd; r++)
        for (size_t c = 0; c < nd; c++) {
            if ((r & ~oldmask_new) != (c & ~oldmask_new)) continue;
            size_t ro = 0, co = 0;
            for (size_t i = 0; i < pos_old.size(); i++) {
                ro |= ((r >> pos_old[i]) & 1) << i;
                co |= ((c >> pos_old[i]) & 1) << i;
            }
            nm[r * nd + c] = b.m[ro * od + co];
        }
    b.bits = nb;
    b.m.swap(nm);
}

static void block_mul_gate(Block& b, const LGate& g, uint32_t nbits) {
    int local_of_bit[64];
    for (uint32_t i = 0; i < nbits && i < 64; i++) local_of_bit[i] = -1;
    for (size_t i = 0; i < b.bits.size(); i++) local_of_bit[b.bits[i]] = (int)i;
    apply_gate_to_block(g, local_of_bit, (size_t)1 << b.bits.size(), b.m.data());
}

// Greedy fusion into blocks of at most k qubits.  A gate joins the most
// recent block that touches any of its qubits when the union still has at
// most k qubits; every block created after that one is disjoint from the
// gate, so the creation order of blocks is a valid application order.
// Consecutive uncontrolled 1-qubit gates on the same bit multiplied into one
// dense 2 x 2 gate (host, FP64): fewer block updates in fuse_blocks.
static void merge_1q_runs(const std::vector<LGate>& prog, std::vector<LGate>& out) {
    out.clear();
    out.reserve(prog.size());
    auto dense2 = [](const LGate& g, Cx* m) {
        if (g.cls == GC_DENSE) {
            for (int i = 0; i < 4; i++) m[i] = g.m[i];
        } else if (g.cls == GC_DIAG) {
            m[0] = g.m[0];
            m[1] = Cx{0, 0};
            m[2] = Cx{0, 0};
            m[3] = g.m[1];
        } else {  // GC_X
            m[0] = Cx{0, 0};
            m[1] = Cx{1, 0};
            m[2] = Cx{1, 0};
            m[3] = Cx{0, 0};
        }
    };
    for (const LGate& g : prog) {
        const bool one = g.k == 1 && g.nc == 0 && (g.cls == GC_DENSE || g.cls == GC_DIAG || g.cls == GC_X);
        if (one && !out.empty()) {
            LGate& p = out.back();
            const bool pone = p.k == 1 && p.nc == 0 && (p.cls == GC_DENSE || p.cls == GC_DIAG || p.cls == GC_X);
            if (pone && p.tb[0] == g.tb[0]) {
                Cx a[4], b[4], c[4];
                dense2(p, a);
                dense2(g, b);
                for (int r = 0; r < 2; r++)  // c = b a (g after p)
                    for (int q = 0; q < 2; q++) {
                        const Cx x = b[r * 2], y = a[q], u = b[r * 2 + 1], v = a[2 + q];
                        c[r * 2 + q] = Cx{x.re * y.re - x.im * y.im + u.re * v.re - u.im * v.im,
                                          x.re * y.im + x.im * y.re + u.re * v.im + u.im * v.re};
                    }
                p.cls = GC_DENSE;
                p.m.assign(c, c + 4);
                continue;
            }
        }
        out.push_back(g);
    }
}

static void fuse_blocks(const std::vector<LGate>& prog_in, uint32_t nbits, int k, std::vector<LGate>& out) {
    std::vector<LGate> prog;
    merge_1q_runs(prog_in, prog);
    std::vector<Block> blocks;
    std::vector<int> last(nbits, -1);
    for (const LGate& g : prog) {
        std::vector<int> S;
        for (int q = 0; q < g.k; q++) S.push_back(g.tb[q]);
        for (int c = 0; c < g.nc; c++) S.push_back(g.cb[c]);
        int B = -1;
        for (int b : S) B = std::max(B, last[b]);
        if ((int)S.size() > kMaxTargets) {
            // too wide to fuse (its block matrix would exceed 2^6 x 2^6)
            Block pb;
            pb.passthrough = true;
            pb.gate = g;
            blocks.push_back(pb);
            for (int b : S) last[b] = (int)blocks.size() - 1;
            continue;
        }
        if (B >= 0 && !blocks[B].passthrough) {
            std::set<int> u(blocks[B].bits.begin(), blocks[B].bits.end());
            for (int b : S) u.insert(b);
            if ((int)u.size() <= std::max<int>(k, (int)blocks[B].bits.size())) {
                block_extend(blocks[B], S);
                block_mul_gate(blocks[B], g, nbits);
                for (int b : S) last[b] = B;
                continue;
            }
        }
        Block nb;
        nb.bits = S;
        std::sort(nb.bits.begin(), nb.bits.end());
        size_t d = (size_t)1 << nb.bits.size();
        nb.m.assign(d * d, Cx{0, 0});
        for (size_t i = 0; i < d; i++) nb.m[i * d + i] = Cx{1, 0};
        block_mul_gate(nb, g, nbits);
        blocks.push_back(nb);
        for (int b : S) last[b] = (int)blocks.size() - 1;
    }
    for (const Block& b : blocks) {
        if (b.passthrough) {
            out.push_back(b.gate);
            continue;
        }
        LGate g;
        g.k = (int)b.bits.size();
        for (int i = 0; i < g.k; i++) g.tb[i] = b.bits[i];
        g.nc = 0;
        size_t d = (size_t)1 << g.k;
        if (matrix_is_diagonal(b.m.data(), (uint32_t)d)) {
            g.cls = GC_DIAG;
            g.m.resize(d);
            for (size_t i = 0; i < d; i++) g.m[i] = b.m[i * d + i];
        } else {
            g.cls = GC_DENSE;
            g.m = b.m;
        }
        out.push_back(g);
    }
}

// ------------------------------------------------------------ execution

// Persistent launch: as many CTAs as fit on the SMs at once (each loops
// over its tiles with the next one in flight), never more than tiles.
template <typename V, bool EXACT, int RB, bool TCK, bool STG, bool DM = false>
static int launch_tile_k(int num_sms, unsigned threads, size_t smem, cudaStream_t s, V* st, const TileHdr& hdr,
                         const TOp* ops, const TSeg* segs, const typename CoefT<V>::C* coef, const float* mmat,
                         int* err, const CUtensorMap& tmap) {
    static bool attr = false;
    if (!attr) {
        int dev = 0, optin = 0;
        YAO_CUDA(cudaGetDevice(&dev));
        YAO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa;
        YAO_CUDA(cudaFuncGetAttributes(&fa, k_tile_pass<V, EXACT, RB, TCK, STG, DM>));
        YAO_CUDA(cudaFuncSetAttribute(k_tile_pass<V, EXACT, RB, TCK, STG, DM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      optin - (int)fa.sharedSizeBytes));
        YAO_CUDA(cudaFuncSetAttribute(k_tile_pass<V, EXACT, RB, TCK, STG, DM>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared));
        attr = true;
    }
    int per_sm = 0;
    YAO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_pass<V, EXACT, RB, TCK, STG, DM>, (int)threads, smem));
    if (per_sm < 1) return fail(YAO_ERR_UNSUPPORTED, "tile pass does not fit on an SM");
    const unsigned grid = (unsigned)std::min<uint64_t>(hdr.ntiles, (uint64_t)per_sm * (uint64_t)num_sms);
    k_tile_pass<V, EXACT, RB, TCK, STG, DM><<<grid, threads, smem, s>>>(st, hdr, ops, segs, coef, mmat, err, tmap);
    return YAO_OK;
}

template <typename V, bool EXACT, int RB>
static int launch_tile_rb(int num_sms, unsigned threads, size_t smem, cudaStream_t s, V* st, const TileHdr& hdr,
                          const TOp* ops, const TSeg* segs, const typename CoefT<V>::C* coef, const float* mmat,
                          int* err, const CUtensorMap& tmap) {
    if constexpr (sizeof(V) == 8 && !EXACT) {
        if (hdr.mma)
            return hdr.staged
                       ? launch_tile_k<V, EXACT, RB, true, true>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap)
                       : launch_tile_k<V, EXACT, RB, true, false>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap);
    }
    if constexpr (sizeof(V) == 16 && !EXACT && RB >= 2) {
        if (hdr.dmma)
            return hdr.staged
                       ? launch_tile_k<V, EXACT, RB, false, true, true>(num_sms, threads, smem, s, st, hdr, ops, segs, coef,
                                                                        mmat, err, tmap)
                       : launch_tile_k<V, EXACT, RB, false, false, true>(num_sms, threads, smem, s, st, hdr, ops, segs,
                                                                         coef, mmat, err, tmap);
    }
    return hdr.staged
               ? launch_tile_k<V, EXACT, RB, false, true>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap)
               : launch_tile_k<V, EXACT, RB, false, false>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap);
}

template <typename V, bool EXACT>
static int launch_tile(int rb, int num_sms, unsigned threads, size_t smem, cudaStream_t s, V* st,
                       const TileHdr& hdr, const TOp* ops, const TSeg* segs, const typename CoefT<V>::C* coef,
                       const float* mmat, int* err, const CUtensorMap& tmap) {
    switch (rb) {
    case 1: return launch_tile_rb<V, EXACT, 1>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap);
    case 2: return launch_tile_rb<V, EXACT, 2>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap);
    case 3: return launch_tile_rb<V, EXACT, 3>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap);
    case 4:
        if constexpr (sizeof(V) == 8)
            return launch_tile_rb<V, EXACT, 4>(num_sms, threads, smem, s, st, hdr, ops, segs, coef, mmat, err, tmap);
        break;
    default: break;
    }
    return fail(YAO_ERR_INVALID_ARGUMENT, "unsupported register-bit count");
}

// Dense complex128 FUSED blocks on the FP64 tensor cores (YAO_DMMA=0 keeps
// them on the CUDA cores).
static bool dmma_enabled() {
    const char* e = getenv("YAO_DMMA");
    return !(e && e[0] == '0');
}

// The coefficients of a pass with every block for the FP64 tensor cores
// stored with a row stride of 2^k + 2 (in place of its plain copy; each op
// owns the range from its offset to the next op's); rewrites the ops'
// offsets.  Returns whether some op was rewritten.
static bool pad_dmma(std::vector<TOp>& ops, const std::vector<Cx>& in, std::vector<Cx>& out, int rb, uint32_t tbits,
                     unsigned threads) {
    out.clear();
    bool any = false;
    const size_t first = ops.empty() ? in.size() : (size_t)ops[0].moff;
    out.insert(out.end(), in.begin(), in.begin() + first);
    for (size_t i = 0; i < ops.size(); i++) {
        TOp& op = ops[i];
        const size_t m0 = (size_t)op.moff, m1 = i + 1 < ops.size() ? (size_t)ops[i + 1].moff : in.size();
        op.moff = (int32_t)out.size();
        if (op.cls == GC_DENSE && op.mma < 0 && dmma_op(op.k, rb, tbits, threads)) {
            const size_t nl = (size_t)1 << op.k;
            for (size_t r = 0; r < nl; r++) {
                out.insert(out.end(), in.begin() + m0 + r * nl, in.begin() + m0 + (r + 1) * nl);
                out.push_back(Cx{0.0, 0.0});
                out.push_back(Cx{0.0, 0.0});
            }
            any = true;
        } else {
            out.insert(out.end(), in.begin() + m0, in.begin() + m1);
        }
    }
    return any;
}

// Coefficient count of a pass after pad_dmma (without building it).
static size_t padded_count(const std::vector<TOp>& ops, size_t ncoef, int rb, uint32_t tbits, unsigned threads) {
    size_t n = ops.empty() ? ncoef : (size_t)ops[0].moff;
    for (size_t i = 0; i < ops.size(); i++) {
        const TOp& op = ops[i];
        const size_t m0 = (size_t)op.moff, m1 = i + 1 < ops.size() ? (size_t)ops[i + 1].moff : ncoef;
        if (op.cls == GC_DENSE && op.mma < 0 && dmma_op(op.k, rb, tbits, threads)) {
            const size_t nl = (size_t)1 << op.k;
            n += nl * (nl + 2);
        } else {
            n += m1 - m0;
        }
    }
    return n;
}

// Grow a kept device / pinned host buffer to at least `bytes` (by 1.25x).
static int grow_dev(void** p, size_t* have, size_t bytes, cudaStream_t s) {
    if (bytes <= *have) return YAO_OK;
    const size_t nb = std::max(bytes, *have + *have / 4);
    if (*p) {
        YAO_CUDA(cudaStreamSynchronize(s));
        YAO_CUDA(cudaFree(*p));
        *p = nullptr;
        *have = 0;
    }
    if (cudaMalloc(p, nb) != cudaSuccess) {
        *p = nullptr;
        return fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate the batch tables");
    }
    *have = nb;
    return YAO_OK;
}
static int grow_host(void** p, size_t* have, size_t bytes) {
    if (bytes <= *have) return YAO_OK;
    const size_t nb = std::max(bytes, *have + *have / 4);
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *have = 0;
    if (cudaMallocHost(p, nb) != cudaSuccess) {
        *p = nullptr;
        return fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate pinned memory for the batch tables");
    }
    *have = nb;
    return YAO_OK;
}

// Tensor-core block variant (kTcVar* bits; YAO_TC_VARIANT overrides).
static int tc_variant() {
    const char* e = getenv("YAO_TC_VARIANT");
    return e ? (atoi(e) & 15) : 0;
}

// ------------------------------------------------------------- TMA maps

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library does not link libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

bool tma_enabled() {
    const char* e = getenv("YAO_TMA");
    return !(e && e[0] == '0');
}

// The TMA plan of a tile (see TmaPlan) whose positions are the global bits
// tb[0] < tb[1] < ... < tb[tbits - 1], and its tensor map over the state
// `st` of 2^nbits amplitudes of `amp` bytes.  Dimension 0 is the lowest c
// bits (128 bytes: c = 4 for complex64, 3 for complex128); then each run of
// consecutive global bits among the next tile positions (at most 8 bits a
// run: a box edge is at most 256) is one dimension, up to 4 of them; tile
// positions beyond those are enumerated (at least 1024 bytes a box, so
// every box lands on a swizzle-atom boundary).  Returns false when the tile
// cannot move by TMA (tiny tiles, low bits 0..c-1 not all in the tile,
// coordinates beyond 31 bits); the caller then moves it with plain copies.
bool tma_make_plan(const int8_t* tb, int tbits, uint32_t nbits, size_t amp, void* st, TmaPlan& p, CUtensorMap* map) {
    const int c = amp == 8 ? 4 : 3;
    int m = 0;
    while (m < tbits && tb[m] == m) m++;
    if (m < c || ((size_t)1 << tbits) * amp < 2048 || nbits > 33) return false;
    struct Run {
        int g0, len;
    };
    std::vector<Run> runs;
    int pos = c, J = c;
    while (pos < tbits && (int)runs.size() < 4) {
        Run r{tb[pos], 1};
        while (pos + r.len < tbits && r.len < 8 && tb[pos + r.len] == r.g0 + r.len) r.len++;
        runs.push_back(r);
        pos += r.len;
        J = pos;
    }
    if (((size_t)1 << J) * amp < 1024 || tbits - J > 6) return false;
    memset(&p, 0, sizeof(p));
    p.nebits = tbits - J;
    for (int q = 0; q < p.nebits; q++) p.ebits[q] = tb[J + q];
    p.copy_bytes = (int32_t)(((size_t)1 << J) * amp);
    cuuint64_t dim[5], stride[4];
    cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
    const int nd = 1 + (int)runs.size();
    for (int r = 0; r < 5; r++) {
        const int sh = r == 0 ? 0 : (r < nd ? runs[r - 1].g0 : (int)nbits);
        const int next = r + 1 < nd ? runs[r].g0 : (int)nbits;
        p.shift[r] = (int8_t)sh;
        p.width[r] = (int8_t)(r < nd ? next - sh : 0);
        dim[r] = (cuuint64_t)1 << p.width[r];
        box[r] = r == 0 ? 1u << c : (r < nd ? 1u << runs[r - 1].len : 1u);
        if (r > 0) stride[r - 1] = ((cuuint64_t)1 << sh) * amp;
    }
    if (p.width[0] > 29) return false;  // c0 = 2 x (bits below the first run) stays a positive int32
    dim[0] *= 2;  // two real elements per amplitude
    box[0] *= 2;
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const CUresult e = enc(map, amp == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, st,
                           dim, stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return e == CUDA_SUCCESS;
}

template <typename V, bool EXACT>
static int run_pass(Ctx* ctx, V* st, uint32_t nbits, const PassPlan& pp) {
    typedef typename CoefT<V>::C C;
    // blocks for the FP64 tensor cores get a copy of their matrix with a
    // row stride of 2^k + 2 (appended; the op points at it)
    std::vector<TOp> ops = pp.ops;
    std::vector<Cx> padded;
    const unsigned threads = (unsigned)(((uint32_t)1 << pp.hdr.tbits) >> pp.rb);
    const bool dm = sizeof(V) == 16 && !EXACT && dmma_enabled() &&
                    pad_dmma(ops, pp.coef, padded, pp.rb, (uint32_t)pp.hdr.tbits, threads);
    const std::vector<Cx>& cx = dm ? padded : pp.coef;
    std::vector<C> hc(cx.size());
    for (size_t i = 0; i < cx.size(); i++) {
        if (sizeof(V) == 16) {
            double2* p = (double2*)&hc[i];
            *p = make_double2(cx[i].re, cx[i].im);
        } else {
            float4* p = (float4*)&hc[i];
            float hr = (float)cx[i].re, hi = (float)cx[i].im;
            *p = make_float4(hr, hi, (float)(cx[i].re - (double)hr), (float)(cx[i].im - (double)hi));
        }
    }
    // one device buffer: ops | segments | coefficients | tensor-core operands
    // (256-byte aligned parts)
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    size_t ob = ops.size() * sizeof(TOp), sb = pp.segs.size() * sizeof(TSeg), cb = hc.size() * sizeof(C),
           mb = pp.mmat.size() * sizeof(float);
    size_t sb_off = al(ob);
    size_t cb_off = sb_off + al(sb);
    size_t mb_off = cb_off + al(cb);
    void* dbuf = nullptr;
    YAO_CUDA(cudaMallocAsync(&dbuf, mb_off + mb, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dbuf, ops.data(), ob, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync((char*)dbuf + sb_off, pp.segs.data(), sb, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync((char*)dbuf + cb_off, hc.data(), cb, cudaMemcpyHostToDevice, ctx->stream));
    if (mb) YAO_CUDA(cudaMemcpyAsync((char*)dbuf + mb_off, pp.mmat.data(), mb, cudaMemcpyHostToDevice, ctx->stream));
    TileHdr hdr = pp.hdr;
    hdr.ncoef = (int32_t)hc.size();
    if (hdr.tbits - hdr.m > kMaxScatterBits) return fail(YAO_ERR_UNSUPPORTED, "tile has too many scattered bits");
    const size_t tile_bytes = ((size_t)1 << hdr.tbits) * sizeof(V);
    const size_t stg = staged_bytes(hdr.nops, hdr.nsegs, hdr.ncoef, sizeof(C));
    // tiles by TMA when the pass has a plan; the pass description is staged
    // when it fits next to two tiles (and the tensor-core operands), and a
    // TMA pass gets a third tile buffer when that fits too; 16 KiB are left
    // for the kernel's static shared memory, 1 KiB for aligning the tiles
    CUtensorMap tmap;
    memset(&tmap, 0, sizeof(tmap));
    hdr.use_tma = tma_enabled() && tma_make_plan(hdr.tb, hdr.tbits, nbits, sizeof(V), st, hdr.tma, &tmap) ? 1 : 0;
    static int optin = 0;
    if (!optin) YAO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const size_t budget = (size_t)optin - 16 * 1024 - 1024;
    // tensor-core passes: X operands and the B operand slots; every op's B
    // stays resident for the pass when the slots fit beside two tiles,
    // else one slot is reloaded per op and tile
    size_t bslot = 0;
    int ntc = 0;
    if (hdr.mma) {
        // YAO_TEST_TC_STALL=1 (failure-path test): the tensor-core ops issue
        // neither their operand copy nor their MMAs, so both bounded waits of
        // each op run out (0.1 s each) and the call reports YAO_ERR_TIMEOUT
        if (const char* e = getenv("YAO_TEST_TC_STALL")) hdr.tc_test = e[0] == '1';
        hdr.tc_variant = tc_variant();
        bslot = hdr.tc_variant & kTcVarInt8 ? (size_t)kTc8BBytes : (hdr.tc_variant & kTcVarB3 ? 3 : 2) * kTcBPart;
        for (const TOp& op : ops) ntc += op.mma >= 0;
    }
    auto tcb = [&](int slots) { return hdr.mma ? 1024 + kTcXBytes + (size_t)slots * bslot : 0; };
    const char* re = getenv("YAO_TC_RESIDENT");
    const bool allow_res = !(re && re[0] == '0');
    hdr.tc_resident = hdr.mma && !hdr.tc_test && allow_res && 2 * tile_bytes + tcb(ntc) + stg <= budget ? ntc : 0;
    const int slots = hdr.tc_resident ? ntc : 1;
    hdr.staged = 2 * tile_bytes + tcb(slots) + stg <= budget ? 1 : 0;
    hdr.nstage = 2;
    // CTAs of at most 256 threads fit twice per SM by registers (128 a
    // thread): take the most tile buffers with which two CTAs fit the SM's
    // shared memory (16 warps instead of 8), else the most one CTA holds
    static int sm_total = 0;
    if (!sm_total)
        YAO_CUDA(cudaDeviceGetAttribute(&sm_total, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
    const size_t half = (size_t)sm_total / 2 - 16 * 1024 - 2048;  // static shared memory, reserve, alignment
    bool two = false;
    const char* te = getenv("YAO_TILE_TWO");  // YAO_TILE_TWO=0: the most buffers one CTA holds
    if (hdr.use_tma && !hdr.mma && threads <= 256 && !(te && te[0] == '0'))
        for (int ns = 3; ns >= 2 && !two; ns--)
            if ((size_t)ns * tile_bytes + (hdr.staged ? stg : 0) <= half) {
                hdr.nstage = ns;
                two = true;
            }
    for (int ns = 4; ns > 2 && hdr.use_tma && !two; ns--)
        if ((size_t)ns * tile_bytes + tcb(slots) + (hdr.staged ? stg : 0) <= budget) {
            hdr.nstage = ns;
            break;
        }
    hdr.dmma = dm ? 1 : 0;
    size_t smem = (size_t)(hdr.use_tma ? hdr.nstage : 1) * tile_bytes + (hdr.staged ? stg : 0);
    if (hdr.mma) smem = ((smem + 1023) & ~(size_t)1023) + kTcXBytes + (size_t)slots * bslot;
    smem += 1024;
    const TOp* dops = (const TOp*)dbuf;
    const TSeg* dsegs = (const TSeg*)((char*)dbuf + sb_off);
    const C* dcoef = (const C*)((char*)dbuf + cb_off);
    const float* dmmat = (const float*)((char*)dbuf + mb_off);
    if (!ctx->d_err) {
        YAO_CUDA(cudaMalloc((void**)&ctx->d_err, sizeof(int)));
        YAO_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    }
    {
        ProfScope prof(ctx, hdr.mma ? "tile_pass_tc" : (EXACT ? "tile_pass_exact" : "tile_pass_fused"),
                       (double)pp.hdr.ntiles * (double)((uint64_t)1 << pp.hdr.tbits) * 2.0 * sizeof(V));
        int s = launch_tile<V, EXACT>(pp.rb, ctx->num_sms, threads, smem, ctx->stream, st, hdr, dops, dsegs, dcoef,
                                      dmmat, ctx->d_err, tmap);
        if (s) return s;
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaFreeAsync(dbuf, ctx->stream));
    return YAO_OK;
}

// Execution choice of a TILED / FUSED run: fusion width k (FUSED), tile
// bits and register bits per thread.
struct TileConfig {
    int k = 0;
    int tbits = 0;
    int rb = 0;
    int tc = 1;  // complex64 FUSED: dense 3..5-qubit blocks may go to the tensor cores
};

// FP32 -> TF32, round to nearest even (low 13 mantissa bits cleared)
static float host_tf32(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0xFFFu + ((u >> 13) & 1u);
    u &= 0xFFFFE000u;
    memcpy(&f, &u, 4);
    return f;
}

// Mark the dense 3..5-qubit ops of a complex64 pass with a 2^12 tile for
// the tensor cores and append their operands.  A block on k < 5 targets is
// widened to 5 with the identity on 5 - k further tile bits (U x I), so every
// tensor-core op is one 128 x 64 x 64 product.  Operand: the block's real
// form B[2i+q][2j+p] (re/im of output i against re/im of input j), split into
// TF32 high and low parts, in the canonical K-major layout.
static void tc_prepare(PassPlan& pp) {
    if (pp.hdr.tbits != kTcTileBits) return;
    for (TOp& op : pp.ops) {
        if (op.cls != GC_DENSE || op.k < 3 || op.k > kTcK || op.lcmask != 0 || op.gcmask != 0) continue;
        const int k0 = op.k, nl0 = 1 << k0;
        // widen: local index bits k0..4 on tile positions outside the block
        uint32_t used = 0;
        for (int q = 0; q < k0; q++) used |= 1u << op.tl[q];
        for (int q = k0, pos = 0; q < kTcK; q++) {
            while (used & (1u << pos)) pos++;
            op.tl[q] = (int8_t)pos;
            used |= 1u << pos;
        }
        op.k = kTcK;
        for (int q = 0; q < kTcK; q++) op.ts[q] = op.tl[q];
        std::sort(op.ts, op.ts + kTcK);
        op.mma = (int32_t)pp.mmat.size();
        pp.mmat.resize(pp.mmat.size() + kTcOpFloats, 0.f);
        float* bh = pp.mmat.data() + op.mma;
        float* bl = bh + kTcN * kTcKr;
        float* bll = bl + kTcN * kTcKr;
        unsigned char* b8dig = (unsigned char*)(bh + kTc8Off);
        const int nl = 1 << kTcK;
        for (int i = 0; i < nl; i++)
            for (int j = 0; j < nl; j++) {
                const bool same_hi = (i >> k0) == (j >> k0);
                const Cx u = same_hi ? pp.coef[(size_t)op.moff + (size_t)(i & (nl0 - 1)) * nl0 + (j & (nl0 - 1))]
                                     : Cx{0.0, 0.0};
                const double v[2][2] = {{u.re, -u.im}, {u.im, u.re}};  // [q][p]
                for (int q = 0; q < 2; q++)
                    for (int p2 = 0; p2 < 2; p2++) {
                        const uint32_t o = 2 * i + q, kk = 2 * j + p2;
                        const size_t at = ((o >> 3) * kTcSbo + (kk >> 2) * 128 + (o & 7) * 16 + (kk & 3) * 4) / 4;
                        const float h = host_tf32((float)v[q][p2]);
                        const float l = host_tf32((float)(v[q][p2] - (double)h));
                        bh[at] = h;
                        bl[at] = l;
                        bll[at] = host_tf32((float)(v[q][p2] - (double)h - (double)l));
                        // integer form: v 2^34 rounded, five balanced base-2^7 digits
                        int64_t r = std::llround(std::ldexp(std::max(-1.0, std::min(1.0, v[q][p2])), 34));
                        const size_t b8 = (size_t)((o >> 3) * kTc8Sbo + (kk >> 4) * 128 + (o & 7) * 16 + (kk & 15));
                        for (int d = 0; d < 5; d++) {
                            const int sh = 7 * (4 - d);
                            const int64_t dig = d < 4 ? (r + ((int64_t)1 << (sh - 1))) >> sh : r;
                            r -= dig << sh;
                            b8dig[(size_t)d * kTc8BDigit + b8] = (unsigned char)(int8_t)dig;
                        }
                    }
            }
        pp.hdr.mma = 1;
    }
}

// The host plan of a TILED / FUSED run: passes (fused blocks, tile shapes,
// register segments, tensor-core operands).
template <typename V>
static void plan_run(uint32_t nbits, const std::vector<LGate>& prog, int32_t mode, const TileConfig& cfg,
                     std::vector<PassPlan>& passes, bool* any_tc) {
    std::vector<LGate> work;
    if (mode == YAO_MODE_FUSED)
        fuse_blocks(prog, nbits, std::min(cfg.k, kMaxTargets), work);
    else
        work = prog;
    passes.clear();
    plan_passes(work, nbits, cfg.tbits, passes, mode == YAO_MODE_FUSED && pass_reorder());
    for (PassPlan& pp : passes)
        if (!pp.single) {
            // at most kTileThreads threads per tile
            const int tb = (int)pp.hdr.tbits;
            const int rb = std::max(tb - 9, std::min(cfg.rb, tb));
            plan_segments(pp, std::min(rb, max_reg_bits<V>()), sizeof(V) == 8);
        }
    // dense 3..5-qubit blocks of complex64 FUSED runs go to the tensor cores
    // (cfg.tc; YAO_TC=0 keeps them on the CUDA cores)
    *any_tc = false;
    if (sizeof(V) == 8 && mode == YAO_MODE_FUSED && cfg.tc) {
        const char* e = getenv("YAO_TC");
        if (!(e && e[0] == '0'))
            for (PassPlan& pp : passes)
                if (!pp.single) {
                    tc_prepare(pp);
                    *any_tc |= pp.hdr.mma != 0;
                }
    }
}

// Launches passes[first], passes[first + step], ... of a plan.
template <typename V>
static int launch_passes(Ctx* ctx, V* st, uint32_t nbits, int32_t precision, int32_t mode,
                         const std::vector<PassPlan>& passes, size_t first = 0, size_t step = 1) {
    const bool exact = (mode == YAO_MODE_TILED) && sizeof(V) == 16;
    for (size_t i = first; i < passes.size(); i += step) {
        const PassPlan& pp = passes[i];
        int s;
        if (pp.single)
            s = launch_gate(ctx, st, precision, nbits, pp.gate);
        else if (exact)
            s = run_pass<V, true>(ctx, st, nbits, pp);
        else
            s = run_pass<V, false>(ctx, st, nbits, pp);
        if (s) return s;
    }
    return YAO_OK;
}

template <typename V>
static int run_program_cfg(Ctx* ctx, V* st, uint32_t nbits, int32_t precision, const std::vector<LGate>& prog,
                           int32_t mode, const TileConfig& cfg, bool check_err = true) {
    std::vector<PassPlan> passes;
    bool any_tc = false;
    plan_run<V>(nbits, prog, mode, cfg, passes, &any_tc);
    int s = launch_passes<V>(ctx, st, nbits, precision, mode, passes);
    if (s) return s;
    ctx->tc_used = any_tc;
    // a bounded wait of some pass (a tile's TMA copies, a tensor-core
    // operand copy or MMA completion) gave up: the run's result is void
    // (check_err false: the caller reads the error word at its own
    // synchronisation)
    if (ctx->d_err && check_err) {
        int herr = 0;
        YAO_CUDA(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        YAO_CUDA(cudaStreamSynchronize(ctx->stream));
        if (herr) {
            YAO_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
            return fail(YAO_ERR_TIMEOUT, "tile pass: a bounded wait (tile copy, tensor-core operand or MMA) gave up");
        }
    }
    return YAO_OK;
}

// ------------------------------------------------------------ autotuner
//
// The tile shape (tile bits, register bits) and, for FUSED with k = 0, the
// fusion width (and, for complex64, whether dense blocks go to the tensor
// cores) are picked by timing candidates on the device.  Every candidate's
// whole program is planned on the host; an evenly spread sample of its
// passes (at most kTuneSample, from the start, middle and end of the
// program alike) runs on a scratch copy of the register, and the sample's
// time scaled by passes / sampled passes estimates the run.  The fastest is
// kept per (device, qubits, precision, mode, requested k).  Choices live in
// memory and, when YAO_TUNE_CACHE names a file, in that file (one
// "key k tbits rb tc" line per entry).  YAO_TILE_BITS / YAO_REG_BITS pin the
// shape and YAO_AUTOTUNE=0 turns tuning off (defaults below).

static std::mutex g_tune_mu;
static std::map<std::string, TileConfig> g_tune;
static bool g_tune_loaded = false;

static std::string tune_key(int device, uint32_t nbits, int32_t prec, int32_t mode, int32_t kreq, const char* what) {
    char b[128];
    snprintf(b, sizeof(b), "%s/dev%d/n%u/p%d/m%d/k%d", what, device, nbits, prec, mode, kreq);
    return b;
}

// FNV-1a over a program's structure (gate classes, target and control bits;
// not the matrix entries): circuits that differ only in their parameters
// share a tuned configuration, other circuits of the same size do not.
static uint64_t program_shape_hash(const std::vector<LGate>& prog) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](uint64_t v) {
        for (int i = 0; i < 8; i++) {
            h ^= (v >> (8 * i)) & 0xff;
            h *= 1099511628211ull;
        }
    };
    mix(prog.size());
    for (const LGate& g : prog) {
        mix((uint64_t)(uint32_t)g.cls | (uint64_t)(uint32_t)g.k << 32);
        for (int i = 0; i < g.k; i++) mix((uint64_t)(uint32_t)g.tb[i]);
        mix(g.cmask());
        mix(g.cval());
    }
    return h;
}

static void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = getenv("YAO_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = fopen(path, "r");
    if (!f) return;
    char line[256], key[128];
    while (fgets(line, sizeof(line), f)) {
        TileConfig c;
        if (sscanf(line, "%127s %d %d %d %d", key, &c.k, &c.tbits, &c.rb, &c.tc) == 5) g_tune[key] = c;
    }
    fclose(f);
}

static void tune_store_locked() {
    const char* path = getenv("YAO_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = fopen(path, "w");
    if (!f) return;
    for (const auto& kv : g_tune)
        fprintf(f, "%s %d %d %d %d\n", kv.first.c_str(), kv.second.k, kv.second.tbits, kv.second.rb, kv.second.tc);
    fclose(f);
}

static bool env_int(const char* name, int lo, int hi, int* out) {
    const char* e = getenv(name);
    if (!e || !*e) return false;
    int v = atoi(e);
    if (v < lo || v > hi) return false;
    *out = v;
    return true;
}

template <typename V>
static TileConfig default_config(int32_t mode, int32_t kreq) {
    TileConfig c;
    c.k = mode == YAO_MODE_FUSED ? (kreq > 0 ? std::min(kreq, kMaxTargets) : 4) : 0;
    c.tbits = 11;
    c.rb = 2;
    env_int("YAO_TILE_BITS", 6, sizeof(V) == 16 ? 12 : 13, &c.tbits);
    env_int("YAO_REG_BITS", 1, max_reg_bits<V>(), &c.rb);
    return c;
}

template <typename V>
static void tile_candidates(uint32_t nbits, std::vector<TileConfig>& out) {
    // tile bits 10..12 (complex128), 10..13 (complex64: passes with little
    // work per tile run fastest on 2^10 tiles, 0.77 of HBM for one 1-qubit
    // block against 0.745 on 2^11)
    const int tmax = sizeof(V) == 16 ? 12 : 13;
    std::set<std::pair<int, int>> seen;
    for (int tb = 10; tb <= tmax; tb++)
        for (int rb = 2; rb <= max_reg_bits<V>(); rb++) {
            const int etb = std::min<int>(tb, (int)nbits);
            if (etb - rb > 9) continue;  // 2^(etb - rb) threads: at most kTileThreads
            if (!seen.insert({etb, rb}).second) continue;
            TileConfig c;
            c.tbits = tb;
            c.rb = rb;
            out.push_back(c);
        }
}

// Time every candidate on a scratch copy of the state; *best receives the
// fastest (left at the default when no scratch memory is available).
constexpr size_t kTuneSample = 12;

template <typename V>
static int tune_program(Ctx* ctx, const Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t kreq,
                        TileConfig* best, double* best_ms) {
    *best = default_config<V>(mode, kreq);
    *best_ms = -1.0;
    const uint32_t n = r->nbits;
    if (prog.empty()) return YAO_OK;
    const size_t bytes = ((size_t)1 << n) * sizeof(V);
    V* scratch = nullptr;
    if (cudaMallocAsync((void**)&scratch, bytes, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return YAO_OK;
    }
    YAO_CUDA(cudaMemcpyAsync(scratch, r->d, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    const bool prof = ctx->prof;
    ctx->prof = false;
    cudaEvent_t a, b;
    YAO_CUDA(cudaEventCreate(&a));
    YAO_CUDA(cudaEventCreate(&b));
    int st = YAO_OK;
    // one plan per candidate (host), then timed samples of its passes
    struct Cand {
        TileConfig c;
        std::vector<PassPlan> passes;
        size_t first = 0, step = 1, nsample = 0;
        float best = 0.f;  // estimated ms of the whole run
    };
    auto make = [&](const TileConfig& c) {
        Cand x;
        x.c = c;
        bool any_tc = false;
        plan_run<V>(n, prog, mode, c, x.passes, &any_tc);
        const size_t P = x.passes.size();
        x.step = P > kTuneSample ? P / kTuneSample : 1;
        x.first = P > kTuneSample ? (P - x.step * (kTuneSample - 1)) / 2 : 0;
        x.nsample = 0;
        for (size_t i = x.first; i < P; i += x.step) x.nsample++;
        return x;
    };
    auto timed = [&](Cand& x, float* ms) -> int {
        YAO_CUDA(cudaEventRecord(a, ctx->stream));
        int s = launch_passes<V>(ctx, scratch, n, r->precision, mode, x.passes, x.first, x.step);
        if (s) return s;
        YAO_CUDA(cudaEventRecord(b, ctx->stream));
        YAO_CUDA(cudaEventSynchronize(b));
        YAO_CUDA(cudaEventElapsedTime(ms, a, b));
        *ms *= (float)x.passes.size() / (float)std::max<size_t>(1, x.nsample);
        return YAO_OK;
    };
    // Candidates are timed in interleaved rounds (every candidate once per
    // round, after a warm-up round: first launches of each kernel variant
    // carry one-time costs), keeping each one's best run.  Under the power
    // cap the SM clock drifts over seconds; interleaving gives every
    // candidate the same clocks, so a drift does not pick a slower one.
    constexpr int kRounds = 3;
    // YAO_TUNE_LOG=1: every candidate's estimate on stderr
    const char* tl = getenv("YAO_TUNE_LOG");
    const bool log = tl && tl[0] == '1';
    auto best_of = [&](std::vector<Cand>& cand, size_t* pick, float* pick_ms) -> int {
        float ms = 0.f;
        for (int round = 0; round <= kRounds; round++)
            for (size_t i = 0; i < cand.size(); i++) {
                int s = timed(cand[i], &ms);
                if (s) return s;
                if (round == 1 || (round > 1 && ms < cand[i].best)) cand[i].best = ms;
            }
        *pick = 0;
        for (size_t i = 1; i < cand.size(); i++)
            if (cand[i].best < cand[*pick].best) *pick = i;
        *pick_ms = cand[*pick].best;
        if (log)
            for (size_t i = 0; i < cand.size(); i++)
                fprintf(stderr,
                        "[yao tune] n=%u %s mode=%d k=%d tbits=%d rb=%d tc=%d: %.3f ms (%zu of %zu passes timed)%s\n",
                        n, sizeof(V) == 8 ? "c64" : "c128", mode, cand[i].c.k, cand[i].c.tbits, cand[i].c.rb,
                        cand[i].c.tc, cand[i].best, cand[i].nsample, cand[i].passes.size(),
                        i == *pick ? "  <- chosen" : "");
        return YAO_OK;
    };
    std::vector<TileConfig> shapes;
    tile_candidates<V>(n, shapes);
    std::vector<Cand> cand;
    for (const TileConfig& sc : shapes) {
        TileConfig c = *best;
        c.tbits = sc.tbits;
        c.rb = sc.rb;
        cand.push_back(make(c));
    }
    size_t pick = 0;
    float bms = 0.f;
    st = best_of(cand, &pick, &bms);
    if (!st) *best = cand[pick].c;
    if (!st && mode == YAO_MODE_FUSED && kreq <= 0) {
        // widths 2..6 with the chosen shape; complex64 widths 3..5 also
        // with the tensor cores' 2^12 tile, on and off the tensor cores
        const TileConfig shape = *best;
        std::vector<TileConfig> cs;
        for (int k = 2; k <= kMaxTargets; k++) {
            TileConfig c = shape;
            c.k = k;
            c.tc = 0;
            cs.push_back(c);
            if (sizeof(V) == 8 && k >= 3 && k <= kTcK)
                for (int rb = 3; rb <= 4; rb++) {  // 512 or 256 threads a tile
                    c.tbits = kTcTileBits;
                    c.rb = rb;
                    c.tc = 1;
                    cs.push_back(c);
                }
        }
        cand.clear();
        for (const TileConfig& c : cs) cand.push_back(make(c));
        st = best_of(cand, &pick, &bms);
        if (!st) *best = cand[pick].c;
    } else if (!st && mode == YAO_MODE_FUSED && sizeof(V) == 8 && kreq >= 3 && kreq <= kTcK) {
        // a requested complex64 width: the tensor cores' 2^12 tile against the
        // chosen shape on the CUDA cores
        TileConfig on = *best, on4 = *best, off = *best;
        on.tbits = on4.tbits = kTcTileBits;
        on.rb = 3;
        on4.rb = 4;
        on.tc = on4.tc = 1;
        off.tc = 0;
        cand.clear();
        cand.push_back(make(on));
        cand.push_back(make(on4));
        cand.push_back(make(off));
        st = best_of(cand, &pick, &bms);
        if (!st) *best = cand[pick].c;
    }
    ctx->prof = prof;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(scratch, ctx->stream);
    if (!st) *best_ms = bms;
    return st;
}

template <typename V>
static int choose_config(Ctx* ctx, const Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t kreq,
                         bool force, TileConfig* out) {
    *out = default_config<V>(mode, kreq);
    if (!force) {
        int pinned = 0;
        if (env_int("YAO_TILE_BITS", 6, 13, &pinned) || env_int("YAO_REG_BITS", 1, 4, &pinned)) return YAO_OK;
        const char* at = getenv("YAO_AUTOTUNE");
        if (at && at[0] == '0') return YAO_OK;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    YAO_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return YAO_OK;  // no synchronising while a graph is captured
    char what[32];
    snprintf(what, sizeof(what), "prog-%016llx", (unsigned long long)program_shape_hash(prog));
    const std::string key = tune_key(ctx->device, r->nbits, r->precision, mode, kreq, what);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_load_locked();
        auto it = g_tune.find(key);
        if (it != g_tune.end() && !force) {
            *out = it->second;
            return YAO_OK;
        }
    }
    double ms;
    int s = tune_program<V>(ctx, r, prog, mode, kreq, out, &ms);
    if (s) return s;
    if (ms >= 0) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune[key] = *out;
        tune_store_locked();
    }
    return YAO_OK;
}

template <typename V>
static int run_program_t(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k, bool check_err) {
    V* st = (V*)r->d;
    if (mode == YAO_MODE_PLAIN) {
        for (const LGate& g : prog) {
            int s = launch_gate(ctx, st, r->precision, r->nbits, g);
            if (s) return s;
        }
        return YAO_OK;
    }
    TileConfig cfg;
    int s = choose_config<V>(ctx, r, prog, mode, k, false, &cfg);
    if (s) return s;
    return run_program_cfg<V>(ctx, st, r->nbits, r->precision, prog, mode, cfg, check_err);
}

int launch_program(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k, bool check_err) {
    if (r->precision == YAO_C128) return run_program_t<double2>(ctx, r, prog, mode, k, check_err);
    return run_program_t<float2>(ctx, r, prog, mode, k, check_err);
}

int read_device_err(Ctx* ctx, const char* what) {
    if (!ctx->d_err) return YAO_OK;
    int herr = 0;
    YAO_CUDA(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!herr) return YAO_OK;
    YAO_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    return fail(YAO_ERR_TIMEOUT, std::string(what) + ": a bounded wait of a kernel gave up");
}

int plan_info(const std::vector<LGate>& prog, uint32_t nbits, int32_t precision, int32_t mode, int32_t k,
              int32_t tbits, int32_t rb, int64_t info[7]) {
    for (int i = 0; i < 7; i++) info[i] = 0;
    std::vector<LGate> work;
    if (mode == YAO_MODE_FUSED)
        fuse_blocks(prog, nbits, std::max(1, std::min<int>(k, kMaxTargets)), work);
    else
        work = prog;
    info[6] = (int64_t)work.size();
    std::vector<PassPlan> passes;
    plan_passes(work, nbits, tbits, passes, mode == YAO_MODE_FUSED && pass_reorder());
    const int maxrb = precision == YAO_C128 ? max_reg_bits<double2>() : max_reg_bits<float2>();
    for (PassPlan& pp : passes) {
        info[0]++;
        if (pp.single) {
            info[1]++;
            continue;
        }
        const int tb = (int)pp.hdr.tbits;
        plan_segments(pp, std::min(std::max(tb - 9, std::min<int>(rb, tb)), maxrb), precision == YAO_C64);
        if (precision == YAO_C64 && mode == YAO_MODE_FUSED) tc_prepare(pp);
        info[2] += (int64_t)pp.ops.size();
        for (const TOp& op : pp.ops) {
            if (op.mma >= 0)
                info[3]++;
            else if (op.cls == GC_DENSE && op.k >= 3)
                info[4]++;
        }
        for (const TSeg& sg : pp.segs) info[5] += sg.wide ? 0 : 1;
    }
    return YAO_OK;
}

int autotune_program(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k, int32_t out[4]) {
    TileConfig c;
    int s = r->precision == YAO_C128 ? choose_config<double2>(ctx, r, prog, mode, k, true, &c)
                                     : choose_config<float2>(ctx, r, prog, mode, k, true, &c);
    if (s) return s;
    out[0] = c.k;
    out[1] = c.tbits;
    out[2] = c.rb;
    out[3] = c.tc;
    return YAO_OK;
}

// ------------------------------------------------------------ batch host

// YAO_BATCH_TIMING=1: host phase times of a batched launch on stderr.
struct PhaseTimer {
    bool on;
    std::chrono::steady_clock::time_point t0;
    PhaseTimer() : on(getenv("YAO_BATCH_TIMING") != nullptr), t0(std::chrono::steady_clock::now()) {}
    void mark(const char* what) {
        if (!on) return;
        const auto t = std::chrono::steady_clock::now();
        fprintf(stderr, "batch %s: %.1f ms\n", what, std::chrono::duration<double, std::milli>(t - t0).count());
        t0 = t;
    }
};

template <typename V>
static int batch_t(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                   int32_t mode, const TileConfig& cfg) {
    typedef typename CoefT<V>::C C;
    PhaseTimer ptimer;
    const int tbits_cap = std::min(cfg.tbits, 12), rb = 3;
    const int k = cfg.k;
    const bool exact = mode == YAO_MODE_TILED && sizeof(V) == 16;
    // plan every circuit (independent: spread over host threads)
    std::vector<std::vector<PassPlan>> plans(progs.size());
    for (size_t c = 0; c < progs.size(); c++)
        if (regs[c]->nbits < 3) return fail(YAO_ERR_UNSUPPORTED, "batched circuits need at least 3 qubits");
    std::vector<int> bad(progs.size(), 0);
    auto plan_one = [&](size_t c) {
        std::vector<LGate> work;
        if (mode == YAO_MODE_FUSED)
            fuse_blocks(*progs[c], regs[c]->nbits, std::max(1, std::min(k, kMaxTargets)), work);
        plan_passes(mode == YAO_MODE_FUSED ? work : *progs[c], regs[c]->nbits, tbits_cap, plans[c],
                    mode == YAO_MODE_FUSED && pass_reorder());
        for (PassPlan& pp : plans[c]) {
            if (pp.single) bad[c] = 1;
            else if (pp.hdr.tbits - pp.hdr.m > kMaxScatterBits) bad[c] = 2;
            else plan_segments(pp, rb, sizeof(V) == 8);
        }
    };
    {
        const size_t nth = std::max<size_t>(1, std::min<size_t>({(size_t)std::thread::hardware_concurrency(),
                                                                  (size_t)32, progs.size() / 8 + 1}));
        std::atomic<size_t> nextc(0);
        auto worker = [&]() {
            for (size_t c; (c = nextc.fetch_add(1)) < progs.size();) plan_one(c);
        };
        std::vector<std::thread> pool;
        for (size_t t = 1; t < nth; t++) pool.emplace_back(worker);
        worker();
        for (std::thread& th : pool) th.join();
    }
    size_t maxpasses = 0;
    for (size_t c = 0; c < progs.size(); c++) {
        if (bad[c] == 1) return fail(YAO_ERR_UNSUPPORTED, "a gate of the batch does not fit a tile");
        if (bad[c] == 2) return fail(YAO_ERR_UNSUPPORTED, "tile has too many scattered bits");
        maxpasses = std::max(maxpasses, plans[c].size());
    }
    ptimer.mark("plan");
    // entries level-major, ops / segments / coefficients concatenated, in
    // one table laid out as on the device: sizes and offsets first, then
    // every entry filled in parallel into pinned memory, one copy up
    const bool use_dm = sizeof(V) == 16 && mode == YAO_MODE_FUSED && dmma_enabled();
    struct Slot {
        uint32_t c, level;
        size_t ops, segs, coef, chunk;  // offsets
        uint32_t nchunk, per;
    };
    std::vector<Slot> slots;
    size_t nops = 0, nsegs = 0, ncoef = 0, nchunks = 0;
    for (size_t level = 0; level < maxpasses; level++)
        for (size_t c = 0; c < progs.size(); c++) {
            if (level >= plans[c].size()) continue;
            const PassPlan& pp = plans[c][level];
            Slot sl;
            sl.c = (uint32_t)c;
            sl.level = (uint32_t)level;
            sl.ops = nops;
            sl.segs = nsegs;
            sl.coef = ncoef;
            sl.chunk = nchunks;
            // chunks of consecutive tiles: about 32 per pass of a large
            // circuit, at most 16 tiles each
            const uint32_t nt = (uint32_t)pp.hdr.ntiles;
            sl.per = std::max<uint32_t>(1, std::min<uint32_t>(16, nt / 32));
            sl.nchunk = (nt + sl.per - 1) / sl.per;
            nops += pp.ops.size();
            nsegs += pp.segs.size();
            ncoef += use_dm ? padded_count(pp.ops, pp.coef.size(), rb, (uint32_t)pp.hdr.tbits, kTileThreads)
                            : pp.coef.size();
            nchunks += sl.nchunk;
            slots.push_back(sl);
        }
    if (nchunks == 0) return YAO_OK;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t b_ent = al(slots.size() * sizeof(BatchEntry)), b_chk = al(nchunks * sizeof(BatchChunk)),
                 b_ops = al(std::max<size_t>(1, nops) * sizeof(TOp)), b_seg = al(std::max<size_t>(1, nsegs) * sizeof(TSeg)),
                 b_coef = al(std::max<size_t>(1, ncoef) * sizeof(C)),
                 b_ctr = al(sizeof(unsigned long long) + sizeof(int) + progs.size() * sizeof(unsigned int));
    const size_t b_tab = b_ent + b_chk + b_ops + b_seg + b_coef;
    int st;
    if ((st = grow_host(&ctx->batch_host, &ctx->batch_host_bytes, b_tab))) return st;
    if ((st = grow_dev(&ctx->batch_dev, &ctx->batch_dev_bytes, b_tab + b_ctr, ctx->stream))) return st;
    char* hp = (char*)ctx->batch_host;
    BatchEntry* h_ent = (BatchEntry*)hp;
    BatchChunk* h_chk = (BatchChunk*)(hp + b_ent);
    TOp* h_ops = (TOp*)(hp + b_ent + b_chk);
    TSeg* h_seg = (TSeg*)(hp + b_ent + b_chk + b_ops);
    C* h_coef = (C*)(hp + b_ent + b_chk + b_ops + b_seg);
    std::atomic<size_t> next_slot(0);
    std::atomic<int> any_dm_a(0), unstaged_a(0);
    std::atomic<size_t> max_stg_a(0);
    auto fill = [&]() {
        std::vector<TOp> eops;
        std::vector<Cx> padded;
        size_t my_max = 0;
        for (size_t e; (e = next_slot.fetch_add(1)) < slots.size();) {
            const Slot& sl = slots[e];
            const PassPlan& pp = plans[sl.c][sl.level];
            BatchEntry be;
            memset(&be, 0, sizeof(be));
            be.hdr = pp.hdr;
            be.state = (uint64_t)(uintptr_t)regs[sl.c]->d;
            be.circuit = sl.c;
            be.pass = sl.level;
            be.ops_off = (int32_t)sl.ops;
            be.segs_off = (int32_t)sl.segs;
            be.coef_off = (int32_t)sl.coef;
            // blocks for the FP64 tensor cores: padded rows (see pad_dmma)
            const std::vector<Cx>* cx = &pp.coef;
            const std::vector<TOp>* po = &pp.ops;
            if (use_dm) {
                eops = pp.ops;
                if (pad_dmma(eops, pp.coef, padded, rb, (uint32_t)pp.hdr.tbits, kTileThreads)) {
                    cx = &padded;
                    po = &eops;
                    any_dm_a.store(1);
                }
            }
            std::copy(po->begin(), po->end(), h_ops + sl.ops);
            std::copy(pp.segs.begin(), pp.segs.end(), h_seg + sl.segs);
            C* dst = h_coef + sl.coef;
            for (const Cx& x : *cx) {
                C cc;
                if (sizeof(V) == 16) {
                    const double2 v = make_double2(x.re, x.im);
                    memcpy(&cc, &v, sizeof(cc));
                } else {
                    float hr = (float)x.re, hi = (float)x.im;
                    const float4 v = make_float4(hr, hi, (float)(x.re - (double)hr), (float)(x.im - (double)hi));
                    memcpy(&cc, &v, sizeof(cc));
                }
                *dst++ = cc;
            }
            be.hdr.ncoef = (int32_t)cx->size();
            const size_t stg = staged_bytes(be.hdr.nops, be.hdr.nsegs, be.hdr.ncoef, sizeof(C));
            be.hdr.staged = stg <= kMaxStagedBytes ? 1 : 0;
            if (be.hdr.staged)
                my_max = std::max(my_max, stg);
            else
                unstaged_a.store(1);
            h_ent[e] = be;
            const uint32_t nt = (uint32_t)pp.hdr.ntiles;
            for (uint32_t q = 0; q < sl.nchunk; q++) {
                BatchChunk ch;
                ch.entry = (uint32_t)e;
                ch.tile0 = q * sl.per;
                ch.ntile = std::min(sl.per, nt - ch.tile0);
                ch.pad = 0;
                h_chk[sl.chunk + q] = ch;
            }
        }
        size_t cur = max_stg_a.load();
        while (my_max > cur && !max_stg_a.compare_exchange_weak(cur, my_max)) {
        }
    };
    {
        const size_t nth = std::max<size_t>(1, std::min<size_t>({(size_t)std::thread::hardware_concurrency(),
                                                                  (size_t)32, slots.size() / 64 + 1}));
        std::vector<std::thread> pool;
        for (size_t t = 1; t < nth; t++) pool.emplace_back(fill);
        fill();
        for (std::thread& th : pool) th.join();
    }
    const size_t max_stg = max_stg_a.load();
    const bool all_staged = unstaged_a.load() == 0, any_dm = any_dm_a.load() != 0;
    // YAO_TEST_BATCH_STALL=1 (failure-path test): circuit 0's second pass
    // waits for a tile count that is never reached, with a 0.2 s limit, so
    // the bounded wait runs out and the call reports YAO_ERR_TIMEOUT
    uint64_t wait_ns = kBatchWaitNs;
    if (const char* e = getenv("YAO_TEST_BATCH_STALL"))
        if (e[0] == '1')
            for (size_t q = 0; q < slots.size(); q++)
                if (h_ent[q].circuit == 0 && h_ent[q].pass == 1) {
                    h_ent[q].pass = 1u << 20;
                    wait_ns = 200000000ull;
                }
    ptimer.mark("entries");
    char* buf = (char*)ctx->batch_dev;
    BatchEntry* d_ent = (BatchEntry*)buf;
    BatchChunk* d_chk = (BatchChunk*)(buf + b_ent);
    TOp* d_ops = (TOp*)(buf + b_ent + b_chk);
    TSeg* d_seg = (TSeg*)(buf + b_ent + b_chk + b_ops);
    C* d_coef = (C*)(buf + b_ent + b_chk + b_ops + b_seg);
    char* p = buf + b_tab;
    unsigned long long* d_next = (unsigned long long*)p;
    int* d_err = (int*)(p + sizeof(unsigned long long));
    unsigned int* d_done = (unsigned int*)(p + sizeof(unsigned long long) + sizeof(int));
    YAO_CUDA(cudaMemcpyAsync(buf, hp, b_tab, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    const size_t smem = ((size_t)1 << tbits_cap) * sizeof(V) + max_stg;
    // complex128 FUSED batches with blocks for the FP64 tensor cores: the
    // DM instantiation, reading a staged description from shared memory only
    // when every entry is staged (the other forms measured no faster so)
    auto kern = exact ? k_batch_tiles<V, true, 3>
                      : any_dm ? (all_staged ? k_batch_tiles<V, false, 3, true, true> : k_batch_tiles<V, false, 3, false, true>)
                               : k_batch_tiles<V, false, 3>;
    YAO_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    YAO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileThreads, smem));
    const unsigned grid = (unsigned)std::max(1, per_sm) * (unsigned)ctx->num_sms;
    ptimer.mark("upload");
    // capture: reset the queue and counters, run the persistent kernel
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    YAO_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(d_next, 0, b_ctr, ctx->stream);
    kern<<<grid, kTileThreads, smem, ctx->stream>>>(d_ent, d_chk, (uint64_t)nchunks, d_next, d_done, d_err,
                                                    d_ops, d_seg, d_coef, wait_ns);
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    if (ce != cudaSuccess) return cuda_fail(ce, "capture of the batch launch");
    YAO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    {
        double bytes = 0;
        for (size_t q = 0; q < slots.size(); q++)
            bytes += (double)h_ent[q].hdr.ntiles * (double)(1u << h_ent[q].hdr.tbits) * 2.0 * sizeof(V);
        ProfScope prof(ctx, exact ? "batch_tiles_exact" : "batch_tiles_fused", bytes);
        YAO_CUDA(cudaGraphLaunch(exec, ctx->stream));
    }
    ctx->launches++;
    int herr = 0;
    YAO_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    ptimer.mark("launch");
    if (herr) return fail(YAO_ERR_TIMEOUT, "batched launch: a chunk waited too long for its circuit's previous pass");
    return YAO_OK;
}

// Batch autotuner: tile bits (10..12) and, for FUSED with k = 0, the fusion
// width (2..6), timed on up to 64 of the batch's circuits (evenly spaced)
// run on scratch copies of their registers; kept per (device, largest
// qubit count, precision, mode, requested k) like the single-circuit choice.
template <typename V>
static int tune_batch(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                      int32_t mode, int32_t kreq, TileConfig* best, bool* tuned) {
    *tuned = false;
    const size_t ns = std::min<size_t>(64, regs.size());
    std::vector<const std::vector<LGate>*> sp(ns);
    std::vector<Reg> sr(ns);
    std::vector<Reg*> srp(ns);
    size_t total = 0;
    for (size_t i = 0; i < ns; i++) {
        const size_t c = i * regs.size() / ns;
        sp[i] = progs[c];
        sr[i] = *regs[c];
        total += (regs[c]->bytes() + 255) / 256 * 256;
    }
    char* scratch = nullptr;
    if (cudaMallocAsync((void**)&scratch, total, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return YAO_OK;
    }
    size_t off = 0;
    for (size_t i = 0; i < ns; i++) {
        YAO_CUDA(cudaMemcpyAsync(scratch + off, sr[i].d, sr[i].bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
        sr[i].d = scratch + off;
        srp[i] = &sr[i];
        off += (sr[i].bytes() + 255) / 256 * 256;
    }
    const bool prof = ctx->prof;
    ctx->prof = false;
    cudaEvent_t a, b;
    YAO_CUDA(cudaEventCreate(&a));
    YAO_CUDA(cudaEventCreate(&b));
    auto timed = [&](const TileConfig& c, float* ms) -> int {
        YAO_CUDA(cudaEventRecord(a, ctx->stream));
        int s = batch_t<V>(ctx, sp, srp, mode, c);
        if (s) return s;
        YAO_CUDA(cudaEventRecord(b, ctx->stream));
        YAO_CUDA(cudaEventSynchronize(b));
        YAO_CUDA(cudaEventElapsedTime(ms, a, b));
        return YAO_OK;
    };
    int st = YAO_OK;
    float ms = 0.f, bms = 0.f;
    bool have = false;
    TileConfig cur = *best;
    for (int tb = 10; !st && tb <= 12; tb++) {
        TileConfig c = cur;
        c.tbits = tb;
        if ((st = timed(c, &ms))) break;  // warm-up of this shape
        if ((st = timed(c, &ms))) break;
        if (!have || ms < bms) {
            bms = ms;
            *best = c;
            have = true;
        }
    }
    if (!st && mode == YAO_MODE_FUSED && kreq <= 0) {
        const TileConfig shape = *best;
        for (int k = 2; k <= kMaxTargets; k++) {
            if (k == shape.k) continue;
            TileConfig c = shape;
            c.k = k;
            float m2 = 0.f;  // the better of two runs (the first also warms up)
            if ((st = timed(c, &ms))) break;
            if ((st = timed(c, &m2))) break;
            ms = std::min(ms, m2);
            if (ms < bms) {
                bms = ms;
                *best = c;
            }
        }
    }
    ctx->prof = prof;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(scratch, ctx->stream);
    *tuned = !st;
    return st;
}

template <typename V>
static int batch_choose(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                        int32_t mode, int32_t kreq, TileConfig* out) {
    *out = default_config<V>(mode, kreq);
    out->tbits = 12;
    if (mode == YAO_MODE_FUSED && kreq <= 0) out->k = 2;
    int pinned = 0;
    if (env_int("YAO_TILE_BITS", 6, 12, &pinned)) {
        out->tbits = pinned;
        return YAO_OK;
    }
    const char* at = getenv("YAO_AUTOTUNE");
    if (at && at[0] == '0') return YAO_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    YAO_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return YAO_OK;
    uint32_t nmax = 0;
    for (const Reg* r : regs) nmax = std::max(nmax, r->nbits);
    const std::string key = tune_key(ctx->device, nmax, regs[0]->precision, mode, kreq, "batch");
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_load_locked();
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            *out = it->second;
            return YAO_OK;
        }
    }
    bool tuned = false;
    int s = tune_batch<V>(ctx, progs, regs, mode, kreq, out, &tuned);
    if (s) return s;
    if (tuned) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune[key] = *out;
        tune_store_locked();
    }
    return YAO_OK;
}

template <typename V>
static int batch_entry(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                       int32_t mode, int32_t k) {
    TileConfig cfg;
    int s = batch_choose<V>(ctx, progs, regs, mode, k, &cfg);
    if (s) return s;
    return batch_t<V>(ctx, progs, regs, mode, cfg);
}

int launch_batch(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                 int32_t mode, int32_t k) {
    if (regs.empty()) return YAO_OK;
    if (regs[0]->precision == YAO_C128) return batch_entry<double2>(ctx, progs, regs, mode, k);
    return batch_entry<float2>(ctx, progs, regs, mode, k);
}

}  // namespace yao
