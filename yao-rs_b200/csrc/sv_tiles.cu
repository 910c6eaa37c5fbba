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
//    qubits (host, FP64); each block is one op of a pass.  On complex64
//    registers the block coefficients are split into an FP32 high part and
//    an FP32 low part (c = hi + lo), and both products are accumulated in
//    FP32 (a two-term compensated product).
#include <algorithm>
#include <cmath>
#include <set>
#include <vector>

#include "device_common.cuh"

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
};

struct TOp {
    int32_t cls;
    int32_t k;
    int8_t tl[kMaxTargets];  // local target positions (-1 = outside the tile, DIAG only)
    int8_t tg[kMaxTargets];  // global target positions
    int32_t all_local;
    uint32_t lcmask, lcval;  // in-tile controls (local bit positions)
    uint64_t gcmask, gcval;  // out-of-tile controls (global bit positions)
    uint64_t active;         // DIAG: non-unit entries
    int32_t moff;            // first coefficient in the pass's coefficient array
    int8_t rp[kMaxTargets];  // register segments: target positions among the segment's register bits
    int8_t pad[2];
};

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
// split-coefficient products for complex64 data: hi*x + lo*x, FP32 accumulate
template <bool EXACT>
__device__ __forceinline__ float2 cmul_c(float4 c, float2 x) {
    float hr = fmaf(c.x, x.x, -c.y * x.y), hi = fmaf(c.x, x.y, c.y * x.x);
    float lr = fmaf(c.z, x.x, -c.w * x.y), li = fmaf(c.z, x.y, c.w * x.x);
    return make_float2(hr + lr, hi + li);
}
template <bool EXACT>
__device__ __forceinline__ float2 cfma_c(float2 acc, float4 c, float2 x) {
    float2 p = cmul_c<EXACT>(c, x);
    return make_float2(acc.x + p.x, acc.y + p.y);
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
constexpr int kMaxItems = 16;  // outputs per thread in a wide op (2^RB <= 16)
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
__device__ __forceinline__ uint32_t swz(uint32_t l, double2*) { return l ^ ((l >> 3) & 7); }
__device__ __forceinline__ uint32_t swz(uint32_t l, float2*) { return l ^ ((l >> 4) & 15); }

template <typename V>
__device__ __forceinline__ uint64_t tile_global(uint64_t base, uint32_t l, const TileHdr& hdr) {
    uint64_t gi = base | (l & ((1u << hdr.m) - 1));
    for (int j = hdr.m; j < hdr.tbits; j++) gi |= (uint64_t)((l >> j) & 1) << hdr.tb[j];
    return gi;
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
#pragma unroll
    for (int j = 0; j < (1 << RB); j++) {
        if (j & (1 << P)) continue;
        const int j1 = j | (1 << P);
        if (((lbase | roff[j]) & op.lcmask) != op.lcval) continue;
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

// One tile of one pass: load, every segment, store.  COHERENT loads bypass
// L1 (the tile may have been written by another SM during the same launch).
template <typename V, bool EXACT, int RB, bool COHERENT>
__device__ __forceinline__ void tile_body(V* __restrict__ st, const TileHdr& hdr, uint64_t t,
                                          const TOp* __restrict__ ops, const TSeg* __restrict__ segs,
                                          const typename CoefT<V>::C* __restrict__ coef, V* s) {
    typedef typename CoefT<V>::C C;
    constexpr int NA = 1 << RB;
    V* tag = nullptr;  // selects the swizzle overload
    const uint32_t T = 1u << hdr.tbits;
    const int nt = blockDim.x;
    {
        const uint64_t base = insert_zeros(t, hdr.tb, hdr.tbits);
        for (uint32_t l = threadIdx.x; l < T; l += nt) {
            const V* src = &st[tile_global<V>(base, l, hdr)];
            s[swz(l, tag)] = COHERENT ? ld_l2(src) : *src;
        }
        __syncthreads();
        for (int si = 0; si < hdr.nsegs; si++) {
            const TSeg sg = segs[si];
            if (!sg.wide && threadIdx.x < (T >> RB)) {
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
                    v[j] = s[swz(lbase | o, tag)];
                }
                for (int oi = sg.op_begin; oi < sg.op_end; oi++) {
                    const TOp& op = ops[oi];
                    if ((base & op.gcmask) != op.gcval) continue;  // uniform over the tile
                    const C* m = coef + op.moff;
                    if (op.cls == GC_DIAG) {
#pragma unroll
                        for (int j = 0; j < NA; j++) {
                            const uint32_t l = lbase | roff[j];
                            if ((l & op.lcmask) != op.lcval) continue;
                            uint32_t dl = 0;
                            if (op.all_local) {
                                for (int i = 0; i < op.k; i++) dl |= ((l >> op.tl[i]) & 1) << i;
                            } else {
                                const uint64_t gi = tile_global<V>(base, l, hdr);
                                for (int i = 0; i < op.k; i++) dl |= (uint32_t)((gi >> op.tg[i]) & 1) << i;
                            }
                            if ((op.active >> dl) & 1) v[j] = cmulassign_c<EXACT>(v[j], m[dl]);
                        }
                    } else if (op.k == 1) {
                        reg1_at<V, EXACT, RB, 0>(op.rp[0], v, lbase, roff, op, m);
                    } else {
                        reg2_at<V, EXACT, RB, 0, 1>(op.rp[0], op.rp[1], v, lbase, roff, op, m);
                    }
                }
#pragma unroll
                for (int j = 0; j < NA; j++) s[swz(lbase | roff[j], tag)] = v[j];
            } else if (sg.wide) {
                // one dense op on k >= 3 targets: item = (group, row); outputs
                // stay in registers until every thread has read its inputs
                const TOp& op = ops[sg.op_begin];
                const bool on = (base & op.gcmask) == op.gcval;
                const C* m = coef + op.moff;
                const int k = op.k, nl = 1 << k;
                int sorted[kMaxTargets];
                for (int i = 0; i < k; i++) sorted[i] = op.tl[i];
                for (int i = 1; i < k; i++)
                    for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; j--) {
                        int tmp = sorted[j];
                        sorted[j] = sorted[j - 1];
                        sorted[j - 1] = tmp;
                    }
                V outv[kMaxItems];
                uint32_t outi[kMaxItems];
                int cnt = 0;
                for (uint32_t it = threadIdx.x; on && it < T; it += nt) {
                    uint32_t g = it >> k, row = it & (nl - 1);
                    uint32_t b = g;
                    for (int i = 0; i < k; i++) b = ins0(b, sorted[i]);
                    const bool act = (b & op.lcmask) == op.lcval;
                    uint32_t ro = 0;
                    for (int i = 0; i < k; i++) ro |= ((row >> i) & 1) << op.tl[i];
                    V acc = VecT<V>::zero();
                    if (act) {
                        const C* mr = m + (size_t)row * nl;
                        for (int c = 0; c < nl; c++) {
                            uint32_t co = 0;
                            for (int i = 0; i < k; i++) co |= ((c >> i) & 1) << op.tl[i];
                            acc = cfma_c<EXACT>(acc, mr[c], s[swz(b | co, tag)]);
                        }
                    }
                    outv[cnt] = acc;
                    outi[cnt] = act ? (b | ro) : 0xffffffffu;
                    cnt++;
                }
                __syncthreads();
                for (int i = 0; i < cnt; i++)
                    if (outi[i] != 0xffffffffu) s[swz(outi[i], tag)] = outv[i];
            }
            __syncthreads();
        }
        for (uint32_t l = threadIdx.x; l < T; l += nt) st[tile_global<V>(base, l, hdr)] = s[swz(l, tag)];
        if (COHERENT) __threadfence();  // the stores are visible device-wide before the tile is marked done
        __syncthreads();
    }
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
__device__ __forceinline__ void stage_pass(const TileHdr& hdr, unsigned char* smem, const TOp*& ops, const TSeg*& segs,
                                           const typename CoefT<V>::C*& coef) {
    typedef typename CoefT<V>::C C;
    if (!hdr.staged) return;
    auto a16 = [](size_t x) { return (x + 15) / 16 * 16; };
    unsigned char* p = smem + ((size_t)1 << hdr.tbits) * sizeof(V);
    TOp* so = (TOp*)p;
    p += a16((size_t)hdr.nops * sizeof(TOp));
    TSeg* ss = (TSeg*)p;
    p += a16((size_t)hdr.nsegs * sizeof(TSeg));
    C* sc = (C*)p;
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

template <typename V, bool EXACT, int RB>
__global__ void __launch_bounds__(kTileThreads, RB <= 2 ? 2 : 1)
    k_tile_pass(V* __restrict__ st, const TileHdr hdr, const TOp* __restrict__ gops, const TSeg* __restrict__ gsegs,
                const typename CoefT<V>::C* __restrict__ gcoef) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TOp* ops = gops;
    const TSeg* segs = gsegs;
    const typename CoefT<V>::C* coef = gcoef;
    stage_pass<V>(hdr, smem_raw, ops, segs, coef);
    for (uint64_t t = blockIdx.x; t < hdr.ntiles; t += gridDim.x)
        tile_body<V, EXACT, RB, false>(st, hdr, t, ops, segs, coef, (V*)smem_raw);
}

// ------------------------------------------------------------- batches
//
// Many circuits (uneven sizes) in one persistent launch.  Every (circuit,
// pass) is an entry; its tiles are jobs.  Entries are ordered level-major
// (every circuit's pass 0, then every circuit's pass 1, ...), jobs are taken
// from a global counter in that order, and a job first waits until all tiles
// of its circuit's previous passes are done (`done[circuit]` counts finished
// tiles).  A job only waits on jobs taken before it, by CTAs that are
// running, so the waits end; each wait is still bounded in time, and a wait
// that gives up sets `*err` and lets the job (and its circuit) fail.
struct BatchEntry {
    TileHdr hdr;
    uint64_t state;      // device address of the circuit's state
    uint64_t job_start;  // first job id of this entry
    uint32_t circuit, pass;
    int32_t ops_off, segs_off, coef_off, pad;
};

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint64_t kBatchWaitNs = 2000000000ull;  // 2 s

template <typename V, bool EXACT, int RB>
__global__ void __launch_bounds__(kTileThreads, 1)
    k_batch_tiles(const BatchEntry* __restrict__ entries, int nentries, uint64_t njobs,
                  unsigned long long* __restrict__ next, unsigned int* __restrict__ done, int* __restrict__ err,
                  const TOp* __restrict__ ops, const TSeg* __restrict__ segs,
                  const typename CoefT<V>::C* __restrict__ coef) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long sj;
    __shared__ int se, sskip;
    for (;;) {
        if (threadIdx.x == 0) sj = atomicAdd(next, 1ull);
        __syncthreads();
        const uint64_t j = sj;
        if (j >= njobs) break;
        if (threadIdx.x == 0) {
            int lo = 0, hi = nentries - 1;  // last entry with job_start <= j
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (entries[mid].job_start <= j)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            se = lo;
            const BatchEntry& e = entries[lo];
            const unsigned int need = (unsigned int)(e.pass * e.hdr.ntiles);
            int skip = 0;
            if (need > 0) {
                const uint64_t t0 = global_ns();
                while (*((volatile unsigned int*)&done[e.circuit]) < need) {
                    if (global_ns() - t0 > kBatchWaitNs) {
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
        const BatchEntry& e = entries[se];
        if (!sskip) {
            const TOp* o = ops + e.ops_off;
            const TSeg* sgs = segs + e.segs_off;
            const typename CoefT<V>::C* cf = coef + e.coef_off;
            stage_pass<V>(e.hdr, smem_raw, o, sgs, cf);
            tile_body<V, EXACT, RB, true>((V*)e.state, e.hdr, j - e.job_start, o, sgs, cf, (V*)smem_raw);
        }
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&done[e.circuit], 1u);
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
static void plan_segments(PassPlan& pp, int rb) {
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
static void moving_bits(const LGate& g, std::vector<int>& out) {
    out.clear();
    if (g.cls == GC_DIAG) return;
    for (int i = 0; i < g.k; i++) out.push_back(g.tb[i]);
}

// Split a gate list into passes: each pass is a maximal contiguous run whose
// moving bits fit in `tbits` tile bits together with the low bits.
static void plan_passes(const std::vector<LGate>& prog, uint32_t nbits, int tbits_max, std::vector<PassPlan>& out) {
    int tbits = std::min<int>((int)nbits, tbits_max);
    size_t i = 0;
    while (i < prog.size()) {
        std::set<int> hi;  // moving bits at or above the low run
        PassPlan pp;
        std::vector<const LGate*> run;
        size_t j = i;
        // The tile is the moving bits plus the lowest other bits, tbits in
        // total.  Keeping at most tbits - 4 moving bits guarantees bits 0..3
        // are in the tile (runs of >= 16 consecutive amplitudes per load).
        const int limit = ((int)nbits <= tbits) ? (int)nbits : tbits - 4;
        for (; j < prog.size(); j++) {
            std::vector<int> mb;
            moving_bits(prog[j], mb);
            std::set<int> nh = hi;
            for (int b : mb) nh.insert(b);
            if ((int)nh.size() > limit || (int)mb.size() > kMaxTargets) break;
            hi = nh;
            run.push_back(&prog[j]);
        }
        if (run.empty()) {
            PassPlan sp;
            sp.single = true;
            sp.gate = prog[i];
            out.push_back(sp);
            i++;
            continue;
        }
        std::set<int> tile = hi;
        for (int b = 0; (int)tile.size() < tbits && b < (int)nbits; b++) tile.insert(b);
        std::vector<int> TB(tile.begin(), tile.end());
        memset(&pp.hdr, 0, sizeof(pp.hdr));
        pp.hdr.tbits = (int32_t)TB.size();
        int m = 0;
        while (m < (int)TB.size() && TB[m] == m) m++;
        pp.hdr.m = m;
        for (size_t q = 0; q < TB.size(); q++) pp.hdr.tb[q] = (int8_t)TB[q];
        pp.hdr.ntiles = (uint64_t)1 << (nbits - TB.size());
        auto local_of = [&](int gbit) -> int {
            for (size_t q = 0; q < TB.size(); q++)
                if (TB[q] == gbit) return (int)q;
            return -1;
        };
        for (const LGate* g : run) {
            TOp op;
            memset(&op, 0, sizeof(op));
            op.cls = g->cls;
            op.k = g->k;
            op.all_local = 1;
            for (int q = 0; q < g->k; q++) {
                op.tg[q] = (int8_t)g->tb[q];
                op.tl[q] = (int8_t)local_of(g->tb[q]);
                if (op.tl[q] < 0) op.all_local = 0;
            }
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
        i = j;
    }
}

// ------------------------------------------------------------- fusion

// Apply an LGate to a small dense vector over the block's local bits
// (host, FP64) -- used to multiply gates into fused block matrices.
static void host_apply(const LGate& g, const std::vector<int>& local_of_bit, std::vector<Cx>& v) {
    const size_t n = v.size();
    auto lb = [&](int gb) { return local_of_bit[gb]; };
    uint64_t cm = 0, cvv = 0;
    for (int c = 0; c < g.nc; c++) {
        cm |= (uint64_t)1 << lb(g.cb[c]);
        if (g.cv[c]) cvv |= (uint64_t)1 << lb(g.cb[c]);
    }
    uint64_t tmask = 0;
    for (int q = 0; q < g.k; q++) tmask |= (uint64_t)1 << lb(g.tb[q]);
    const int nl = 1 << g.k;
    std::vector<Cx> old(nl);
    for (size_t b = 0; b < n; b++) {
        if (b & tmask) continue;
        if ((b & cm) != cvv) continue;
        std::vector<size_t> idx(nl);
        for (int l = 0; l < nl; l++) {
            size_t o = b;
            for (int q = 0; q < g.k; q++)
                if ((l >> q) & 1) o |= (size_t)1 << lb(g.tb[q]);
            idx[l] = o;
            old[l] = v[o];
        }
        if (g.cls == GC_X) {
            v[idx[0]] = old[1];
            v[idx[1]] = old[0];
        } else if (g.cls == GC_SWAP) {
            v[idx[1]] = old[2];
            v[idx[2]] = old[1];
        } else if (g.cls == GC_DIAG) {
            for (int l = 0; l < nl; l++) {
                Cx a = old[l], d = g.m[l];
                v[idx[l]] = Cx{a.re * d.re - a.im * d.im, a.re * d.im + a.im * d.re};
            }
        } else {
            for (int r = 0; r < nl; r++) {
                Cx acc{0, 0};
                for (int c = 0; c < nl; c++) {
                    Cx m = g.m[(size_t)r * nl + c], x = old[c];
                    acc.re += m.re * x.re - m.im * x.im;
                    acc.im += m.re * x.im + m.im * x.re;
                }
                v[idx[r]] = acc;
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
    std::vector<int> local_of_bit(nbits, -1);
    for (size_t i = 0; i < b.bits.size(); i++) local_of_bit[b.bits[i]] = (int)i;
    size_t d = (size_t)1 << b.bits.size();
    std::vector<Cx> col(d);
    for (size_t c = 0; c < d; c++) {
        for (size_t r = 0; r < d; r++) col[r] = b.m[r * d + c];
        host_apply(g, local_of_bit, col);
        for (size_t r = 0; r < d; r++) b.m[r * d + c] = col[r];
    }
}

// Greedy fusion into blocks of at most k qubits.  A gate joins the most
// recent block that touches any of its qubits when the union still has at
// most k qubits; every block created after that one is disjoint from the
// gate, so the creation order of blocks is a valid application order.
static void fuse_blocks(const std::vector<LGate>& prog, uint32_t nbits, int k, std::vector<LGate>& out) {
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

template <typename V, bool EXACT, int RB>
static int launch_tile_rb(unsigned grid, unsigned threads, size_t smem, cudaStream_t s, V* st, const TileHdr& hdr,
                          const TOp* ops, const TSeg* segs, const typename CoefT<V>::C* coef) {
    static bool attr = false;
    if (!attr) {
        YAO_CUDA(cudaFuncSetAttribute(k_tile_pass<V, EXACT, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      160 * 1024));
        YAO_CUDA(cudaFuncSetAttribute(k_tile_pass<V, EXACT, RB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared));
        attr = true;
    }
    k_tile_pass<V, EXACT, RB><<<grid, threads, smem, s>>>(st, hdr, ops, segs, coef);
    return YAO_OK;
}

template <typename V, bool EXACT>
static int launch_tile(int rb, unsigned grid, unsigned threads, size_t smem, cudaStream_t s, V* st,
                       const TileHdr& hdr, const TOp* ops, const TSeg* segs, const typename CoefT<V>::C* coef) {
    switch (rb) {
    case 1: return launch_tile_rb<V, EXACT, 1>(grid, threads, smem, s, st, hdr, ops, segs, coef);
    case 2: return launch_tile_rb<V, EXACT, 2>(grid, threads, smem, s, st, hdr, ops, segs, coef);
    case 3: return launch_tile_rb<V, EXACT, 3>(grid, threads, smem, s, st, hdr, ops, segs, coef);
    case 4:
        if constexpr (sizeof(V) == 8) return launch_tile_rb<V, EXACT, 4>(grid, threads, smem, s, st, hdr, ops, segs, coef);
        break;
    default: break;
    }
    return fail(YAO_ERR_INVALID_ARGUMENT, "unsupported register-bit count");
}

template <typename V, bool EXACT>
static int run_pass(Ctx* ctx, V* st, uint32_t nbits, const PassPlan& pp) {
    typedef typename CoefT<V>::C C;
    std::vector<C> hc(pp.coef.size());
    for (size_t i = 0; i < pp.coef.size(); i++) {
        if (sizeof(V) == 16) {
            double2* p = (double2*)&hc[i];
            *p = make_double2(pp.coef[i].re, pp.coef[i].im);
        } else {
            float4* p = (float4*)&hc[i];
            float hr = (float)pp.coef[i].re, hi = (float)pp.coef[i].im;
            *p = make_float4(hr, hi, (float)(pp.coef[i].re - (double)hr), (float)(pp.coef[i].im - (double)hi));
        }
    }
    // one device buffer: ops | segments | coefficients (256-byte aligned parts)
    size_t ob = pp.ops.size() * sizeof(TOp), sb = pp.segs.size() * sizeof(TSeg), cb = hc.size() * sizeof(C);
    size_t sb_off = (ob + 255) / 256 * 256;
    size_t cb_off = sb_off + (sb + 255) / 256 * 256;
    void* dbuf = nullptr;
    YAO_CUDA(cudaMallocAsync(&dbuf, cb_off + cb, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dbuf, pp.ops.data(), ob, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync((char*)dbuf + sb_off, pp.segs.data(), sb, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync((char*)dbuf + cb_off, hc.data(), cb, cudaMemcpyHostToDevice, ctx->stream));
    TileHdr hdr = pp.hdr;
    hdr.ncoef = (int32_t)hc.size();
    const size_t tile_bytes = ((size_t)1 << hdr.tbits) * sizeof(V);
    const size_t stg = staged_bytes(hdr.nops, hdr.nsegs, hdr.ncoef, sizeof(C));
    hdr.staged = stg <= kMaxStagedBytes ? 1 : 0;
    const size_t smem = tile_bytes + (hdr.staged ? stg : 0);
    const unsigned threads = (unsigned)(((uint32_t)1 << pp.hdr.tbits) >> pp.rb);
    const unsigned grid = (unsigned)std::min<uint64_t>(pp.hdr.ntiles, (uint64_t)ctx->num_sms * 4);
    const TOp* dops = (const TOp*)dbuf;
    const TSeg* dsegs = (const TSeg*)((char*)dbuf + sb_off);
    const C* dcoef = (const C*)((char*)dbuf + cb_off);
    {
        ProfScope prof(ctx, EXACT ? "tile_pass_exact" : "tile_pass_fused",
                       (double)pp.hdr.ntiles * (double)((uint64_t)1 << pp.hdr.tbits) * 2.0 * sizeof(V));
        int s = launch_tile<V, EXACT>(pp.rb, grid, threads, smem, ctx->stream, st, hdr, dops, dsegs, dcoef);
        if (s) return s;
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaFreeAsync(dbuf, ctx->stream));
    return YAO_OK;
}

template <typename V>
static int run_program_t(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k) {
    V* st = (V*)r->d;
    if (mode == YAO_MODE_PLAIN) {
        for (const LGate& g : prog) {
            int s = launch_gate(ctx, st, r->precision, r->nbits, g);
            if (s) return s;
        }
        return YAO_OK;
    }
    // tile size: 2^12 complex128 (64 KiB) or 2^13 complex64 (64 KiB) per CTA
    // tile: 2^tbits amplitudes per CTA (shared memory = 2^tbits * sizeof(V));
    // YAO_TILE_BITS overrides the default for tuning runs
    int tbits = sizeof(V) == 16 ? 12 : 13;
    if (const char* e = getenv("YAO_TILE_BITS")) {
        int v = atoi(e);
        if (v >= 6 && v <= (sizeof(V) == 16 ? 12 : 13)) tbits = v;
    }
    std::vector<LGate> work;
    bool exact = (mode == YAO_MODE_TILED) && sizeof(V) == 16;
    if (mode == YAO_MODE_FUSED) {
        int kk = k > 0 ? std::min(k, kMaxTargets) : 5;
        fuse_blocks(prog, r->nbits, kk, work);
    } else {
        work = prog;
    }
    std::vector<PassPlan> passes;
    plan_passes(work, r->nbits, tbits, passes);
    // register bits: 3 (8 amplitudes per thread) unless YAO_REG_BITS says
    // otherwise, more only when the tile would need more than kTileThreads
    // threads
    int rb_pref = 3;
    if (const char* e = getenv("YAO_REG_BITS")) {
        int v = atoi(e);
        if (v >= 1 && v <= 4) rb_pref = v;
    }
    for (PassPlan& pp : passes)
        if (!pp.single) {
            int tb = (int)pp.hdr.tbits;
            int rb = std::max(tb - 9, std::min(rb_pref, tb));
            plan_segments(pp, std::min(rb, max_reg_bits<V>()));
        }
    for (const PassPlan& pp : passes) {
        int s;
        if (pp.single)
            s = launch_gate(ctx, st, r->precision, r->nbits, pp.gate);
        else if (exact)
            s = run_pass<V, true>(ctx, st, r->nbits, pp);
        else
            s = run_pass<V, false>(ctx, st, r->nbits, pp);
        if (s) return s;
    }
    return YAO_OK;
}

int launch_program(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k) {
    if (r->precision == YAO_C128) return run_program_t<double2>(ctx, r, prog, mode, k);
    return run_program_t<float2>(ctx, r, prog, mode, k);
}

// ------------------------------------------------------------ batch host

template <typename V>
static int batch_t(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                   int32_t mode, int32_t k) {
    typedef typename CoefT<V>::C C;
    const int tbits_cap = 12, rb = 3;
    const bool exact = mode == YAO_MODE_TILED && sizeof(V) == 16;
    // plan every circuit
    std::vector<std::vector<PassPlan>> plans(progs.size());
    size_t maxpasses = 0;
    for (size_t c = 0; c < progs.size(); c++) {
        if (regs[c]->nbits < 3) return fail(YAO_ERR_UNSUPPORTED, "batched circuits need at least 3 qubits");
        std::vector<LGate> work;
        if (mode == YAO_MODE_FUSED)
            fuse_blocks(*progs[c], regs[c]->nbits, k > 0 ? std::min(k, kMaxTargets) : 2, work);
        else
            work = *progs[c];
        plan_passes(work, regs[c]->nbits, tbits_cap, plans[c]);
        for (PassPlan& pp : plans[c]) {
            if (pp.single) return fail(YAO_ERR_UNSUPPORTED, "a gate of the batch does not fit a tile");
            plan_segments(pp, rb);
        }
        maxpasses = std::max(maxpasses, plans[c].size());
    }
    // entries level-major, ops / segments / coefficients concatenated
    std::vector<BatchEntry> entries;
    std::vector<TOp> ops;
    std::vector<TSeg> segs;
    std::vector<C> coef;
    uint64_t njobs = 0;
    for (size_t level = 0; level < maxpasses; level++)
        for (size_t c = 0; c < progs.size(); c++) {
            if (level >= plans[c].size()) continue;
            const PassPlan& pp = plans[c][level];
            BatchEntry e;
            memset(&e, 0, sizeof(e));
            e.hdr = pp.hdr;
            e.state = (uint64_t)(uintptr_t)regs[c]->d;
            e.job_start = njobs;
            e.circuit = (uint32_t)c;
            e.pass = (uint32_t)level;
            e.ops_off = (int32_t)ops.size();
            e.segs_off = (int32_t)segs.size();
            e.coef_off = (int32_t)coef.size();
            ops.insert(ops.end(), pp.ops.begin(), pp.ops.end());
            segs.insert(segs.end(), pp.segs.begin(), pp.segs.end());
            for (const Cx& x : pp.coef) {
                C cc;
                if (sizeof(V) == 16) {
                    *(double2*)&cc = make_double2(x.re, x.im);
                } else {
                    float hr = (float)x.re, hi = (float)x.im;
                    *(float4*)&cc = make_float4(hr, hi, (float)(x.re - (double)hr), (float)(x.im - (double)hi));
                }
                coef.push_back(cc);
            }
            entries.push_back(e);
            njobs += pp.hdr.ntiles;
        }
    if (njobs == 0) return YAO_OK;
    if (coef.empty()) coef.resize(1);
    if (ops.empty()) ops.resize(1);
    if (segs.empty()) segs.resize(1);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t b_ent = al(entries.size() * sizeof(BatchEntry)), b_ops = al(ops.size() * sizeof(TOp)),
                 b_seg = al(segs.size() * sizeof(TSeg)), b_coef = al(coef.size() * sizeof(C)),
                 b_ctr = al(sizeof(unsigned long long) + sizeof(int) + progs.size() * sizeof(unsigned int));
    char* buf = nullptr;
    YAO_CUDA(cudaMallocAsync((void**)&buf, b_ent + b_ops + b_seg + b_coef + b_ctr, ctx->stream));
    char* p = buf;
    BatchEntry* d_ent = (BatchEntry*)p;
    p += b_ent;
    TOp* d_ops = (TOp*)p;
    p += b_ops;
    TSeg* d_seg = (TSeg*)p;
    p += b_seg;
    C* d_coef = (C*)p;
    p += b_coef;
    unsigned long long* d_next = (unsigned long long*)p;
    int* d_err = (int*)(p + sizeof(unsigned long long));
    unsigned int* d_done = (unsigned int*)(p + sizeof(unsigned long long) + sizeof(int));
    YAO_CUDA(cudaMemcpyAsync(d_ent, entries.data(), entries.size() * sizeof(BatchEntry), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(d_ops, ops.data(), ops.size() * sizeof(TOp), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(d_seg, segs.data(), segs.size() * sizeof(TSeg), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(d_coef, coef.data(), coef.size() * sizeof(C), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    // every entry's description is staged in shared memory when the largest fits
    size_t max_stg = 0;
    std::vector<int32_t> ncoefs(entries.size());
    {
        // coefficient counts per entry (entries are laid out in order)
        for (size_t i = 0; i < entries.size(); i++) {
            int32_t end = (i + 1 < entries.size()) ? entries[i + 1].coef_off : (int32_t)coef.size();
            ncoefs[i] = end - entries[i].coef_off;
            max_stg = std::max(max_stg, staged_bytes(entries[i].hdr.nops, entries[i].hdr.nsegs, ncoefs[i], sizeof(C)));
        }
        const int st = max_stg <= kMaxStagedBytes ? 1 : 0;
        for (size_t i = 0; i < entries.size(); i++) {
            entries[i].hdr.ncoef = ncoefs[i];
            entries[i].hdr.staged = st;
        }
        YAO_CUDA(cudaMemcpyAsync(d_ent, entries.data(), entries.size() * sizeof(BatchEntry), cudaMemcpyHostToDevice,
                                 ctx->stream));
        YAO_CUDA(cudaStreamSynchronize(ctx->stream));
        if (!st) max_stg = 0;
    }
    const size_t smem = ((size_t)1 << tbits_cap) * sizeof(V) + max_stg;
    auto kern = exact ? k_batch_tiles<V, true, 3> : k_batch_tiles<V, false, 3>;
    YAO_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    YAO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileThreads, smem));
    const unsigned grid = (unsigned)std::max(1, per_sm) * (unsigned)ctx->num_sms;
    // capture: reset the queue and counters, run the persistent kernel
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    YAO_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(d_next, 0, b_ctr, ctx->stream);
    kern<<<grid, kTileThreads, smem, ctx->stream>>>(d_ent, (int)entries.size(), njobs, d_next, d_done, d_err, d_ops,
                                                    d_seg, d_coef);
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    if (ce != cudaSuccess) return cuda_fail(ce, "capture of the batch launch");
    YAO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    {
        double bytes = 0;
        for (const BatchEntry& e : entries) bytes += (double)e.hdr.ntiles * (double)(1u << e.hdr.tbits) * 2.0 * sizeof(V);
        ProfScope prof(ctx, exact ? "batch_tiles_exact" : "batch_tiles_fused", bytes);
        YAO_CUDA(cudaGraphLaunch(exec, ctx->stream));
    }
    ctx->launches++;
    int herr = 0;
    YAO_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    YAO_CUDA(cudaFreeAsync(buf, ctx->stream));
    if (herr) return fail(YAO_ERR_TIMEOUT, "batched launch: a job waited too long for its circuit's previous pass");
    return YAO_OK;
}

int launch_batch(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                 int32_t mode, int32_t k) {
    if (regs.empty()) return YAO_OK;
    if (regs[0]->precision == YAO_C128) return batch_t<double2>(ctx, progs, regs, mode, k);
    return batch_t<float2>(ctx, progs, regs, mode, k);
}

}  // namespace yao
