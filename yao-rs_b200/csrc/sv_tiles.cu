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
    int32_t pad;
    int8_t tb[16];
    uint64_t ntiles;
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
    int32_t pad;
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
constexpr int kMaxItems = 16;  // outputs per thread in a dense k >= 3 op (tile <= 8192)

template <typename V, bool EXACT>
__global__ void __launch_bounds__(kTileThreads) k_tile_pass(V* __restrict__ st, const TileHdr hdr,
                                                            const TOp* __restrict__ ops,
                                                            const typename CoefT<V>::C* __restrict__ coef) {
    typedef typename CoefT<V>::C C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* s = (V*)smem_raw;
    const uint32_t T = 1u << hdr.tbits;
    const uint32_t lowmask = (1u << hdr.m) - 1;
    const int nt = blockDim.x;
    for (uint64_t t = blockIdx.x; t < hdr.ntiles; t += gridDim.x) {
        const uint64_t base = insert_zeros(t, hdr.tb, hdr.tbits);
        // ---- load
        for (uint32_t l = threadIdx.x; l < T; l += nt) {
            uint64_t gi = base | (l & lowmask);
            for (int j = hdr.m; j < hdr.tbits; j++) gi |= (uint64_t)((l >> j) & 1) << hdr.tb[j];
            s[l] = st[gi];
        }
        __syncthreads();
        // ---- ops
        for (int oi = 0; oi < hdr.nops; oi++) {
            const TOp& op = ops[oi];
            if ((base & op.gcmask) != op.gcval) continue;  // uniform over the tile
            const C* m = coef + op.moff;
            if (op.cls == GC_X) {
                const int tq = op.tl[0];
                for (uint32_t p = threadIdx.x; p < T / 2; p += nt) {
                    uint32_t i0 = ins0(p, tq);
                    if ((i0 & op.lcmask) != op.lcval) continue;
                    uint32_t i1 = i0 | (1u << tq);
                    V a = s[i0];
                    s[i0] = s[i1];
                    s[i1] = a;
                }
            } else if (op.cls == GC_SWAP) {
                const int t0 = op.tl[0], t1 = op.tl[1];
                for (uint32_t q = threadIdx.x; q < T / 4; q += nt) {
                    uint32_t b = ins0(ins0(q, min(t0, t1)), max(t0, t1));
                    if ((b & op.lcmask) != op.lcval) continue;
                    uint32_t i1 = b | (1u << t0), i2 = b | (1u << t1);
                    V a = s[i1];
                    s[i1] = s[i2];
                    s[i2] = a;
                }
            } else if (op.cls == GC_DIAG) {
                for (uint32_t l = threadIdx.x; l < T; l += nt) {
                    if ((l & op.lcmask) != op.lcval) continue;
                    uint32_t dl = 0;
                    if (op.all_local) {
                        for (int i = 0; i < op.k; i++) dl |= ((l >> op.tl[i]) & 1) << i;
                    } else {
                        uint64_t gi = base | (l & lowmask);
                        for (int j = hdr.m; j < hdr.tbits; j++) gi |= (uint64_t)((l >> j) & 1) << hdr.tb[j];
                        for (int i = 0; i < op.k; i++) dl |= (uint32_t)((gi >> op.tg[i]) & 1) << i;
                    }
                    if (!((op.active >> dl) & 1)) continue;
                    s[l] = cmulassign_c<EXACT>(s[l], m[dl]);
                }
            } else if (op.k == 1) {
                const int tq = op.tl[0];
                const C a = m[0], b = m[1], c = m[2], d = m[3];
                for (uint32_t p = threadIdx.x; p < T / 2; p += nt) {
                    uint32_t i0 = ins0(p, tq);
                    if ((i0 & op.lcmask) != op.lcval) continue;
                    uint32_t i1 = i0 | (1u << tq);
                    V w = s[i0], x = s[i1];
                    s[i0] = cfma_c<EXACT>(cmul_c<EXACT>(a, w), b, x);
                    s[i1] = cfma_c<EXACT>(cmul_c<EXACT>(c, w), d, x);
                }
            } else if (op.k == 2) {
                const int t0 = op.tl[0], t1 = op.tl[1];  // t0 < t1 (sorted by the lowering)
                for (uint32_t q = threadIdx.x; q < T / 4; q += nt) {
                    uint32_t b = ins0(ins0(q, t0), t1);
                    if ((b & op.lcmask) != op.lcval) continue;
                    uint32_t idx[4] = {b, b | (1u << t0), b | (1u << t1), b | (1u << t0) | (1u << t1)};
                    V old[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) old[j] = s[idx[j]];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        V acc = VecT<V>::zero();
#pragma unroll
                        for (int j = 0; j < 4; j++) acc = cfma_c<EXACT>(acc, m[i * 4 + j], old[j]);
                        s[idx[i]] = acc;
                    }
                }
            } else {
                // dense k >= 3: item it = (group, row); outputs kept in registers
                // until every thread has read its inputs.
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
                for (uint32_t it = threadIdx.x; it < T; it += nt) {
                    uint32_t g = it >> k, row = it & (nl - 1);
                    uint32_t b = g;
                    for (int i = 0; i < k; i++) b = ins0(b, sorted[i]);
                    bool act = (b & op.lcmask) == op.lcval;
                    uint32_t ro = 0;
                    for (int i = 0; i < k; i++) ro |= ((row >> i) & 1) << op.tl[i];
                    V acc = VecT<V>::zero();
                    if (act) {
                        const C* mr = m + (size_t)row * nl;
                        for (int c = 0; c < nl; c++) {
                            uint32_t co = 0;
                            for (int i = 0; i < k; i++) co |= ((c >> i) & 1) << op.tl[i];
                            acc = cfma_c<EXACT>(acc, mr[c], s[b | co]);
                        }
                    }
                    outv[cnt] = acc;
                    outi[cnt] = act ? (b | ro) : 0xffffffffu;
                    cnt++;
                }
                __syncthreads();
                for (int i = 0; i < cnt; i++)
                    if (outi[i] != 0xffffffffu) s[outi[i]] = outv[i];
            }
            __syncthreads();
        }
        // ---- store
        for (uint32_t l = threadIdx.x; l < T; l += nt) {
            uint64_t gi = base | (l & lowmask);
            for (int j = hdr.m; j < hdr.tbits; j++) gi |= (uint64_t)((l >> j) & 1) << hdr.tb[j];
            st[gi] = s[l];
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
    std::vector<Cx> coef;
};

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
    size_t ob = pp.ops.size() * sizeof(TOp), cb = hc.size() * sizeof(C);
    size_t cb_off = (ob + 255) / 256 * 256;
    void* dbuf = nullptr;
    YAO_CUDA(cudaMallocAsync(&dbuf, cb_off + cb, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dbuf, pp.ops.data(), ob, cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync((char*)dbuf + cb_off, hc.data(), cb, cudaMemcpyHostToDevice, ctx->stream));
    size_t smem = ((size_t)1 << pp.hdr.tbits) * sizeof(V);
    static bool attr_set[2][2] = {{false, false}, {false, false}};
    bool& a = attr_set[sizeof(V) == 16][EXACT];
    if (!a) {
        YAO_CUDA(cudaFuncSetAttribute(k_tile_pass<V, EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        a = true;
    }
    unsigned grid = (unsigned)std::min<uint64_t>(pp.hdr.ntiles, (uint64_t)ctx->num_sms * 4);
    {
        ProfScope prof(ctx, EXACT ? "tile_pass_exact" : "tile_pass_fused",
                       (double)pp.hdr.ntiles * (double)((uint64_t)1 << pp.hdr.tbits) * 2.0 * sizeof(V));
        k_tile_pass<V, EXACT><<<grid, kTileThreads, smem, ctx->stream>>>(st, pp.hdr, (const TOp*)dbuf,
                                                                          (const C*)((char*)dbuf + cb_off));
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
    int tbits = sizeof(V) == 16 ? 12 : 13;
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

}  // namespace yao
