// sv_gates.cu — gate application kernels for state vectors.
//
// PLAIN form: one kernel launch per gate.  The amplitudes a gate touches are
// enumerated as groups: a group index g gets a zero bit inserted at every
// locked position (targets and controls, ascending), the control values are
// OR-ed in, and the 2^k group members sit at base + off[l], where local index
// bit i selects target bit tb[i].  This enumerates exactly the index set of
// yao-rs's itercontrol / for_each_single_control_base
// (bitbasis/src/iterate_control.rs:82-159, src/instruct_qubit.rs:38-79), and
// each member is updated with the same arithmetic as the matching instruct_*
// function, so the double-precision result equals the CPU path's.
//
// Consecutive threads take consecutive groups: when the lowest locked bit is
// >= 4, each warp reads and writes contiguous 512-byte runs (double2).
#include <algorithm>
#include <vector>

#include "device_common.cuh"

namespace yao {

struct DOp {
    int32_t cls;
    int32_t k;
    int32_t nlocked;
    int32_t pad;
    uint64_t cval;
    uint64_t active;  // DIAG: local indices whose entry is not exactly 1
    int8_t locked[64];
    uint64_t off[4];
    double2 m[16];
};

template <typename V>
struct DOpT {
    int32_t cls, k, nlocked, pad;
    uint64_t cval, active;
    int8_t locked[64];
    uint64_t off[4];
    V m[16];
};

static void make_locked(const LGate& g, int8_t* locked, int32_t& n) {
    std::vector<int> pos;
    for (int i = 0; i < g.k; i++) pos.push_back(g.tb[i]);
    for (int i = 0; i < g.nc; i++) pos.push_back(g.cb[i]);
    std::sort(pos.begin(), pos.end());
    n = (int32_t)pos.size();
    for (size_t i = 0; i < pos.size(); i++) locked[i] = (int8_t)pos[i];
}

static bool is_one(const Cx& c) { return c.re == 1.0 && c.im == 0.0; }

// ------------------------------------------------------------ k <= 2 kernel
template <typename V, int CLS, int K, int U>
__global__ void __launch_bounds__(256) k_gate_small(V* __restrict__ st, uint64_t ngroups, const DOpT<V> op) {
    constexpr int NL = 1 << K;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g0 < ngroups; g0 += stride * U) {
        V v[U][NL];
        uint64_t base[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            uint64_t g = g0 + (uint64_t)u * stride;
            ok[u] = g < ngroups;
            base[u] = insert_zeros(g, op.locked, op.nlocked) | op.cval;
            if (ok[u]) {
                if (CLS == GC_SWAP) {
                    v[u][1] = st[base[u] + op.off[1]];
                    v[u][2] = st[base[u] + op.off[2]];
                } else if (CLS == GC_DIAG) {
#pragma unroll
                    for (int l = 0; l < NL; l++)
                        if ((op.active >> l) & 1) v[u][l] = st[base[u] + op.off[l]];
                } else {
#pragma unroll
                    for (int l = 0; l < NL; l++) v[u][l] = st[base[u] + op.off[l]];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (!ok[u]) continue;
            if (CLS == GC_X) {
                // instruct_x: swap the pair
                st[base[u] + op.off[0]] = v[u][1];
                st[base[u] + op.off[1]] = v[u][0];
            } else if (CLS == GC_SWAP) {
                st[base[u] + op.off[1]] = v[u][2];
                st[base[u] + op.off[2]] = v[u][1];
            } else if (CLS == GC_DIAG) {
#pragma unroll
                for (int l = 0; l < NL; l++)
                    if ((op.active >> l) & 1) st[base[u] + op.off[l]] = cmulassign_x(v[u][l], op.m[l]);
            } else if (K == 1) {
                // u1rows: a*w + b*v, c*w + d*v
                V w = v[u][0], x = v[u][1];
                st[base[u] + op.off[0]] = cadd_x(cmul_x(op.m[0], w), cmul_x(op.m[1], x));
                st[base[u] + op.off[1]] = cadd_x(cmul_x(op.m[2], w), cmul_x(op.m[3], x));
            } else {
                // unrows: acc = 0; acc += g[i][j] * old[j]
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    V acc = VecT<V>::zero();
#pragma unroll
                    for (int j = 0; j < 4; j++) acc = cadd_x(acc, cmul_x(op.m[i * 4 + j], v[u][j]));
                    st[base[u] + op.off[i]] = acc;
                }
            }
        }
    }
}

// ------------------------------------------------------ k >= 3 kernels
// DIAG with k >= 3: one thread per group, members loaded one at a time.
template <typename V>
__global__ void __launch_bounds__(256) k_gate_diag_n(V* __restrict__ st, uint64_t ngroups, int k,
                                                     const int32_t* __restrict__ tb, const int8_t* __restrict__ locked,
                                                     int nlocked, uint64_t cval, uint64_t active,
                                                     const V* __restrict__ d) {
    __shared__ int8_t slock[64];
    __shared__ int32_t stb[kMaxTargets];
    if (threadIdx.x < nlocked) slock[threadIdx.x] = locked[threadIdx.x];
    if (threadIdx.x < k) stb[threadIdx.x] = tb[threadIdx.x];
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const int nl = 1 << k;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += stride) {
        uint64_t base = insert_zeros(g, slock, nlocked) | cval;
        for (int l = 0; l < nl; l++) {
            if (!((active >> l) & 1)) continue;  // entry exactly 1: value unchanged
            V dl = d[l];
            uint64_t off = 0;
            for (int i = 0; i < k; i++) off |= (uint64_t)((l >> i) & 1) << stb[i];
            st[base + off] = cmulassign_x(st[base + off], dl);
        }
    }
}

// DENSE with k >= 3 (instruct_nq): a block stages 256 / 2^k groups in shared
// memory, then each thread produces one output row:
// temp[row] = 0; temp[row] += g[row][col] * x[col] (col ascending).
template <typename V>
__global__ void __launch_bounds__(256) k_gate_dense_n(V* __restrict__ st, uint64_t ngroups, int k,
                                                      const int32_t* __restrict__ tb,
                                                      const int8_t* __restrict__ locked, int nlocked, uint64_t cval,
                                                      const V* __restrict__ m) {
    __shared__ V sx[256];
    __shared__ int8_t slock[64];
    __shared__ int32_t stb[kMaxTargets];
    if (threadIdx.x < nlocked) slock[threadIdx.x] = locked[threadIdx.x];
    if (threadIdx.x < k) stb[threadIdx.x] = tb[threadIdx.x];
    __syncthreads();
    const int nl = 1 << k;
    const int gpb = 256 >> k;  // groups per block iteration (k <= 6 -> >= 4)
    const int lg = threadIdx.x >> k, row = threadIdx.x & (nl - 1);
    for (uint64_t gb = (uint64_t)blockIdx.x * gpb; gb < ngroups; gb += (uint64_t)gridDim.x * gpb) {
        uint64_t g = gb + lg;
        bool ok = g < ngroups && lg < gpb;
        uint64_t base = 0, off = 0;
        if (ok) {
            base = insert_zeros(g, slock, nlocked) | cval;
            for (int i = 0; i < k; i++) off |= (uint64_t)((row >> i) & 1) << stb[i];
            sx[threadIdx.x] = st[base + off];
        }
        __syncthreads();
        if (ok) {
            V acc = VecT<V>::zero();
            const V* xr = sx + lg * nl;
            const V* mr = m + (size_t)row * nl;
            for (int c = 0; c < nl; c++) acc = cadd_x(acc, cmul_x(mr[c], xr[c]));
            st[base + off] = acc;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- dispatch

template <typename V>
static void to_v(const Cx& c, V& out);
template <>
void to_v<double2>(const Cx& c, double2& out) {
    out = make_double2(c.re, c.im);
}
template <>
void to_v<float2>(const Cx& c, float2& out) {
    out = make_float2((float)c.re, (float)c.im);
}

// Device copy of the coefficients of a k >= 3 gate: cached per LGate
// pointer+content would need invalidation; the k >= 3 path is rare, so the
// coefficients are staged through a small per-call buffer.
template <typename V>
static int launch_gate_n(Ctx* ctx, V* st, uint32_t nbits, const LGate& g, uint64_t ngroups, int8_t* locked,
                         int32_t nlocked) {
    size_t nm = g.m.size();
    size_t bytes = nm * sizeof(V) + 64 + sizeof(int32_t) * kMaxTargets;
    std::vector<uint8_t> host(bytes);
    V* hm = (V*)host.data();
    for (size_t i = 0; i < nm; i++) to_v<V>(g.m[i], hm[i]);
    memcpy(host.data() + nm * sizeof(V), locked, 64);
    memcpy(host.data() + nm * sizeof(V) + 64, g.tb, sizeof(int32_t) * kMaxTargets);
    void* dbuf = nullptr;
    YAO_CUDA(cudaMallocAsync(&dbuf, bytes, ctx->stream));
    YAO_CUDA(cudaMemcpyAsync(dbuf, host.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
    // the pageable source is consumed before cudaMemcpyAsync returns
    const V* dm = (const V*)dbuf;
    const int8_t* dl = (const int8_t*)((uint8_t*)dbuf + nm * sizeof(V));
    const int32_t* dtb = (const int32_t*)((uint8_t*)dbuf + nm * sizeof(V) + 64);
    uint64_t cval = g.cval();
    ProfScope prof(ctx, g.cls == GC_DIAG ? "gate_diag_n" : "gate_dense_n",
                   (double)ngroups * (1 << g.k) * 2.0 * sizeof(V));
    if (g.cls == GC_DIAG) {
        unsigned grid = grid_for(ngroups, 256, ctx->num_sms);
        uint64_t active = 0;
        for (size_t l = 0; l < g.m.size(); l++)
            if (!is_one(g.m[l])) active |= (uint64_t)1 << l;
        k_gate_diag_n<V><<<grid, 256, 0, ctx->stream>>>(st, ngroups, g.k, dtb, dl, nlocked, cval, active, dm);
    } else {
        int gpb = 256 >> g.k;
        unsigned grid = grid_for((ngroups + gpb - 1) / gpb, 1, ctx->num_sms, 16);
        k_gate_dense_n<V><<<grid, 256, 0, ctx->stream>>>(st, ngroups, g.k, dtb, dl, nlocked, cval, dm);
    }
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    YAO_CUDA(cudaFreeAsync(dbuf, ctx->stream));
    return YAO_OK;
}

// nsets > 1: the gate acts on nsets registers of nbits qubits stored back to
// back; the register index sits above every locked bit, so the groups of all
// registers are enumerated as one range.
template <typename V, int U>
static int launch_small(const LGate& g, unsigned grid, cudaStream_t s, V* st, uint64_t ngroups, const DOpT<V>& op) {
    if (g.cls == GC_X)
        k_gate_small<V, GC_X, 1, U><<<grid, 256, 0, s>>>(st, ngroups, op);
    else if (g.cls == GC_SWAP)
        k_gate_small<V, GC_SWAP, 2, U><<<grid, 256, 0, s>>>(st, ngroups, op);
    else if (g.cls == GC_DIAG && g.k == 1)
        k_gate_small<V, GC_DIAG, 1, U><<<grid, 256, 0, s>>>(st, ngroups, op);
    else if (g.cls == GC_DIAG && g.k == 2)
        k_gate_small<V, GC_DIAG, 2, U><<<grid, 256, 0, s>>>(st, ngroups, op);
    else if (g.cls == GC_DENSE && g.k == 1)
        k_gate_small<V, GC_DENSE, 1, U><<<grid, 256, 0, s>>>(st, ngroups, op);
    else if (g.cls == GC_DENSE && g.k == 2)
        k_gate_small<V, GC_DENSE, 2, U><<<grid, 256, 0, s>>>(st, ngroups, op);
    else
        return fail(YAO_ERR_INVALID_ARGUMENT, "unsupported gate class");
    return YAO_OK;
}

template <typename V>
static int launch_gate_t(Ctx* ctx, V* st, uint32_t nbits, const LGate& g, uint64_t nsets = 1) {
    DOpT<V> op;
    memset(&op, 0, sizeof(op));
    op.cls = g.cls;
    op.k = g.k;
    make_locked(g, op.locked, op.nlocked);
    if (op.nlocked > (int)nbits) return fail(YAO_ERR_INVALID_ARGUMENT, "gate locks more bits than the register has");
    op.cval = g.cval();
    uint64_t ngroups = nsets << (nbits - op.nlocked);
    if (g.k >= 3 && (g.cls == GC_DIAG || g.cls == GC_DENSE))
        return launch_gate_n<V>(ctx, st, nbits, g, ngroups, op.locked, op.nlocked);
    int nl = 1 << g.k;
    for (int l = 0; l < nl && l < 4; l++) {
        uint64_t off = 0;
        for (int i = 0; i < g.k; i++) off |= (uint64_t)((l >> i) & 1) << g.tb[i];
        op.off[l] = off;
    }
    for (size_t i = 0; i < g.m.size() && i < 16; i++) to_v<V>(g.m[i], op.m[i]);
    if (g.cls == GC_DIAG) {
        op.active = 0;
        for (int l = 0; l < nl; l++)
            if (!is_one(g.m[l])) op.active |= (uint64_t)1 << l;
        if (op.active == 0) return YAO_OK;  // identity
    }
    // groups per thread per sweep (loads of all of them in flight together)
    // and CTAs per SM of the grid; YAO_PLAIN_GROUPS / YAO_PLAIN_CTAS override
    // the defaults for tuning runs
    static const int U = [] {
        const char* e = getenv("YAO_PLAIN_GROUPS");
        const int v = e ? atoi(e) : 2;
        return (v == 1 || v == 2 || v == 4) ? v : 2;
    }();
    static const int per_sm = [] {
        const char* e = getenv("YAO_PLAIN_CTAS");
        const int v = e ? atoi(e) : 48;
        return (v >= 1 && v <= 64) ? v : 48;
    }();
    unsigned grid = grid_for((ngroups + U - 1) / U, 256, ctx->num_sms, per_sm);
    cudaStream_t s = ctx->stream;
    // algorithmic traffic: every touched amplitude is read and written once
    int touched = g.cls == GC_DIAG ? __builtin_popcountll(op.active) : (g.cls == GC_SWAP ? 2 : nl);
    static const char* names[4][3] = {{"gate_x", "gate_x", "gate_x"},
                                      {"gate_swap", "gate_swap", "gate_swap"},
                                      {"gate_diag1", "gate_diag1", "gate_diag2"},
                                      {"gate_dense1", "gate_dense1", "gate_dense2"}};
    ProfScope prof(ctx, names[g.cls][g.k], (double)ngroups * touched * 2.0 * sizeof(V));
    int st_ = 0;
    if (U == 1)
        st_ = launch_small<V, 1>(g, grid, s, st, ngroups, op);
    else if (U == 4)
        st_ = launch_small<V, 4>(g, grid, s, st, ngroups, op);
    else
        st_ = launch_small<V, 2>(g, grid, s, st, ngroups, op);
    if (st_) return st_;
    ctx->launches++;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

int launch_gate(Ctx* ctx, void* state, int32_t precision, uint32_t nbits, const LGate& g) {
    if (precision == YAO_C128) return launch_gate_t<double2>(ctx, (double2*)state, nbits, g);
    return launch_gate_t<float2>(ctx, (float2*)state, nbits, g);
}

int launch_gate_sets(Ctx* ctx, void* state, uint32_t nbits, const LGate& g, uint64_t nsets) {
    return launch_gate_t<double2>(ctx, (double2*)state, nbits, g, nsets);
}

}  // namespace yao
