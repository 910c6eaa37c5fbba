// capi.cpp — the extern "C" entry points of include/yao_gpu.h.
//
// Host-side responsibilities: argument validation with yao-rs's error
// semantics (a panic or Err there is a negative status and a message here),
// the conversion of the circuit wire format into lowered gates, and the
// sequencing of device launches.  All device work runs on the context's
// stream; functions that return host values synchronise it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <set>
#include <sstream>

#include "yao_internal.h"

namespace yao {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
void clear_error() { g_err.clear(); }
int fail(int st, const std::string& m) {
    g_err = m;
    return st;
}
int cuda_fail(cudaError_t e, const char* what) {
    std::string m = std::string("CUDA error: ") + cudaGetErrorString(e) + " (" + what + ")";
    g_err = m;
    return e == cudaErrorMemoryAllocation ? YAO_ERR_OUT_OF_MEMORY : YAO_ERR_CUDA;
}

// ----------------------------------------------------------------- context
// cudaMalloc; when it fails, the freed memory that the device's default pool
// keeps is released (after this context's queued frees) and it is tried once
// more.
static cudaError_t alloc_device(Ctx* ctx, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaErrorMemoryAllocation) return e;
    cudaGetLastError();
    cudaMemPool_t pool;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess ||
        cudaDeviceGetDefaultMemPool(&pool, ctx->device) != cudaSuccess || cudaMemPoolTrimTo(pool, 0) != cudaSuccess)
        return e;
    return cudaMalloc(p, bytes);
}

int Ctx::ensure_scratch(size_t bytes) {
    if (bytes <= scratch_bytes) return 0;
    size_t nb = std::max<size_t>(bytes, 1 << 20);
    if (scratch) {
        cudaStreamSynchronize(stream);
        cudaFree(scratch);
        scratch = nullptr;
        scratch_bytes = 0;
    }
    if (alloc_device(this, &scratch, nb) != cudaSuccess) {
        cudaGetLastError();
        scratch = nullptr;
        fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate reduction scratch");
        return -1;
    }
    scratch_bytes = nb;
    return 0;
}

int Ctx::ensure_host_pinned(size_t bytes) {
    if (bytes <= host_pinned_bytes) return 0;
    size_t nb = std::max<size_t>(bytes, 4096);
    if (host_pinned) cudaFreeHost(host_pinned);
    if (cudaMallocHost(&host_pinned, nb) != cudaSuccess) {
        host_pinned = nullptr;
        host_pinned_bytes = 0;
        fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate pinned host memory");
        return -1;
    }
    host_pinned_bytes = nb;
    return 0;
}

cudaEvent_t Ctx::take_event() {
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void Ctx::prof_begin(const char* name, double bytes) {
    ProfRec r;
    r.name = name;
    r.bytes = bytes;
    r.a = take_event();
    r.b = take_event();
    cudaEventRecord(r.a, stream);
    recs.push_back(r);
}

void Ctx::prof_end() {
    if (!recs.empty()) cudaEventRecord(recs.back().b, stream);
}

static int use_device(const Ctx* c) {
    YAO_CUDA(cudaSetDevice(c->device));
    return YAO_OK;
}

// ---------------------------------------------------------- wire format

static int read_element(const yao_element& e, Element& out) {
    out.kind = e.kind;
    if (e.kind == YAO_ELEM_GATE) {
        GateElem& g = out.g;
        g.type = e.type;
        if (e.type < YAO_GATE_X || e.type > YAO_GATE_CUSTOM) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown gate type");
        g.targets.assign(e.targets, e.targets + e.ntargets);
        g.ctrls.assign(e.ctrl_locs, e.ctrl_locs + e.nctrl);
        if (e.ctrl_configs)
            g.cfgs.assign(e.ctrl_configs, e.ctrl_configs + e.nconfigs);
        else
            g.cfgs.assign(e.nctrl, 1);
        for (int i = 0; i < 4; i++) g.params[i] = e.params[i];
        if (e.type == YAO_GATE_CUSTOM) {
            if (!e.matrix || e.matrix_dim == 0) return fail(YAO_ERR_INVALID_ARGUMENT, "Custom gate needs a matrix");
            g.custom_dim = e.matrix_dim;
            const Cx* m = (const Cx*)e.matrix;
            g.custom.assign(m, m + (size_t)e.matrix_dim * e.matrix_dim);
            g.custom_diag = e.is_diagonal != 0;
        }
    } else if (e.kind == YAO_ELEM_CHANNEL) {
        ChannelElem& c = out.ch;
        c.type = e.type;
        if (e.type < YAO_NOISE_BIT_FLIP || e.type > YAO_NOISE_CUSTOM)
            return fail(YAO_ERR_INVALID_ARGUMENT, "unknown noise channel type");
        c.locs.assign(e.targets, e.targets + e.ntargets);
        for (int i = 0; i < 4; i++) c.params[i] = e.params[i];
        c.depol_n = e.depol_n;
        if (e.type == YAO_NOISE_COHERENT || e.type == YAO_NOISE_CUSTOM) {
            if (!e.matrix || e.matrix_dim == 0) return fail(YAO_ERR_INVALID_ARGUMENT, "channel needs matrices");
            c.dim = e.matrix_dim;
            c.nkraus = e.type == YAO_NOISE_CUSTOM ? e.nkraus : 1;
            const Cx* m = (const Cx*)e.matrix;
            c.mats.assign(m, m + (size_t)c.dim * c.dim * c.nkraus);
        }
    } else if (e.kind == YAO_ELEM_ANNOTATION) {
        if (e.ntargets < 1 || !e.targets) return fail(YAO_ERR_INVALID_ARGUMENT, "annotation needs a location");
        out.annot_loc = e.targets[0];
    } else {
        return fail(YAO_ERR_INVALID_ARGUMENT, "unknown element kind");
    }
    return YAO_OK;
}

static int ilog2_exact(uint32_t d) {
    int n = 0;
    uint32_t p = 1;
    while (p < d) p *= 2, n++;
    return p == d ? n : -1;
}

static uint32_t channel_num_qubits(const ChannelElem& c) {
    if (c.type == YAO_NOISE_DEPOLARIZING) return (uint32_t)c.depol_n;
    if (c.type == YAO_NOISE_CUSTOM || c.type == YAO_NOISE_COHERENT) {
        int n = ilog2_exact(c.dim);
        return n < 0 ? 0xffffffffu : (uint32_t)n;
    }
    return 1;
}

static std::string locs_str(const std::vector<uint32_t>& v) {
    std::ostringstream o;
    o << "[";
    for (size_t i = 0; i < v.size(); i++) o << (i ? ", " : "") << v[i];
    o << "]";
    return o.str();
}

// Circuit::new validation (src/circuit.rs:150-272), same rule order.
static int validate(const std::vector<uint32_t>& dims, const std::vector<Element>& elems, int32_t* ce) {
    const uint32_t ns = (uint32_t)dims.size();
    auto err = [&](int kind, const std::string& m) {
        if (ce) *ce = kind;
        return fail(YAO_ERR_CIRCUIT, m);
    };
    for (const Element& el : elems) {
        if (el.kind == YAO_ELEM_GATE) {
            const GateElem& g = el.g;
            if (g.cfgs.size() != g.ctrls.size())
                return err(YAO_CE_CONTROL_CONFIG_LENGTH_MISMATCH, "control_configs length does not match control_locs length");
            for (uint32_t l : g.targets)
                if (l >= ns)
                    return err(YAO_CE_LOC_OUT_OF_RANGE, "location " + std::to_string(l) + " is out of range (num_sites = " + std::to_string(ns) + ")");
            for (uint32_t l : g.ctrls)
                if (l >= ns)
                    return err(YAO_CE_LOC_OUT_OF_RANGE, "location " + std::to_string(l) + " is out of range (num_sites = " + std::to_string(ns) + ")");
            std::vector<uint32_t> ov;
            for (uint32_t t : g.targets)
                if (std::find(g.ctrls.begin(), g.ctrls.end(), t) != g.ctrls.end() &&
                    std::find(ov.begin(), ov.end(), t) == ov.end())
                    ov.push_back(t);
            if (!ov.empty())
                return err(YAO_CE_OVERLAPPING_LOCS, "target_locs and control_locs overlap at locations: " + locs_str(ov));
            for (uint32_t l : g.ctrls)
                if (dims[l] != 2)
                    return err(YAO_CE_CONTROL_SITE_NOT_QUBIT, "control site at location " + std::to_string(l) + " has dimension " + std::to_string(dims[l]) + " (must be 2)");
            if (g.type != YAO_GATE_CUSTOM)
                for (uint32_t l : g.targets)
                    if (dims[l] != 2)
                        return err(YAO_CE_NAMED_GATE_TARGET_NOT_QUBIT, "named gate target site at location " + std::to_string(l) + " has dimension " + std::to_string(dims[l]) + " (must be 2)");
            uint64_t prod = 1;
            for (uint32_t l : g.targets) prod *= dims[l];
            uint32_t msize = g.type == YAO_GATE_CUSTOM ? g.custom_dim : (g.type == YAO_GATE_SWAP || g.type == YAO_GATE_ISWAP || g.type == YAO_GATE_FSIM ? 4 : 2);
            if (msize != prod)
                return err(YAO_CE_MATRIX_SIZE_MISMATCH, "gate matrix size " + std::to_string(msize) + " does not match product of target site dimensions " + std::to_string(prod));
        } else if (el.kind == YAO_ELEM_CHANNEL) {
            const ChannelElem& c = el.ch;
            for (uint32_t l : c.locs)
                if (l >= ns)
                    return err(YAO_CE_LOC_OUT_OF_RANGE, "location " + std::to_string(l) + " is out of range (num_sites = " + std::to_string(ns) + ")");
            uint32_t nq = channel_num_qubits(c);
            if (nq == 0xffffffffu) return fail(YAO_ERR_INVALID_ARGUMENT, "channel dimension is not a power of 2");
            if (c.locs.size() != nq)
                return err(YAO_CE_MATRIX_SIZE_MISMATCH, "gate matrix size " + std::to_string(c.locs.size()) + " does not match product of target site dimensions " + std::to_string(nq));
            for (uint32_t l : c.locs)
                if (dims[l] != 2)
                    return err(YAO_CE_NAMED_GATE_TARGET_NOT_QUBIT, "named gate target site at location " + std::to_string(l) + " has dimension " + std::to_string(dims[l]) + " (must be 2)");
            std::vector<uint32_t> seen, ov;
            for (uint32_t l : c.locs) {
                if (std::find(seen.begin(), seen.end(), l) != seen.end()) {
                    if (std::find(ov.begin(), ov.end(), l) == ov.end()) ov.push_back(l);
                } else {
                    seen.push_back(l);
                }
            }
            if (!ov.empty())
                return err(YAO_CE_OVERLAPPING_LOCS, "target_locs and control_locs overlap at locations: " + locs_str(ov));
        } else {
            if (el.annot_loc >= ns)
                return err(YAO_CE_LOC_OUT_OF_RANGE, "location " + std::to_string(el.annot_loc) + " is out of range (num_sites = " + std::to_string(ns) + ")");
        }
    }
    return YAO_OK;
}

// The lowered gate list of a circuit (pure-state path, apply.rs:123-147).
static const std::vector<LGate>& lowered(Circuit* c) {
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = c->lowered.find(c->nbits);
    if (it != c->lowered.end()) return it->second;
    std::vector<LGate> prog;
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_GATE) lower_gate(el.g, c->nbits, 0, false, prog);
    return c->lowered.emplace(c->nbits, std::move(prog)).first->second;
}

// The kernels take at most kMaxTargets targets per gate (a 64 x 64 matrix).
static int check_widths(const Circuit* c) {
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_GATE && el.g.targets.size() > (size_t)kMaxTargets)
            return fail(YAO_ERR_UNSUPPORTED, "gates on more than 6 target qubits are not supported");
    return YAO_OK;
}

static int check_apply(const Circuit* c, const Reg* r) {
    if (!c->qubit_only) return fail(YAO_ERR_QUBIT_ONLY, "ArrayReg only supports qubit-only circuits");
    if (c->nbits != r->nbits) return fail(YAO_ERR_NBITS_MISMATCH, "Register and circuit qubit count mismatch");
    return check_widths(c);
}

static int alloc_reg(Ctx* ctx, uint32_t nbits, int32_t prec, Reg** out) {
    if (nbits > (uint32_t)kMaxQubits) return fail(YAO_ERR_INVALID_ARGUMENT, "too many qubits");
    if (prec != YAO_C128 && prec != YAO_C64) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown precision");
    int s = use_device(ctx);
    if (s) return s;
    std::unique_ptr<yao_reg> r(new yao_reg());
    r->ctx = ctx;
    r->nbits = nbits;
    r->precision = prec;
    cudaError_t e = alloc_device(ctx, &r->d, r->bytes());
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate a " + std::to_string(nbits) + "-qubit register (" +
                                               std::to_string(r->bytes()) + " bytes)");
    }
    *out = r.release();
    return YAO_OK;
}

static int alloc_dm(Ctx* ctx, uint32_t nbits, DM** out) {
    if (2 * nbits > (uint32_t)kMaxQubits) return fail(YAO_ERR_INVALID_ARGUMENT, "too many qubits");
    int s = use_device(ctx);
    if (s) return s;
    std::unique_ptr<yao_dm> d(new yao_dm());
    d->ctx = ctx;
    d->nbits = nbits;
    if (alloc_device(ctx, &d->d, d->bytes()) != cudaSuccess) {
        cudaGetLastError();
        return fail(YAO_ERR_OUT_OF_MEMORY, "cannot allocate the density matrix");
    }
    *out = d.release();
    return YAO_OK;
}

static int check_measure_locs(uint32_t nbits, const uint32_t* locs, uint32_t n) {
    std::set<uint32_t> seen;
    for (uint32_t i = 0; i < n; i++) {
        if (locs[i] >= nbits)
            return fail(YAO_ERR_MEASURE_LOCS, "measurement location " + std::to_string(locs[i]) +
                                                  " is out of range for " + std::to_string(nbits) + " qubits");
        if (!seen.insert(locs[i]).second)
            return fail(YAO_ERR_MEASURE_LOCS, "duplicate measurement location " + std::to_string(locs[i]));
    }
    return YAO_OK;
}

static Cx cxmul(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

}  // namespace yao

using namespace yao;

#define CHECK_NULL(p)                                                                \
    do {                                                                             \
        if (!(p)) return fail(YAO_ERR_INVALID_ARGUMENT, "null argument: " #p);        \
    } while (0)

extern "C" {

const char* yao_last_error(void) { return g_err.c_str(); }
int yao_abi_version(void) { return YAO_GPU_ABI_VERSION; }

// ------------------------------------------------------------------ context
int yao_ctx_create(int device, yao_ctx** out) {
    CHECK_NULL(out);
    clear_error();
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(YAO_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= n) return fail(YAO_ERR_INVALID_ARGUMENT, "device index out of range");
    YAO_CUDA(cudaSetDevice(device));
    std::unique_ptr<yao_ctx> c(new yao_ctx());
    c->device = device;
    YAO_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    // the stream-ordered work buffers (expect_grad's psi and lambda, tile
    // tables) come from the device's default pool: let it keep up to 4 GiB
    // of freed memory across calls instead of unmapping it at every
    // synchronisation (alloc_device trims it when an allocation fails)
    cudaMemPool_t pool;
    YAO_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = (uint64_t)4 << 30;
    YAO_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    int sms = 0;
    YAO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    c->num_sms = sms;
    *out = c.release();
    return YAO_OK;
}

int yao_ctx_destroy(yao_ctx* c) {
    if (!c) return YAO_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->scratch) cudaFree(c->scratch);
    if (c->d_err) cudaFree(c->d_err);
    if (c->host_pinned) cudaFreeHost(c->host_pinned);
    if (c->batch_dev) cudaFree(c->batch_dev);
    if (c->batch_host) cudaFreeHost(c->batch_host);
    cudaStreamDestroy(c->stream);
    delete c;
    return YAO_OK;
}

int yao_ctx_synchronize(yao_ctx* c) {
    CHECK_NULL(c);
    YAO_CUDA(cudaStreamSynchronize(c->stream));
    return YAO_OK;
}

int yao_ctx_launch_count(const yao_ctx* c, uint64_t* out) {
    CHECK_NULL(c);
    CHECK_NULL(out);
    *out = c->launches;
    return YAO_OK;
}

int yao_ctx_stream(const yao_ctx* c, void** out) {
    CHECK_NULL(c);
    CHECK_NULL(out);
    *out = (void*)c->stream;
    return YAO_OK;
}

int yao_ctx_profile(yao_ctx* c, int enable) {
    CHECK_NULL(c);
    YAO_CUDA(cudaStreamSynchronize(c->stream));
    for (auto& r : c->recs) {
        c->event_pool.push_back(r.a);
        c->event_pool.push_back(r.b);
    }
    c->recs.clear();
    c->prof = enable != 0;
    return YAO_OK;
}

int yao_ctx_profile_report(yao_ctx* c, char* buf, size_t cap) {
    CHECK_NULL(c);
    CHECK_NULL(buf);
    YAO_CUDA(cudaStreamSynchronize(c->stream));
    struct Agg {
        uint64_t n = 0;
        double ms = 0, bytes = 0;
    };
    std::map<std::string, Agg> agg;
    std::vector<std::string> order;
    for (auto& r : c->recs) {
        float ms = 0.f;
        YAO_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        if (!agg.count(r.name)) order.push_back(r.name);
        Agg& a = agg[r.name];
        a.n++;
        a.ms += ms;
        a.bytes += r.bytes;
    }
    std::ostringstream o;
    o.precision(17);
    o << "[";
    for (size_t i = 0; i < order.size(); i++) {
        const Agg& a = agg[order[i]];
        o << (i ? "," : "") << "{\"kernel\":\"" << order[i] << "\",\"launches\":" << a.n << ",\"ms\":" << a.ms
          << ",\"bytes\":" << a.bytes << "}";
    }
    o << "]";
    std::string s = o.str();
    if (s.size() + 1 > cap) return fail(YAO_ERR_INVALID_ARGUMENT, "report buffer too small");
    memcpy(buf, s.c_str(), s.size() + 1);
    return YAO_OK;
}

// ------------------------------------------------------------------ circuit
int yao_circuit_create(const uint32_t* dims, uint32_t nsites, const yao_element* elems, size_t nelems,
                       yao_circuit** out, int32_t* ce_kind) {
    CHECK_NULL(out);
    clear_error();
    if (ce_kind) *ce_kind = YAO_CE_NONE;
    if (nsites && !dims) return fail(YAO_ERR_INVALID_ARGUMENT, "null dims");
    if (nelems && !elems) return fail(YAO_ERR_INVALID_ARGUMENT, "null elements");
    std::unique_ptr<yao_circuit> c(new yao_circuit());
    c->dims.assign(dims, dims + nsites);
    c->nbits = nsites;
    c->qubit_only = std::all_of(c->dims.begin(), c->dims.end(), [](uint32_t d) { return d == 2; });
    c->elems.resize(nelems);
    for (size_t i = 0; i < nelems; i++) {
        int s = read_element(elems[i], c->elems[i]);
        if (s) return s;
    }
    int s = validate(c->dims, c->elems, ce_kind);
    if (s) return s;
    *out = c.release();
    return YAO_OK;
}

void yao_circuit_free(yao_circuit* c) { delete c; }

int yao_circuit_num_params(const yao_circuit* c, size_t* out) {
    CHECK_NULL(c);
    CHECK_NULL(out);
    size_t n = 0;
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_GATE) n += (size_t)gate_num_params(el.g.type);
    *out = n;
    return YAO_OK;
}

int yao_circuit_parameters(const yao_circuit* c, double* out, size_t n) {
    CHECK_NULL(c);
    size_t np;
    yao_circuit_num_params(c, &np);
    if (n != np) return fail(YAO_ERR_INVALID_ARGUMENT, "parameter buffer length does not match num_params");
    size_t k = 0;
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_GATE)
            for (int i = 0; i < gate_num_params(el.g.type); i++) out[k++] = el.g.params[i];
    return YAO_OK;
}

// Circuit::dispatch (src/circuit.rs:332-352)
int yao_circuit_dispatch(yao_circuit* c, const double* params, size_t n) {
    CHECK_NULL(c);
    size_t np;
    yao_circuit_num_params(c, &np);
    if (n != np)
        return fail(YAO_ERR_INVALID_ARGUMENT, "dispatch length " + std::to_string(n) + " does not match num_params " +
                                                  std::to_string(np));
    size_t k = 0;
    for (Element& el : c->elems)
        if (el.kind == YAO_ELEM_GATE)
            for (int i = 0; i < gate_num_params(el.g.type); i++) el.g.params[i] = params[k++];
    std::lock_guard<std::mutex> lk(c->mu);
    c->lowered.clear();
    c->unitary.clear();
    c->version++;
    return YAO_OK;
}

// Circuit::dagger (src/circuit.rs:360-378)
int yao_circuit_dagger(const yao_circuit* c, yao_circuit** out) {
    CHECK_NULL(c);
    CHECK_NULL(out);
    std::unique_ptr<yao_circuit> d(new yao_circuit());
    d->dims = c->dims;
    d->nbits = c->nbits;
    d->qubit_only = c->qubit_only;
    for (size_t i = c->elems.size(); i-- > 0;) {
        Element e = c->elems[i];
        if (e.kind == YAO_ELEM_GATE) e.g = gate_dagger(e.g);
        d->elems.push_back(e);
    }
    int s = validate(d->dims, d->elems, nullptr);
    if (s) return s;
    *out = d.release();
    return YAO_OK;
}

int yao_gate_matrix(int32_t gate, const double* params, double* out, uint32_t* dim) {
    CHECK_NULL(out);
    CHECK_NULL(dim);
    double zero[4] = {0, 0, 0, 0};
    std::vector<Cx> m;
    if (named_gate_matrix(gate, params ? params : zero, m, *dim) != 0)
        return fail(YAO_ERR_INVALID_ARGUMENT, "not a named gate");
    memcpy(out, m.data(), sizeof(Cx) * m.size());
    return YAO_OK;
}

// Gate::generator_matrix (src/gate.rs:153-193): G = (dU/dtheta_i) U^-1, a
// constant matrix; its assert on i (:155-159) is an error with its message.
int yao_gate_generator_matrix(int32_t gate, uint32_t i, double* out, uint32_t* dim) {
    CHECK_NULL(out);
    CHECK_NULL(dim);
    clear_error();
    const int np = gate_num_params(gate);
    if ((int64_t)i >= np)
        return fail(YAO_ERR_INVALID_ARGUMENT, "generator_matrix index " + std::to_string(i) +
                                                  " out of range (num_params=" + std::to_string(np) + ")");
    GateElem g;
    g.type = gate;
    std::vector<Cx> m;
    gate_generator(g, (int)i, m, *dim);
    memcpy(out, m.data(), sizeof(Cx) * m.size());
    return YAO_OK;
}

int yao_noise_kraus(const yao_element* ch, double* out, uint32_t max_kraus, uint32_t* nkraus, uint32_t* dim) {
    CHECK_NULL(ch);
    CHECK_NULL(nkraus);
    CHECK_NULL(dim);
    Element el;
    int s = read_element(*ch, el);
    if (s) return s;
    std::vector<Cx> k;
    s = channel_kraus(el.ch, k, *nkraus, *dim);
    if (s) return s;
    if (*nkraus > max_kraus) return fail(YAO_ERR_INVALID_ARGUMENT, "output buffer too small");
    if (out) memcpy(out, k.data(), sizeof(Cx) * k.size());
    return YAO_OK;
}

// NoiseChannel::superop (src/noise.rs:359-379): S = sum_i kron(conj(K_i), K_i)
int yao_noise_superop(const yao_element* ch, double* out, uint32_t* dim2) {
    CHECK_NULL(ch);
    CHECK_NULL(out);
    CHECK_NULL(dim2);
    Element el;
    int s = read_element(*ch, el);
    if (s) return s;
    std::vector<Cx> S;
    uint32_t d2;
    s = channel_superop(el.ch, S, d2);
    if (s) return s;
    memcpy(out, S.data(), S.size() * sizeof(Cx));
    *dim2 = d2;
    return YAO_OK;
}

// ---------------------------------------------------------------- registers
int yao_reg_zero_state(yao_ctx* ctx, uint32_t nbits, int32_t precision, yao_reg** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    Reg* r;
    int s = alloc_reg(ctx, nbits, precision, &r);
    if (s) return s;
    s = launch_fill_zero_state(ctx, r, 0);
    if (s) {
        cudaFree(r->d);
        delete r;
        return s;
    }
    *out = static_cast<yao_reg*>(r);
    return YAO_OK;
}

int yao_reg_product_state(yao_ctx* ctx, uint32_t nbits, uint64_t basis, yao_reg** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    if (nbits < 64 && basis >= ((uint64_t)1 << nbits)) return fail(YAO_ERR_INVALID_ARGUMENT, "basis index out of range");
    Reg* r;
    int s = alloc_reg(ctx, nbits, YAO_C128, &r);
    if (s) return s;
    s = launch_fill_zero_state(ctx, r, basis);
    *out = static_cast<yao_reg*>(r);
    return s;
}

int yao_reg_from_host(yao_ctx* ctx, uint32_t nbits, const double* amps, yao_reg** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(amps);
    CHECK_NULL(out);
    Reg* r;
    int s = alloc_reg(ctx, nbits, YAO_C128, &r);
    if (s) return s;
    cudaError_t e = cudaMemcpyAsync(r->d, amps, r->bytes(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(r->d);
        delete r;
        return cuda_fail(e, "upload");
    }
    *out = static_cast<yao_reg*>(r);
    return YAO_OK;
}

int yao_reg_uniform_state(yao_ctx* ctx, uint32_t nbits, yao_reg** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    Reg* r;
    int s = alloc_reg(ctx, nbits, YAO_C128, &r);
    if (s) return s;
    s = launch_uniform_state(ctx, r);
    *out = static_cast<yao_reg*>(r);
    return s;
}

// ArrayReg::ghz_state (src/register.rs:56-63)
int yao_reg_ghz_state(yao_ctx* ctx, uint32_t nbits, yao_reg** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    Reg* r;
    int s = alloc_reg(ctx, nbits, YAO_C128, &r);
    if (s) return s;
    s = launch_fill_zero_state(ctx, r, 0);
    if (!s) {
        double amp[2] = {1.0 / std::sqrt(2.0), 0.0};
        uint64_t last = ((uint64_t)1 << nbits) - 1;
        YAO_CUDA(cudaMemcpyAsync(r->d, amp, 16, cudaMemcpyHostToDevice, ctx->stream));
        YAO_CUDA(cudaMemcpyAsync((char*)r->d + 16 * last, amp, 16, cudaMemcpyHostToDevice, ctx->stream));
        YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    *out = static_cast<yao_reg*>(r);
    return s;
}

int yao_reg_deterministic_state(yao_ctx* ctx, uint32_t nbits, yao_reg** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    Reg* r;
    int s = alloc_reg(ctx, nbits, YAO_C128, &r);
    if (s) return s;
    s = launch_deterministic_state(ctx, r);
    *out = static_cast<yao_reg*>(r);
    return s;
}

void yao_reg_free(yao_reg* r) {
    if (!r) return;
    cudaSetDevice(r->ctx->device);
    cudaStreamSynchronize(r->ctx->stream);
    cudaFree(r->d);
    delete r;
}

int yao_reg_clone(const yao_reg* r, yao_reg** out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    Reg* c;
    int s = alloc_reg(r->ctx, r->nbits, r->precision, &c);
    if (s) return s;
    YAO_CUDA(cudaMemcpyAsync(c->d, r->d, r->bytes(), cudaMemcpyDeviceToDevice, r->ctx->stream));
    *out = static_cast<yao_reg*>(c);
    return YAO_OK;
}

int yao_reg_convert(const yao_reg* r, int32_t precision, yao_reg** out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    Reg* c;
    int s = alloc_reg(r->ctx, r->nbits, precision, &c);
    if (s) return s;
    s = launch_convert(r->ctx, r, c);
    *out = static_cast<yao_reg*>(c);
    return s;
}

int yao_reg_nbits(const yao_reg* r, uint32_t* out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    *out = r->nbits;
    return YAO_OK;
}

int yao_reg_precision(const yao_reg* r, int32_t* out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    *out = r->precision;
    return YAO_OK;
}

int yao_reg_to_host(const yao_reg* r, void* amps) {
    CHECK_NULL(r);
    CHECK_NULL(amps);
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    YAO_CUDA(cudaMemcpyAsync(amps, r->d, r->bytes(), cudaMemcpyDeviceToHost, r->ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(r->ctx->stream));
    return YAO_OK;
}

int yao_reg_upload(yao_reg* r, const void* amps) {
    CHECK_NULL(r);
    CHECK_NULL(amps);
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    YAO_CUDA(cudaMemcpyAsync(r->d, amps, r->bytes(), cudaMemcpyHostToDevice, r->ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(r->ctx->stream));
    return YAO_OK;
}

int yao_reg_device_ptr(const yao_reg* r, void** out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    *out = r->d;
    return YAO_OK;
}

int yao_reg_norm(const yao_reg* r, double* out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    double ns;
    int s = reduce_norm_sqr(r->ctx, r, &ns);
    if (s) return s;
    *out = std::sqrt(ns);
    return YAO_OK;
}

int yao_reg_normalize(yao_reg* r) {
    double nrm;
    int s = yao_reg_norm(r, &nrm);
    if (s) return s;
    if (nrm > 0.0) return launch_scale(r->ctx, r, nrm);
    return YAO_OK;
}

int yao_reg_fidelity(const yao_reg* a, const yao_reg* b, double* out) {
    CHECK_NULL(a);
    CHECK_NULL(b);
    CHECK_NULL(out);
    if (a->nbits != b->nbits) return fail(YAO_ERR_NBITS_MISMATCH, "fidelity of registers with different qubit counts");
    if (a->ctx != b->ctx) return fail(YAO_ERR_INVALID_ARGUMENT, "registers of different contexts");
    YAO_CUDA(cudaSetDevice(a->ctx->device));
    Cx inner;
    int s = reduce_inner(a->ctx, a, b, &inner);
    if (s) return s;
    *out = inner.re * inner.re + inner.im * inner.im;
    return YAO_OK;
}

int yao_reg_max_abs_diff(const yao_reg* a, const yao_reg* b, double* out) {
    CHECK_NULL(a);
    CHECK_NULL(b);
    CHECK_NULL(out);
    if (a->nbits != b->nbits) return fail(YAO_ERR_NBITS_MISMATCH, "registers with different qubit counts");
    YAO_CUDA(cudaSetDevice(a->ctx->device));
    return reduce_max_abs_diff(a->ctx, a, b, out);
}

// --------------------------------------------------------------------- apply
// Every lowered gate is unitary to 1e-12 (named gates are; a Custom matrix
// is checked).
static bool program_is_unitary(const std::vector<LGate>& prog) {
    for (const LGate& g : prog) {
        if (g.cls == GC_X || g.cls == GC_SWAP) continue;
        const size_t d = (size_t)1 << g.k;
        if (g.cls == GC_DIAG) {
            for (const Cx& x : g.m)
                if (std::fabs(x.re * x.re + x.im * x.im - 1.0) > 1e-12) return false;
            continue;
        }
        for (size_t i = 0; i < d; i++)
            for (size_t j = 0; j < d; j++) {
                double re = 0, im = 0;
                for (size_t r = 0; r < d; r++) {
                    const Cx a = g.m[r * d + i], b = g.m[r * d + j];
                    re += a.re * b.re + a.im * b.im;
                    im += a.re * b.im - a.im * b.re;
                }
                if (std::fabs(re - (i == j ? 1.0 : 0.0)) > 1e-12 || std::fabs(im) > 1e-12) return false;
            }
    }
    return true;
}

// program_is_unitary of the circuit's lowered program, cached per width.
static bool circuit_is_unitary(Circuit* c) {
    const std::vector<LGate>& prog = lowered(c);
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = c->unitary.find(c->nbits);
    if (it != c->unitary.end()) return it->second;
    const bool u = program_is_unitary(prog);
    c->unitary[c->nbits] = u;
    return u;
}

int yao_apply_inplace_mode(const yao_circuit* cc, yao_reg* r, int32_t mode, int32_t k) {
    CHECK_NULL(cc);
    CHECK_NULL(r);
    clear_error();
    yao_circuit* c = const_cast<yao_circuit*>(cc);
    int s = check_apply(c, r);
    if (s) return s;
    if (mode < YAO_MODE_PLAIN || mode > YAO_MODE_FUSED) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown apply mode");
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    const std::vector<LGate>& prog = lowered(c);
    // FUSED on complex64: the FP32 arithmetic drifts the norm by a few 1e-7
    // over thousands of gates, and the tensor cores' FP32 accumulation
    // shrinks it by up to about 1e-7 per block; a unitary circuit keeps the
    // input's norm, so the FP64 norm of the input is restored afterwards
    // when blocks ran on the tensor cores or the circuit has 256 gates or
    // more (shorter CUDA-core runs drift by less than an FP32 ulp).
    // YAO_NORM_RESTORE=0 leaves the norm as the arithmetic produced it (for
    // measuring the drift)
    const char* nr_env = getenv("YAO_NORM_RESTORE");
    const bool renorm = mode == YAO_MODE_FUSED && r->precision == YAO_C64 && circuit_is_unitary(c) &&
                        !(nr_env && nr_env[0] == '0');
    double n0 = 0.0;
    if (renorm && (s = reduce_norm_sqr(r->ctx, r, &n0))) return s;
    r->ctx->tc_used = false;
    s = launch_program(r->ctx, r, prog, mode, k);
    if (s) return s;
    if (renorm && n0 > 0.0 && (r->ctx->tc_used || prog.size() >= 256)) {
        double n1 = 0.0;
        if ((s = reduce_norm_sqr(r->ctx, r, &n1))) return s;
        if (n1 > 0.0 && (s = launch_scale(r->ctx, r, std::sqrt(n1 / n0)))) return s;
    }
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

int yao_autotune(const yao_circuit* cc, yao_reg* r, int32_t mode, int32_t k, int32_t* choice) {
    CHECK_NULL(cc);
    CHECK_NULL(r);
    CHECK_NULL(choice);
    clear_error();
    yao_circuit* c = const_cast<yao_circuit*>(cc);
    int s = check_apply(c, r);
    if (s) return s;
    if (mode != YAO_MODE_TILED && mode != YAO_MODE_FUSED)
        return fail(YAO_ERR_INVALID_ARGUMENT, "autotuning applies to the TILED and FUSED modes");
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    return autotune_program(r->ctx, r, lowered(c), mode, k, choice);
}

int yao_plan_info(const yao_circuit* cc, int32_t precision, int32_t mode, int32_t k, int32_t tile_bits,
                  int32_t reg_bits, int64_t* info) {
    CHECK_NULL(cc);
    CHECK_NULL(info);
    clear_error();
    yao_circuit* c = const_cast<yao_circuit*>(cc);
    if (!c->qubit_only) return fail(YAO_ERR_QUBIT_ONLY, "ArrayReg only supports qubit-only circuits");
    int s = check_widths(c);
    if (s) return s;
    if (mode != YAO_MODE_TILED && mode != YAO_MODE_FUSED)
        return fail(YAO_ERR_INVALID_ARGUMENT, "plans exist for the TILED and FUSED modes");
    if (precision != YAO_C128 && precision != YAO_C64) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown precision");
    if (tile_bits < 6 || tile_bits > 13 || reg_bits < 1 || reg_bits > 4)
        return fail(YAO_ERR_INVALID_ARGUMENT, "tile bits 6..13, register bits 1..4");
    return plan_info(lowered(c), c->nbits, precision, mode, k, tile_bits, reg_bits, info);
}

int yao_grad_plan_info(const yao_circuit* cc, int64_t info[3]) {
    CHECK_NULL(cc);
    CHECK_NULL(info);
    clear_error();
    yao_circuit* c = const_cast<yao_circuit*>(cc);
    if (!c->qubit_only) return fail(YAO_ERR_QUBIT_ONLY, "ArrayReg only supports qubit-only circuits");
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_CHANNEL) return fail(YAO_ERR_CHANNEL_IN_AD, "expect_grad: circuit contains a noise channel");
    size_t np = 0;
    yao_circuit_num_params(c, &np);
    int st = YAO_OK;
    AdjPlan* p = adjoint_plan_new(c, c->nbits, YAO_C128, np, &st);
    if (!p) return fail(st, "expect_grad runs this circuit one gate at a time (no tiled plan)");
    adjoint_plan_counts(p, info);
    adjoint_plan_free(p);
    return YAO_OK;
}

int yao_apply_inplace(const yao_circuit* c, yao_reg* r) { return yao_apply_inplace_mode(c, r, YAO_MODE_PLAIN, 0); }

int yao_apply(const yao_circuit* c, const yao_reg* r, yao_reg** out) {
    CHECK_NULL(c);
    CHECK_NULL(r);
    CHECK_NULL(out);
    int s = check_apply(c, r);
    if (s) return s;
    yao_reg* n;
    s = yao_reg_clone(r, &n);
    if (s) return s;
    s = yao_apply_inplace(c, n);
    if (s) {
        yao_reg_free(n);
        return s;
    }
    *out = n;
    return YAO_OK;
}

// ------------------------------------------------------------ density matrix
int yao_dm_from_reg(const yao_reg* r, yao_dm** out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    if (r->precision != YAO_C128) return fail(YAO_ERR_UNSUPPORTED, "density matrices are complex128");
    DM* d;
    int s = alloc_dm(r->ctx, r->nbits, &d);
    if (s) return s;
    s = launch_dm_from_reg(r->ctx, r, d);
    *out = static_cast<yao_dm*>(d);
    return s;
}

int yao_dm_zero_state(yao_ctx* ctx, uint32_t nbits, yao_dm** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    yao_reg* r;
    int s = yao_reg_zero_state(ctx, nbits, YAO_C128, &r);
    if (s) return s;
    s = yao_dm_from_reg(r, out);
    yao_reg_free(r);
    return s;
}

int yao_dm_from_host(yao_ctx* ctx, uint32_t nbits, const double* rho, yao_dm** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(rho);
    CHECK_NULL(out);
    DM* d;
    int s = alloc_dm(ctx, nbits, &d);
    if (s) return s;
    YAO_CUDA(cudaMemcpyAsync(d->d, rho, d->bytes(), cudaMemcpyHostToDevice, ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = static_cast<yao_dm*>(d);
    return YAO_OK;
}

int yao_dm_mixed(yao_ctx* ctx, const double* weights, const yao_reg* const* regs, size_t n, yao_dm** out) {
    CHECK_NULL(ctx);
    CHECK_NULL(out);
    if (n == 0 || !weights || !regs) return fail(YAO_ERR_INVALID_ARGUMENT, "mixed needs at least one register");
    uint32_t nb = regs[0]->nbits;
    for (size_t i = 0; i < n; i++)
        if (regs[i]->nbits != nb || regs[i]->precision != YAO_C128)
            return fail(YAO_ERR_INVALID_ARGUMENT, "registers differ in size or precision");
    DM* d;
    int s = alloc_dm(ctx, nb, &d);
    if (s) return s;
    YAO_CUDA(cudaMemsetAsync(d->d, 0, d->bytes(), ctx->stream));
    for (size_t i = 0; i < n && !s; i++) s = launch_dm_mixed_accum(ctx, regs[i], weights[i], d);
    *out = static_cast<yao_dm*>(d);
    return s;
}

void yao_dm_free(yao_dm* d) {
    if (!d) return;
    cudaSetDevice(d->ctx->device);
    cudaStreamSynchronize(d->ctx->stream);
    cudaFree(d->d);
    delete d;
}

int yao_dm_clone(const yao_dm* d, yao_dm** out) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    DM* c;
    int s = alloc_dm(d->ctx, d->nbits, &c);
    if (s) return s;
    YAO_CUDA(cudaMemcpyAsync(c->d, d->d, d->bytes(), cudaMemcpyDeviceToDevice, d->ctx->stream));
    *out = static_cast<yao_dm*>(c);
    return YAO_OK;
}

int yao_dm_nbits(const yao_dm* d, uint32_t* out) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    *out = d->nbits;
    return YAO_OK;
}

int yao_dm_to_host(const yao_dm* d, double* rho) {
    CHECK_NULL(d);
    CHECK_NULL(rho);
    YAO_CUDA(cudaSetDevice(d->ctx->device));
    YAO_CUDA(cudaMemcpyAsync(rho, d->d, d->bytes(), cudaMemcpyDeviceToHost, d->ctx->stream));
    YAO_CUDA(cudaStreamSynchronize(d->ctx->stream));
    return YAO_OK;
}

// FUSED density-matrix form: rho is a 2n-qubit vector (row bits above the
// column bits), a gate is U on its row bits and conj(U) on its column bits,
// a channel is one dense 2k-qubit op, its superoperator
// S[(a, b), (c, e)] = sum_q K_q[a][c] conj(K_q)[b][e] (local index a + 2^k b,
// row bits then column bits), and the program runs through the FUSED
// tile-pass engine (FP64 blocks of up to 6 of the 2n bits, autotuned).
static int dm_apply_fused(yao_dm* d, const Circuit* c) {
    const uint32_t n = d->nbits, nb = 2 * n;
    std::vector<LGate> prog;
    for (const Element& el : c->elems) {
        if (el.kind == YAO_ELEM_GATE) {
            lower_gate(el.g, nb, 0, false, prog);
            lower_gate(el.g, nb, n, true, prog);
        } else if (el.kind == YAO_ELEM_CHANNEL) {
            std::vector<Cx> kraus;
            uint32_t nk, dim;
            int s = channel_kraus(el.ch, kraus, nk, dim);
            if (s) return s;
            std::vector<LGate> rows, cols;
            for (uint32_t q = 0; q < nk; q++) {
                std::vector<Cx> K(kraus.begin() + (size_t)q * dim * dim, kraus.begin() + (size_t)(q + 1) * dim * dim);
                const bool diag = matrix_is_diagonal(K.data(), dim);
                std::vector<Cx> Kc(K);
                for (auto& v : Kc) v.im = -v.im;
                rows.push_back(lower_matrix(K, dim, diag, el.ch.locs, {}, {}, nb, 0));
                cols.push_back(lower_matrix(Kc, dim, diag, el.ch.locs, {}, {}, nb, n));
            }
            const int k = rows[0].k, NL = 1 << k, D = NL * NL;
            if (2 * k > kMaxTargets) return fail(YAO_ERR_UNSUPPORTED, "channels on more than 3 qubits");
            auto entry = [&](const LGate& g, int r, int cc) -> Cx {
                if (g.cls == GC_DIAG) return r == cc ? g.m[r] : Cx{0.0, 0.0};
                return g.m[(size_t)r * NL + cc];
            };
            LGate sop;
            sop.cls = GC_DENSE;
            sop.k = 2 * k;
            sop.nc = 0;
            for (int i = 0; i < k; i++) {
                sop.tb[i] = rows[0].tb[i];
                sop.tb[k + i] = cols[0].tb[i];
            }
            sop.m.assign((size_t)D * D, Cx{0.0, 0.0});
            for (uint32_t q = 0; q < nk; q++)
                for (int a = 0; a < NL; a++)
                    for (int b = 0; b < NL; b++)
                        for (int cc = 0; cc < NL; cc++)
                            for (int e = 0; e < NL; e++) {
                                const Cx x = entry(rows[q], a, cc), y = entry(cols[q], b, e);
                                Cx& t = sop.m[(size_t)(a + (b << k)) * D + (cc + (e << k))];
                                t.re += x.re * y.re - x.im * y.im;
                                t.im += x.re * y.im + x.im * y.re;
                            }
            prog.push_back(std::move(sop));
        }
    }
    Reg v;
    v.ctx = d->ctx;
    v.nbits = nb;
    v.precision = YAO_C128;
    v.d = d->d;
    int s = launch_program(d->ctx, &v, prog, YAO_MODE_FUSED, 0);
    if (s) return s;
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

int yao_dm_apply(yao_dm* d, const yao_circuit* cc) { return yao_dm_apply_mode(d, cc, YAO_MODE_PLAIN); }

int yao_dm_apply_mode(yao_dm* d, const yao_circuit* cc, int32_t mode) {
    CHECK_NULL(d);
    CHECK_NULL(cc);
    clear_error();
    if (mode != YAO_MODE_PLAIN && mode != YAO_MODE_FUSED)
        return fail(YAO_ERR_INVALID_ARGUMENT, "density-matrix apply modes are PLAIN and FUSED");
    const Circuit* c = cc;
    if (!c->qubit_only) return fail(YAO_ERR_QUBIT_ONLY, "DensityMatrix only supports qubit-only circuits");
    if (c->nbits != d->nbits) return fail(YAO_ERR_NBITS_MISMATCH, "Register and circuit qubit count mismatch");
    int sw = check_widths(c);
    if (sw) return sw;
    YAO_CUDA(cudaSetDevice(d->ctx->device));
    const uint32_t n = d->nbits, nb = 2 * n;
    if (mode == YAO_MODE_FUSED) return dm_apply_fused(d, c);
    for (const Element& el : c->elems) {
        if (el.kind == YAO_ELEM_GATE) {
            std::vector<LGate> rows, cols;
            lower_gate(el.g, nb, 0, false, rows);
            lower_gate(el.g, nb, n, true, cols);
            for (size_t i = 0; i < rows.size(); i++) {
                int s = launch_dm_gate(d->ctx, d, rows[i], cols[i]);
                if (s) return s;
            }
        } else if (el.kind == YAO_ELEM_CHANNEL) {
            std::vector<Cx> kraus;
            uint32_t nk, dim;
            int s = channel_kraus(el.ch, kraus, nk, dim);
            if (s) return s;
            std::vector<LGate> rows, cols;
            for (uint32_t q = 0; q < nk; q++) {
                std::vector<Cx> K(kraus.begin() + (size_t)q * dim * dim, kraus.begin() + (size_t)(q + 1) * dim * dim);
                bool diag = matrix_is_diagonal(K.data(), dim);
                std::vector<Cx> Kc(K);
                for (auto& v : Kc) v.im = -v.im;
                rows.push_back(lower_matrix(K, dim, diag, el.ch.locs, {}, {}, nb, 0));
                cols.push_back(lower_matrix(Kc, dim, diag, el.ch.locs, {}, {}, nb, n));
            }
            s = launch_dm_channel(d->ctx, d, rows, cols, {}, {});
            if (s) return s;
        }
    }
    YAO_CUDA(cudaGetLastError());
    return YAO_OK;
}

int yao_dm_trace(const yao_dm* d, double out[2]) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    YAO_CUDA(cudaSetDevice(d->ctx->device));
    Cx t;
    int s = reduce_dm_trace(d->ctx, d, &t);
    out[0] = t.re;
    out[1] = t.im;
    return s;
}

int yao_dm_purity(const yao_dm* d, double* out) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    YAO_CUDA(cudaSetDevice(d->ctx->device));
    return reduce_dm_purity(d->ctx, d, out);
}

int yao_dm_partial_tr(const yao_dm* d, const uint32_t* traced, uint32_t n, yao_dm** out) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    if (n && !traced) return fail(YAO_ERR_INVALID_ARGUMENT, "null traced locs");
    std::set<uint32_t> tr;
    for (uint32_t i = 0; i < n; i++) {
        if (traced[i] >= d->nbits) return fail(YAO_ERR_INVALID_ARGUMENT, "traced location out of range");
        tr.insert(traced[i]);
    }
    DM* o;
    int s = alloc_dm(d->ctx, d->nbits - (uint32_t)tr.size(), &o);
    if (s) return s;
    s = launch_dm_partial_tr(d->ctx, d, traced, n, o);
    *out = static_cast<yao_dm*>(o);
    return s;
}

// --------------------------------------------------------------- observables
int yao_expect_arrayreg(const yao_reg* r, const yao_term* terms, size_t nterms, double out[2]) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    clear_error();
    std::vector<MonoTerm> mt;
    int s = build_mono_terms(terms, nterms, r->nbits, true, mt);
    if (s) return s;
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    std::vector<Cx> vals;
    s = expect_terms(r->ctx, r, mt, vals);
    if (s) return s;
    Cx acc{0, 0};
    for (size_t t = 0; t < mt.size(); t++) {
        Cx p = cxmul(mt[t].coeff, vals[t]);
        acc.re += p.re;
        acc.im += p.im;
    }
    out[0] = acc.re;
    out[1] = acc.im;
    return YAO_OK;
}

int yao_expect_arrayreg_noalloc(const yao_reg* r, const yao_term* terms, size_t nterms, double out[2]) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    clear_error();
    YAO_CUDA(cudaSetDevice(r->ctx->device));
    return expect_noalloc(r->ctx, r, terms, nterms, out);
}

int yao_expect_dm(const yao_dm* d, const yao_term* terms, size_t nterms, double out[2]) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    clear_error();
    std::vector<MonoTerm> mt;
    int s = build_mono_terms(terms, nterms, d->nbits, false, mt);
    if (s) return s;
    YAO_CUDA(cudaSetDevice(d->ctx->device));
    std::vector<Cx> vals;
    s = reduce_dm_expect(d->ctx, d, mt, vals);
    if (s) return s;
    Cx acc{0, 0};
    for (size_t t = 0; t < mt.size(); t++) {
        Cx p = cxmul(mt[t].coeff, vals[t]);
        acc.re += p.re;
        acc.im += p.im;
    }
    out[0] = acc.re;
    out[1] = acc.im;
    return YAO_OK;
}

// expect_grad (src/ad.rs:75-156)
int yao_expect_grad(const yao_term* terms, size_t nterms, const yao_circuit* cc, const yao_reg* psi0,
                    double* value, double* grad, size_t ngrad) {
    CHECK_NULL(cc);
    CHECK_NULL(psi0);
    CHECK_NULL(value);
    clear_error();
    yao_circuit* c = const_cast<yao_circuit*>(cc);
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_CHANNEL)
            return fail(YAO_ERR_CHANNEL_IN_AD,
                        "expect_grad: circuit contains a noise channel; AD is unsupported for channels");
    int s = check_apply(c, psi0);
    if (s) return s;
    if (psi0->precision != YAO_C128) return fail(YAO_ERR_UNSUPPORTED, "expect_grad runs on complex128 registers");
    size_t np;
    yao_circuit_num_params(c, &np);
    if (ngrad != np) return fail(YAO_ERR_INVALID_ARGUMENT, "gradient buffer length does not match num_params");
    if (np && !grad) return fail(YAO_ERR_INVALID_ARGUMENT, "null gradient buffer");
    std::vector<MonoTerm> mt;
    s = build_mono_terms(terms, nterms, psi0->nbits, true, mt);
    if (s) return s;
    Ctx* ctx = psi0->ctx;
    YAO_CUDA(cudaSetDevice(ctx->device));
    // psi (a copy of psi0) and lambda in stream-ordered memory: nothing below
    // synchronises before the reverse sweep's readback
    Reg psi_r = *static_cast<const Reg*>(psi0), lam_r = *static_cast<const Reg*>(psi0);
    psi_r.d = lam_r.d = nullptr;
    struct Pool {
        Ctx* ctx;
        void* a = nullptr;
        void* b = nullptr;
        ~Pool() {
            if (a) cudaFreeAsync(a, ctx->stream);
            if (b) cudaFreeAsync(b, ctx->stream);
        }
    } pool{ctx};
    const size_t bytes = psi_r.bytes();
    if (cudaMallocAsync(&pool.a, bytes, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        pool.a = nullptr;
        return fail(YAO_ERR_OUT_OF_MEMORY, "expect_grad: cannot allocate the forward state");
    }
    psi_r.d = pool.a;
    YAO_CUDA(cudaMemcpyAsync(psi_r.d, psi0->d, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    // forward pass: FUSED (FP64 blocks; within ~1e-15 of the PLAIN state);
    // its error word is read with the sweep's
    s = launch_program(ctx, &psi_r, lowered(c), YAO_MODE_FUSED, 0, false);
    if (s) return s;
    // the reverse sweep's plan, on the host while the forward pass runs
    // (YAO_ADJ_TILES=0, or a wider gate: the per-gate form below)
    struct PlanHold {
        AdjPlan* p = nullptr;
        ~PlanHold() {
            if (p) adjoint_plan_free(p);
        }
    } plan;
    const char* at = getenv("YAO_ADJ_TILES");
    if (np && !(at && at[0] == '0')) {
        int pst = YAO_OK;
        plan.p = adjoint_plan_new(c, psi0->nbits, YAO_C128, np, &pst);
        if (!plan.p && pst != YAO_ERR_UNSUPPORTED) return pst;
    }
    if (np == 0) {
        std::vector<Cx> vals;
        s = read_device_err(ctx, "expect_grad");
        if (s) return s;
        s = expect_terms(ctx, &psi_r, mt, vals);
        if (s) return s;
        Cx acc{0, 0};
        for (size_t t = 0; t < mt.size(); t++) {
            Cx p = cxmul(mt[t].coeff, vals[t]);
            acc.re += p.re;
            acc.im += p.im;
        }
        *value = acc.re;
        return YAO_OK;
    }
    if (cudaMallocAsync(&pool.b, bytes, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        pool.b = nullptr;
        return fail(YAO_ERR_OUT_OF_MEMORY, "expect_grad: cannot allocate lambda");
    }
    lam_r.d = pool.b;
    Reg* psi = &psi_r;
    Reg* lam = &lam_r;
    // lambda = H psi, and the energy Re <psi|lambda> = <psi|H|psi>.re in the
    // same pass (read back with the gradient)
    s = build_lambda_energy(ctx, psi, mt, lam);
    if (s) return s;
    // reverse sweep over shared-memory tiles of psi and lambda
    if (plan.p) {
        s = adjoint_run(ctx, psi, lam, plan.p, grad);
        if (s) return s;
        *value = lambda_energy_collect(ctx);  // adjoint_run synchronised
        return YAO_OK;
    }
    // the per-gate form reuses the reduction buffers: collect first
    s = read_device_err(ctx, "expect_grad");
    if (s) return s;
    *value = lambda_energy_collect(ctx);
    size_t slot = np;
    for (size_t ei = c->elems.size(); ei-- > 0;) {
        const Element& el = c->elems[ei];
        if (el.kind != YAO_ELEM_GATE) continue;
        const GateElem& g = el.g;
        std::vector<LGate> dag;
        lower_gate(gate_dagger(g), psi0->nbits, 0, false, dag);
        int npar = gate_num_params(g.type);
        if (npar > 0) {
            LGate gens[2];
            gens[0].k = 0;
            gens[1].k = 0;
            for (int i = 0; i < npar; i++) {
                std::vector<Cx> gm;
                uint32_t gd;
                gate_generator(g, i, gm, gd);
                gens[i] = lower_matrix(gm, gd, false, g.targets, g.ctrls, g.cfgs, psi0->nbits, 0);
            }
            Cx dots[2];
            s = adjoint_step(ctx, psi, lam, gens, dag, dots);
            if (s) return s;
            for (int i = 0; i < npar; i++) grad[slot - npar + i] = 2.0 * dots[i].re;
            slot -= npar;
        } else {
            for (const LGate& dg : dag) {
                s = launch_gate(ctx, psi->d, YAO_C128, psi0->nbits, dg);
                if (s) return s;
                s = launch_gate(ctx, lam->d, YAO_C128, psi0->nbits, dg);
                if (s) return s;
            }
        }
    }
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    return YAO_OK;
}

int yao_expect_grad_batch(const yao_term* terms, size_t nterms, const yao_circuit* cc, const double* params,
                          size_t nsets, const yao_reg* psi0, double* values, double* grads) {
    CHECK_NULL(cc);
    CHECK_NULL(psi0);
    CHECK_NULL(values);
    clear_error();
    const Circuit* c = cc;
    for (const Element& el : c->elems)
        if (el.kind == YAO_ELEM_CHANNEL)
            return fail(YAO_ERR_CHANNEL_IN_AD,
                        "expect_grad: circuit contains a noise channel; AD is unsupported for channels");
    int s = check_apply(c, psi0);
    if (s) return s;
    if (psi0->precision != YAO_C128) return fail(YAO_ERR_UNSUPPORTED, "expect_grad runs on complex128 registers");
    size_t np;
    yao_circuit_num_params(cc, &np);
    if (nsets == 0) return YAO_OK;
    if (np && (!params || !grads)) return fail(YAO_ERR_INVALID_ARGUMENT, "null params or grads");
    std::vector<MonoTerm> mt;
    s = build_mono_terms(terms, nterms, psi0->nbits, true, mt);
    if (s) return s;
    YAO_CUDA(cudaSetDevice(psi0->ctx->device));
    return expect_grad_batch(psi0->ctx, mt, c, params, nsets, psi0, values, grads);
}

// --------------------------------------------------------------- measurement
int yao_probs(const yao_reg* r, const uint32_t* locs, int32_t nlocs, double* out) {
    CHECK_NULL(r);
    CHECK_NULL(out);
    clear_error();
    Ctx* ctx = r->ctx;
    YAO_CUDA(cudaSetDevice(ctx->device));
    if (nlocs < 0) {
        uint64_t n = (uint64_t)1 << r->nbits;
        if (ctx->ensure_scratch(sizeof(double) * n)) return YAO_ERR_OUT_OF_MEMORY;
        int s = launch_probs_full(ctx, r, (double*)ctx->scratch);
        if (s) return s;
        YAO_CUDA(cudaMemcpyAsync(out, ctx->scratch, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        YAO_CUDA(cudaStreamSynchronize(ctx->stream));
        return YAO_OK;
    }
    int s = check_measure_locs(r->nbits, locs, (uint32_t)nlocs);
    if (s) return s;
    std::vector<uint32_t> bits(nlocs);
    for (int32_t i = 0; i < nlocs; i++) bits[i] = r->nbits - 1 - locs[i];
    return reduce_marginal(ctx, r, bits.data(), (uint32_t)nlocs, out);
}

int yao_dm_probs(const yao_dm* d, const uint32_t* locs, int32_t nlocs, double* out) {
    CHECK_NULL(d);
    CHECK_NULL(out);
    clear_error();
    YAO_CUDA(cudaSetDevice(d->ctx->device));
    std::vector<uint32_t> bits;
    if (nlocs >= 0) {
        int s = check_measure_locs(d->nbits, locs, (uint32_t)nlocs);
        if (s) return s;
        for (int32_t i = 0; i < nlocs; i++) bits.push_back(d->nbits - 1 - locs[i]);
    }
    return reduce_dm_marginal(d->ctx, d, bits.data(), nlocs, out);
}

// measure_with_postprocess (src/measure.rs:243-274)
int yao_measure_with_postprocess(yao_reg* r, const uint32_t* locs, uint32_t nlocs, int32_t post, uint64_t reset_val,
                                 double rand01, uint8_t* outcome, yao_reg** removed) {
    CHECK_NULL(r);
    clear_error();
    int s = check_measure_locs(r->nbits, locs, nlocs);
    if (s) return s;
    if (nlocs && (!locs || !outcome)) return fail(YAO_ERR_INVALID_ARGUMENT, "null locs or outcome");
    if (post == YAO_POST_REMOVE_MEASURED && !removed) return fail(YAO_ERR_INVALID_ARGUMENT, "null removed");
    Ctx* ctx = r->ctx;
    YAO_CUDA(cudaSetDevice(ctx->device));
    uint64_t np = (uint64_t)1 << nlocs;
    std::vector<double> probs(np);
    std::vector<uint32_t> bits(nlocs);
    for (uint32_t i = 0; i < nlocs; i++) bits[i] = r->nbits - 1 - locs[i];
    s = reduce_marginal(ctx, r, bits.data(), nlocs, probs.data());
    if (s) return s;
    // sample_from_probs (:140-150): sequential cumsum, first r < cumsum
    uint64_t idx = np - 1;
    double cumsum = 0.0;
    for (uint64_t i = 0; i < np; i++) {
        cumsum += probs[i];
        if (rand01 < cumsum) {
            idx = i;
            break;
        }
    }
    // decode_outcome_bits (:152-156): MSB first
    uint64_t mask = 0, value = 0;
    for (uint32_t i = 0; i < nlocs; i++) {
        outcome[i] = (uint8_t)((idx >> (nlocs - 1 - i)) & 1);
        mask |= (uint64_t)1 << bits[i];
        if (outcome[i]) value |= (uint64_t)1 << bits[i];
    }
    if (post == YAO_POST_NONE) return YAO_OK;
    if (post == YAO_POST_RESET_TO && reset_val >= np)
        return fail(YAO_ERR_INVALID_ARGUMENT, "reset value " + std::to_string(reset_val) + " does not fit in " +
                                                  std::to_string(nlocs) + " measured qubits");
    if (post != YAO_POST_RESET_TO && post != YAO_POST_REMOVE_MEASURED)
        return fail(YAO_ERR_INVALID_ARGUMENT, "unknown post-processing");
    // collapse_qubits_to (:158-185)
    double norm_sq;
    s = launch_collapse(ctx, r, mask, value, &norm_sq);
    if (s) return s;
    double nrm = std::sqrt(norm_sq);
    if (nrm > 1e-15) {
        s = launch_scale(ctx, r, nrm);
        if (s) return s;
    }
    if (post == YAO_POST_RESET_TO) {
        // reset_qubits_to (:187-215)
        uint64_t swap = 0;
        for (uint32_t i = 0; i < nlocs; i++) {
            uint8_t to = (uint8_t)((reset_val >> (nlocs - 1 - i)) & 1);
            if (to != outcome[i]) swap |= (uint64_t)1 << bits[i];
        }
        if (swap) s = launch_reset_move(ctx, r, mask, value, swap);
        if (!s) YAO_CUDA(cudaStreamSynchronize(ctx->stream));
        return s;
    }
    // remove_measured_qubits (:217-240)
    std::vector<uint32_t> kept;
    for (uint32_t loc = 0; loc < r->nbits; loc++)
        if (std::find(locs, locs + nlocs, loc) == locs + nlocs) kept.push_back(r->nbits - 1 - loc);
    Reg* nr;
    s = alloc_reg(ctx, (uint32_t)kept.size(), r->precision, &nr);
    if (s) return s;
    s = launch_remove_gather_fixed(ctx, r, nr, kept.data(), (uint32_t)kept.size(), value);
    if (!s) {
        double ns2;
        s = reduce_norm_sqr(ctx, nr, &ns2);
        if (!s && std::sqrt(ns2) > 0.0) s = launch_scale(ctx, nr, std::sqrt(ns2));
    }
    if (s) {
        yao_reg_free(static_cast<yao_reg*>(nr));
        return s;
    }
    YAO_CUDA(cudaStreamSynchronize(ctx->stream));
    *removed = static_cast<yao_reg*>(nr);
    return YAO_OK;
}

// ------------------------------------------------------------------ batched
int yao_batch_apply(const yao_circuit* const* circuits, yao_reg* const* regs, size_t n, int32_t mode, int32_t k) {
    if (n && (!circuits || !regs)) return fail(YAO_ERR_INVALID_ARGUMENT, "null batch arrays");
    if (mode < YAO_MODE_PLAIN || mode > YAO_MODE_FUSED) return fail(YAO_ERR_INVALID_ARGUMENT, "unknown apply mode");
    for (size_t i = 0; i < n; i++) {
        int s = check_apply(circuits[i], regs[i]);
        if (s) return s;
        if (regs[i]->ctx != regs[0]->ctx || regs[i]->precision != regs[0]->precision)
            return fail(YAO_ERR_INVALID_ARGUMENT, "batched registers must share one context and precision");
    }
    if (n == 0) return YAO_OK;
    bool small = false;
    for (size_t i = 0; i < n; i++) small |= regs[i]->nbits < 3;
    if (mode == YAO_MODE_PLAIN || small) {
        // one kernel per gate, circuit after circuit
        for (size_t i = 0; i < n; i++) {
            int s = yao_apply_inplace_mode(circuits[i], regs[i], mode, k);
            if (s) return s;
        }
        return YAO_OK;
    }
    std::vector<const std::vector<LGate>*> progs(n);
    std::vector<Reg*> rs(n);
    for (size_t i = 0; i < n; i++) {
        progs[i] = &lowered(const_cast<yao_circuit*>(circuits[i]));
        rs[i] = regs[i];
    }
    YAO_CUDA(cudaSetDevice(regs[0]->ctx->device));
    Ctx* ctx = regs[0]->ctx;
    // the norm rule of yao_apply_inplace_mode, batched: the FP64 input norm
    // of every unitary circuit's register is restored when blocks ran on the
    // tensor cores or a circuit of the batch has 256 gates or more
    std::vector<Reg*> nr;
    bool long_prog = false;
    if (mode == YAO_MODE_FUSED && regs[0]->precision == YAO_C64)
        for (size_t i = 0; i < n; i++)
            if (circuit_is_unitary(const_cast<yao_circuit*>(circuits[i]))) {
                nr.push_back(rs[i]);
                long_prog |= progs[i]->size() >= 256;
            }
    double* d_norm = nullptr;
    int s;
    if (!nr.empty()) {
        YAO_CUDA(cudaMallocAsync((void**)&d_norm, 2 * nr.size() * sizeof(double), ctx->stream));
        if ((s = launch_batch_norm_sqr(ctx, nr, d_norm))) {
            cudaFreeAsync(d_norm, ctx->stream);
            return s;
        }
    }
    ctx->tc_used = false;
    s = launch_batch(ctx, progs, rs, mode, k);
    if (!s && !nr.empty() && (ctx->tc_used || long_prog)) {
        s = launch_batch_norm_sqr(ctx, nr, d_norm + nr.size());
        if (!s) s = launch_batch_rescale(ctx, nr, d_norm, d_norm + nr.size());
    }
    if (d_norm) {
        cudaFreeAsync(d_norm, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
    return s;
}

}  // extern "C"
