// yao_internal.h — shared host/device declarations of the B200 simulation
// library (everything behind include/yao_gpu.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/yao_gpu.h"

namespace yao {

struct Cx {
    double re, im;
};

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
void clear_error();
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define YAO_CUDA(call)                                    \
    do {                                                  \
        cudaError_t e__ = (call);                         \
        if (e__ != cudaSuccess) return cuda_fail(e__, #call); \
    } while (0)

// Largest qubit count of one state vector (2^34 complex128 = 256 GiB would
// not fit; the limit is the device memory, checked at allocation).
constexpr int kMaxQubits = 34;
// Largest number of targets of one lowered gate (2^6 x 2^6 matrix).
constexpr int kMaxTargets = 6;

// ------------------------------------------------------------------ gates
// A gate after dispatch_arrayreg_gate's decision (yao-rs src/apply.rs:7-120),
// expressed on bit positions (bit = nbits - 1 - loc).
enum GateClass : int32_t {
    GC_X = 0,     // amplitude-pair swap on one target bit (instruct_x[_controlled])
    GC_SWAP = 1,  // swap of the |01> / |10> amplitudes of two bits (instruct_swap)
    GC_DIAG = 2,  // elementwise product by d[local index] (instruct_*_diag*)
    GC_DENSE = 3  // dense 2^k x 2^k product (instruct_1q / _2q / _nq [+controlled])
};

struct LGate {
    int32_t cls = GC_DENSE;
    int32_t k = 1;                   // number of target bits
    int32_t tb[kMaxTargets] = {0};   // local index bit i <-> global bit tb[i]
    int32_t nc = 0;                  // controls
    int32_t cb[64] = {0};            // control bit positions
    int32_t cv[64] = {0};            // control values (0/1)
    std::vector<Cx> m;               // dense: 2^k x 2^k row-major; diag: 2^k entries
    uint64_t cmask() const;
    uint64_t cval() const;
};

// A gate of the circuit (yao-rs PositionedGate) kept in wire form plus the
// data needed to lower it (matrix of named gates is rebuilt on dispatch).
struct GateElem {
    int32_t type = 0;                // enum yao_gate_kind
    std::vector<uint32_t> targets;   // locs
    std::vector<uint32_t> ctrls;     // locs
    std::vector<uint8_t> cfgs;       // 0/1
    double params[4] = {0, 0, 0, 0};
    std::vector<Cx> custom;          // Custom matrix
    uint32_t custom_dim = 0;
    bool custom_diag = false;
};

struct ChannelElem {
    int32_t type = 0;                // enum yao_noise_kind
    std::vector<uint32_t> locs;
    double params[4] = {0, 0, 0, 0};
    int32_t depol_n = 1;
    std::vector<Cx> mats;            // Coherent / Custom matrices
    uint32_t dim = 0;
    uint32_t nkraus = 0;
};

struct Element {
    int32_t kind = YAO_ELEM_GATE;
    GateElem g;
    ChannelElem ch;
    uint32_t annot_loc = 0;
};

// host-side gate algebra (gate.rs / noise.rs restated), host_gate.cpp
int named_gate_matrix(int32_t type, const double* params, std::vector<Cx>& m, uint32_t& dim);
bool named_gate_is_diagonal(int32_t type);
int gate_num_params(int32_t type);
void gate_matrix(const GateElem& g, std::vector<Cx>& m, uint32_t& dim, bool& diag);
GateElem gate_dagger(const GateElem& g);
void gate_generator(const GateElem& g, int i, std::vector<Cx>& m, uint32_t& dim);
int channel_kraus(const ChannelElem& ch, std::vector<Cx>& kraus, uint32_t& nkraus, uint32_t& dim);
int channel_superop(const ChannelElem& ch, std::vector<Cx>& S, uint32_t& d2);
bool matrix_is_diagonal(const Cx* m, uint32_t d);

// Lower one gate on an nbits-qubit register with location offset `shift`
// (density-matrix column copies use shift = n); conj = use conj(matrix).
// Appends one or more LGates (a multi-target X becomes one per target).
void lower_gate(const GateElem& g, uint32_t nbits, uint32_t shift, bool conj, std::vector<LGate>& out);
// Lower an explicit matrix (Kraus operator, generator) placed like g.
LGate lower_matrix(const std::vector<Cx>& m, uint32_t dim, bool diag, const std::vector<uint32_t>& targets,
                   const std::vector<uint32_t>& ctrls, const std::vector<uint8_t>& cfgs, uint32_t nbits,
                   uint32_t shift);

// ---------------------------------------------------------------- circuit
struct Circuit {
    std::vector<uint32_t> dims;
    std::vector<Element> elems;
    uint32_t nbits = 0;
    bool qubit_only = true;
    // lowered program cache (per register width); built lazily
    std::mutex mu;
    std::map<uint32_t, std::vector<LGate>> lowered;
    std::map<uint32_t, bool> unitary;  // every lowered gate unitary (cached beside `lowered`)
    uint64_t version = 0;  // bumped by dispatch()
};

// ---------------------------------------------------------------- context
struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    // device scratch for reductions (grown on demand)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // pinned host mirror of small reduction results
    void* host_pinned = nullptr;
    size_t host_pinned_bytes = 0;
    uint64_t launches = 0;
    // device word a kernel sets when one of its bounded waits gave up
    int* d_err = nullptr;
    // the last TILED / FUSED run put some blocks on the tensor cores
    bool tc_used = false;
    // tables of the batched launch (device and pinned host copies), kept and
    // grown across calls; freed with the context
    void* batch_dev = nullptr;
    size_t batch_dev_bytes = 0;
    void* batch_host = nullptr;
    size_t batch_host_bytes = 0;
    int ensure_scratch(size_t bytes);
    int ensure_host_pinned(size_t bytes);
    // optional per-launch timing (CUDA events on `stream` around each launch)
    struct ProfRec {
        const char* name;
        cudaEvent_t a, b;
        double bytes;
    };
    bool prof = false;
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t take_event();
    void prof_begin(const char* name, double bytes);
    void prof_end();
};

// Records one launch when profiling is on: construct right before the
// launch, destroy right after it.
struct ProfScope {
    Ctx* c;
    bool on;
    ProfScope(Ctx* ctx, const char* name, double bytes) : c(ctx), on(ctx->prof) {
        if (on) c->prof_begin(name, bytes);
    }
    ~ProfScope() {
        if (on) c->prof_end();
    }
};

struct Reg {
    Ctx* ctx = nullptr;
    uint32_t nbits = 0;
    int32_t precision = YAO_C128;
    void* d = nullptr;  // double2* (C128) or float2* (C64)
    size_t bytes() const { return ((size_t)1 << nbits) * (precision == YAO_C128 ? 16 : 8); }
};

struct DM {
    Ctx* ctx = nullptr;
    uint32_t nbits = 0;
    void* d = nullptr;  // double2*, 4^n
    size_t bytes() const { return ((size_t)1 << (2 * nbits)) * 16; }
};

// ------------------------------------------------------- device launchers
// All launchers enqueue on ctx->stream and return YAO_OK or an error.
int launch_gate(Ctx* ctx, void* state, int32_t precision, uint32_t nbits, const LGate& g);
// check_err false: the error word of the passes' bounded waits is left for
// the caller to read (read_device_err) at its own synchronisation
int launch_program(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k, bool check_err = true);
// Synchronises, and turns a set error word into YAO_ERR_TIMEOUT (clearing it)
int read_device_err(Ctx* ctx, const char* what);
// Time TILED / FUSED candidates for this program and register (always
// re-tunes); out = {k, tile bits, register bits}.
int autotune_program(Ctx* ctx, Reg* r, const std::vector<LGate>& prog, int32_t mode, int32_t k, int32_t out[4]);
// Host-only plan of a TILED / FUSED run (see yao_plan_info).
int plan_info(const std::vector<LGate>& prog, uint32_t nbits, int32_t precision, int32_t mode, int32_t k,
              int32_t tbits, int32_t rb, int64_t info[7]);
// Many circuits (one register each, same context and precision) in one
// persistent, graph-captured launch (TILED or FUSED forms).
int launch_batch(Ctx* ctx, const std::vector<const std::vector<LGate>*>& progs, const std::vector<Reg*>& regs,
                 int32_t mode, int32_t k);

int launch_fill_zero_state(Ctx* ctx, Reg* r, uint64_t basis);
int launch_uniform_state(Ctx* ctx, Reg* r);
int launch_deterministic_state(Ctx* ctx, Reg* r);
int launch_convert(Ctx* ctx, const Reg* src, Reg* dst);
int reduce_norm_sqr(Ctx* ctx, const Reg* r, double* out);
int launch_scale(Ctx* ctx, Reg* r, double inv_norm);
int adjoint_tiles(Ctx* ctx, Reg* psi, Reg* lam, const Circuit* c, double* grad, size_t np);
// adjoint_tiles in two halves: the host plan (null with *status
// YAO_ERR_UNSUPPORTED when the per-gate form must run) and its sweep
struct AdjPlan;
AdjPlan* adjoint_plan_new(const Circuit* c, uint32_t n, int32_t precision, size_t np, int* status);
void adjoint_plan_free(AdjPlan* p);
void adjoint_plan_counts(const AdjPlan* p, int64_t out[3]);  // passes, ops, generator dots
int adjoint_run(Ctx* ctx, Reg* psi, Reg* lam, const AdjPlan* plan, double* grad);
int launch_batch_norm_sqr(Ctx* ctx, const std::vector<Reg*>& regs, double* out);
int launch_batch_rescale(Ctx* ctx, const std::vector<Reg*>& regs, const double* n0, const double* n1);
int reduce_inner(Ctx* ctx, const Reg* a, const Reg* b, Cx* out);
int reduce_max_abs_diff(Ctx* ctx, const Reg* a, const Reg* b, double* out);

// Pauli-monomial term: (O psi)[i] = i^phase(i) * psi[i ^ xmask] (or 0)
struct MonoTerm {
    uint64_t xmask = 0;
    uint64_t d1mask = 0, d2mask = 0;  // per-bit quarter-turn increments when the bit is 1
    uint64_t need1 = 0, need0 = 0;    // bits that must be 1 / 0 for a nonzero entry
    int32_t base = 0;                 // quarter turns when all bits are 0
    int32_t zero = 0;                 // identically zero operator
    Cx coeff{0, 0};
};
// Build monomial terms from yao_term[] with sites mapped to bit positions
// by bit = msb_first ? nbits-1-site : site.
int build_mono_terms(const yao_term* terms, size_t nterms, uint32_t nbits, bool msb_first,
                     std::vector<MonoTerm>& out);
int expect_terms(Ctx* ctx, const Reg* r, const std::vector<MonoTerm>& terms, std::vector<Cx>& values);
// expect_terms in two halves (the sums land in ctx->host_pinned once the
// stream has passed the launch half's copy)
struct ExpectPending {
    size_t nterms = 0;
    std::vector<size_t> idx;  // term of each result pair, group by group
    std::vector<int> nv;      // doubles per group
};
int expect_terms_launch(Ctx* ctx, const Reg* r, const std::vector<MonoTerm>& terms, ExpectPending& pend);
void expect_terms_collect(Ctx* ctx, const ExpectPending& pend, std::vector<Cx>& values);
// The allocation-free expectation value (static device scratch), sv_reduce.cu.
int expect_noalloc(Ctx* ctx, const Reg* r, const yao_term* terms, size_t nterms, double* out);
int build_lambda(Ctx* ctx, const Reg* psi, const std::vector<MonoTerm>& terms, Reg* lambda);
int build_lambda_sets(Ctx* ctx, const void* psi_d, void* lam_d, uint32_t nbits, uint64_t nsets,
                      const std::vector<MonoTerm>& terms);
// lambda = H psi and, in the same pass, Re <psi|lambda> = <psi|H|psi>.re,
// queued for ctx->host_pinned[0]; lambda_energy_collect reads it once the
// stream has passed that copy (sv_reduce.cu).
int build_lambda_energy(Ctx* ctx, const Reg* psi, const std::vector<MonoTerm>& terms, Reg* lambda);
double lambda_energy_collect(Ctx* ctx);
// A gate on nsets complex128 registers of nbits qubits stored back to back.
int launch_gate_sets(Ctx* ctx, void* state, uint32_t nbits, const LGate& g, uint64_t nsets);
// Energies and adjoint gradients of nsets parameter vectors of one circuit.
int expect_grad_batch(Ctx* ctx, const std::vector<MonoTerm>& terms, const Circuit* c, const double* params,
                      size_t nsets, const Reg* psi0, double* values, double* grads);
int adjoint_step(Ctx* ctx, Reg* psi, Reg* lambda, const LGate* gen, const std::vector<LGate>& dag,
                 Cx* dot_out);

int launch_probs_full(Ctx* ctx, const Reg* r, double* dprobs);
int reduce_marginal(Ctx* ctx, const Reg* r, const uint32_t* bits, uint32_t nl, double* host_out);
int launch_collapse(Ctx* ctx, Reg* r, uint64_t mask, uint64_t value, double* norm_sq_out);
int launch_reset_move(Ctx* ctx, Reg* r, uint64_t mask, uint64_t value, uint64_t swap_mask);
int launch_remove_gather_fixed(Ctx* ctx, const Reg* src, Reg* dst, const uint32_t* kept_bits, uint32_t nk,
                               uint64_t fixed);

// density matrices
int launch_dm_from_reg(Ctx* ctx, const Reg* r, DM* d);
int launch_dm_mixed_accum(Ctx* ctx, const Reg* r, double w, DM* d);
int launch_dm_gate(Ctx* ctx, DM* d, const LGate& row, const LGate& col);
int launch_dm_channel(Ctx* ctx, DM* d, const std::vector<LGate>& rows, const std::vector<LGate>& cols,
                      const std::vector<uint32_t>& row_bits, const std::vector<uint32_t>& col_bits);
int reduce_dm_trace(Ctx* ctx, const DM* d, Cx* out);
int reduce_dm_purity(Ctx* ctx, const DM* d, double* out);
int reduce_dm_expect(Ctx* ctx, const DM* d, const std::vector<MonoTerm>& terms, std::vector<Cx>& values);
int reduce_dm_marginal(Ctx* ctx, const DM* d, const uint32_t* bits, int32_t nl, double* host_out);
int launch_dm_partial_tr(Ctx* ctx, const DM* d, const uint32_t* traced, uint32_t nt, DM* out);

}  // namespace yao

// The opaque handle types of the C ABI; every object is created as one of
// these, so the casts between the handle and its base type are valid.
struct yao_ctx : yao::Ctx {};
struct yao_circuit : yao::Circuit {};
struct yao_reg : yao::Reg {};
struct yao_dm : yao::DM {};
