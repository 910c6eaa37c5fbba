/*
 * yao_gpu.h — C ABI of the B200 simulation library for the yao-rs hot path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (YAO_OK = 0, negative = error; the message is in
 * yao_last_error()).  No C++ or torch type crosses this boundary.
 *
 * Conventions kept from yao-rs:
 *   - A state is 2^n complex amplitudes, interleaved {re, im} doubles
 *     (num_complex::Complex64 is #[repr(C)] {re, im}), index
 *     sum_loc q_loc * 2^(n-1-loc): loc 0 is the most significant bit
 *     (yao-rs src/instruct_qubit.rs:15-18).
 *   - A density matrix is row-major 4^n complex, rho[row*dim + col]
 *     (src/density_matrix.rs:7-12).
 *   - Gate matrices are row-major; in a multi-target gate, target_locs[0]
 *     is the least significant bit of the gate-local index
 *     (src/instruct_qubit.rs:215-231, 346-355).
 *
 * Each function cites the yao-rs interface it replaces (path:line inside
 * the yao-rs repository).
 */
#ifndef YAO_GPU_H
#define YAO_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define YAO_GPU_ABI_VERSION 1

/* ---------------------------------------------------------------- status */
enum yao_status {
    YAO_OK = 0,
    YAO_ERR_INVALID_ARGUMENT = -1,
    YAO_ERR_CIRCUIT = -2,          /* Circuit::new -> Err(CircuitError), src/circuit.rs:41-57 */
    YAO_ERR_QUBIT_ONLY = -3,       /* "ArrayReg only supports qubit-only circuits", src/apply.rs:124-127 */
    YAO_ERR_NBITS_MISMATCH = -4,   /* "Register and circuit qubit count mismatch", src/apply.rs:128-132 */
    YAO_ERR_CHANNEL_IN_AD = -5,    /* "expect_grad: circuit contains a noise channel", src/ad.rs:80-84 */
    YAO_ERR_NOISE_PARAM = -6,      /* NoiseChannel::validate_params panics, src/noise.rs:90-176 */
    YAO_ERR_MEASURE_LOCS = -7,     /* validate_measure_locs panics, src/measure.rs:124-133 */
    YAO_ERR_OUT_OF_MEMORY = -8,
    YAO_ERR_CUDA = -9,
    YAO_ERR_NO_DEVICE = -10,
    YAO_ERR_UNSUPPORTED = -11,
    YAO_ERR_TIMEOUT = -12
};

/* CircuitError variants (src/circuit.rs:41-57), reported by yao_circuit_create */
enum yao_circuit_error_kind {
    YAO_CE_NONE = 0,
    YAO_CE_CONTROL_CONFIG_LENGTH_MISMATCH = 1,
    YAO_CE_LOC_OUT_OF_RANGE = 2,
    YAO_CE_OVERLAPPING_LOCS = 3,
    YAO_CE_CONTROL_SITE_NOT_QUBIT = 4,
    YAO_CE_NAMED_GATE_TARGET_NOT_QUBIT = 5,
    YAO_CE_MATRIX_SIZE_MISMATCH = 6
};

/* ------------------------------------------------------- circuit wire format */
/* CircuitElement (src/circuit.rs:33-38) */
enum yao_elem_kind { YAO_ELEM_GATE = 0, YAO_ELEM_CHANNEL = 1, YAO_ELEM_ANNOTATION = 2 };

/* Gate enum (src/gate.rs:7-35) */
enum yao_gate_kind {
    YAO_GATE_X = 0, YAO_GATE_Y, YAO_GATE_Z, YAO_GATE_H, YAO_GATE_S, YAO_GATE_T,
    YAO_GATE_SWAP, YAO_GATE_PHASE, YAO_GATE_RX, YAO_GATE_RY, YAO_GATE_RZ,
    YAO_GATE_SQRTX, YAO_GATE_SQRTY, YAO_GATE_SQRTW, YAO_GATE_ISWAP, YAO_GATE_FSIM,
    YAO_GATE_CUSTOM
};

/* NoiseChannel enum (src/noise.rs:16-60) */
enum yao_noise_kind {
    YAO_NOISE_BIT_FLIP = 0,            /* params[0] = p */
    YAO_NOISE_PHASE_FLIP,              /* params[0] = p */
    YAO_NOISE_DEPOLARIZING,            /* depol_n = n, params[0] = p */
    YAO_NOISE_PAULI_CHANNEL,           /* params = px, py, pz */
    YAO_NOISE_RESET,                   /* params = p0, p1 */
    YAO_NOISE_AMPLITUDE_DAMPING,       /* params = gamma, excited_population */
    YAO_NOISE_PHASE_DAMPING,           /* params[0] = gamma */
    YAO_NOISE_PHASE_AMPLITUDE_DAMPING, /* params = amplitude, phase, excited_population */
    YAO_NOISE_THERMAL_RELAXATION,      /* params = t1, t2, time, excited_population */
    YAO_NOISE_COHERENT,                /* matrix (matrix_dim x matrix_dim) */
    YAO_NOISE_CUSTOM                   /* nkraus matrices back to back */
};

/* Op enum (src/operator.rs:8-17) */
enum yao_op { YAO_OP_I = 0, YAO_OP_X, YAO_OP_Y, YAO_OP_Z, YAO_OP_P0, YAO_OP_P1, YAO_OP_PU, YAO_OP_PD };

/* PostProcess enum (src/measure.rs:18-23) */
enum yao_postprocess { YAO_POST_NONE = 0, YAO_POST_RESET_TO = 1, YAO_POST_REMOVE_MEASURED = 2 };

/* Element precision of a register. */
enum yao_precision { YAO_C128 = 0, YAO_C64 = 1 };

/* Execution form of yao_apply_inplace_mode.
 *   PLAIN     one kernel per gate, arithmetic identical to yao-rs (bit-exact);
 *   TILED     runs of gates applied per shared-memory tile, same arithmetic
 *             and order as PLAIN (bit-exact), fewer HBM passes;
 *   FUSED     gates multiplied into dense k-qubit blocks on the host (FP64),
 *             each block one tiled pass; not bit-exact, report 1 - fidelity.
 *             On a YAO_C64 register the blocks are applied with split
 *             (hi + lo) FP32 products accumulated in FP32 (dense 3..5-qubit
 *             blocks: three TF32 tensor-core products), and when every gate
 *             is unitary and blocks ran on the tensor cores or the circuit
 *             has 256 gates or more, the input's FP64 norm is restored at
 *             the end (yao_apply_inplace_mode; the batched form does not). */
enum yao_apply_mode { YAO_MODE_PLAIN = 0, YAO_MODE_TILED = 1, YAO_MODE_FUSED = 2 };

/* One circuit element: PositionedGate (src/circuit.rs:103-109),
 * PositionedChannel (:26-30) or PositionedAnnotation (:19-23). */
typedef struct yao_element {
    int32_t kind;               /* enum yao_elem_kind */
    int32_t type;               /* enum yao_gate_kind (gate) / enum yao_noise_kind (channel) */
    uint32_t ntargets;          /* target_locs (gate) / locs (channel); annotation: 1 (targets[0] = loc) */
    uint32_t nctrl;             /* control_locs */
    const uint32_t* targets;
    const uint32_t* ctrl_locs;
    const uint8_t* ctrl_configs; /* control_configs, 0/1 each; NULL = all active-high */
    const double* matrix;       /* interleaved complex, row-major (Custom gate, Coherent, Custom channel) */
    uint32_t matrix_dim;        /* rows of each matrix */
    uint32_t nkraus;            /* Custom channel: number of Kraus matrices */
    int32_t is_diagonal;        /* Custom gate flag */
    int32_t depol_n;            /* Depolarizing { n } */
    uint32_t nconfigs;          /* length of ctrl_configs (must equal nctrl unless ctrl_configs is NULL) */
    uint32_t reserved;
    double params[4];
} yao_element;

/* One term c * OperatorString of an OperatorPolynomial (src/operator.rs:21-33,69-73):
 * (sites[i], ops[i]) pairs in any order; OperatorString::new sorts them by site
 * and drops Op::I. */
typedef struct yao_term {
    double coeff_re;
    double coeff_im;
    uint32_t nops;
    uint32_t reserved;
    const uint32_t* sites;
    const int32_t* ops;         /* enum yao_op */
} yao_term;

typedef struct yao_ctx yao_ctx;
typedef struct yao_circuit yao_circuit;
typedef struct yao_reg yao_reg;
typedef struct yao_dm yao_dm;

/* ------------------------------------------------------------------ misc */
/* Message of the last failed call on this thread ("" if none). */
const char* yao_last_error(void);
int yao_abi_version(void);

/* ------------------------------------------------------------- context */
/* A context owns one CUDA device, one stream and the device scratch of
 * the reductions.  yao-rs has no counterpart (it is single-threaded CPU). */
int yao_ctx_create(int device, yao_ctx** out);
int yao_ctx_destroy(yao_ctx* ctx);
int yao_ctx_synchronize(yao_ctx* ctx);
/* Number of kernels this context has launched so far. */
int yao_ctx_launch_count(const yao_ctx* ctx, uint64_t* out);
/* The cudaStream_t all of this context's work is enqueued on. */
int yao_ctx_stream(const yao_ctx* ctx, void** out);
/* Per-launch timing: with profiling on, every kernel launch is bracketed by
 * CUDA events on the context stream.  Enabling (or disabling) clears the
 * records.  The report is a JSON array of {kernel, launches, ms, bytes},
 * bytes being the launches' algorithmic HBM traffic (reads + writes of the
 * amplitudes they update). */
int yao_ctx_profile(yao_ctx* ctx, int enable);
int yao_ctx_profile_report(yao_ctx* ctx, char* buf, size_t cap);

/* --------------------------------------------------------------- circuit */
/* Circuit::new (src/circuit.rs:150-272).  dims[i] is the local dimension
 * of site i.  On YAO_ERR_CIRCUIT, *ce_kind (if non-NULL) receives the
 * CircuitError variant. */
int yao_circuit_create(const uint32_t* dims, uint32_t nsites, const yao_element* elems,
                       size_t nelems, yao_circuit** out, int32_t* ce_kind);
void yao_circuit_free(yao_circuit* c);
/* Circuit::num_params / parameters / dispatch / dagger (src/circuit.rs:308-378) */
int yao_circuit_num_params(const yao_circuit* c, size_t* out);
int yao_circuit_parameters(const yao_circuit* c, double* out, size_t n);
int yao_circuit_dispatch(yao_circuit* c, const double* params, size_t n);
int yao_circuit_dagger(const yao_circuit* c, yao_circuit** out);
/* Gate::matrix (src/gate.rs:63-68) for a named gate; out holds dim*dim
 * interleaved complex (dim <= 4). */
int yao_gate_matrix(int32_t gate, const double* params, double* out, uint32_t* dim);
/* Gate::generator_matrix (src/gate.rs:153-193): the constant generator
 * G = (dU/dtheta_i) U^-1 of parameter i of a named parametric gate (Rx, Ry,
 * Rz, Phase: i = 0; FSim: i = 0 theta, 1 phi); out holds dim*dim interleaved
 * complex (dim <= 4).  i >= num_params (every non-parametric gate) is
 * YAO_ERR_INVALID_ARGUMENT with yao-rs's panic message. */
int yao_gate_generator_matrix(int32_t gate, uint32_t i, double* out, uint32_t* dim);
/* NoiseChannel::kraus_operators / superop (src/noise.rs:183-379).
 * kraus_out holds up to max_kraus matrices of dim x dim. */
int yao_noise_kraus(const yao_element* channel, double* kraus_out, uint32_t max_kraus,
                    uint32_t* nkraus, uint32_t* dim);
int yao_noise_superop(const yao_element* channel, double* out, uint32_t* dim2);

/* --------------------------------------------------------------- ArrayReg */
/* ArrayReg::zero_state / from_vec / uniform_state / ghz_state /
 * deterministic_state / product_state (src/register.rs:21-96). */
int yao_reg_zero_state(yao_ctx* ctx, uint32_t nbits, int32_t precision, yao_reg** out);
int yao_reg_from_host(yao_ctx* ctx, uint32_t nbits, const double* amps, yao_reg** out);
int yao_reg_uniform_state(yao_ctx* ctx, uint32_t nbits, yao_reg** out);
int yao_reg_ghz_state(yao_ctx* ctx, uint32_t nbits, yao_reg** out);
int yao_reg_deterministic_state(yao_ctx* ctx, uint32_t nbits, yao_reg** out);
int yao_reg_product_state(yao_ctx* ctx, uint32_t nbits, uint64_t basis, yao_reg** out);
void yao_reg_free(yao_reg* r);
int yao_reg_clone(const yao_reg* r, yao_reg** out);
/* Copy to another precision (C128 <-> C64). */
int yao_reg_convert(const yao_reg* r, int32_t precision, yao_reg** out);
int yao_reg_nbits(const yao_reg* r, uint32_t* out);
int yao_reg_precision(const yao_reg* r, int32_t* out);
/* state_vec: 2*2^n doubles (C128) or 2*2^n floats (C64). */
int yao_reg_to_host(const yao_reg* r, void* amps);
int yao_reg_upload(yao_reg* r, const void* amps);
int yao_reg_device_ptr(const yao_reg* r, void** out);
/* ArrayReg::norm / normalize / fidelity (src/register.rs:98-125). */
int yao_reg_norm(const yao_reg* r, double* out);
int yao_reg_normalize(yao_reg* r);
int yao_reg_fidelity(const yao_reg* a, const yao_reg* b, double* out);
/* Largest |a_i - b_i| over both components. */
int yao_reg_max_abs_diff(const yao_reg* a, const yao_reg* b, double* out);

/* apply_inplace / apply (src/apply.rs:123-154).  Channels are skipped,
 * annotations are no-ops, exactly as in the CPU path. */
int yao_apply_inplace(const yao_circuit* c, yao_reg* r);
int yao_apply(const yao_circuit* c, const yao_reg* r, yao_reg** out);
/* The same with an explicit execution form (enum yao_apply_mode); k is the
 * fusion width of YAO_MODE_FUSED (1..6; 0 = autotuned). */
int yao_apply_inplace_mode(const yao_circuit* c, yao_reg* r, int32_t mode, int32_t k);
/* Autotuner of the TILED / FUSED forms (no yao-rs counterpart): times tile
 * shapes (and, for FUSED with k = 0, fusion widths 2..6) on a prefix of c
 * applied to a scratch copy of r (r is not changed) and records the fastest
 * for r's qubit count, precision and mode; later apply calls with the same
 * (qubits, precision, mode, k) use it.  choice[4] = {k, tile bits, register
 * bits, 1 when complex64 FUSED blocks may run on the tensor cores}.  Apply calls tune on first use by themselves unless YAO_AUTOTUNE=0;
 * YAO_TUNE_CACHE=<file> keeps the choices across processes. */
int yao_autotune(const yao_circuit* c, yao_reg* r, int32_t mode, int32_t k, int32_t* choice);
/* The TILED / FUSED plan of c for a given shape, computed on the host only
 * (no device needed): info[7] = {passes, single-gate passes, ops,
 * tensor-core ops, wide CUDA-core ops, register segments, fused blocks}. */
int yao_plan_info(const yao_circuit* c, int32_t precision, int32_t mode, int32_t k, int32_t tile_bits,
                  int32_t reg_bits, int64_t* info);

/* ---------------------------------------------------------- DensityMatrix */
/* DensityMatrix::from_reg / zero_state / mixed (src/density_matrix.rs:19-57). */
int yao_dm_from_reg(const yao_reg* r, yao_dm** out);
int yao_dm_zero_state(yao_ctx* ctx, uint32_t nbits, yao_dm** out);
int yao_dm_from_host(yao_ctx* ctx, uint32_t nbits, const double* rho, yao_dm** out);
int yao_dm_mixed(yao_ctx* ctx, const double* weights, const yao_reg* const* regs, size_t n,
                 yao_dm** out);
void yao_dm_free(yao_dm* d);
int yao_dm_clone(const yao_dm* d, yao_dm** out);
int yao_dm_nbits(const yao_dm* d, uint32_t* out);
int yao_dm_to_host(const yao_dm* d, double* rho);
/* Register::apply for DensityMatrix (src/density_matrix.rs:249-259):
 * gates rho -> U rho U^dagger, channels rho -> sum_i K_i rho K_i^dagger. */
int yao_dm_apply(yao_dm* d, const yao_circuit* c);
/* The same with an execution form: YAO_MODE_PLAIN (= yao_dm_apply, the exact
 * Kraus sum of yao-rs) or YAO_MODE_FUSED: rho as a 2n-qubit vector, each
 * gate as U on the row bits and conj(U) on the column bits, each channel as
 * its superoperator sum_i K_i (x) conj(K_i) (a dense op on 2k bits), all run
 * through the FUSED tile-pass engine in FP64 (not bit-identical; agrees to
 * ~1e-14). */
int yao_dm_apply_mode(yao_dm* d, const yao_circuit* c, int32_t mode);
/* trace / purity / partial_tr (src/density_matrix.rs:63-112). */
int yao_dm_trace(const yao_dm* d, double out[2]);
int yao_dm_purity(const yao_dm* d, double* out);
int yao_dm_partial_tr(const yao_dm* d, const uint32_t* traced_locs, uint32_t n, yao_dm** out);

/* ------------------------------------------------------------- observables */
/* expect_arrayreg / expect_dm (src/expect.rs:7-72); out = {re, im}.
 * expect_dm keeps yao-rs's site convention of that function: site s is bit s
 * of the row/column index (least significant first). */
int yao_expect_arrayreg(const yao_reg* r, const yao_term* terms, size_t nterms, double out[2]);
/* The same value as yao_expect_arrayreg, computed without allocating any
 * memory.  No yao-rs counterpart: it exists for callers that cannot allocate
 * at call time -- an application whose memory pool already holds nearly all
 * of the GPU's memory for its state vectors (a cudaMalloc would fail or make
 * the pool give memory back), or one that must not stall the GPU (cudaFree
 * synchronises the device).  The reduction scratch is a 131,200-byte
 * file-scope device array that every GPU loading the library keeps until
 * exit; its address is looked up on the first call on each device (make
 * that first call before any stream capture; a lookup that fails is tried
 * again on the next call).  Limits: at most 64 terms of
 * at most 64 ops each, else YAO_ERR_INVALID_ARGUMENT.  All calls share the
 * array: calls that overlap on the GPU race and must be serialised. */
int yao_expect_arrayreg_noalloc(const yao_reg* r, const yao_term* terms, size_t nterms, double out[2]);
int yao_expect_dm(const yao_dm* d, const yao_term* terms, size_t nterms, double out[2]);
/* expect_grad (src/ad.rs:75-156): value = Re <psi|H|psi>, grad in
 * Circuit::parameters() order; ngrad must equal num_params.  The forward
 * state is computed in FUSED form (within ~1e-15 of the PLAIN state) and the
 * reverse sweep runs over shared-memory tiles of psi and lambda (circuits
 * with gates on more than 2 qubits, or YAO_ADJ_TILES=0: one step per gate). */
/* The plan of expect_grad's tiled reverse sweep for c, computed on the host
 * only (no device needed): info[3] = {passes, ops, generator dots}.  Steps
 * on disjoint qubits may share a pass out of sweep order (YAO_ADJ_REORDER=0:
 * consecutive steps only).  YAO_ERR_UNSUPPORTED when c takes the per-gate
 * form (a gate on more than 2 qubits). */
int yao_grad_plan_info(const yao_circuit* c, int64_t info[3]);
int yao_expect_grad(const yao_term* terms, size_t nterms, const yao_circuit* c,
                    const yao_reg* psi0, double* value, double* grad, size_t ngrad);

/* ------------------------------------------------------------ measurement */
/* probs (src/measure.rs:82-122).  nlocs < 0 means None (all 2^n
 * probabilities); otherwise the marginal over locs with locs[0] as the most
 * significant bit of the outcome index. */
int yao_probs(const yao_reg* r, const uint32_t* locs, int32_t nlocs, double* out);
int yao_dm_probs(const yao_dm* d, const uint32_t* locs, int32_t nlocs, double* out);
/* measure_with_postprocess (src/measure.rs:243-274) with the uniform draw r
 * in [0,1) supplied by the caller (yao-rs draws it from its Rng).
 * outcome receives nlocs bits (MSB-first decode, :152-156).  For
 * YAO_POST_REMOVE_MEASURED, *removed receives the new register. */
int yao_measure_with_postprocess(yao_reg* r, const uint32_t* locs, uint32_t nlocs,
                                 int32_t post, uint64_t reset_val, double rand01,
                                 uint8_t* outcome, yao_reg** removed);

/* ---------------------------------------------------------------- batched */
/* Many circuits of uneven size applied in one persistent launch.  Each
 * circuit i runs on its own register regs[i] (all C128 or all C64, one
 * context).  The context keeps the launch's tables (a device buffer and a
 * pinned host buffer, grown as batches need) until yao_ctx_destroy.  No
 * yao-rs counterpart: yao-rs applies circuits one at a time
 * (src/apply.rs:123). */
int yao_batch_apply(const yao_circuit* const* circuits, yao_reg* const* regs, size_t n,
                    int32_t mode, int32_t k);
/* expect_grad (src/ad.rs:75-156) for nsets parameter vectors of one circuit:
 * params is nsets x num_params (row-major, Circuit::parameters() order),
 * values receives nsets energies, grads nsets x num_params.  The circuit's
 * own parameters are not used or changed.  All sets start from psi0. */
int yao_expect_grad_batch(const yao_term* terms, size_t nterms, const yao_circuit* c,
                          const double* params, size_t nsets, const yao_reg* psi0,
                          double* values, double* grads);

/* ------------------------------------------------------- tensor networks */
/* A tensor network: tensors with labelled legs (row-major data, first leg
 * slowest, interleaved complex), a size per label, output labels. */
typedef struct yao_tn yao_tn;

/* Network builders of src/einsum.rs. */
enum yao_tn_kind {
    YAO_TN_EINSUM = 0,         /* circuit_to_einsum (src/einsum.rs:34-119): input legs 0..n-1 open */
    YAO_TN_BOUNDARY = 1,       /* circuit_to_einsum_with_boundary (:151-252): |0> inputs, `pinned` outputs <0| */
    YAO_TN_OVERLAP = 2,        /* circuit_to_overlap (:127-131): <0|U|0> */
    YAO_TN_EXPECTATION = 3,    /* circuit_to_expectation (:274-500): <0|U^dagger O U|0>, single-term O */
    YAO_TN_DM = 4,             /* circuit_to_einsum_dm (:519-665): ket labels 1..n, bra labels negative */
    YAO_TN_EXPECTATION_DM = 5  /* circuit_to_expectation_dm (:673-761): tr(O rho), single-term O */
};
/* The network of a circuit (kind: enum yao_tn_kind).  `pinned` is used by
 * YAO_TN_BOUNDARY, `terms` (exactly one term, or none for the zero
 * operator) by the expectation kinds. */
int yao_tn_from_circuit(const yao_circuit* c, int32_t kind, const uint32_t* pinned, uint32_t npinned,
                        const yao_term* terms, size_t nterms, yao_tn** out);
/* A network from arrays (TensorNetwork { code, tensors, size_dict },
 * src/einsum.rs:16-21): tensor t has ranks[t] legs, its labels next in
 * `labels` and its data next in `data` (2 doubles per element, nelems
 * elements over all tensors); the sizes are label_dims[i] for label_ids[i]. */
int yao_tn_create(size_t ntensors, const uint32_t* ranks, const int64_t* labels, const double* data, size_t nelems,
                  size_t nlabels, const int64_t* label_ids, const uint32_t* label_dims, uint32_t nout,
                  const int64_t* out_labels, yao_tn** out);
void yao_tn_free(yao_tn* tn);
/* Sizes of the arrays yao_tn_export fills: tensors, legs over all tensors,
 * elements over all tensors, output labels, labels with a size. */
int yao_tn_counts(const yao_tn* tn, size_t* ntensors, size_t* nlegs, size_t* nelems, uint32_t* nout,
                  size_t* nlabels);
int yao_tn_export(const yao_tn* tn, uint32_t* ranks, int64_t* labels, double* data, int64_t* out_labels,
                  int64_t* label_ids, uint32_t* label_dims);
/* Elements of the contraction result (product of the output legs' sizes). */
int yao_tn_output_len(const yao_tn* tn, size_t* out);
/* Contracts the network on the context's GPU (src/contractor.rs contract,
 * src/torch_contractor.rs:33 contract on Device::Cuda): pairwise in a greedy
 * order, complex128; `out` receives the result, legs in the order of the
 * output labels, row-major (2 * out_len doubles). */
int yao_tn_contract(yao_ctx* ctx, const yao_tn* tn, double* out, size_t out_len);
/* The same in a given order (src/contractor.rs:20-32 contract_with_tree and
 * contract_dm_with_tree: the contraction tree as its post-order list of
 * pairs).  A network of T tensors takes exactly T - 1 pairs; pair s
 * contracts path[2s] and path[2s + 1], where 0..T-1 are the network's
 * tensors and T + r is the result of pair r < s; every tensor is used once.
 * Paths that break these rules fail with YAO_ERR_INVALID_ARGUMENT before
 * anything reaches the GPU. */
int yao_tn_contract_path(yao_ctx* ctx, const yao_tn* tn, const uint32_t* path, size_t npairs, double* out,
                         size_t out_len);

#ifdef __cplusplus
}
#endif

#endif /* YAO_GPU_H */
