/*
 * oracle.h — CPU restatement of yao-rs's simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: the tests, the smoke
 * check and the CPU-baseline leg of the benchmark call it to produce the
 * numbers the CUDA library must match.  Nothing in the product links or
 * calls it.
 *
 * It restates the Rust loops of yao-rs one to one (same loop order, same
 * operation order, num_complex's (ac-bd, ad+bc) multiply, no FMA: built with
 * -ffp-contract=off), so its outputs are bit-identical to the Rust code's
 * for the same inputs.  Pinned against the golden vectors committed by
 * yao-rs (tests/data/<name>.json), see tests/test_oracle_golden.py.
 *
 * States are interleaved {re, im} doubles.
 */
#ifndef YAO_ORACLE_H
#define YAO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/yao_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* bitbasis (bitbasis/src/iterate_control.rs, bit_ops.rs) */
typedef struct orc_iterctl {
    uint64_t n;
    uint64_t base;
    int32_t nchunks;
    int32_t pad;
    uint64_t masks[64];
    uint64_t factors[64];
} orc_iterctl;

int orc_itercontrol(uint32_t nbits, const uint64_t* positions, const uint64_t* configs,
                    uint32_t npos, orc_iterctl* out);
uint64_t orc_itercontrol_get(const orc_iterctl* ic, uint64_t k);
int orc_group_shift(uint32_t nbits, const uint64_t* positions, uint32_t npos,
                    uint64_t* masks, uint64_t* factors, int32_t* nchunks);
int orc_controller(const uint64_t* cbits, const uint64_t* cvals, uint32_t n, uint64_t basis);
uint64_t orc_bmask(const uint64_t* positions, uint32_t n);
uint64_t orc_bmask_range(uint64_t start, uint64_t stop);
uint64_t orc_swapbits(uint64_t b, uint64_t i, uint64_t j);
uint64_t orc_breflect(uint64_t b, uint64_t nbits);
uint64_t orc_neg(uint64_t b, uint64_t nbits);
uint64_t orc_btruncate(uint64_t b, uint64_t n);

/* instruct_qubit.rs (all take the yao-rs loc convention, loc 0 = MSB) */
void orc_instruct_x(double* st, uint32_t nbits, uint32_t loc);
void orc_instruct_x_controlled(double* st, uint32_t nbits, uint32_t loc, const uint64_t* ctrl_locs,
                               const uint64_t* ctrl_bits, uint32_t nctrl);
void orc_instruct_1q(double* st, uint32_t nbits, uint32_t loc, const double* m /* a,b,c,d */);
void orc_instruct_1q_diag(double* st, uint32_t nbits, uint32_t loc, const double* d /* d0,d1 */);
void orc_instruct_2q(double* st, uint32_t nbits, const uint64_t* locs, const double* gate);
void orc_instruct_2q_diag(double* st, uint32_t nbits, const uint64_t* locs, const double* diag);
void orc_instruct_swap(double* st, uint32_t nbits, const uint64_t* locs);
void orc_instruct_nq(double* st, uint32_t nbits, const uint64_t* locs, uint32_t nlocs,
                     const double* gate, const uint64_t* ctrl_locs, const uint64_t* ctrl_bits,
                     uint32_t nctrl);
void orc_instruct_1q_controlled(double* st, uint32_t nbits, uint32_t loc, const double* m,
                                const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl);
void orc_instruct_2q_controlled(double* st, uint32_t nbits, const uint64_t* locs, const double* gate,
                                const uint64_t* ctrl_locs, const uint64_t* ctrl_bits, uint32_t nctrl);
void orc_instruct_1q_diag_controlled(double* st, uint32_t nbits, uint32_t loc, const double* d,
                                     const uint64_t* ctrl_locs, const uint64_t* ctrl_bits,
                                     uint32_t nctrl);
void orc_instruct_2q_diag_controlled(double* st, uint32_t nbits, const uint64_t* locs,
                                     const double* diag, const uint64_t* ctrl_locs,
                                     const uint64_t* ctrl_bits, uint32_t nctrl);

/* gate.rs */
int orc_gate_matrix(int32_t gate, const double* params, double* out, uint32_t* dim);
int orc_gate_is_diagonal(int32_t gate);
int orc_gate_num_params(int32_t gate);
int orc_gate_generator(int32_t gate, uint32_t i, double* out, uint32_t* dim);

/* noise.rs */
int orc_noise_kraus(const yao_element* ch, double* out, uint32_t max_kraus, uint32_t* nkraus,
                    uint32_t* dim);
int orc_noise_superop(const yao_element* ch, double* out, uint32_t* dim2);

/* register.rs / apply.rs (elements use the C ABI wire format) */
int orc_apply_inplace(uint32_t nbits, const yao_element* elems, size_t n, double* st);
void orc_deterministic_state(uint32_t nbits, double* st);
double orc_norm(uint32_t nbits, const double* st);
double orc_fidelity(uint32_t nbits, const double* a, const double* b);

/* density_matrix.rs */
void orc_dm_from_reg(uint32_t nbits, const double* psi, double* rho);
int orc_dm_apply(uint32_t nbits, const yao_element* elems, size_t n, double* rho);
void orc_dm_trace(uint32_t nbits, const double* rho, double* out);
double orc_dm_purity(uint32_t nbits, const double* rho);
void orc_dm_partial_tr(uint32_t nbits, const double* rho, const uint32_t* traced, uint32_t ntraced,
                       double* out);

/* expect.rs / ad.rs */
void orc_expect_arrayreg(uint32_t nbits, const double* psi, const yao_term* terms, size_t nterms,
                         double* out);
void orc_expect_dm(uint32_t nbits, const double* rho, const yao_term* terms, size_t nterms,
                   double* out);
int orc_expect_grad(uint32_t nbits, const yao_term* terms, size_t nterms, const yao_element* elems,
                    size_t nelems, const double* psi0, double* value, double* grad, size_t ngrad);

/* measure.rs */
void orc_probs(uint32_t nbits, const double* psi, const uint32_t* locs, int32_t nlocs, double* out);
void orc_dm_probs(uint32_t nbits, const double* rho, const uint32_t* locs, int32_t nlocs, double* out);
uint64_t orc_sample_from_probs(const double* probs, uint64_t n, double r);
int orc_measure_with_postprocess(uint32_t nbits, double* psi, const uint32_t* locs, uint32_t nlocs,
                                 int32_t post, uint64_t reset_val, double r, uint8_t* outcome,
                                 double* removed_out);

#ifdef __cplusplus
}
#endif

#endif
