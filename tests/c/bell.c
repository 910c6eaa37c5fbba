/* A C caller of the library, compiled against include/yao_gpu.h alone: a
 * Bell pair (H on loc 0, CNOT 0 -> 1) on a 2-qubit register, then <Z0 Z1>
 * and the probabilities.  Prints the four amplitudes, the expectation value
 * and the probabilities; exits non-zero on any failed call. */
#include <stdio.h>
#include <stdint.h>

#include "yao_gpu.h"

#define CK(x)                                                              \
    do {                                                                   \
        int s_ = (x);                                                      \
        if (s_ != YAO_OK) {                                                \
            fprintf(stderr, "%s -> %d: %s\n", #x, s_, yao_last_error());   \
            return 1;                                                      \
        }                                                                  \
    } while (0)

int main(void) {
    yao_ctx* ctx = NULL;
    CK(yao_ctx_create(0, &ctx));
    const uint32_t dims[2] = {2, 2};
    const uint32_t t0 = 0, t1 = 1, c0 = 0;
    yao_element els[2] = {{0}, {0}};
    els[0].kind = YAO_ELEM_GATE;
    els[0].type = YAO_GATE_H;
    els[0].ntargets = 1;
    els[0].targets = &t0;
    els[1].kind = YAO_ELEM_GATE;
    els[1].type = YAO_GATE_X;
    els[1].ntargets = 1;
    els[1].targets = &t1;
    els[1].nctrl = 1;
    els[1].ctrl_locs = &c0;
    yao_circuit* c = NULL;
    int32_t ce = 0;
    CK(yao_circuit_create(dims, 2, els, 2, &c, &ce));
    yao_reg* r = NULL;
    CK(yao_reg_zero_state(ctx, 2, YAO_C128, &r));
    CK(yao_apply_inplace(c, r));
    double amps[8];
    CK(yao_reg_to_host(r, amps));
    const uint32_t sites[2] = {0, 1};
    const int32_t ops[2] = {YAO_OP_Z, YAO_OP_Z};
    yao_term zz = {1.0, 0.0, 2, 0, sites, ops};
    double e[2];
    CK(yao_expect_arrayreg(r, &zz, 1, e));
    double p[4];
    CK(yao_probs(r, NULL, -1, p));
    for (int i = 0; i < 4; i++) printf("amp %d %.17g %.17g\n", i, amps[2 * i], amps[2 * i + 1]);
    printf("zz %.17g %.17g\n", e[0], e[1]);
    for (int i = 0; i < 4; i++) printf("prob %d %.17g\n", i, p[i]);
    yao_reg_free(r);
    yao_circuit_free(c);
    CK(yao_ctx_destroy(ctx));
    return 0;
}
