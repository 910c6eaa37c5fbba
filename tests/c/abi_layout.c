/* Prints the layout of the wire structs of include/yao_gpu.h as seen by a C
 * compiler: one "name value" line per size and field offset.  The Python
 * binding's ctypes mirror must agree with every line. */
#include <stddef.h>
#include <stdio.h>

#include "yao_gpu.h"

#define F(s, f) printf(#s "." #f " %zu\n", offsetof(s, f))

int main(void) {
    printf("yao_element.sizeof %zu\n", sizeof(yao_element));
    F(yao_element, kind);
    F(yao_element, type);
    F(yao_element, ntargets);
    F(yao_element, nctrl);
    F(yao_element, targets);
    F(yao_element, ctrl_locs);
    F(yao_element, ctrl_configs);
    F(yao_element, matrix);
    F(yao_element, matrix_dim);
    F(yao_element, nkraus);
    F(yao_element, is_diagonal);
    F(yao_element, depol_n);
    F(yao_element, nconfigs);
    F(yao_element, reserved);
    F(yao_element, params);
    printf("yao_term.sizeof %zu\n", sizeof(yao_term));
    F(yao_term, coeff_re);
    F(yao_term, coeff_im);
    F(yao_term, nops);
    F(yao_term, reserved);
    F(yao_term, sites);
    F(yao_term, ops);
    printf("abi_version %d\n", YAO_GPU_ABI_VERSION);
    return 0;
}
