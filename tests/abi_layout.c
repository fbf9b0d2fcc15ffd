/* A C consumer of include/chai_b200.h: compiled as C99 by tests/test_abi.py,
 * it prints the size of every structure of the C ABI and the offset of every
 * field, which the test compares with the ctypes binding (chai_b200/_lib.py). */
#include <stddef.h>
#include <stdio.h>

#include "chai_b200.h"

#define S(T) printf("%s %zu\n", #T, sizeof(T))
#define F(T, f) printf("%s.%s %zu\n", #T, #f, offsetof(T, f))

int main(void)
{
    S(chai_bc); F(chai_bc, kind); F(chai_bc, code); F(chai_bc, version); F(chai_bc, scalar); F(chai_bc, buffer);
    S(chai_stmt); F(chai_stmt, lhs_variable); F(chai_stmt, lhs_version); F(chai_stmt, n_cells); F(chai_stmt, cells);
    S(chai_kernel_arg); F(chai_kernel_arg, kind); F(chai_kernel_arg, prec); F(chai_kernel_arg, variable);
    F(chai_kernel_arg, version); F(chai_kernel_arg, value);
    S(chai_inline_kernel); F(chai_inline_kernel, source); F(chai_inline_kernel, name); F(chai_inline_kernel, n_args);
    F(chai_inline_kernel, args); F(chai_inline_kernel, global_size); F(chai_inline_kernel, local_size);
    S(chai_trace_desc); F(chai_trace_desc, num_traces); F(chai_trace_desc, n_stmts); F(chai_trace_desc, stmts);
    F(chai_trace_desc, hash); F(chai_trace_desc, kernels); F(chai_trace_desc, n_kernels);
    S(chai_buffer_binding); F(chai_buffer_binding, variable); F(chai_buffer_binding, prec);
    F(chai_buffer_binding, width); F(chai_buffer_binding, height); F(chai_buffer_binding, slots);
    F(chai_buffer_binding, buffer);
    S(chai_value_shape); F(chai_value_shape, variable); F(chai_value_shape, version); F(chai_value_shape, prec);
    F(chai_value_shape, slots); F(chai_value_shape, width); F(chai_value_shape, height);
    S(chai_rng_desc); F(chai_rng_desc, variant); F(chai_rng_desc, prec); F(chai_rng_desc, dist);
    F(chai_rng_desc, vec_len); F(chai_rng_desc, seed); F(chai_rng_desc, width); F(chai_rng_desc, height);
    F(chai_rng_desc, slots); F(chai_rng_desc, has_limits); F(chai_rng_desc, min_limit); F(chai_rng_desc, max_limit);
    S(chai_gemm_desc); F(chai_gemm_desc, precision); F(chai_gemm_desc, trans_a); F(chai_gemm_desc, trans_b);
    F(chai_gemm_desc, m); F(chai_gemm_desc, n); F(chai_gemm_desc, k); F(chai_gemm_desc, a); F(chai_gemm_desc, lda);
    F(chai_gemm_desc, b); F(chai_gemm_desc, ldb); F(chai_gemm_desc, c); F(chai_gemm_desc, ldc);
    F(chai_gemm_desc, alpha); F(chai_gemm_desc, beta); F(chai_gemm_desc, batch); F(chai_gemm_desc, stride_a);
    F(chai_gemm_desc, stride_b); F(chai_gemm_desc, stride_c);
    S(chai_gemm_problem); F(chai_gemm_problem, m); F(chai_gemm_problem, n); F(chai_gemm_problem, k);
    F(chai_gemm_problem, a); F(chai_gemm_problem, b); F(chai_gemm_problem, c);
    S(chai_gemm_key); F(chai_gemm_key, m); F(chai_gemm_key, n); F(chai_gemm_key, k); F(chai_gemm_key, precision);
    F(chai_gemm_key, is_gemv);
    S(chai_gemm_cfg); F(chai_gemm_cfg, block_m); F(chai_gemm_cfg, block_n); F(chai_gemm_cfg, block_k);
    F(chai_gemm_cfg, stages); F(chai_gemm_cfg, vec_width); F(chai_gemm_cfg, cluster_m); F(chai_gemm_cfg, cluster_n);
    F(chai_gemm_cfg, group_m); F(chai_gemm_cfg, measured_us);
    return 0;
}
