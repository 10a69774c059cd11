// Solver kernels of libddagpu: operation codes and launchers.
#pragma once
#include "internal.h"

namespace ddagpu {

enum FieldOp {
    OP_STEP0_CG = 1, OP_STEP0_AA, OP_STEP0_BICG, OP_STEP0_SIMPLE,
    OP_CG1, OP_CG2, OP_CG3,
    OP_AA1, OP_AA2, OP_AA3,
    OP_B_RHO, OP_B_S, OP_B_GH, OP_B_R, OP_B_WW, OP_B_P,
    OP_SIMPLE, OP_ERR, OP_COPY_RS
};

enum ScalarStage {
    SC_STEP0_ERR1 = 1, SC_STEP0_AA, SC_B_RHO1,
    SC_CG1, SC_CG2, SC_AA1, SC_AA2, SC_B1, SC_B2, SC_B3, SC_B4, SC_ERR1,
    SC_START, SC_TOP, SC_FINAL
};

struct FieldArgs {
    size_t N;
    int nrhs;
    int ni, nj, nl;
    const signed char *occ;   // [N], or [nrhs][N] with occ_stride = N
    size_t occ_stride;        // 0: one occupancy shared by every right-hand side
    const int *mv;            // [nmat1]
    const float2 *alpha;      // [nrhs][nmat1]
    int nmat1;
    RhsState *st;             // [nrhs]
    const int *rhs_active;    // [nrhs] or null
    float2 *p, *pmin, *r, *s, *g, *h, *w;  // [nrhs][3][N]
    const double *kinc;       // [nrhs][3]
    const double *einc;       // [nrhs][6]
    double d0;
    float tau;
    // iterative refinement (FP64 solution and residual)
    const float2 *b;          // [nrhs][3][N] right-hand side of the outer system (p_inc)
    float2 *rb;               // [nrhs][3][N] right-hand side of the inner solve (float r)
    double2 *x64;             // [nrhs][3][N] FP64 solution
    const float2 *rhs_in;     // step 0 starts from p = rhs_in instead of p_inc when set
    const int *step_gate;     // OP_COPY_RS runs only when *step_gate == 1 (if set)
};

cudaError_t launch_field_op(int op, const FieldArgs &a, cudaStream_t st);
cudaError_t launch_first_approx(const FieldArgs &a, cudaStream_t st);
// phase tables [nrhs][nj + nl + ni] of the incident field (y, z, x), the values first_approx uses
cudaError_t launch_inc_tables(const FieldArgs &a, float2 *tab, cudaStream_t st);
// step_dev (may be null): read the step number from device memory; `step` then holds
// Max_Step, past which SC_TOP only clears the copy flag
cudaError_t launch_scalar(RhsState *st_, const int *act_in, int *act_out, int nrhs, int stage,
                          int step, double *trace, int trace_len, cudaStream_t st,
                          const int *step_dev = nullptr);
// last node of a graph-recorded iteration: condition = any active && *step_dev <= max_step
cudaError_t launch_loop_control(const int *active, int nrhs, const int *step_dev, int max_step,
                                cudaGraphConditionalHandle h, cudaStream_t st);
cudaError_t launch_step_advance(int *step_dev, cudaStream_t st);
cudaError_t launch_step_set(int *step_dev, int value, cudaStream_t st);
cudaError_t launch_init_state(RhsState *st_, int *active, int nrhs, double err_max, const int *nact,
                              cudaStream_t st);
cudaError_t launch_gated_copy(const FieldArgs &a, int dir, cudaStream_t st);

// refinement passes: 0 x64 = b; 1 r = b - (x64 - alpha conv) with conv in w, error into
// acc[0], inner rhs rb = float(r); 2 x64 += p; 3 p = float(x64); 4 p = rhs_in
cudaError_t launch_refine(int op, const FieldArgs &a, cudaStream_t st);

}  // namespace ddagpu
