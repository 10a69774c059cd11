// Solver vector kernels: the incident dipoles (FirstApproximation, dda_func.cpp:654-689),
// the masked linear combinations of the four iterative methods (LinearComb,
// dda_func.cpp:813-974, and the inline loops of DDA_FFT, dda_func.cpp:1114-1521) and their
// reductions (ldcScalMul 724-755, ldScalMulConj 757-782, ldError 784-811), each fused
// into one pass over the fields with FP64 warp-shuffle reductions.  The scalar kernels
// turn the reductions into the float coefficients the reference applies, on the device.
#include "common.cuh"
#include "internal.h"
#include "solver.h"

namespace ddagpu {

namespace {

DDA_DEV double2 dmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
DDA_DEV double2 ddiv(double2 a, double2 b)
{
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
DDA_DEV float2 fcast(double2 a) { return make_float2((float)a.x, (float)a.y); }

// bilinear product sum over the 3 components (no conjugation), exact float products
DDA_DEV void bil_acc(const float2 (&a)[3], const float2 (&b)[3], double &re, double &im)
{
#pragma unroll
    for (int c = 0; c < 3; c++) {
        re += (double)a[c].x * b[c].x - (double)a[c].y * b[c].y;
        im += (double)a[c].x * b[c].y + (double)a[c].y * b[c].x;
    }
}
DDA_DEV double herm_acc(const float2 (&a)[3], const float2 (&b)[3])
{
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) s += (double)a[c].x * b[c].x + (double)a[c].y * b[c].y;
    return s;
}
DDA_DEV double norm_cell(const float2 (&r)[3])
{
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) s += (double)r[c].x * r[c].x + (double)r[c].y * r[c].y;
    return sqrt(s);
}

DDA_DEV void ld3(const float2 *f, size_t N, size_t q, float2 (&v)[3])
{
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = f[c * N + q];
}
DDA_DEV void st3(float2 *f, size_t N, size_t q, const float2 (&v)[3])
{
#pragma unroll
    for (int c = 0; c < 3; c++) f[c * N + q] = v[c];
}
DDA_DEV void z3(float2 (&v)[3])
{
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = czero();
}
DDA_DEV void axpy3(float2 (&y)[3], float2 a, const float2 (&x)[3])
{
#pragma unroll
    for (int c = 0; c < 3; c++) y[c] = cadd(y[c], cmul(a, x[c]));
}

// A warp takes FB x 32 consecutive cells per pass: lane t has cells q0 + t + 32 k, k < FB,
// so every access of the warp stays one contiguous run and a thread has the loads of its
// FB cells in flight together.
constexpr int FB = 4;
DDA_DEV void occ_batch(const signed char *occ, size_t N, size_t q0, int (&m)[FB])
{
#pragma unroll
    for (int k = 0; k < FB; k++) m[k] = q0 + 32 * k < N ? (int)occ[q0 + 32 * k] : 0;
}
// first cell of this thread and the stride between passes
DDA_DEV size_t fb_first()
{
    const size_t gt = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    return (gt >> 5) * (32 * FB) + (gt & 31);
}
DDA_DEV size_t fb_stride() { return (size_t)gridDim.x * blockDim.x * FB; }

// ------------------------------------------------------------------ field pass
template <int OP>
__global__ void __launch_bounds__(256) field_op(FieldArgs a)
{
    __shared__ double scratch[8 * 4];
    const int rhs = blockIdx.y;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    if (OP == OP_COPY_RS && a.step_gate && *a.step_gate != 1) return;   // first iteration only
    RhsState &S = a.st[rhs];
    const size_t N = a.N, off = (size_t)rhs * 3 * N;
    float2 *p = a.p ? a.p + off : nullptr, *r = a.r ? a.r + off : nullptr;
    float2 *s = a.s ? a.s + off : nullptr, *g = a.g ? a.g + off : nullptr;
    float2 *h = a.h ? a.h + off : nullptr, *w = a.w ? a.w + off : nullptr;
    const float2 cA = S.cA, cB = S.cB, cW = S.cW, c2 = S.c2;
    const float rA = S.rA, rB = S.rB, tau = a.tau;
    const signed char *occ = a.occ + (size_t)rhs * a.occ_stride;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const bool act = a.mv[(int)occ[q]] != 0;
        float2 P[3], R[3], Sv[3], X[3], Y[3];
        if (OP == OP_STEP0_CG) { // s = r; error
            ld3(r, N, q, R);
            st3(s, N, q, R);
            if (act) v[0] += norm_cell(R);
        } else if (OP == OP_STEP0_AA) { // RR_1 = <r,r>_H; error
            ld3(r, N, q, R);
            if (act) { v[0] += herm_acc(R, R); v[1] += norm_cell(R); }
        } else if (OP == OP_STEP0_BICG) { // g = r; s = r; rho_1 = <r,g>
            ld3(r, N, q, R);
            st3(g, N, q, R);
            st3(s, N, q, R);
            if (act) bil_acc(R, R, v[0], v[1]);
        } else if (OP == OP_STEP0_SIMPLE) { // s = p; p = s - r (all cells); error
            ld3(p, N, q, P);
            ld3(r, N, q, R);
            st3(s, N, q, P);
#pragma unroll
            for (int c = 0; c < 3; c++) X[c] = csub(P[c], R[c]);
            st3(p, N, q, X);
            if (act) v[0] += norm_cell(R);
        } else if (OP == OP_CG1) { // <s,W>, <r,s>
            if (act) {
                ld3(s, N, q, Sv); ld3(w, N, q, X); ld3(r, N, q, R);
                bil_acc(Sv, X, v[0], v[1]);
                bil_acc(R, Sv, v[2], v[3]);
            }
        } else if (OP == OP_CG2) { // p -= cA s; r -= cA W; <r,W>; error
            if (act) {
                ld3(p, N, q, P); ld3(s, N, q, Sv); ld3(r, N, q, R); ld3(w, N, q, X);
                const float2 m = make_float2(-cA.x, -cA.y);
                axpy3(P, m, Sv);
                axpy3(R, m, X);
                st3(p, N, q, P);
                st3(r, N, q, R);
                bil_acc(R, X, v[0], v[1]);
                v[2] += norm_cell(R);
            }
        } else if (OP == OP_CG3) { // s = r - cB s
            if (act) {
                ld3(r, N, q, R); ld3(s, N, q, Sv);
#pragma unroll
                for (int c = 0; c < 3; c++) Sv[c] = cadd(R[c], cmul(make_float2(-cB.x, -cB.y), Sv[c]));
                st3(s, N, q, Sv);
            }
        } else if (OP == OP_AA1) { // SS = <s,s>_H
            if (act) { ld3(s, N, q, Sv); v[0] += herm_acc(Sv, Sv); }
        } else if (OP == OP_AA2) { // r += rA W; p += rA s; RR = <r,r>_H; error
            if (act) {
                ld3(p, N, q, P); ld3(s, N, q, Sv); ld3(r, N, q, R); ld3(w, N, q, X);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    R[c] = cadd(R[c], cscale(X[c], rA));
                    P[c] = cadd(P[c], cscale(Sv[c], rA));
                }
                st3(p, N, q, P);
                st3(r, N, q, R);
                v[0] += herm_acc(R, R);
                v[1] += norm_cell(R);
            }
        } else if (OP == OP_AA3) { // s = W + rB s
            if (act) {
                ld3(w, N, q, X); ld3(s, N, q, Sv);
#pragma unroll
                for (int c = 0; c < 3; c++) Sv[c] = cadd(X[c], cscale(Sv[c], rB));
                st3(s, N, q, Sv);
            }
        } else if (OP == OP_B_RHO) { // rho = <r,g>
            if (act) { ld3(r, N, q, R); ld3(g, N, q, X); bil_acc(R, X, v[0], v[1]); }
        } else if (OP == OP_B_S) { // s = r + cB s + c2 h (0 on inactive cells)
            if (act) {
                ld3(r, N, q, R); ld3(s, N, q, Sv); ld3(h, N, q, X);
#pragma unroll
                for (int c = 0; c < 3; c++)
                    Y[c] = cadd(cadd(R[c], cmul(cB, Sv[c])), cmul(c2, X[c]));
            } else {
                z3(Y);
            }
            st3(s, N, q, Y);
        } else if (OP == OP_B_GH) { // <g,h>
            if (act) { ld3(g, N, q, X); ld3(h, N, q, Y); bil_acc(X, Y, v[0], v[1]); }
        } else if (OP == OP_B_R) { // r -= cA h
            if (act) {
                ld3(r, N, q, R); ld3(h, N, q, X);
                axpy3(R, make_float2(-cA.x, -cA.y), X);
                st3(r, N, q, R);
            }
        } else if (OP == OP_B_WW) { // <W,r>, <W,W>
            if (act) {
                ld3(w, N, q, X); ld3(r, N, q, R);
                bil_acc(X, R, v[0], v[1]);
                bil_acc(X, X, v[2], v[3]);
            }
        } else if (OP == OP_B_P) { // p = p - cA s - cW r (0 on inactive); r -= cW W; error
            if (act) {
                ld3(p, N, q, P); ld3(s, N, q, Sv); ld3(r, N, q, R); ld3(w, N, q, X);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    // the 4-vector LinearComb evaluates cv1 + c1 cv2 first, then adds c2 cv3
                    Y[c] = cadd(cmul(make_float2(-cW.x, -cW.y), R[c]),
                                cadd(P[c], cmul(make_float2(-cA.x, -cA.y), Sv[c])));
                }
                axpy3(R, make_float2(-cW.x, -cW.y), X);
                st3(r, N, q, R);
                v[0] += norm_cell(R);
            } else {
                z3(Y);
            }
            st3(p, N, q, Y);
        } else if (OP == OP_SIMPLE) { // r = W - s; p -= tau r on active; p = r = 0 elsewhere
            if (act) {
                ld3(p, N, q, P); ld3(s, N, q, Sv); ld3(w, N, q, X);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    R[c] = csub(X[c], Sv[c]);
                    P[c] = csub(P[c], cscale(R[c], tau));
                }
                v[0] += norm_cell(R);
            } else {
                z3(P);
                z3(R);
            }
            st3(p, N, q, P);
            st3(r, N, q, R);
        } else if (OP == OP_ERR) { // error only
            if (act) { ld3(r, N, q, R); v[0] += norm_cell(R); }
        } else if (OP == OP_COPY_RS) { // s = r (CG step 0, deferred to the first iteration)
            ld3(r, N, q, R);
            st3(s, N, q, R);
        }
    }
    constexpr int NV = (OP == OP_CG1 || OP == OP_B_WW) ? 4
                     : (OP == OP_CG2)                              ? 3
                     : (OP == OP_STEP0_AA || OP == OP_STEP0_BICG || OP == OP_AA2 ||
                        OP == OP_B_RHO || OP == OP_B_GH)           ? 2
                     : (OP == OP_STEP0_CG || OP == OP_STEP0_SIMPLE || OP == OP_AA1 ||
                        OP == OP_B_P || OP == OP_SIMPLE || OP == OP_ERR) ? 1
                                                                    : 0;
    constexpr int NVA = (NV > 0) ? NV : 1;
    if (NV > 0) {
        double t[NVA];
#pragma unroll
        for (int k = 0; k < NVA; k++) t[k] = v[k];
        block_sum_atomic<NVA>(t, scratch, S.acc);
    }
}

// ------------------------------------------------------------ incident dipoles
// p = alpha_m exp(i k.(r - c)) E_inc on active cells, c = (n-1) d0 / 2 per axis; the
// phase is separable: entry e of the tables [nj] y, [nl] z, [ni] x is exp(i k_a (x_a - c_a)).
DDA_DEV float2 inc_phase(const FieldArgs &a, const double *k, int e)
{
    const int ni = a.ni, nj = a.nj, nl = a.nl;
    const double cx = (ni - 1) * a.d0 / 2, cy = (nj - 1) * a.d0 / 2, cz = (nl - 1) * a.d0 / 2;
    const double ph = e < nj        ? k[1] * (e * a.d0 - cy)
                    : e < nj + nl   ? k[2] * ((e - nj) * a.d0 - cz)
                                    : k[0] * ((e - nj - nl) * a.d0 - cx);
    return expi_reduced(ph);
}

// The phase tables of every right-hand side, [nrhs][nj + nl + ni], for the forward pass that
// computes the incident dipoles itself (step 0 of a solve on the compile-time-sized passes).
__global__ void __launch_bounds__(256) inc_tables(FieldArgs a, float2 *tab)
{
    const int rhs = blockIdx.x, n = a.nj + a.nl + a.ni;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    for (int e = threadIdx.x; e < n; e += blockDim.x) tab[(size_t)rhs * n + e] = inc_phase(a, a.kinc + 3 * rhs, e);
}

__global__ void __launch_bounds__(256) first_approx(FieldArgs a)
{
    extern __shared__ float2 tab[];   // [nj] y, [nl] z, then [ni] x
    const int rhs = blockIdx.y;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    const int ni = a.ni, nj = a.nj, nl = a.nl;
    const double *k = a.kinc + 3 * rhs, *E = a.einc + 6 * rhs;
    for (int e = threadIdx.x; e < nj + nl + ni; e += blockDim.x) tab[e] = inc_phase(a, k, e);
    __syncthreads();
    const size_t N = a.N, off = (size_t)rhs * 3 * N;
    const float2 *al = a.alpha + (size_t)rhs * a.nmat1;
    const signed char *occ = a.occ + (size_t)rhs * a.occ_stride;
    const float2 Ef[3] = {make_float2((float)E[0], (float)E[1]), make_float2((float)E[2], (float)E[3]),
                          make_float2((float)E[4], (float)E[5])};
    for (size_t q0 = fb_first(); q0 < N; q0 += fb_stride()) {
        int mk[FB];
        occ_batch(occ, N, q0, mk);
        // lattice position of the first cell; the others are 32 cells further along l
        // (wrapping rows)
        const unsigned q0u = (unsigned)q0, row = q0u / (unsigned)nl;   // lattices below 2^32 cells
        int l = (int)(q0u - row * (unsigned)nl), j = (int)(row % (unsigned)nj), i = (int)(row / (unsigned)nj);
#pragma unroll
        for (int k = 0; k < FB; k++) {
            const size_t q = q0 + 32 * k;
            if (q >= N) break;
            const int m = mk[k];
            float2 out[3];
            if (a.mv[m]) {
                const float2 ph = cmul(cmul(tab[nj + nl + i], tab[j]), tab[nj + l]);
                const float2 c1 = cmul(ph, al[m]);
#pragma unroll
                for (int c = 0; c < 3; c++) out[c] = cmul(c1, Ef[c]);
            } else {
                z3(out);
            }
            st3(a.p + off, N, q, out);
            for (l += 32; l >= nl; l -= nl) {
                if (++j == nj) {
                    j = 0;
                    ++i;
                }
            }
        }
    }
}

// ---------------------------------------------------------------- scalar stages
__device__ float2 fmul_ref(float2 a, float2 b)
{
    // float complex product without contraction, as the reference's cplx operator*
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

__global__ void scalar_stage(RhsState *st, const int *rhs_active_in, int *rhs_active, int nrhs,
                             int stage, int step_arg, const int *step_dev, double *trace,
                             int trace_len)
{
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    // with step_dev the step comes from device memory and step_arg holds Max_Step
    const int step = step_dev ? *step_dev : step_arg;
    if (rhs >= nrhs) return;
    RhsState &S = st[rhs];
    const bool run = rhs_active_in ? rhs_active_in[rhs] != 0 : true;
    if (!run) return;
    double *A = S.acc;
    const double nact = (double)(S.nact > 0 ? S.nact : 1);
    switch (stage) {
    case SC_STEP0_ERR1: // error in acc[0]
        S.err = A[0] / nact;
        break;
    case SC_STEP0_AA: // RR_1 = acc0, error acc1
        S.RR1 = A[0];
        S.err = A[1] / nact;
        break;
    case SC_B_RHO1: // rho_1 = rho = <r,g>
        S.rho1 = make_double2(A[0], A[1]);
        S.rho = S.rho1;
        break;
    case SC_CG1: // den = <s,W>; a = <r,s>/den
        S.den = make_double2(A[0], A[1]);
        S.ldA = ddiv(make_double2(A[2], A[3]), S.den);
        S.cA = fcast(S.ldA);
        break;
    case SC_CG2: // b = <r,W>/den; error
        S.cB = fcast(ddiv(make_double2(A[0], A[1]), S.den));
        S.err = A[2] / nact;
        break;
    case SC_AA1: // rA = -RR_1/SS
        S.rA = (float)(-S.RR1 / A[0]);
        break;
    case SC_AA2: { // rB = RR/RR_1; RR_1 = RR; error
        const double RR = A[0];
        S.rB = (float)(RR / S.RR1);
        S.RR1 = RR;
        S.err = A[1] / nact;
        break;
    }
    case SC_B1: { // rho; b = (rho a)/(rho_1 w); c2 = -(cB cW) in float
        S.rho = make_double2(A[0], A[1]);
        const double2 b = ddiv(dmul(S.rho, S.ldA), dmul(S.rho1, S.ldW));
        S.cB = fcast(b);
        const float2 t = fmul_ref(S.cB, S.cW);
        S.c2 = make_float2(-t.x, -t.y);
        break;
    }
    case SC_B2: // a = rho/<g,h>
        S.ldA = ddiv(S.rho, make_double2(A[0], A[1]));
        S.cA = fcast(S.ldA);
        break;
    case SC_B3: // w = <W,r>/<W,W>
        S.ldW = ddiv(make_double2(A[0], A[1]), make_double2(A[2], A[3]));
        S.cW = fcast(S.ldW);
        break;
    case SC_B4: // error; rho_1 = rho
        S.err = A[0] / nact;
        S.rho1 = S.rho;
        break;
    case SC_ERR1:
        S.err = A[0] / nact;
        break;
    case SC_START: // after step 0: best iterate is step 0 (dda_func.cpp:1280-1293)
        S.err_min = S.err;
        S.step_min = 0;
        S.steps = 0;
        S.restored = 0;
        break;
    case SC_TOP: // dda_func.cpp:1301-1313
        S.need_copy = 0;
        if (step_dev && step > step_arg) {
            // a graph-recorded iteration past Max_Step (step_arg): the host loop has ended
            // here, so only the copy flag is cleared
        } else if (S.err <= S.err_max) {
            S.active = 0;
        } else if (step == 1) {
            // the step-0 iterate is the best one so far (dda_func.cpp:1286-1293); it is
            // stored only now, when an iteration is about to overwrite it
            S.need_copy = 1;
        } else if (S.err < S.err_min) {
            S.err_min = S.err;
            S.step_min = step - 1;
            S.need_copy = 1;
        }
        break;
    case SC_FINAL: // dda_func.cpp:1537-1548
        S.need_copy = (S.err > S.err_min) ? 1 : 0;
        S.restored = S.need_copy;
        break;
    }
    for (int k = 0; k < kAcc; k++) A[k] = 0.0;
    const bool new_err = stage == SC_STEP0_ERR1 || stage == SC_STEP0_AA || stage == SC_CG2 ||
                         stage == SC_AA2 || stage == SC_B4 || stage == SC_ERR1;
    if (new_err) {
        if (trace && step < trace_len) trace[(size_t)rhs * trace_len + step] = S.err;
        S.steps = step;
    }
    if (rhs_active) rhs_active[rhs] = S.active;
}

// need_copy-gated copies (best iterate p -> p_min, rollback p_min -> p)
__global__ void __launch_bounds__(256) gated_copy(FieldArgs a, int dir)
{
    const int rhs = blockIdx.y;
    const RhsState &S = a.st[rhs];
    if (!S.need_copy) return;
    const size_t n3 = 3 * a.N, off = (size_t)rhs * n3;
    const float4 *src = reinterpret_cast<const float4 *>((dir ? a.pmin : a.p) + off);
    float4 *dst = reinterpret_cast<float4 *>((dir ? a.p : a.pmin) + off);
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n3 / 2;
         q += (size_t)gridDim.x * blockDim.x)
        dst[q] = src[q];
}

// Iterative refinement passes over all 3 components of every cell.
__global__ void __launch_bounds__(256) refine_op(FieldArgs a, int op)
{
    __shared__ double scratch[8];
    const int rhs = blockIdx.y;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    const size_t N = a.N, off = (size_t)rhs * 3 * N;
    double v[1] = {0.0};
    const signed char *occ = a.occ + (size_t)rhs * a.occ_stride;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const int m = occ[q];
        const bool act = a.mv[m] != 0;
        if (op == 0) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float2 x = a.b[off + c * N + q];
                a.x64[off + c * N + q] = make_double2(x.x, x.y);
            }
        } else if (op == 1) {
            const float2 al = a.alpha[(size_t)rhs * a.nmat1 + m];
            double nrm = 0.0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t o = off + c * N + q;
                double rr = 0.0, ri = 0.0;
                if (act) {
                    const float2 cv = a.w[o], bb = a.b[o];
                    const double2 x = a.x64[o];
                    // A x = x - alpha conv, r = b - A x
                    const double acr = (double)al.x * cv.x - (double)al.y * cv.y;
                    const double aci = (double)al.x * cv.y + (double)al.y * cv.x;
                    rr = (double)bb.x - (x.x - acr);
                    ri = (double)bb.y - (x.y - aci);
                }
                nrm += rr * rr + ri * ri;
                a.rb[o] = make_float2((float)rr, (float)ri);
            }
            if (act) v[0] += sqrt(nrm);
        } else if (op == 2) {
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const size_t o = off + c * N + q;
                    const float2 d = a.p[o];
                    double2 x = a.x64[o];
                    x.x += d.x;
                    x.y += d.y;
                    a.x64[o] = x;
                }
            }
        } else if (op == 3) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t o = off + c * N + q;
                const double2 x = a.x64[o];
                a.p[o] = make_float2((float)x.x, (float)x.y);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t o = off + c * N + q;
                a.p[o] = act ? a.rhs_in[o] : czero();
            }
        }
    }
    if (op == 1) block_sum_atomic<1>(v, scratch, a.st[rhs].acc);
}

}  // namespace

cudaError_t launch_refine(int op, const FieldArgs &a, cudaStream_t st)
{
    const unsigned bx = (unsigned)((a.N + 1023) / 1024);
    refine_op<<<dim3(bx < 1 ? 1 : bx, a.nrhs), 256, 0, st>>>(a, op);
    return cudaGetLastError();
}

// Blocks of field_op<OP> resident on the whole GPU at once (looked up once per operation).
template <int OP>
unsigned field_op_wave()
{
    static unsigned w = 0;
    if (!w) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, field_op<OP>, 256, 0);
        w = (unsigned)(sms > 0 && per > 0 ? sms * per : 1);
    }
    return w;
}

template <int OP>
void launch_field_op_t(const FieldArgs &a, cudaStream_t st)
{
    // the residual norm of step 0 (a read of r on active cells and one sum) runs one
    // resident wave of blocks over all right-hand sides: each thread strides over several
    // cells, so the block reduction is amortised (85 vs 104 us at 128 x 64^3); the other
    // passes keep four cells per thread, which measured faster for them (BiCGStab at
    // 32 x 64^3: 465 vs 474 ms)
    unsigned bx = (unsigned)((a.N + 1023) / 1024);
    if (OP == OP_ERR) {
        const unsigned want = field_op_wave<OP>() / (unsigned)(a.nrhs > 0 ? a.nrhs : 1);
        if (bx > want) bx = want;
    }
    field_op<OP><<<dim3(bx < 1 ? 1 : bx, a.nrhs), 256, 0, st>>>(a);
}

cudaError_t launch_field_op(int op, const FieldArgs &a, cudaStream_t st)
{
    switch (op) {
#define CASE(X) case X: launch_field_op_t<X>(a, st); break;
        CASE(OP_STEP0_CG) CASE(OP_STEP0_AA) CASE(OP_STEP0_BICG) CASE(OP_STEP0_SIMPLE)
        CASE(OP_CG1) CASE(OP_CG2) CASE(OP_CG3) CASE(OP_AA1) CASE(OP_AA2) CASE(OP_AA3)
        CASE(OP_B_RHO) CASE(OP_B_S) CASE(OP_B_GH) CASE(OP_B_R) CASE(OP_B_WW) CASE(OP_B_P)
        CASE(OP_SIMPLE) CASE(OP_ERR) CASE(OP_COPY_RS)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_inc_tables(const FieldArgs &a, float2 *tab, cudaStream_t st)
{
    inc_tables<<<a.nrhs, 256, 0, st>>>(a, tab);
    return cudaGetLastError();
}

cudaError_t launch_first_approx(const FieldArgs &a, cudaStream_t st)
{
    const unsigned bx = (unsigned)((a.N + 256 * FB - 1) / (256 * FB));
    first_approx<<<dim3(bx < 1 ? 1 : bx, a.nrhs), 256, (a.ni + a.nj + a.nl) * sizeof(float2), st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_scalar(RhsState *st_, const int *act_in, int *act_out, int nrhs, int stage,
                          int step, double *trace, int trace_len, cudaStream_t st,
                          const int *step_dev)
{
    scalar_stage<<<(nrhs + 127) / 128, 128, 0, st>>>(st_, act_in, act_out, nrhs, stage, step, step_dev,
                                                     trace, trace_len);
    return cudaGetLastError();
}

// Last kernel of one iteration of a solve recorded in a CUDA graph, after the convergence
// test of the next step: keep looping while some right-hand side is active and the step
// has not passed Max_Step (the host loop's test, dda_func.cpp:1301-1313).
__global__ void __launch_bounds__(256) loop_control(const int *active, int nrhs, const int *step_dev,
                                                    int max_step, cudaGraphConditionalHandle h)
{
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    int mine = 0;
    for (int r = threadIdx.x; r < nrhs; r += blockDim.x) mine |= active[r] != 0;
    if (mine) atomicOr(&any, 1);
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(h, (any && *step_dev <= max_step) ? 1u : 0u);
}

// ++*step_dev, or *step_dev = value
__global__ void step_advance(int *step_dev, int set, int value)
{
    *step_dev = set ? value : *step_dev + 1;
}

cudaError_t launch_step_advance(int *step_dev, cudaStream_t st)
{
    step_advance<<<1, 1, 0, st>>>(step_dev, 0, 0);
    return cudaGetLastError();
}

cudaError_t launch_step_set(int *step_dev, int value, cudaStream_t st)
{
    step_advance<<<1, 1, 0, st>>>(step_dev, 1, value);
    return cudaGetLastError();
}

// Fresh solver state for a solve recorded in a graph (the host loop uploads it instead):
// all scalars zero, the threshold, active, and the active-cell count of each right-hand side.
__global__ void init_state(RhsState *st, int *active, int nrhs, double err_max, const int *nact)
{
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    if (rhs >= nrhs) return;
    RhsState S;
    memset(&S, 0, sizeof S);
    S.err_max = err_max;
    S.active = 1;
    S.nact = nact[rhs];
    st[rhs] = S;
    active[rhs] = 1;
}

cudaError_t launch_init_state(RhsState *st_, int *active, int nrhs, double err_max, const int *nact,
                              cudaStream_t st)
{
    init_state<<<(nrhs + 127) / 128, 128, 0, st>>>(st_, active, nrhs, err_max, nact);
    return cudaGetLastError();
}

cudaError_t launch_loop_control(const int *active, int nrhs, const int *step_dev, int max_step,
                                cudaGraphConditionalHandle h, cudaStream_t st)
{
    loop_control<<<1, 256, 0, st>>>(active, nrhs, step_dev, max_step, h);
    return cudaGetLastError();
}

cudaError_t launch_gated_copy(const FieldArgs &a, int dir, cudaStream_t st)
{
    // most right-hand sides copy nothing at a given step: a capped grid (grid-stride loop)
    // keeps the launch of the idle blocks cheap
    unsigned bx = (unsigned)((3 * a.N / 2 + 1023) / 1024);
    const unsigned cap = (unsigned)(4096 / (a.nrhs > 0 ? a.nrhs : 1));
    if (bx > (cap < 8 ? 8 : cap)) bx = cap < 8 ? 8 : cap;
    gated_copy<<<dim3(bx < 1 ? 1 : bx, a.nrhs), 256, 0, st>>>(a, dir);
    return cudaGetLastError();
}

}  // namespace ddagpu
