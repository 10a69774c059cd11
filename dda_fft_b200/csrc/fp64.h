// FP64 solve of one polarisation (fp64.cu): the reference's DDA_FFT in double on the GPU,
// the oracle solve of the precision pattern.
#pragma once
#include <functional>

#include "internal.h"

namespace ddagpu {

// FP64 octant of the Green tensor FFT, [comp][kx][ky][kz] for k in [0, n]^3 (green.cu)
cudaError_t green_build_octant64(int ni, int nj, int nl, double kd, double2 *out, cudaStream_t st);

// Device buffers of the FP64 solve for one lattice, built on first use and kept.
struct Fp64Buffers {
    int ni = 0, nj = 0, nl = 0;
    double kd = 0;
    double2 *g = nullptr, *tw = nullptr, *work = nullptr;
    double2 *p = nullptr, *pmin = nullptr, *r = nullptr, *s = nullptr, *gg = nullptr, *h = nullptr,
            *w = nullptr, *b = nullptr, *alpha = nullptr;
    double *acc = nullptr;
    ~Fp64Buffers();
    void release();
    cudaError_t ensure(int ni, int nj, int nl, double kd, cudaStream_t st);
};

struct Fp64Problem {
    int solver;               // 0 CG, 1 AA*, 2 BiCGStab, 3 simple iteration
    double tau;
    int nmat1;
    const double2 *alpha;     // host [nmat1]
    const signed char *occ;   // device [N] (the context's occupancy)
    const int *mv;            // device [nmat1]
    int nact;
    double d0;
    double kinc[3], einc[6];
    const double2 *rhs;       // host [3][N] or null (b = p_inc)
    const double2 *x0;        // host [3][N] or null (start from b)
    int max_step;
    double err_max;
    int ndir;
    const double *ksc;        // host [ndir][3]
};

struct Fp64Result {
    int steps = 0, step_min = -1, rolled_back = 0, matvecs = 0;
    double err = 0, err_min = 0;
    double cabs = 0, cext = 0;
    double *esc = nullptr;    // host [ndir][6]
    double2 *p = nullptr;     // host [3][N] or null
    double *trace = nullptr;  // host, trace_len entries, or null
    int trace_len = 0;
};

cudaError_t solve_fp64(Fp64Buffers &B, const Fp64Problem &P, cudaStream_t st, Fp64Result &R,
                       long long *launches);

// ---- mixed precision: FP64 fields, scalars and residuals around the FP32 FFT matvec

// One right-hand side's lattice as the FP64 field kernels see it (device pointers).
struct Field64View {
    size_t N;
    int ni, nj, nl;
    const signed char *occ;   // [N]
    const int *mv;            // [nmat1]
    const double2 *alpha;     // [nmat1]
};

// out = alpha_m exp(i k.(r - c)) E on active cells (FirstApproximation in FP64), 0 elsewhere;
// from_f32 (may be null): out = the float field on active cells instead
cudaError_t f64_right_hand_side(const Field64View &f, double d0, const double *kinc,
                                const double *einc, const float2 *from_f32, double2 *out,
                                cudaStream_t st);

// Iterative refinement whose inner solver is the reference's CG (COCG, dda_func.cpp:
// 1137-1138, 1359-1371) with FP64 fields and FP64 scalars (no float casts), every
// convolution on the FP32 FFT passes.  The true residual b - (x - alpha G*x) is computed
// when the updated residual has fallen to inner_rel times the last true one, meets
// Error_max, or after inner_max_step iterations; unless it meets Error_max, CG restarts
// from the current FP64 solution with the true residual (a fresh search direction).
// Restarting matters: the FP64 reductions sum in a varying order, so runs differ in their
// last bits, and COCG's occasional near-breakdown steps (very large coefficients) can
// then inject FP32 matvec error far above the residual; keeping the old direction after
// such a step made the iteration diverge, a restart does not.  Stops when a true residual
// meets Error_max or after max_outer outer steps; the best true-residual iterate is kept.
struct MixedCgBuffers {
    size_t n3 = 0;
    double2 *x = nullptr, *r = nullptr, *s = nullptr, *w = nullptr, *b = nullptr, *best = nullptr,
            *alpha = nullptr;
    double *acc = nullptr;
    ~MixedCgBuffers();
    void release();
    cudaError_t ensure(size_t n3);
};

struct MixedCgResult {
    int outer = 0, iterations = 0, matvecs = 0;
    double err = 0;
    double history[64] = {};
};

// conv(src, out): out = G * src on the lattice (FP32 passes, raw convolution)
using ConvFn = std::function<cudaError_t(const float2 *src, float2 *out)>;

// B.b holds the FP64 right-hand side; f.alpha must point at B.alpha (filled from
// alpha_host); three float buffers of 3N are scratch.  Leaves x in B.x and float(x) in p32.
cudaError_t mixed_cg(MixedCgBuffers &B, const Field64View &f, const double2 *alpha_host, int nmat1,
                     int nact, double err_max, int max_outer, double inner_rel, int inner_max_step,
                     const ConvFn &conv, float2 *s32, float2 *conv32, float2 *x32, float2 *p32,
                     cudaStream_t st, MixedCgResult &R, long long *launches);

}  // namespace ddagpu
