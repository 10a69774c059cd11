// Internal types shared by the kernels and the host driver of libddagpu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ddagpu {

// Maximum lattice edge per axis handled by the fused FFT passes (powers of two).
constexpr int kMaxEdge = 128;
constexpr int kMinEdge = 2;
constexpr int kMaxMaterials = 255;   // occupancy bytes index materials 0..255
constexpr int kAcc = 8;              // FP64 reduction slots per right-hand side

// Per right-hand-side solver scalars, resident on the device.  The reference keeps
// these in long double and casts each coefficient to float before use
// (dda_func.cpp:1219,1260,1319,1362,1368,1375,1381,1424,1464); here the full-precision
// values are FP64 and the applied coefficients are the float casts.
struct RhsState {
    double acc[kAcc];       // reduction accumulators, consumed and zeroed by scalar kernels
    double2 ldA, ldW, rho1, rho, den;  // complex scalars of CG / BiCGStab
    double RR1;             // AA*: <r, r>_H of the previous step
    float2 cA, cB, cW, c2;  // float coefficients currently applied
    float rA, rB;           // AA* real coefficients
    double err, err_min;    // mean residual norm (ldError) and best so far
    double err_max;         // stopping threshold (float value of Error_max)
    int step_min;           // step of the best iterate
    int active;             // 1 while iterating
    int need_copy;          // 1: copy p -> p_min at this step
    int restored;           // 1: final p was replaced by p_min
    int steps;              // last completed step
    int nact;               // active cells
};

// Geometry of one lattice and its device-resident tables.
struct Lat {
    int ni, nj, nl;
    size_t N;               // ni * nj * nl
    const float2 *tw_i, *tw_j, *tw_l;   // [W_n^k, k<n ; W_2n^j, j<n] per axis
};

// Epilogue of the inverse pass: out = sv * v - a_m * conv on active cells, 0 elsewhere;
// mode 0 writes conv unchanged (plain convolution).
struct Epilogue {
    int mode;               // 0 raw convolution, 1 masked solver form
    int conj;               // use conj(alpha)
    float sv;               // scale of v
    const float2 *v;        // field v, same layout as out (may be null if sv == 0)
    const signed char *occ; // [N] material per cell (per right-hand side if occ_stride)
    size_t occ_stride;      // bytes between the occupancies of consecutive right-hand sides
    const float2 *alpha;    // [nrhs][nmat1] polarisability per material
    const int *mv;          // [nmat1] active material flags
    int nmat1;              // materials including index 0
};

struct MatvecArgs {
    Lat L;
    int nrhs;
    const float2 *src;      // [nrhs][3][N] input field
    size_t fstride;         // 3 N
    float2 *work;           // [nrhs][3][ni][2nj][2nl]
    size_t wstride;
    const float2 *ahat;     // octant Green tensor [ni+1][nj+1][nl+1][6] (z in parity order)
    int conj;               // use conj(Ahat)
    float2 *out;            // [nrhs][3][N]
    Epilogue ep;
    const int *rhs_active;  // [nrhs] or null
    int tile_x;             // columns per CTA of the x pass (generic kernels)
    int rows_g;             // rows per staging group of the y/z passes (generic kernels)
    int fast;               // 1: compile-time-sized kernels of matvec_fast.cu
    int fx, fyz;            // launch variants of the fast x pass (0..5) and y/z passes (0..2)
    int *err;               // device flag set by a kernel whose bounded wait gave up (or null)
    const void *tmaps;      // host CUtensorMap[3] of the work buffer (TMA x variants), or null
    int wait_selftest;      // 1: the bulk-copy wait waits (briefly) for a phase that never completes
    // step 0 from the incident field (compile-time-sized passes only): the forward y/z pass
    // computes its input p = alpha_m exp(i k.(r - c)) E_inc on active cells (0 elsewhere)
    // from the occupancy and materials of ep instead of reading src, and writes it to inc_out
    int inc;
    // with inc: right-hand sides 2k, 2k+1 are the two polarisations of one orientation with
    // the same polarisabilities, so p_inc = phi(r) E_q with one scalar phi = alpha_m
    // exp(i k.(r - c)); the forward passes transform phi once per pair (into component slot
    // 0 of right-hand side 2k) and the x pass forms G * (phi E_q) for both polarisations
    int pair;
    const float2 *inc_tab;  // [nrhs][nj + nl + ni] phase tables (y, z, x)
    const double *einc;     // [nrhs][6] incident field
    float2 *inc_out;        // [nrhs][3][N]
};

// Dynamic shared memory limit of a kernel on the current device, raised to at least
// `bytes` and never lowered: the limit is a per-process property of the kernel, shared by
// every context, so a context on a smaller lattice must not shrink what a larger one set
// (matvec.cu).
cudaError_t raise_smem_limit(const void *kernel, int bytes);

// kernels (matvec.cu)
cudaError_t kernel_binary_version(int *version);   // of the loaded module, e.g. 100
cudaError_t launch_matvec(const MatvecArgs &a, cudaStream_t st);
size_t matvec_smem_yz(const Lat &L, int rows_g);
size_t matvec_smem_x(const Lat &L, int tile_x);
cudaError_t matvec_prepare(const Lat &L, int tile_x, int rows_g);

// compile-time-sized passes for edges in {16, 32, 64} (matvec_fast.cu)
bool matvec_fast_supported(const Lat &L);
constexpr int kXVariants = 12;     // launch variants of the fast x pass (9..11: TMA tensor tiles)
constexpr int kYZVariants = 3;     // launch variants of the fast y/z passes
cudaError_t matvec_fast_prepare(const Lat &L);
int matvec_fast_x_tile(int ni, int x_variant);   // spectral columns per CTA of an x variant
cudaError_t launch_matvec_fast(const MatvecArgs &a, cudaStream_t st);

// Green tensor (green.cu)
cudaError_t green_build_octant(int ni, int nj, int nl, double kd, float2 *ahat, cudaStream_t st);
cudaError_t green_project_dense(int ni, int nj, int nl, const float2 *dense_dev, float2 *ahat,
                                cudaStream_t st);
size_t ahat_elems(int ni, int nj, int nl);

}  // namespace ddagpu
