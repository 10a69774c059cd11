/*
 * ddagpu.h -- C ABI of libddagpu, the B200 (sm_100a) implementation of the DDA-FFT hot
 * path of physicist2018/dda-fft v7.2: the zero-padded FFT convolution A*p inside the
 * CG / AA* / BiCGStab / simple-iteration solvers, the solver updates and reductions,
 * the far-field sums, the cross sections and the Jones -> Mueller averaging.
 *
 * Plain pointers and sizes only.  Unless a name ends in _dev, array arguments are HOST
 * memory in the reference's own layouts:
 *   field    [i_max][j_max][l_max] cvector  = 6 floats per cell (x.re x.im y.re y.im z.re z.im)
 *   cmA      [2 i_max][2 j_max][2 l_max] cmatrix = 12 floats per cell (e00 e01 e02 e11 e12 e22)
 *   cAlpha   [i_max][j_max][l_max] signed char material index, 0 = empty cell
 *   ksc      [planes][angles] vector (3 floats), Esc [planes][angles] cvector (6 floats)
 * _dev entry points take DEVICE pointers in the structure-of-arrays layout
 * [rhs][component][i][j][l] of complex float.
 *
 * Every function returns DDAGPU_OK (0) or a negative code; ddagpu_last_error() gives the
 * message of the last failure on the calling thread.  The reference never returns an error
 * (it exits on out-of-memory and on a workspace mismatch, dda_func.cpp:1006-1008,
 * 1091-1094); a host adapter maps the codes to those exits.  A context may be used from one
 * thread at a time (calls on one context are serialised by a lock); separate contexts on
 * the same device run concurrently, like the reference's worker workspaces
 * (main.cpp:777-995).
 */
#ifndef DDAGPU_H
#define DDAGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DDAGPU_OK 0
#define DDAGPU_EINVAL (-1)     /* invalid argument (sizes, solver, null pointer)          */
#define DDAGPU_ENOMEM (-2)     /* device allocation failed (reference: exit(1))          */
#define DDAGPU_ECUDA (-3)      /* a CUDA call failed                                       */
#define DDAGPU_EMISMATCH (-4)  /* lattice differs from the context (reference: exit(1)) */
#define DDAGPU_ENOTBUILT (-5)  /* no CUDA device / library built without kernels           */

typedef struct ddagpu_ctx ddagpu_ctx;

/* Result details of one solve (the reference prints these, dda_func.cpp:1281,1524-1548). */
typedef struct {
    int steps;          /* iterations performed after step 0                           */
    int step_min;       /* step of the best iterate                                     */
    int rolled_back;    /* 1 if the final iterate was replaced by the best one          */
    int matvecs;        /* convolutions performed                                       */
    double err;         /* final discrepancy (mean residual norm, ldError)              */
    double err_min;     /* smallest discrepancy seen                                    */
} ddagpu_solve_info;

const char *ddagpu_version(void);
const char *ddagpu_last_error(void);
/* Architecture the library's kernels were compiled for, as the CUDA runtime reports it for
 * the module loaded on `device` (major * 10 + minor: 100 for sm_100a).  No counterpart in
 * the reference. */
int ddagpu_binary_version(int device, int *version);

/* Creates a context for one lattice on one CUDA device, builds the Green tensor FFT from kd
 * on the device, and reserves work space for up to max_rhs right-hand sides solved
 * together.  Replaces CreateAMatrix + FFT_3D(cmA) (main.cpp:466-486, dda_func.cpp:85-148,
 * fft_func.cpp:317-416) and dda_workspace_create (dda_func.cpp:1031-1054).
 * Lattice edges: powers of two in [2, 128]. */
int ddagpu_create(ddagpu_ctx **ctx, int device, int i_max, int j_max, int l_max, double kd,
                  int max_rhs);
int ddagpu_destroy(ddagpu_ctx *ctx);

/* Replaces the Green tensor with a host-built cmA (the reference's own, main.cpp:466-486),
 * e.g. for bit-level comparisons.  It is projected on the symmetric octant the kernels
 * store; the projection changes only convolution outputs outside the lattice. */
int ddagpu_set_green(ddagpu_ctx *ctx, const float *cmA);

/* Convolution sub-seam (dda_func.cpp:150-187; conj != 0: Convolution_conj, 227-437):
 * out = G * p on the lattice, p and out host fields. */
int ddagpu_convolution(ddagpu_ctx *ctx, const float *p, float *out, int conj);

/* The DDA_FFT seam (function.hpp:153-160, dda_func.cpp:1075-1570): solves one
 * polarisation with solver 0 CG, 1 AA*, 2 BiCGStab, 3 simple iteration (weight rTau), to
 * the reference's absolute Error_max rule with best-iterate rollback, then CabsCext and the
 * far field at every (plane, angle).  cListMaterials: n_mat+1 complex polarisabilities
 * (index 0 = empty); iListMV: n_mat+1 active flags.  The FFT tables of the reference's
 * signature are not needed; iMode_FFT is accepted for both CT (0) and RB (1), which give
 * the same convolution.  trace (optional, Max_Step+1 doubles) receives the discrepancy of
 * every step. */
int ddagpu_dda_fft(ddagpu_ctx *ctx, int iNoIllumination, int iMode_SolutionMethod, float rTau,
                   int i_max, int j_max, int l_max, const float *cListMaterials,
                   const int *iListMV, int n_mat, const signed char *cAlpha, int Max_Step,
                   float Error_max, float d0, const float *kinc, const float *Einc,
                   int iMode_FFT, int iNoScPl, int iNoA, const float *ksc, float *Esc,
                   float *rCabs, float *rCext, ddagpu_solve_info *info, double *trace);

/* Iterative refinement around DDA_FFT's solvers, every convolution on the FP32 FFT passes,
 * the solution and the true residual r = p_inc - (p - alpha G*p) in FP64.  Stops when the
 * mean true residual norm (the reference's discrepancy, dda_func.cpp:784-811, of the true
 * instead of the recursively updated residual) is <= Error_max, or after max_outer outer
 * steps; info reports the true residual of every outer step.  Outputs as ddagpu_dda_fft.
 *   iMode_SolutionMethod 0 (CG): the inner solver is the reference's CG (dda_func.cpp:
 *     1359-1371) with FP64 fields and FP64 scalars; an outer step computes the true
 *     residual when the updated one has fallen to inner_rel x the last true one, meets
 *     Error_max, or after inner_max_step iterations, and restarts CG from the current FP64
 *     solution.  Reaches a discrepancy near 1e-8 on a 128^3 sphere at x = 16,
 *     m = 1.6+0.0005i (inner_rel 1e-3).
 *   1..3: each outer step solves A d = r in FP32 with that solver (restarted from d = r, to
 *     inner_rel x the current residual, at most inner_max_step iterations, best iterate
 *     kept) and adds d to p. */
typedef struct {
    int outer;               /* outer steps taken                                       */
    int inner_steps;         /* inner solver iterations, all outer steps                */
    int matvecs;             /* convolutions, inner and outer                           */
    double err;              /* final mean true residual norm                           */
    double err_history[64];  /* mean true residual norm before each outer step          */
} ddagpu_refine_info;

int ddagpu_dda_fft_refined(ddagpu_ctx *ctx, int iMode_SolutionMethod, float rTau,
                           const float *cListMaterials, const int *iListMV, int n_mat,
                           const signed char *cAlpha, float d0, const float *kinc,
                           const float *Einc, double Error_max, int max_outer, double inner_rel,
                           int inner_max_step, int iNoScPl, int iNoA, const float *ksc,
                           float *Esc, float *rCabs, float *rCext, ddagpu_refine_info *info);

/* A x = rhs for an arbitrary right-hand side (A = I - D_alpha G of the context's lattice):
 * the solver of DDA_FFT started from x = rhs instead of p_inc (dda_func.cpp:1103-1104),
 * to the discrepancy Error_max in max_step steps, or with refine != 0 by the FP64
 * refinement above (max_step = outer steps).  rhs and x_out are host fields.  Used for
 * adjoint solves: A^T = I - G D_alpha, so A^T l = g is A m = D_alpha g with l = m / alpha. */
int ddagpu_solve_linear(ddagpu_ctx *ctx, int iMode_SolutionMethod, float rTau,
                        const float *cListMaterials, const int *iListMV, int n_mat,
                        const signed char *cAlpha, const float *rhs, double Error_max,
                        int max_step, int refine, double inner_rel, int inner_max_step,
                        float *x_out, ddagpu_refine_info *info);

/* FP64 solve: DDA_FFT (dda_func.cpp:1075-1570) with every field, transform, product and
 * scalar in double -- the reference's FP64 build (complex.hpp:10 as `typedef double real`)
 * run on the GPU, without its float casts of the solver coefficients.  It is the oracle
 * solve that the precision pattern measures a float solve against, at sizes where the CPU
 * FP64 build takes hours.  alpha: 2 (n_mat + 1) doubles; kinc, Einc, ksc [ndir][3] and
 * Esc [ndir][6] doubles; rhs (optional) solves A p = rhs instead of A p = p_inc, x0
 * (optional) starts the solver from x0 instead of the right-hand side; rhs, x0 and p_out
 * (optional, the final dipoles) are fields of 6 doubles per cell; ndir <= 65535.  Same stopping rule,
 * rollback and outputs as ddagpu_dda_fft.  The FP64 work space (about 100 bytes per padded
 * cell plus 10 fields) is allocated on the first call and kept until ddagpu_release_fp64 or
 * ddagpu_destroy. */
int ddagpu_solve_fp64(ddagpu_ctx *ctx, int iMode_SolutionMethod, double rTau, const double *alpha,
                      const int *iListMV, int n_mat, const signed char *cAlpha, double d0,
                      const double *kinc, const double *Einc, const double *rhs, const double *x0,
                      int Max_Step, double Error_max, int ndir, const double *ksc, double *Esc,
                      double *Cabs, double *Cext, double *p_out, ddagpu_solve_info *info,
                      double *trace);
int ddagpu_release_fp64(ddagpu_ctx *ctx);

/* FarField sub-seam (dda_func.cpp:1576-1625) for ndir directions at once. */
int ddagpu_farfield(ddagpu_ctx *ctx, const int *iListMV, int n_mat, const signed char *cAlpha,
                    float d0, const float *p, int ndir, const float *ksc, float *Esc);

/* CabsCext sub-seam (dda_func.cpp:1679-1727). */
int ddagpu_cabscext(ddagpu_ctx *ctx, float d0, const float *kinc, const float *Einc,
                    const float *cListMaterials, int n_mat, const signed char *cAlpha,
                    const float *p, float *Cabs, float *Cext);

/* BuildMatrixJones + JonesToMuller averaged over planes (mmuller.cpp:175-314,
 * main.cpp:943-954) for one orientation: esc0/esc1 [planes][angles] cvector of the two
 * polarisations, ksc [planes][angles] vector, normals [planes] vector; out [angles][16]. */
int ddagpu_mueller(ddagpu_ctx *ctx, const float *kinc, const float *einc0, const float *einc1,
                   int nplanes, int nangles, const float *ksc, const float *normals,
                   const float *esc0, const float *esc1, float *out);

/* ---------------------------------------------------------------- batched solves
 * One call runs many orientations of one target: both polarisations of every orientation
 * are right-hand sides of one batched solve that shares the Green tensor, the occupancy
 * and the FFT passes (the sample loop of main.cpp:806-985 for targets whose geometry does
 * not change between samples). */
typedef struct {
    int solver;              /* 0..3                                                   */
    float tau;               /* simple-iteration weight                                */
    int max_step;            /* Max_Step                                               */
    float err_max;           /* Error_max (absolute, dda_func.cpp:1302)                */
    int polarizability;      /* 1 CM, 2 CMRR, 3 CMNR, 4 ILDR, 5 LDR                    */
    int n_mat;               /* materials 1..n_mat                                     */
    const float *m;          /* refractive indices, 2 n_mat floats (re, im)            */
    const signed char *occ;  /* host occupancy [i][j][l]; NULL reuses the occupancy of
                                the previous batched call, still resident on the device */
    int nplanes;             /* scattering planes (main.cpp:377-387)                   */
    float theta_min, theta_max, theta_step; /* degrees (main.cpp:195-200)              */
} ddagpu_batch_cfg;

typedef struct {
    int n_rhs;               /* right-hand sides solved                               */
    int max_steps;           /* largest iteration count of any right-hand side        */
    int rolled_back;         /* right-hand sides whose best iterate was restored      */
    double max_err;          /* largest final discrepancy                              */
} ddagpu_batch_info;

/* n_orient rotations rot[n_orient][9] (row-major VectTrans of main.cpp:885-898, or the
 * fixed Z(-psi) Y(-iota) X(-kappa) product of main.cpp:516-541) -> per orientation
 * Cabs, Cext (averages of the two polarisations, main.cpp:939) and the plane-averaged
 * Mueller matrix mueller[n_orient][angles][16]. */
int ddagpu_orientation_solves(ddagpu_ctx *ctx, const ddagpu_batch_cfg *cfg, int n_orient,
                              const double *rot, double *cabs, double *cext, double *mueller,
                              ddagpu_batch_info *info);

/* Realisation batch: n_real targets on this context's lattice, each with its own occupancy
 * occ[n_real][i][j][l] (host; cfg->occ is not used) -- the sample loop of main.cpp:806-985
 * for targets that change between samples (random and agglomerate targets, or shape files).
 * Right-hand sides of one batched solve carry different occupancies.  rot[n_real][9] as for
 * ddagpu_orientation_solves, or NULL for the fixed orientation psi = iota = kappa = 0. */
int ddagpu_realization_solves(ddagpu_ctx *ctx, const ddagpu_batch_cfg *cfg, int n_real,
                              const signed char *occ, const double *rot, double *cabs,
                              double *cext, double *mueller, ddagpu_batch_info *info);

/* Agglomerate realisations (target 6, particle.cpp:21-85): realisation k is the monomer
 * list monomers[first_k .. first_k + counts[k])[13] of ddagpu_anthrax_place, rasterised on
 * the GPU straight into the batch (no occupancy crosses the host).  One material
 * (cfg->n_mat = 1); ndip[n_real] (may be NULL) receives each realisation's dipole count. */
int ddagpu_agglomerate_solves(ddagpu_ctx *ctx, const ddagpu_batch_cfg *cfg, int n_real,
                              const float *monomers, const int *counts, const double *rot,
                              double *cabs, double *cext, double *mueller, int *ndip,
                              ddagpu_batch_info *info);

/* Groups: contexts of different lattice sizes on one device whose batched agglomerate
 * solves run as ONE graph launch per call -- the sample loop of main.cpp:806-985 for
 * realisations whose lattices differ (main.cpp:812-858), each lattice with its own Green
 * tensor (main.cpp:466-486).  Member k's whole solve (state set-up, step 0, its iterations
 * as a conditional while node, rollback, far field, cross sections, Mueller matrices) is an
 * independent branch of the group's graph, recorded once per solve shape and replayed; the
 * members' inputs are uploaded on their own streams first.  No counterpart in the reference.
 * A context may belong to several groups and still be used on its own; a call locks every
 * member (in address order, so calls of groups that share members do not deadlock).  Per-member arrays are indexed by member: n_real[k] (0 leaves member k out;
 * at most max_rhs / 2 of that member), monomers[k], counts[k] as ddagpu_agglomerate_solves,
 * rot[k] (or rot == NULL: fixed orientation), outputs cabs[k], cext[k], mueller[k], ndip[k]
 * (each array of pointers may be NULL) and info[k]. */
typedef struct ddagpu_group ddagpu_group;
int ddagpu_group_create(ddagpu_group **grp, ddagpu_ctx *const *ctxs, int nctx);
int ddagpu_group_destroy(ddagpu_group *grp);
long long ddagpu_group_graph_runs(ddagpu_group *grp);   /* group graph launches so far */
int ddagpu_group_agglomerate_solves(ddagpu_group *grp, const ddagpu_batch_cfg *cfg, const int *n_real,
                                    const float *const *monomers, const int *const *counts,
                                    const double *const *rot, double *const *cabs, double *const *cext,
                                    double *const *mueller, int *const *ndip, ddagpu_batch_info *info);

/* Number of scattering angles for a configuration (rounding of main.cpp:201). */
int ddagpu_num_angles(float theta_min, float theta_max, float theta_step);

/* Rotation matrices of the reference's Monte-Carlo orientation sampler: worker `worker` of
 * a run seeded base_seed (main.cpp:803-804, 876-898, randomize.cpp:44-58). */
int ddagpu_mc_rotations(unsigned long long base_seed, int worker, int count, double *rot);
/* Random stream of worker `worker` of a run seeded base_seed (main.cpp:803-804): the state
 * to pass to ddagpu_anthrax_place; samples drawn one after another keep updating it. */
unsigned long long ddagpu_rng_seed(unsigned long long base_seed, int worker);

/* Agglomerates of capsule monomers (target 6, iGenerateAnthrax, particle.cpp:21-85).
 * Monomer count as main.cpp:585-586; placement on the host with the reference's random
 * stream and float geometry (monomers[count][13] = r, l, begin[3], end[3], axis[3], 0, 0;
 * returns DDAGPU_EINVAL if the packing is too dense to place them); rasterisation of the
 * monomers into the lattice on the GPU (occ host output, 1 = filled). */
long long ddagpu_anthrax_count(int i_max, int j_max, int l_max, float packing,
                               float monomer_radius, float length_ratio);
int ddagpu_anthrax_place(unsigned long long *rng_state, int i_max, float monomer_radius,
                         float monomer_length, int count, float *monomers);
int ddagpu_anthrax_rasterize(int device, int i_max, int j_max, int l_max, const float *monomers,
                             int count, signed char *occ, int *ndip);

/* Launch variants of the compile-time-sized matvec passes (edges 16..128): x_variant
 * 0/1/2 = 32, 16 or 8 spectral columns per x-pass CTA (16, 8, 4 at edge 128), 3/4/5 = the
 * same with the input rows moved into shared memory by bulk asynchronous copies, 6/7/8 =
 * the same tiles with the x lines' second factorisation (16 = 8 x 2, 32 = 4 x 8,
 * 64 = 16 x 4, 128 = 8 x 16 instead of 4 x 4, 8 x 4, 8 x 8, 16 x 8: the radix schedule),
 * 9/10/11 = the tiles of 0/1/2 moved into shared memory as one TMA tensor tile per
 * component (cp.async.bulk.tensor over a tensor map of the work buffer; offered where the
 * driver provides the encoder);
 * yz_variant 0/1/2 = the default block size of the y/z passes, the other of 256 / 512, or
 * 128 threads.
 * ddagpu_autotune times every combination (and the generic passes) and keeps the
 * fastest.  No counterpart in the reference. */
int ddagpu_set_fast_variant(ddagpu_ctx *ctx, int x_variant, int yz_variant);

/* Form of the far-field sum (FarField, dda_func.cpp:1576-1625).  When the scattering
 * directions of a right-hand side take few distinct z components (the planes of a fixed
 * orientation turn about the incident direction, the lattice z axis: every plane's
 * direction at one angle has the same kz), the z sum of the separable phase is done once
 * per distinct kz and the x/y sum once per direction; otherwise every direction sums over
 * every active dipole.  mode 0 (default): the grouped form where it does at most half the
 * work of the direct one; 1: always the direct form; 2: the grouped form whenever its group
 * sums fit in 1 GiB.  The two forms agree to FP32 rounding.  No counterpart in the
 * reference, whose sum is per direction. */
int ddagpu_set_farfield_mode(ddagpu_ctx *ctx, int mode);

/* How a far field of these directions is summed, without a device: ksc [nrhs][ndir][3]
 * (pairs != 0: right-hand sides 2k, 2k+1 share theirs), lattice ni x nj x nl, nact active
 * cells per right-hand side, mode as ddagpu_set_farfield_mode.  *groups receives the most
 * distinct kz of a right-hand side (or pair) when the grouped form is chosen, else 0;
 * *items (may be null) the most work items (at most 16 directions of one group each). */
int ddagpu_farfield_plan(const double *ksc, int nrhs, int ndir, int pairs, int ni, int nj, int nl,
                         double nact, int mode, int *groups, int *items);
int ddagpu_get_fast_variant(ddagpu_ctx *ctx, int *x_variant, int *yz_variant);

/* Self-test of the bounded device waits: on != 0 makes the bulk-copy x-pass variants
 * (ddagpu_set_fast_variant x 3..5) wait briefly for a barrier phase that nothing completes,
 * so that the wait runs out; the call then fails with DDAGPU_ECUDA ("a device wait ran
 * out") and the context stays usable once the self-test is switched off.  Diagnostic
 * only; no counterpart in the reference. */
int ddagpu_selftest_wait_timeout(ddagpu_ctx *ctx, int on);

/* Solves as CUDA graphs (no counterpart in the reference, whose loop is on the host,
 * dda_func.cpp:1301-1535).  On (the default): every chunk of a batched call
 * (ddagpu_orientation_solves, ddagpu_realization_solves, ddagpu_agglomerate_solves) is one
 * graph launch -- state set-up, step 0, the iterations as a conditional while node whose
 * body ends with a kernel that stops the loop when no right-hand side is active or
 * Max_Step is reached, the rollback and the post-processing; the single-solve entry
 * points run iterations 2..Max_Step that way.  The host no longer reads the active flags
 * back every iteration.  Graphs are kept per context and rebuilt when the solve's shape
 * (solver, right-hand sides, Max_Step, materials, kernels, directions) changes.  Results
 * are the same kernels in the same order as with the host loop (off). */
int ddagpu_set_solver_graph(ddagpu_ctx *ctx, int on);
long long ddagpu_solver_graph_runs(ddagpu_ctx *ctx);   /* graph launches so far */

/* Random (Voronoi) ellipsoids (targets 4 and 5, iGenerateRandomEllipsoid,
 * particle.cpp:531-614): seeds[n_seeds][3] drawn on the host from the reference's random
 * stream (returns DDAGPU_EINVAL if the ellipsoid b/a, c/a does not fit the lattice); then
 * every cell inside the ellipsoid takes the material of its nearest seed (the first on
 * ties), seeds_per_material[m] seeds for material m + 1 in order, on the GPU.  ndip
 * receives the reference's count: cells of material 1. */
int ddagpu_random_ellipsoid_seeds(unsigned long long *rng_state, int i_max, int j_max, int l_max,
                                  float b_a, float c_a, int n_seeds, float *seeds);
int ddagpu_random_ellipsoid_fill(int device, int i_max, int j_max, int l_max, float b_a, float c_a,
                                 const float *seeds, const int *seeds_per_material, int n_mat,
                                 signed char *occ, int *ndip);

/* ---------------------------------------------------------------- state and result files
 * The sample loop's files in the float build's layout.  .dst: int counter, float Cabs and
 * Cext sums, n_angles x 16 float Mueller sums (main.cpp:214-274, 961-981); .dat: the sums
 * divided by the counter in the reference's text format (main.cpp:1085-1118).  I/O
 * failures return DDAGPU_EINVAL with the reason (the reference exits with codes 2 and 4). */

/* Open the state like main.cpp:214-274: restart != 0 removes it first; a missing file is
 * created with a zero state; the state is then read back into the outputs. */
int ddagpu_state_read(const char *path, int n_angles, int restart, int *counter, float *cabs,
                      float *cext, float *mueller);
/* Rewrite the state from its first byte and flush (main.cpp:966-981). */
int ddagpu_state_write(const char *path, int counter, float cabs, float cext, int n_angles,
                       const float *mueller);
/* Add n finished samples, in order, to the float sums and the counter (main.cpp:961-966):
 * cabs[n], cext[n], mueller[n][n_angles][16] as returned by the batched solves. */
int ddagpu_state_accumulate(int n, const double *cabs, const double *cext, int n_angles,
                            const double *mueller, int *counter, float *cabs_sum,
                            float *cext_sum, float *mueller_sum);
/* Write the .dat (main.cpp:1085-1118); theta_min / theta_step in degrees. */
int ddagpu_write_dat(const char *path, int counter, float cabs, float cext, int n_angles,
                     float theta_min, float theta_step, const float *mueller);

/* Fixed orientation (degrees), main.cpp:516-541. */
int ddagpu_fixed_rotation(double psi, double iota, double kappa, double *rot);

/* Far field that allocates nothing, for callers that must not allocate device memory
 * (code under CUDA graph capture, real-time loops that forbid allocator calls, hosts that
 * hand the library only pre-allocated buffers).  No counterpart in the reference.  Needs no
 * context: the caller passes device pointers to the occupancy occ_dev [i][j][l], the
 * material activity flags mv_dev (n_mat + 1 ints, index 0 = empty; cells whose material
 * index exceeds n_mat count as empty and mv_dev is never read past n_mat), the
 * dipoles p_dev ([3][i][j][l] complex float, structure of arrays), the directions
 * ksc_dev [ndir][3] float, and receives esc_dev [ndir][6] float (cvector per direction),
 * all on `stream` (cudaStream_t; NULL = legacy default stream).  At most 8192 directions
 * per call; more returns DDAGPU_EINVAL.  The FP64 accumulators live in a fixed 576 KiB
 * device array that every GPU loading the library holds until exit; the first call on a
 * device looks up that array's address, so make it before any stream capture.  Calls
 * that overlap on the GPU share the array and race: serialise them (one stream). */
int ddagpu_farfield_noalloc(int device, int i_max, int j_max, int l_max, float d0,
                            const signed char *occ_dev, const int *mv_dev, int n_mat,
                            const void *p_dev, int ndir, const float *ksc_dev, float *esc_dev,
                            void *stream);

/* ---------------------------------------------------------------- device-resident form
 * G*p for nrhs fields already in device memory ([nrhs][3][i][j][l] complex float, SoA),
 * on the context's stream; nrhs <= max_rhs. */
int ddagpu_convolution_dev(ddagpu_ctx *ctx, const void *p_dev, void *out_dev, int nrhs, int conj);
/* The context's CUDA stream (cudaStream_t), for callers that time or order work on it. */
void *ddagpu_stream(ddagpu_ctx *ctx);
/* Number of CUDA kernels this context has launched so far. */
long long ddagpu_kernel_launches(ddagpu_ctx *ctx);
/* Kernel launch parameters: columns per CTA of the x pass and rows per staging group of
 * the y/z passes of the generic kernels; 0 keeps the current value.  ddagpu_autotune
 * times the generic tilings and the specialised passes on the context's lattice and keeps
 * the fastest. */
int ddagpu_set_tiling(ddagpu_ctx *ctx, int tile_x, int rows_g);
int ddagpu_get_tiling(ddagpu_ctx *ctx, int *tile_x, int *rows_g);
/* Kernel family of the matvec: 1 = passes specialised at compile time for lattice edges in
 * {16, 32, 64, 128} (the default where they apply), 0 = the generic passes (any edge 2..128). */
int ddagpu_set_kernels(ddagpu_ctx *ctx, int fast);
int ddagpu_get_kernels(ddagpu_ctx *ctx);
int ddagpu_autotune(ddagpu_ctx *ctx, int nrhs);

#ifdef __cplusplus
}
#endif

#endif /* DDAGPU_H */
