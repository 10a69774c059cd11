/*
 * dda_oracle.h -- TEST INFRASTRUCTURE ONLY.  A plain-C, FP64 restatement of the
 * reference DDA-FFT hot path (physicist2018/dda-fft v7.2) used as the checker for
 * the B200 kernels.  Nothing in the product links, loads or calls it; it is loaded
 * only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm.  Every function cites the reference file:line whose semantics it restates.
 *
 * Parity of this restatement is pinned against the reference itself: the float
 * build (oracle/_ref/libddaref.so) through golden fixtures in tests/golden/, and the
 * reference's FP64 build (oracle/_ref/libddaref64.so) directly in tests.
 *
 * Dense layouts (all double):
 *   field  [ni][nj][nl][3] complex  (x, y, z), 6 doubles per cell
 *   Ahat   [2ni][2nj][2nl][6] complex (e00,e01,e02,e11,e12,e22), 12 doubles per cell
 *   occ    [ni][nj][nl] signed char material index, 0 = empty
 */
#ifndef DDA_ORACLE_H
#define DDA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Ahat = DFT(G on the 2n grid) / (8 ni nj nl).  zero_n_planes != 0 zeroes the index-n
   planes of G first (they only feed discarded outputs), which makes Ahat exactly even
   or odd along each axis. */
int or_green_hat(int ni, int nj, int nl, double kd, int zero_n_planes, double *ahat);

/* G*p on the valid block (Convolution, dda_func.cpp:150-187; conj != 0: Convolution_conj,
   dda_func.cpp:227-437, which uses conj(Ahat(-k))). */
int or_convolution(int ni, int nj, int nl, const double *ahat, const double *p, double *out,
                   int conj);

/* 1-D DFT, natural order; inverse = conj(DFT(conj(x))) with no 1/N (fft_kernel.hpp:291-320). */
int or_dft_line(int n, int inverse, const double *in, double *out);

/* polarisability of one material: model 1 CM, 2 CMRR, 3 CMNR, 4 ILDR, 5 LDR
   (dda_func.cpp:1631-1677, selection main.cpp:606-642, 926-931) */
int or_polarizability(int model, double d0, double m_re, double m_im, const double *kinc3,
                      const double *einc6, double *out2);

typedef struct {
    int ni, nj, nl;
    int solver;              /* 0 CG, 1 AA*, 2 BiCGStab, 3 simple iteration        */
    double tau;              /* weight factor of the simple iteration               */
    int nmat;                /* alpha[0..nmat], listmv[0..nmat]; index 0 = empty    */
    const double *alpha;     /* complex polarisabilities, 2*(nmat+1) doubles        */
    const int *listmv;       /* 1 = active material                                 */
    const signed char *occ;
    int max_step;
    double err_max;
    double d0;
    double kinc[3];
    double einc[6];
    const double *ahat;      /* dense Green tensor, see or_green_hat                */
    int nplanes, nangles;
    const double *ksc;       /* [plane][angle][3]                                   */
    int cast_scalars_float;  /* 1: round solver scalars to float like the float build */
    const double *rhs;       /* if not NULL: solve A p = rhs from p = rhs instead of the
                                incident field (adjoint solves); field layout            */
} or_solve_in;

typedef struct {
    double *p;               /* final dipole moments (may be NULL)                  */
    double *esc;             /* [plane][angle][6]                                   */
    double cabs, cext;
    double *trace;           /* discrepancy after each step, max_step+1 entries     */
    int ntrace;
    int step_min;            /* rolled-back step, -1 if none                        */
    int matvecs;             /* number of convolutions performed                    */
} or_solve_out;

/* DDA_FFT, dda_func.cpp:1075-1570 */
int or_dda_fft(const or_solve_in *in, or_solve_out *out);

int or_first_approximation(int ni, int nj, int nl, const int *listmv, const double *alpha,
                           const signed char *occ, double d0, const double *kinc3,
                           const double *einc6, double *p);
int or_farfield(int ni, int nj, int nl, const int *listmv, const signed char *occ, double d0,
                const double *p, const double *ksc3, double *out6);
int or_cabscext(int ni, int nj, int nl, const double *alpha, const signed char *occ, double d0,
                const double *kinc3, const double *einc6, const double *p, double *cabs,
                double *cext);
int or_jones_mueller(const double *kinc3, const double *ksc3, const double *normal3,
                     const double *einc0, const double *einc1, const double *esc0,
                     const double *esc1, double *jones8, double *out16);

/* xorshift64* stream of randomize.cpp:44-58 */
int or_rng(unsigned long long seed, int count, int *out);
/* Monte-Carlo Euler draws of main.cpp:876-898 for worker `worker` of a run seeded
   `base_seed`: T[count][9] row-major rotation matrices */
int or_mc_rotations(unsigned long long base_seed, int worker, int count, double *T);
int or_gen_ellipsoid(int ni, int nj, int nl, double b_a, double c_a, signed char *occ);

/* scattering geometry of main.cpp:336-387 (before rotation):
   normals[nplanes][3], ksc[nplanes][nangles][3] */
int or_scattering_geometry(int nplanes, int nangles, double theta_min, double theta_step,
                           double *normals, double *ksc);

#ifdef __cplusplus
}
#endif
#endif
