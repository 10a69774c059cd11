/*
 * dda_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 restatement of the reference DDA-FFT hot path (physicist2018/dda-fft v7.2).
 * Written from the reference's semantics, function by function; each function cites
 * the reference file:line it follows.  The arithmetic is plain double precision with
 * straightforward loops: a radix-2 FFT over the full zero-padded grid instead of the
 * reference's padding-aware mixed-radix passes (identical in exact arithmetic), and
 * double accumulators where the reference uses long double.
 */
#include "dda_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cd;

static const double PI_D = 3.14159265358979323846264338327950288;

static size_t idx3(int i, int j, int l, int nj, int nl)
{
    return ((size_t)i * nj + j) * nl + l;
}

/* ----------------------------------------------------------------------------- FFT */

/* In-place radix-2 DFT of n (power of two) points with stride; sign -1 forward. */
static void fft_pow2(cd *a, int n, size_t stride, int sign)
{
    int j = 0;
    for (int i = 1; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            cd t = a[(size_t)i * stride];
            a[(size_t)i * stride] = a[(size_t)j * stride];
            a[(size_t)j * stride] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        for (int k = 0; k < len / 2; k++) {
            double ang = sign * 2.0 * PI_D * (double)k / (double)len;
            cd w = cos(ang) + I * sin(ang);
            for (int s = 0; s < n; s += len) {
                cd u = a[(size_t)(s + k) * stride];
                cd v = a[(size_t)(s + k + len / 2) * stride] * w;
                a[(size_t)(s + k) * stride] = u + v;
                a[(size_t)(s + k + len / 2) * stride] = u - v;
            }
        }
    }
}

/* 3-D DFT over an (m0,m1,m2) grid of `ncomp` interleaved components. */
static void fft3(cd *a, int m0, int m1, int m2, int ncomp, int sign)
{
    for (int c = 0; c < ncomp; c++) {
        for (int i = 0; i < m0; i++)
            for (int j = 0; j < m1; j++)
                fft_pow2(a + (((size_t)i * m1 + j) * m2) * ncomp + c, m2, (size_t)ncomp, sign);
        for (int i = 0; i < m0; i++)
            for (int l = 0; l < m2; l++)
                fft_pow2(a + ((size_t)i * m1 * m2 + l) * ncomp + c, m1, (size_t)m2 * ncomp, sign);
        for (int j = 0; j < m1; j++)
            for (int l = 0; l < m2; l++)
                fft_pow2(a + ((size_t)j * m2 + l) * ncomp + c, m0, (size_t)m1 * m2 * ncomp, sign);
    }
}

int or_dft_line(int n, int inverse, const double *in, double *out)
{
    /* direct O(n^2) DFT of a cvector line (3 components), fft_kernel.hpp:291-320 */
    for (int k = 0; k < n; k++)
        for (int c = 0; c < 3; c++) {
            cd s = 0;
            for (int j = 0; j < n; j++) {
                double ang = (inverse ? 2.0 : -2.0) * PI_D * (double)((long long)j * k % n) / n;
                s += (in[6 * j + 2 * c] + I * in[6 * j + 2 * c + 1]) * (cos(ang) + I * sin(ang));
            }
            out[6 * k + 2 * c] = creal(s);
            out[6 * k + 2 * c + 1] = cimag(s);
        }
    return 0;
}

/* ---------------------------------------------------------------- Green tensor */

/* CreateAMatrix (dda_func.cpp:85-148) on the 2n grid with the wrap-around index
   i >= n -> i - 2n, then FFT_3D(cmatrix) with the 1/(8 ni nj nl) factor
   (fft_func.cpp:317-416). */
int or_green_hat(int ni, int nj, int nl, double kd, int zero_n_planes, double *ahat)
{
    const int m0 = 2 * ni, m1 = 2 * nj, m2 = 2 * nl;
    cd *g = (cd *)ahat; /* 6 complex per cell */
    for (int i = 0; i < m0; i++) {
        double x = (i < ni ? i : i - m0) * kd;
        for (int j = 0; j < m1; j++) {
            double y = (j < nj ? j : j - m1) * kd;
            for (int l = 0; l < m2; l++) {
                double z = (l < nl ? l : l - m2) * kd;
                cd *e = g + idx3(i, j, l, m1, m2) * 6;
                double r2 = x * x + y * y + z * z;
                int on_n = (i == ni) || (j == nj) || (l == nl);
                if (r2 < 1e-10 || (zero_n_planes && on_n)) {
                    for (int q = 0; q < 6; q++) e[q] = 0;
                    continue;
                }
                double r1 = sqrt(r2);
                cd c2 = (cos(r1) + I * sin(r1)) / (r1 * r2);
                cd diag = c2 * ((r2 - 1.0) + I * r1);
                cd off = c2 * ((3.0 - r2) - 3.0 * I * r1) / r2;
                e[0] = off * x * x + diag;
                e[1] = off * x * y;
                e[2] = off * x * z;
                e[3] = off * y * y + diag;
                e[4] = off * y * z;
                e[5] = off * z * z + diag;
            }
        }
    }
    fft3(g, m0, m1, m2, 6, -1);
    double norm = 1.0 / ((double)m0 * m1 * m2);
    for (size_t q = 0; q < (size_t)m0 * m1 * m2 * 6; q++) g[q] *= norm;
    return 0;
}

/* ------------------------------------------------------------------ convolution */

int or_convolution(int ni, int nj, int nl, const double *ahat, const double *p, double *out,
                   int conj_mode)
{
    const int m0 = 2 * ni, m1 = 2 * nj, m2 = 2 * nl;
    const size_t P = (size_t)m0 * m1 * m2;
    cd *w = (cd *)calloc(P * 3, sizeof(cd));
    const cd *A = (const cd *)ahat;
    const cd *pp = (const cd *)p;
    if (!w) return -1;
    /* CopyingBack: zero padding (dda_func.cpp:702-718) */
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int l = 0; l < nl; l++)
                for (int c = 0; c < 3; c++)
                    w[idx3(i, j, l, m1, m2) * 3 + c] = pp[idx3(i, j, l, nj, nl) * 3 + c];
    fft3(w, m0, m1, m2, 3, -1);
    /* pointwise symmetric 3x3 product (dda_func.cpp:157-181); the conj variant uses
       conj(Ahat(-k)) (dda_func.cpp:235-434) */
    for (int i = 0; i < m0; i++)
        for (int j = 0; j < m1; j++)
            for (int l = 0; l < m2; l++) {
                cd e[6];
                if (conj_mode) {
                    const cd *s =
                        A + idx3((m0 - i) % m0, (m1 - j) % m1, (m2 - l) % m2, m1, m2) * 6;
                    for (int q = 0; q < 6; q++) e[q] = conj(s[q]);
                } else {
                    const cd *s = A + idx3(i, j, l, m1, m2) * 6;
                    for (int q = 0; q < 6; q++) e[q] = s[q];
                }
                cd *v = w + idx3(i, j, l, m1, m2) * 3;
                cd a = v[0], b = v[1], c = v[2];
                v[0] = e[0] * a + e[1] * b + e[2] * c;
                v[1] = e[1] * a + e[3] * b + e[4] * c;
                v[2] = e[2] * a + e[4] * b + e[5] * c;
            }
    /* iFFT_3D: conj-DFT-conj with no 1/N (fft_func.cpp:556-653) */
    fft3(w, m0, m1, m2, 3, +1);
    cd *o = (cd *)out;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int l = 0; l < nl; l++)
                for (int c = 0; c < 3; c++)
                    o[idx3(i, j, l, nj, nl) * 3 + c] = w[idx3(i, j, l, m1, m2) * 3 + c];
    free(w);
    return 0;
}

/* --------------------------------------------------------------- polarisability */

int or_polarizability(int model, double d0, double m_re, double m_im, const double *kinc3,
                      const double *einc6, double *out2)
{
    cd m = m_re + I * m_im, eps = m * m;
    /* Polarizability_CM, dda_func.cpp:1631-1637 */
    cd a = d0 * d0 * d0 * (0.75 / PI_D) * (eps - 1.0) / (eps + 2.0);
    const double b1 = -1.8915316, b2 = 0.1648469, b3 = -1.7700004;
    if (model == 2) /* CMRR, dda_func.cpp:1639-1645 */
        a = a / (1.0 - (2.0 / 3.0) * I * a);
    else if (model == 3) { /* CMNR, dda_func.cpp:1647-1656 */
        double b = -sqrt(4.0 * PI_D / 3.0) / d0;
        cd c1 = a / (1.0 + a * b);
        a = c1 / (1.0 - (2.0 / 3.0) * I * c1);
    } else if (model == 4 || model == 5) {
        double S = 0.2; /* ILDR, dda_func.cpp:1658-1665 */
        if (model == 5) { /* LDR, dda_func.cpp:1667-1677 */
            double rx = kinc3[0] * einc6[0], ry = kinc3[1] * einc6[2], rz = kinc3[2] * einc6[4];
            S = rx * rx + ry * ry + rz * rz;
        }
        a = a / (1.0 + (a / d0) * (b1 + b2 * eps + S * b3 * eps - (2.0 / 3.0) * d0 * I));
    }
    out2[0] = creal(a);
    out2[1] = cimag(a);
    return 0;
}

/* ------------------------------------------------------------- field operations */

int or_first_approximation(int ni, int nj, int nl, const int *listmv, const double *alpha,
                           const signed char *occ, double d0, const double *kinc3,
                           const double *einc6, double *p)
{
    /* FirstApproximation, dda_func.cpp:654-689: centre (n-1) d0 / 2 per axis */
    double cx = (ni - 1) * d0 / 2, cy = (nj - 1) * d0 / 2, cz = (nl - 1) * d0 / 2;
    cd *o = (cd *)p;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int l = 0; l < nl; l++) {
                size_t q = idx3(i, j, l, nj, nl);
                int m = occ[q];
                if (!listmv[m]) {
                    o[3 * q] = o[3 * q + 1] = o[3 * q + 2] = 0;
                    continue;
                }
                double ph = kinc3[0] * (i * d0 - cx) + kinc3[1] * (j * d0 - cy) +
                            kinc3[2] * (l * d0 - cz);
                cd c1 = (cos(ph) + I * sin(ph)) * (alpha[2 * m] + I * alpha[2 * m + 1]);
                for (int c = 0; c < 3; c++) o[3 * q + c] = c1 * (einc6[2 * c] + I * einc6[2 * c + 1]);
            }
    return 0;
}

int or_farfield(int ni, int nj, int nl, const int *listmv, const signed char *occ, double d0,
                const double *p, const double *ksc3, double *out6)
{
    /* FarField, dda_func.cpp:1576-1625 */
    double cx = (ni - 1) * d0 / 2, cy = (nj - 1) * d0 / 2, cz = (nl - 1) * d0 / 2;
    const cd *P = (const cd *)p;
    cd acc[3] = {0, 0, 0};
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int l = 0; l < nl; l++) {
                size_t q = idx3(i, j, l, nj, nl);
                if (!listmv[(int)occ[q]]) continue;
                double ph = ksc3[0] * (i * d0 - cx) + ksc3[1] * (j * d0 - cy) +
                            ksc3[2] * (l * d0 - cz);
                cd e = cos(ph) + I * sin(ph);
                cd kp = ksc3[0] * P[3 * q] + ksc3[1] * P[3 * q + 1] + ksc3[2] * P[3 * q + 2];
                for (int c = 0; c < 3; c++) acc[c] += e * (P[3 * q + c] - ksc3[c] * kp);
            }
    for (int c = 0; c < 3; c++) {
        out6[2 * c] = creal(acc[c]);
        out6[2 * c + 1] = cimag(acc[c]);
    }
    return 0;
}

int or_cabscext(int ni, int nj, int nl, const double *alpha, const signed char *occ, double d0,
                const double *kinc3, const double *einc6, const double *p, double *cabs,
                double *cext)
{
    /* CabsCext, dda_func.cpp:1679-1727.  The phase centre is n d0 / 2 here, unlike
       FirstApproximation and FarField ((n-1) d0 / 2); the skip test is alpha == 0. */
    double e2 = 0;
    for (int c = 0; c < 3; c++) e2 += einc6[2 * c] * einc6[2 * c] + einc6[2 * c + 1] * einc6[2 * c + 1];
    double r0 = 4.0 * PI_D / e2, r1 = 0, r2 = 0;
    double cx = ni * d0 / 2, cy = nj * d0 / 2, cz = nl * d0 / 2;
    const cd *P = (const cd *)p;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int l = 0; l < nl; l++) {
                size_t q = idx3(i, j, l, nj, nl);
                int m = occ[q];
                cd a = alpha[2 * m] + I * alpha[2 * m + 1];
                if (creal(a) == 0.0 && cimag(a) == 0.0) continue;
                double ph = -(kinc3[0] * (i * d0 - cx) + kinc3[1] * (j * d0 - cy) +
                              kinc3[2] * (l * d0 - cz));
                cd pe = 0;
                double pp = 0;
                for (int c = 0; c < 3; c++) {
                    pe += P[3 * q + c] * (einc6[2 * c] - I * einc6[2 * c + 1]);
                    pp += creal(P[3 * q + c]) * creal(P[3 * q + c]) +
                          cimag(P[3 * q + c]) * cimag(P[3 * q + c]);
                }
                r1 += cimag((cos(ph) + I * sin(ph)) * pe);
                r2 += cimag(pp / conj(a)) - (2.0 / 3.0) * pp;
            }
    *cext = r0 * r1;
    *cabs = r0 * r2;
    return 0;
}

/* ------------------------------------------------------------------ Jones/Mueller */

static void cross3(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

static cd rdot(const double *v, const double *e6)
{
    return v[0] * (e6[0] + I * e6[1]) + v[1] * (e6[2] + I * e6[3]) + v[2] * (e6[4] + I * e6[5]);
}

int or_jones_mueller(const double *kinc3, const double *ksc3, const double *normal3,
                     const double *einc0, const double *einc1, const double *esc0,
                     const double *esc1, double *jones8, double *out16)
{
    /* BuildMatrixJones, mmuller.cpp:175-252: components of the incident and scattered
       fields across (normal) and along the scattering plane, Jones matrix by Cramer */
    double v[3], pin[3], psc[3], nn;
    cross3(kinc3, normal3, v);
    nn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int c = 0; c < 3; c++) pin[c] = v[c] / nn;
    cross3(ksc3, normal3, v);
    nn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int c = 0; c < 3; c++) psc[c] = -v[c] / nn;
    cd i0n = rdot(normal3, einc0), i1n = rdot(normal3, einc1);
    cd i0p = rdot(pin, einc0), i1p = rdot(pin, einc1);
    cd den = I * (i0n * i1p - i1n * i0p);
    cd s0n = rdot(normal3, esc0), s1n = rdot(normal3, esc1);
    cd s0p = rdot(psc, esc0), s1p = rdot(psc, esc1);
    cd J[2][2];
    J[0][0] = (s1p * i0n - s0p * i1n) / den;
    J[0][1] = (s0p * i1p - s1p * i0p) / den;
    J[1][0] = (s1n * i0n - s0n * i1n) / den;
    J[1][1] = (s0n * i1p - s1n * i0p) / den;
    if (jones8)
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                jones8[4 * a + 2 * b] = creal(J[a][b]);
                jones8[4 * a + 2 * b + 1] = cimag(J[a][b]);
            }
    /* JonesToMuller, mmuller.cpp:254-314 */
    cd A = J[0][0], B = J[0][1], C = J[1][0], D = J[1][1];
    double aa = creal(A * conj(A)), bb = creal(B * conj(B)), cc = creal(C * conj(C)),
           dd = creal(D * conj(D));
    double *M = out16;
    M[0] = 0.5 * (aa + bb + cc + dd);
    M[1] = 0.5 * (aa - bb + cc - dd);
    M[2] = creal(A * conj(B) + D * conj(C));
    M[3] = cimag(A * conj(B) - D * conj(C));
    M[4] = 0.5 * (aa + bb - cc - dd);
    M[5] = 0.5 * (aa - bb - cc + dd);
    M[6] = creal(A * conj(B) - D * conj(C));
    M[7] = cimag(A * conj(B) + D * conj(C));
    M[8] = creal(A * conj(C) + D * conj(B));
    M[9] = creal(A * conj(C) - D * conj(B));
    M[10] = creal(D * conj(A) + B * conj(C));
    M[11] = cimag(A * conj(D) + C * conj(B));
    M[12] = cimag(C * conj(A) + D * conj(B));
    M[13] = cimag(C * conj(A) - D * conj(B));
    M[14] = cimag(D * conj(A) - B * conj(C));
    M[15] = creal(D * conj(A) - B * conj(C));
    return 0;
}

/* --------------------------------------------------------------------- RNG, geometry */

static unsigned long long rng_next(unsigned long long *s)
{
    /* xorshift64*, randomize.cpp:50-58; returns 31 bits like rand() */
    *s ^= *s >> 12;
    *s ^= *s << 25;
    *s ^= *s >> 27;
    return (*s * 2685821657736338717ULL) >> 33;
}

int or_rng(unsigned long long seed, int count, int *out)
{
    unsigned long long s = seed ? seed : 0x9E3779B97F4A7C15ULL; /* randomize.cpp:44-48 */
    for (int k = 0; k < count; k++) out[k] = (int)rng_next(&s);
    return 0;
}

int or_mc_rotations(unsigned long long base_seed, int worker, int count, double *T)
{
    /* per-worker seeding main.cpp:803-804; draws and matrix main.cpp:876-898 */
    unsigned long long s = base_seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(worker + 1);
    if (!s) s = 0x9E3779B97F4A7C15ULL;
    const double RMAX = 2147483647.0;
    for (int k = 0; k < count; k++) {
        double cps = (double)rng_next(&s) * 2.0 / RMAX - 1.0;
        double psi = acos(cps), sps = sin(psi);
        double io = (double)rng_next(&s) * 2.0 * PI_D / RMAX;
        double ka = (double)rng_next(&s) * 2.0 * PI_D / RMAX;
        double cio = cos(io), sio = sin(io), cka = cos(ka), ska = sin(ka);
        double *t = T + 9 * (size_t)k;
        t[0] = cio * cka - cps * sio * ska;
        t[1] = sio * cka + cps * cio * ska;
        t[2] = sps * ska;
        t[3] = -cio * ska - cps * sio * cka;
        t[4] = -sio * ska + cps * cio * cka;
        t[5] = sps * cka;
        t[6] = sps * sio;
        t[7] = -sps * cio;
        t[8] = cps;
    }
    return 0;
}

int or_gen_ellipsoid(int ni, int nj, int nl, double b_a, double c_a, signed char *occ)
{
    /* iGenerateEllipsoid, particle.cpp:408-444 (cell centres, semi-axes from i_max) */
    double cx = ni / 2.0 - 0.5, cy = nj / 2.0 - 0.5, cz = nl / 2.0 - 0.5;
    double a = ni, b = a * b_a, c = a * c_a;
    if (b > nj || c > nl) return -1;
    a = a / 2 * (a / 2);
    b = b / 2 * (b / 2);
    c = c / 2 * (c / 2);
    int n = 0;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            for (int l = 0; l < nl; l++) {
                double x = i - cx, y = j - cy, z = l - cz;
                int in = (x * x) / a + (y * y) / b + (z * z) / c <= 1.0;
                occ[idx3(i, j, l, nj, nl)] = (signed char)in;
                n += in;
            }
    return n;
}

int or_scattering_geometry(int nplanes, int nangles, double theta_min, double theta_step,
                           double *normals, double *ksc)
{
    /* main.cpp:336-387: plane 0 has normal y and directions (sin t, 0, cos t); plane m is
       plane 0 turned about z by m * 180 / nplanes degrees (Rotation_z, dda_func.cpp:27-34) */
    for (int pl = 0; pl < nplanes; pl++) {
        double ang = pl * (180.0 / nplanes) * PI_D / 180.0, c = cos(ang), s = sin(ang);
        double n0[3] = {0, 1, 0};
        normals[3 * pl + 0] = c * n0[0] + s * n0[1];
        normals[3 * pl + 1] = -s * n0[0] + c * n0[1];
        normals[3 * pl + 2] = n0[2];
        for (int a = 0; a < nangles; a++) {
            double th = (theta_min + theta_step * a) * PI_D / 180.0;
            double k0[3] = {sin(th), 0.0, cos(th)};
            double *k = ksc + 3 * ((size_t)pl * nangles + a);
            k[0] = c * k0[0] + s * k0[1];
            k[1] = -s * k0[0] + c * k0[1];
            k[2] = k0[2];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ solver */

typedef struct {
    int ni, nj, nl;
    size_t n;
    const signed char *occ;
    const int *mv;
    const cd *alpha;
} lat;

static int act(const lat *L, size_t q) { return L->mv[(int)L->occ[q]] != 0; }

/* ldcScalMul, dda_func.cpp:724-755: bilinear sum over active cells */
static cd dot_bil(const lat *L, const cd *a, const cd *b)
{
    cd s = 0;
    for (size_t q = 0; q < L->n; q++)
        if (act(L, q))
            for (int c = 0; c < 3; c++) s += a[3 * q + c] * b[3 * q + c];
    return s;
}

/* ldScalMulConj, dda_func.cpp:757-782: Re of the Hermitian product */
static double dot_herm(const lat *L, const cd *a, const cd *b)
{
    double s = 0;
    for (size_t q = 0; q < L->n; q++)
        if (act(L, q))
            for (int c = 0; c < 3; c++) s += creal(a[3 * q + c] * conj(b[3 * q + c]));
    return s;
}

/* ldError, dda_func.cpp:784-811: mean of the per-cell residual norm over active cells */
static double err_mean(const lat *L, const cd *r)
{
    double s = 0;
    long nact = 0;
    for (size_t q = 0; q < L->n; q++)
        if (act(L, q)) {
            double t = 0;
            for (int c = 0; c < 3; c++) t += creal(r[3 * q + c] * conj(r[3 * q + c]));
            s += sqrt(t);
            nact++;
        }
    return s / (double)nact;
}

/* out = v - alpha_m * conv(v) on active cells, 0 elsewhere (dda_func.cpp:1325-1357);
   conj_mode uses the conjugate operator and conj(alpha) (dda_func.cpp:1388-1413) */
static void apply_A(const lat *L, const double *ahat, const cd *v, cd *out, int conj_mode,
                    cd *tmp)
{
    or_convolution(L->ni, L->nj, L->nl, ahat, (const double *)v, (double *)tmp, conj_mode);
    for (size_t q = 0; q < L->n; q++) {
        int m = L->occ[q];
        if (act(L, q)) {
            cd a = conj_mode ? conj(L->alpha[m]) : L->alpha[m];
            for (int c = 0; c < 3; c++) out[3 * q + c] = v[3 * q + c] - a * tmp[3 * q + c];
        } else
            for (int c = 0; c < 3; c++) out[3 * q + c] = 0;
    }
}

static cd rnd_c(cd z, int cast)
{
    return cast ? (double)(float)creal(z) + I * (double)(float)cimag(z) : z;
}
static double rnd_r(double x, int cast) { return cast ? (double)(float)x : x; }

/* masked updates (LinearComb, dda_func.cpp:813-974) */
static void axpy_keep(const lat *L, cd *y, cd c, const cd *x) /* y += c x on active */
{
    for (size_t q = 0; q < L->n; q++)
        if (act(L, q))
            for (int k = 0; k < 3; k++) y[3 * q + k] += c * x[3 * q + k];
}
static void xpay_keep(const lat *L, const cd *x, cd c, cd *y) /* y = x + c y on active */
{
    for (size_t q = 0; q < L->n; q++)
        if (act(L, q))
            for (int k = 0; k < 3; k++) y[3 * q + k] = x[3 * q + k] + c * y[3 * q + k];
}
static void lin3_mask(const lat *L, const cd *x, cd c1, const cd *y, cd c2, const cd *z, cd *o)
{ /* o = x + c1 y + c2 z on active, 0 elsewhere */
    for (size_t q = 0; q < L->n; q++)
        for (int k = 0; k < 3; k++)
            o[3 * q + k] = act(L, q) ? x[3 * q + k] + c1 * y[3 * q + k] + c2 * z[3 * q + k] : 0;
}

int or_dda_fft(const or_solve_in *in, or_solve_out *out)
{
    lat L;
    L.ni = in->ni;
    L.nj = in->nj;
    L.nl = in->nl;
    L.n = (size_t)in->ni * in->nj * in->nl;
    L.occ = in->occ;
    L.mv = in->listmv;
    L.alpha = (const cd *)in->alpha;
    const int cast = in->cast_scalars_float, solver = in->solver;
    const size_t bytes = L.n * 3 * sizeof(cd);
    cd *p = malloc(bytes), *pmin = malloc(bytes), *r = malloc(bytes), *s = malloc(bytes),
       *g = malloc(bytes), *h = malloc(bytes), *w = malloc(bytes), *tmp = malloc(bytes);
    if (!p || !pmin || !r || !s || !g || !h || !w || !tmp) return -1;
    int mv = 0;

    /* step 0 (dda_func.cpp:1102-1278); with a given right-hand side y the same recurrences
       solve A p = y starting from p = y (y vanishes on inactive cells) */
    if (in->rhs) {
        const cd *y = (const cd *)in->rhs;
        for (size_t q = 0; q < L.n; q++)
            for (int c3 = 0; c3 < 3; c3++) p[3 * q + c3] = act(&L, q) ? y[3 * q + c3] : 0;
    } else {
        or_first_approximation(L.ni, L.nj, L.nl, in->listmv, in->alpha, in->occ, in->d0,
                               in->kinc, in->einc, (double *)p);
    }
    or_convolution(L.ni, L.nj, L.nl, in->ahat, (const double *)p, (double *)tmp, 0);
    mv++;
    for (size_t q = 0; q < L.n; q++)
        for (int c = 0; c < 3; c++)
            r[3 * q + c] = act(&L, q) ? -L.alpha[(int)L.occ[q]] * tmp[3 * q + c] : 0;

    cd cA = 0, cW = 0, ldA = 0, ldW = 0, rho1 = 0;
    double RR1 = 0;
    if (solver == 0) memcpy(s, r, bytes);
    if (solver == 1) {
        RR1 = dot_herm(&L, r, r);
        apply_A(&L, in->ahat, r, s, 1, tmp);
        mv++;
    }
    if (solver == 2) {
        memcpy(g, r, bytes);
        memcpy(s, r, bytes);
        rho1 = dot_bil(&L, r, g);
        apply_A(&L, in->ahat, s, h, 0, tmp);
        mv++;
        ldA = rho1 / dot_bil(&L, g, h);
        cA = rnd_c(ldA, cast);
        axpy_keep(&L, r, -cA, h);
        apply_A(&L, in->ahat, r, w, 0, tmp);
        mv++;
        ldW = dot_bil(&L, w, r) / dot_bil(&L, w, w);
        cW = rnd_c(ldW, cast);
        lin3_mask(&L, p, -cA, s, -cW, r, p);
        axpy_keep(&L, r, -cW, w);
    }
    if (solver == 3) {
        memcpy(s, p, bytes);
        for (size_t q = 0; q < 3 * L.n; q++) p[q] = s[q] - r[q];
    }

    double err = err_mean(&L, r), err_min = err;
    int step_min = 0, nt = 0;
    if (out->trace) out->trace[nt] = err;
    nt++;
    memcpy(pmin, p, bytes);

    for (int o = 1; o <= in->max_step; o++) { /* dda_func.cpp:1301-1535 */
        if (err <= in->err_max) break;
        if (err < err_min) {
            err_min = err;
            step_min = o - 1;
            memcpy(pmin, p, bytes);
        }
        if (solver == 2) {
            cd rho = dot_bil(&L, r, g);
            cd ldB = (rho * ldA) / (rho1 * ldW);
            cd cB = rnd_c(ldB, cast);
            cd c2 = rnd_c(-(cB * cW), cast);
            lin3_mask(&L, r, cB, s, c2, h, s);
            rho1 = rho; /* rho of this step; the update rho_1 = rho happens below */
            apply_A(&L, in->ahat, s, h, 0, tmp); /* W -> h (Copying at 1421) */
            mv++;
            ldA = rho / dot_bil(&L, g, h);
            cA = rnd_c(ldA, cast);
            axpy_keep(&L, r, -cA, h);
            apply_A(&L, in->ahat, r, w, 0, tmp);
            mv++;
            ldW = dot_bil(&L, w, r) / dot_bil(&L, w, w);
            cW = rnd_c(ldW, cast);
            lin3_mask(&L, p, -cA, s, -cW, r, p);
            axpy_keep(&L, r, -cW, w);
        } else if (solver == 0) {
            apply_A(&L, in->ahat, s, w, 0, tmp);
            mv++;
            cd den = dot_bil(&L, s, w);
            cA = rnd_c(dot_bil(&L, r, s) / den, cast);
            axpy_keep(&L, p, -cA, s);
            axpy_keep(&L, r, -cA, w);
            cd cB = rnd_c(dot_bil(&L, r, w) / den, cast);
            xpay_keep(&L, r, -cB, s);
        } else if (solver == 1) {
            apply_A(&L, in->ahat, s, w, 0, tmp);
            mv++;
            double SS = dot_herm(&L, s, s);
            double rA = rnd_r(-RR1 / SS, cast);
            axpy_keep(&L, r, rA, w);
            axpy_keep(&L, p, rA, s);
            double RR = dot_herm(&L, r, r);
            double rB = rnd_r(RR / RR1, cast);
            RR1 = RR;
            apply_A(&L, in->ahat, r, w, 1, tmp);
            mv++;
            xpay_keep(&L, w, rB, s);
        } else if (solver == 3) {
            or_convolution(L.ni, L.nj, L.nl, in->ahat, (const double *)p, (double *)tmp, 0);
            mv++;
            double tau = rnd_r(in->tau, cast);
            for (size_t q = 0; q < L.n; q++) {
                int m = L.occ[q];
                for (int c = 0; c < 3; c++) {
                    if (act(&L, q)) {
                        cd ap = p[3 * q + c] - L.alpha[m] * tmp[3 * q + c];
                        r[3 * q + c] = ap - s[3 * q + c];
                        p[3 * q + c] = p[3 * q + c] - tau * r[3 * q + c];
                    } else {
                        p[3 * q + c] = 0;
                        r[3 * q + c] = 0;
                    }
                }
            }
        }
        err = err_mean(&L, r);
        if (out->trace && nt <= in->max_step) out->trace[nt] = err;
        nt++;
    }
    out->step_min = -1;
    if (err > err_min) { /* best-iterate rollback, dda_func.cpp:1537-1548 */
        memcpy(p, pmin, bytes);
        out->step_min = step_min;
    }
    out->ntrace = nt;
    out->matvecs = mv;

    double ce, ca;
    or_cabscext(L.ni, L.nj, L.nl, in->alpha, in->occ, in->d0, in->kinc, in->einc,
                (const double *)p, &ca, &ce);
    out->cabs = ca;
    out->cext = ce;
    for (int pl = 0; pl < in->nplanes; pl++)
        for (int a = 0; a < in->nangles; a++) {
            size_t k = (size_t)pl * in->nangles + a;
            or_farfield(L.ni, L.nj, L.nl, in->listmv, in->occ, in->d0, (const double *)p,
                        in->ksc + 3 * k, out->esc + 6 * k);
        }
    if (out->p) memcpy(out->p, p, bytes);
    free(p);
    free(pmin);
    free(r);
    free(s);
    free(g);
    free(h);
    free(w);
    free(tmp);
    return 0;
}
