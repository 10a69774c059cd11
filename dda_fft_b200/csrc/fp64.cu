// FP64 solve of one polarisation: the reference's DDA_FFT (dda_func.cpp:1075-1570) with every
// field, transform, product and scalar in double -- the reference's FP64 build
// (complex.hpp:10 with `typedef double real`) run on the GPU.  It is the oracle solve of the
// precision pattern: the error of a float solve (with or without FP64-residual refinement)
// is measured against it, on lattices where a CPU FP64 solve would take hours.
//
// The convolution runs as five passes of zero-padded 2n-point transforms over a work buffer
// [3][ni][2nj][2nl] (only the i < ni planes of the padded grid exist, as in the float
// passes), with the Green tensor's FP64 octant [6][ni+1][nj+1][nl+1] (green.cu) unfolded by
// its parities:
//   Z  forward along l of every lattice row (c, i, j < nj), rows zero-padded to 2nl
//   Y  forward along j of tiles of spectral columns (c, i, kz), zero-padded to 2nj
//   X  forward along i, the symmetric 3x3 product, inverse along i (i < ni kept), per
//      tile of (ky, kz) columns with all 3 components
//   YI inverse along j (j < nj kept)
//   ZI inverse along l (l < nl kept) with the solver epilogue out = sv v - alpha_m conv
// Each line lives in shared memory and is transformed by an iterative radix-2 FFT with an
// FP64 twiddle table built on the host.  Throughput is not the aim of this path; exactness
// is: a 128^3 FP64 matvec takes a few milliseconds.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "fp64.h"

namespace ddagpu {

namespace {

constexpr int kT = 256;      // threads per block of every pass
constexpr int kTZ = 8;       // spectral columns per block of the Y, X and YI passes
constexpr int kLJ = 8;       // lattice rows per block of the Z and ZI passes

__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 dsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 dmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 dconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 dzero() { return make_double2(0.0, 0.0); }

// In-place radix-2 FFT of `nlines` lines of M points (M a power of two, 2..256) in shared
// memory, element k of line t at buf[t * LS + k]: bit reversal, then log2 M butterfly
// stages.  tw[k] = exp(-2 pi i k / M) for k < M / 2; inv conjugates them (the reference's
// inverse is conj(DFT(conj x)) with no 1/M, fft_func.cpp:556-653).  Every thread of the
// block calls it; it synchronises before and after.
__device__ void fft_lines_d(double2 *buf, int M, int LS, int nlines, const double2 *__restrict__ tw,
                            bool inv)
{
    __syncthreads();
    const int logM = __ffs(M) - 1;
    for (int e = threadIdx.x; e < nlines * M; e += blockDim.x) {
        const int t = e / M, k = e - t * M;
        const int r = (int)(__brev((unsigned)k) >> (32 - logM));
        if (r > k) {
            double2 *b = buf + (size_t)t * LS;
            const double2 x = b[k];
            b[k] = b[r];
            b[r] = x;
        }
    }
    __syncthreads();
    const int half = M >> 1;
    for (int hs = 1; hs < M; hs <<= 1) {
        const int step = half / hs;
        for (int e = threadIdx.x; e < nlines * half; e += blockDim.x) {
            const int t = e / half, b = e - t * half;
            const int j = b % hs, i0 = (b / hs) * 2 * hs + j, i1 = i0 + hs;
            double2 w = tw[j * step];
            if (inv) w.y = -w.y;
            double2 *L = buf + (size_t)t * LS;
            const double2 u = L[i0], v = dmul(L[i1], w);
            L[i0] = dadd(u, v);
            L[i1] = dsub(u, v);
        }
        __syncthreads();
    }
}

struct Mv64 {
    int ni, nj, nl;
    size_t N;
    const double2 *twi, *twj, *twl;   // exp(-2 pi i k / 2n), k < n, per axis
    const double2 *g;                 // [6][ni+1][nj+1][nl+1]
    double2 *work;                    // [3][ni][2nj][2nl]
    int conj;
};

struct Ep64 {
    int mode;                 // 0 raw convolution, 1 sv v - alpha_m conv on active cells
    double sv;
    const double2 *v;         // [3][N]
    const signed char *occ;   // [N]
    const int *mv;            // [nmat1]
    const double2 *alpha;     // [nmat1]
    int conj;
};

__device__ __forceinline__ size_t wrow(const Mv64 &a, int c, int i, int js)
{
    return (((size_t)c * a.ni + i) * (2 * a.nj) + js) * (2 * a.nl);
}

// Z: rows (c, i, j0 .. j0 + kLJ) of the field, zero-padded, forward along l
__global__ void __launch_bounds__(kT) z_fwd(Mv64 a, const double2 *__restrict__ src)
{
    extern __shared__ double2 smd[];
    const int M = 2 * a.nl, LS = M + 1, j0 = blockIdx.x * kLJ, i = blockIdx.y, c = blockIdx.z;
    const int nr = a.nj - j0 < kLJ ? a.nj - j0 : kLJ;
    const double2 *s = src + (size_t)c * a.N + ((size_t)i * a.nj + j0) * a.nl;
    for (int e = threadIdx.x; e < nr * M; e += blockDim.x) {
        const int t = e / M, l = e - t * M;
        smd[t * LS + l] = l < a.nl ? s[(size_t)t * a.nl + l] : dzero();
    }
    fft_lines_d(smd, M, LS, nr, a.twl, false);
    for (int e = threadIdx.x; e < nr * M; e += blockDim.x) {
        const int t = e / M, k = e - t * M;
        a.work[wrow(a, c, i, j0 + t) + k] = smd[t * LS + k];
    }
}

// Y / YI: spectral columns kz0 .. kz0 + tz of plane (c, i), along j
__global__ void __launch_bounds__(kT) y_pass(Mv64 a, int inv, int tz)
{
    extern __shared__ double2 smd[];
    const int M = 2 * a.nj, LS = M + 1, kz0 = blockIdx.x * tz, i = blockIdx.y, c = blockIdx.z;
    const int nload = inv ? M : a.nj, nstore = inv ? a.nj : M;
    for (int e = threadIdx.x; e < M * tz; e += blockDim.x) {
        const int j = e / tz, t = e - j * tz;
        smd[t * LS + j] = j < nload ? a.work[wrow(a, c, i, j) + kz0 + t] : dzero();
    }
    fft_lines_d(smd, M, LS, tz, a.twj, inv != 0);
    for (int e = threadIdx.x; e < nstore * tz; e += blockDim.x) {
        const int j = e / tz, t = e - j * tz;
        a.work[wrow(a, c, i, j) + kz0 + t] = smd[t * LS + j];
    }
}

// X: columns (ky, kz0 .. kz0 + tz), 3 components: forward along i, G product, inverse
__global__ void __launch_bounds__(kT) x_pass(Mv64 a, int tz)
{
    extern __shared__ double2 smd[];
    const int M = 2 * a.ni, LS = M + 1, kz0 = blockIdx.x * tz, ky = blockIdx.y;
    // line (c, t) at (c * tz + t) * LS
    for (int e = threadIdx.x; e < 3 * M * tz; e += blockDim.x) {
        const int t = e % tz, i = (e / tz) % M, c = e / (tz * M);
        smd[(c * tz + t) * LS + i] = i < a.ni ? a.work[wrow(a, c, i, ky) + kz0 + t] : dzero();
    }
    fft_lines_d(smd, M, LS, 3 * tz, a.twi, false);
    const int nj = a.nj, nl = a.nl, ni = a.ni;
    const bool my = ky > nj;
    const int oy = my ? 2 * nj - ky : ky;
    const size_t per = (size_t)(ni + 1) * (nj + 1) * (nl + 1);
    for (int e = threadIdx.x; e < M * tz; e += blockDim.x) {
        const int t = e % tz, kx = e / tz, kz = kz0 + t;
        const bool mx = kx > ni, mz = kz > nl;
        const int ox = mx ? 2 * ni - kx : kx, oz = mz ? 2 * nl - kz : kz;
        const size_t q = ((size_t)ox * (nj + 1) + oy) * (nl + 1) + oz;
        double2 g[6];
#pragma unroll
        for (int k = 0; k < 6; k++) g[k] = a.g[k * per + q];
        if (mx ^ my) g[1] = make_double2(-g[1].x, -g[1].y);
        if (mx ^ mz) g[2] = make_double2(-g[2].x, -g[2].y);
        if (my ^ mz) g[4] = make_double2(-g[4].x, -g[4].y);
        if (a.conj)
#pragma unroll
            for (int k = 0; k < 6; k++) g[k] = dconj(g[k]);
        double2 *bx = smd + (size_t)(0 * tz + t) * LS + kx, *by = smd + (size_t)(1 * tz + t) * LS + kx,
                *bz = smd + (size_t)(2 * tz + t) * LS + kx;
        const double2 vx = *bx, vy = *by, vz = *bz;
        *bx = dadd(dadd(dmul(g[0], vx), dmul(g[1], vy)), dmul(g[2], vz));
        *by = dadd(dadd(dmul(g[1], vx), dmul(g[3], vy)), dmul(g[4], vz));
        *bz = dadd(dadd(dmul(g[2], vx), dmul(g[4], vy)), dmul(g[5], vz));
    }
    fft_lines_d(smd, M, LS, 3 * tz, a.twi, true);
    for (int e = threadIdx.x; e < 3 * a.ni * tz; e += blockDim.x) {
        const int t = e % tz, i = (e / tz) % a.ni, c = e / (tz * a.ni);
        a.work[wrow(a, c, i, ky) + kz0 + t] = smd[(c * tz + t) * LS + i];
    }
}

// ZI: rows (c, i, j0 .. j0 + kLJ), inverse along l, l < nl kept, epilogue
__global__ void __launch_bounds__(kT) z_inv(Mv64 a, Ep64 ep, double2 *__restrict__ out)
{
    extern __shared__ double2 smd[];
    const int M = 2 * a.nl, LS = M + 1, j0 = blockIdx.x * kLJ, i = blockIdx.y, c = blockIdx.z;
    const int nr = a.nj - j0 < kLJ ? a.nj - j0 : kLJ;
    for (int e = threadIdx.x; e < nr * M; e += blockDim.x) {
        const int t = e / M, k = e - t * M;
        smd[t * LS + k] = a.work[wrow(a, c, i, j0 + t) + k];
    }
    fft_lines_d(smd, M, LS, nr, a.twl, true);
    for (int e = threadIdx.x; e < nr * a.nl; e += blockDim.x) {
        const int t = e / a.nl, l = e - t * a.nl;
        const size_t q = ((size_t)i * a.nj + j0 + t) * a.nl + l, o = (size_t)c * a.N + q;
        const double2 conv = smd[t * LS + l];
        double2 res = conv;
        if (ep.mode == 1) {
            const int m = ep.occ[q];
            if (!ep.mv[m]) {
                res = dzero();
            } else {
                double2 al = ep.alpha[m];
                if (ep.conj) al = dconj(al);
                const double2 sv = ep.sv != 0.0 ? make_double2(ep.v[o].x * ep.sv, ep.v[o].y * ep.sv) : dzero();
                res = dsub(sv, dmul(al, conv));
            }
        }
        out[o] = res;
    }
}

// ---------------------------------------------------------------- field operations
using F64 = Field64View;

__device__ __forceinline__ bool active(const F64 &f, size_t q) { return f.mv[f.occ[q]] != 0; }

// p = alpha_m exp(i k.(r - c)) E_inc on active cells, c = (n - 1) d0 / 2 (FirstApproximation,
// dda_func.cpp:654-689); with rhs: p = rhs on active cells
__global__ void first_approx64(F64 f, double d0, double k0, double k1, double k2, double2 e0,
                               double2 e1, double2 e2, const double2 *rhs, double2 *p)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= f.N) return;
    const int l = (int)(q % f.nl), j = (int)((q / f.nl) % f.nj), i = (int)(q / ((size_t)f.nl * f.nj));
    double2 o[3] = {dzero(), dzero(), dzero()};
    if (active(f, q)) {
        if (rhs) {
            for (int c = 0; c < 3; c++) o[c] = rhs[c * f.N + q];
        } else {
            const double ph = k0 * (i * d0 - (f.ni - 1) * d0 / 2) + k1 * (j * d0 - (f.nj - 1) * d0 / 2) +
                              k2 * (l * d0 - (f.nl - 1) * d0 / 2);
            double s, co;
            sincos(ph, &s, &co);
            const double2 c1 = dmul(make_double2(co, s), f.alpha[f.occ[q]]);
            o[0] = dmul(c1, e0);
            o[1] = dmul(c1, e1);
            o[2] = dmul(c1, e2);
        }
    }
    for (int c = 0; c < 3; c++) p[c * f.N + q] = o[c];
}

// Block sums of (a) the bilinear product sum a b (ldcScalMul, dda_func.cpp:724-755),
// (b) Re sum a conj(b) (ldScalMulConj, 757-782) and (c) sum over cells of |r| (ldError's
// numerator, 784-811), over active cells, added to acc[0..1] in FP64.
__global__ void __launch_bounds__(kT) reduce64(F64 f, int kind, const double2 *a, const double2 *b,
                                               double *acc)
{
    double s0 = 0.0, s1 = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < f.N; q += (size_t)gridDim.x * blockDim.x) {
        if (!active(f, q)) continue;
        if (kind == 2) {
            double t = 0.0;
            for (int c = 0; c < 3; c++) {
                const double2 v = a[c * f.N + q];
                t += v.x * v.x + v.y * v.y;
            }
            s0 += sqrt(t);
        } else {
            for (int c = 0; c < 3; c++) {
                const double2 x = a[c * f.N + q], y = b[c * f.N + q];
                if (kind == 0) {
                    s0 += x.x * y.x - x.y * y.y;
                    s1 += x.x * y.y + x.y * y.x;
                } else {
                    s0 += x.x * y.x + x.y * y.y;
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    __shared__ double sh[2][kT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = s0;
        sh[1][w] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            t0 += sh[0][k];
            t1 += sh[1][k];
        }
        atomicAdd(acc, t0);
        atomicAdd(acc + 1, t1);
    }
}

// o = x + c1 y + c2 z on active cells; inactive cells: o = 0 when mask_zero, else unchanged
// (the reference's LinearComb forms, dda_func.cpp:813-974)
__global__ void lin3_64(F64 f, const double2 *x, double2 c1, const double2 *y, double2 c2,
                        const double2 *z, double2 *o, int mask_zero)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= f.N) return;
    const bool act = active(f, q);
    for (int c = 0; c < 3; c++) {
        const size_t k = c * f.N + q;
        if (act) {
            double2 v = x[k];
            if (y) v = dadd(v, dmul(c1, y[k]));
            if (z) v = dadd(v, dmul(c2, z[k]));
            o[k] = v;
        } else if (mask_zero) {
            o[k] = dzero();
        }
    }
}

// simple iteration (dda_func.cpp:1471-1521): r = (p - alpha conv) - s, p -= tau r on active
// cells (w holds p - alpha conv there), both zero elsewhere
__global__ void simple64(F64 f, const double2 *w, const double2 *s, double2 *r, double2 *p, double tau)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= f.N) return;
    const bool act = active(f, q);
    for (int c = 0; c < 3; c++) {
        const size_t k = c * f.N + q;
        if (act) {
            const double2 rr = dsub(w[k], s[k]);
            r[k] = rr;
            p[k] = dsub(p[k], make_double2(tau * rr.x, tau * rr.y));
        } else {
            r[k] = dzero();
            p[k] = dzero();
        }
    }
}

// far field of one direction per block row (FarField, dda_func.cpp:1576-1625) and CabsCext
// (1679-1727, centre n d0 / 2, cells skipped where alpha == 0), summed in FP64
__global__ void __launch_bounds__(kT) farfield64(F64 f, double d0, const double *ksc, const double2 *p,
                                                 double *esc)
{
    const double *k = ksc + 3 * blockIdx.y;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < f.N; q += (size_t)gridDim.x * blockDim.x) {
        if (!active(f, q)) continue;
        const int l = (int)(q % f.nl), j = (int)((q / f.nl) % f.nj), i = (int)(q / ((size_t)f.nl * f.nj));
        const double ph = k[0] * (i * d0 - (f.ni - 1) * d0 / 2) + k[1] * (j * d0 - (f.nj - 1) * d0 / 2) +
                          k[2] * (l * d0 - (f.nl - 1) * d0 / 2);
        double s, co;
        sincos(ph, &s, &co);
        const double2 P[3] = {p[q], p[f.N + q], p[2 * f.N + q]};
        const double2 kp = make_double2(k[0] * P[0].x + k[1] * P[1].x + k[2] * P[2].x,
                                        k[0] * P[0].y + k[1] * P[1].y + k[2] * P[2].y);
        for (int c = 0; c < 3; c++) {
            const double2 v = make_double2(P[c].x - k[c] * kp.x, P[c].y - k[c] * kp.y);
            acc[2 * c] += co * v.x - s * v.y;
            acc[2 * c + 1] += co * v.y + s * v.x;
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int c = 0; c < 6; c++) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    __shared__ double sh[6][kT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int c = 0; c < 6; c++) sh[c][w] = acc[c];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0.0;
        for (int u = 0; u < (int)(blockDim.x >> 5); u++) t += sh[threadIdx.x][u];
        atomicAdd(esc + 6 * blockIdx.y + threadIdx.x, t);
    }
}

__global__ void __launch_bounds__(kT) cabscext64(F64 f, int nmat1, double d0, double k0, double k1,
                                                 double k2, double2 e0, double2 e1, double2 e2,
                                                 const double2 *p, double *acc)
{
    double r1 = 0.0, r2 = 0.0;
    const double cx = f.ni * d0 / 2, cy = f.nj * d0 / 2, cz = f.nl * d0 / 2;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < f.N; q += (size_t)gridDim.x * blockDim.x) {
        const int m = f.occ[q];
        if (m < 0 || m >= nmat1) continue;
        const double2 a = f.alpha[m];
        if (a.x == 0.0 && a.y == 0.0) continue;
        const int l = (int)(q % f.nl), j = (int)((q / f.nl) % f.nj), i = (int)(q / ((size_t)f.nl * f.nj));
        const double ph = -(k0 * (i * d0 - cx) + k1 * (j * d0 - cy) + k2 * (l * d0 - cz));
        double s, co;
        sincos(ph, &s, &co);
        const double2 P[3] = {p[q], p[f.N + q], p[2 * f.N + q]};
        const double2 E[3] = {dconj(e0), dconj(e1), dconj(e2)};
        double2 pe = dzero();
        double pp = 0.0;
        for (int c = 0; c < 3; c++) {
            pe = dadd(pe, dmul(P[c], E[c]));
            pp += P[c].x * P[c].x + P[c].y * P[c].y;
        }
        r1 += dmul(make_double2(co, s), pe).y;
        // Im(pp / conj(a)) = pp Im(a) / |a|^2
        r2 += pp * a.y / (a.x * a.x + a.y * a.y) - (2.0 / 3.0) * pp;
    }
    for (int o = 16; o > 0; o >>= 1) {
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    }
    __shared__ double sh[2][kT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = r1;
        sh[1][w] = r2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int u = 0; u < (int)(blockDim.x >> 5); u++) {
            t0 += sh[0][u];
            t1 += sh[1][u];
        }
        atomicAdd(acc, t0);
        atomicAdd(acc + 1, t1);
    }
}

// ---------------------------------------------------------------- mixed precision (COCG)
// block sums of NV doubles per thread, added to acc[0 .. NV)
template <int NV>
__device__ void block_add(double (&v)[NV], double *acc)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __shared__ double sh[NV][kT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k][w] = v[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int u = 0; u < (int)(blockDim.x >> 5); u++) t += sh[threadIdx.x][u];
        atomicAdd(acc + threadIdx.x, t);
    }
}

__global__ void to_f32(const double2 *x, float2 *y, size_t n)
{
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        y[q] = make_float2((float)x[q].x, (float)x[q].y);
}

__global__ void from_f32_masked(F64 f, const float2 *x, double2 *y)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= f.N) return;
    const bool act = active(f, q);
    for (int c = 0; c < 3; c++) {
        const float2 v = x[c * f.N + q];
        y[c * f.N + q] = act ? make_double2(v.x, v.y) : dzero();
    }
}

// out = v - alpha_m conv (- sub) on active cells, 0 elsewhere, in FP64 from the float
// convolution; acc (may be null): acc[0] += sum over cells of |out| (ldError's numerator)
__global__ void __launch_bounds__(kT) mixed_apply(F64 f, const double2 *v, const float2 *conv,
                                                  const double2 *sub, double2 *out, double *acc)
{
    double e[1] = {0.0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < f.N; q += (size_t)gridDim.x * blockDim.x) {
        const int m = f.occ[q];
        if (!f.mv[m]) {
            for (int c = 0; c < 3; c++) out[c * f.N + q] = dzero();
            continue;
        }
        const double2 al = f.alpha[m];
        double t = 0.0;
        for (int c = 0; c < 3; c++) {
            const size_t k = c * f.N + q;
            const float2 g = conv[k];
            double2 o = dsub(v[k], dmul(al, make_double2(g.x, g.y)));
            if (sub) o = dsub(o, sub[k]);
            out[k] = o;
            t += o.x * o.x + o.y * o.y;
        }
        e[0] += sqrt(t);
    }
    if (acc) block_add<1>(e, acc);
}

// acc[0..1] += sum s w (bilinear), acc[2..3] += sum r s, over active cells
__global__ void __launch_bounds__(kT) cg_dots(F64 f, const double2 *s, const double2 *w, const double2 *r,
                                              double *acc)
{
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < f.N; q += (size_t)gridDim.x * blockDim.x) {
        if (!active(f, q)) continue;
        for (int c = 0; c < 3; c++) {
            const size_t k = c * f.N + q;
            const double2 a = s[k], b = w[k], d = r[k];
            v[0] += a.x * b.x - a.y * b.y;
            v[1] += a.x * b.y + a.y * b.x;
            v[2] += d.x * a.x - d.y * a.y;
            v[3] += d.x * a.y + d.y * a.x;
        }
    }
    block_add<4>(v, acc);
}

// x -= a s; r -= a w on active cells; acc[0..1] += sum r w, acc[2] += sum |r| (the new r)
__global__ void __launch_bounds__(kT) cg_update(F64 f, double2 a, double2 *x, double2 *r, const double2 *s,
                                                const double2 *w, double *acc)
{
    double v[3] = {0.0, 0.0, 0.0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < f.N; q += (size_t)gridDim.x * blockDim.x) {
        if (!active(f, q)) continue;
        double t = 0.0;
        for (int c = 0; c < 3; c++) {
            const size_t k = c * f.N + q;
            const double2 sv = s[k], wv = w[k];
            x[k] = dsub(x[k], dmul(a, sv));
            const double2 rv = dsub(r[k], dmul(a, wv));
            r[k] = rv;
            v[0] += rv.x * wv.x - rv.y * wv.y;
            v[1] += rv.x * wv.y + rv.y * wv.x;
            t += rv.x * rv.x + rv.y * rv.y;
        }
        v[2] += sqrt(t);
    }
    block_add<3>(v, acc);
}

// s = r - b s on active cells (inactive cells keep their zeros); s32 = float(s)
__global__ void cg_dir(F64 f, double2 b, const double2 *r, double2 *s, float2 *s32)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= f.N) return;
    const bool act = active(f, q);
    for (int c = 0; c < 3; c++) {
        const size_t k = c * f.N + q;
        double2 v = s[k];
        if (act) v = dsub(r[k], dmul(b, v));
        s[k] = v;
        s32[k] = make_float2((float)v.x, (float)v.y);
    }
}

inline unsigned nb(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ------------------------------------------------------------------ host side

Fp64Buffers::~Fp64Buffers() { release(); }

void Fp64Buffers::release()
{
    void *ptrs[] = {g, tw, work, p, pmin, r, s, gg, h, w, b, alpha, acc};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    g = tw = work = p = pmin = r = s = gg = h = w = b = alpha = nullptr;
    acc = nullptr;
    ni = nj = nl = 0;
}

cudaError_t Fp64Buffers::ensure(int ni_, int nj_, int nl_, double kd_, cudaStream_t st)
{
    if (g && ni == ni_ && nj == nj_ && nl == nl_ && kd == kd_) return cudaSuccess;
    release();
    const size_t N = (size_t)ni_ * nj_ * nl_, n3 = 3 * N;
    const size_t oct = (size_t)6 * (ni_ + 1) * (nj_ + 1) * (nl_ + 1);
    const size_t wst = (size_t)3 * ni_ * (2 * nj_) * (2 * nl_);
    cudaError_t e = cudaSuccess;
    auto A = [&](double2 **q, size_t n) {
        if (e == cudaSuccess) e = cudaMalloc((void **)q, n * sizeof(double2));
    };
    A(&g, oct);
    A(&tw, (size_t)ni_ + nj_ + nl_);
    A(&work, wst);
    A(&p, n3);
    A(&pmin, n3);
    A(&r, n3);
    A(&s, n3);
    A(&gg, n3);
    A(&h, n3);
    A(&w, n3);
    A(&b, n3);
    A(&alpha, 256);
    if (e == cudaSuccess) e = cudaMalloc((void **)&acc, 8 * sizeof(double));
    if (e != cudaSuccess) {
        release();
        return e;
    }
    ni = ni_;
    nj = nj_;
    nl = nl_;
    kd = kd_;
    // twiddles exp(-2 pi i k / 2n), k < n, per axis, in FP64
    std::vector<double2> t((size_t)ni + nj + nl);
    const double pi = 3.14159265358979323846264338327950288;
    const int ns[3] = {ni, nj, nl};
    size_t o = 0;
    for (int ax = 0; ax < 3; ax++)
        for (int k = 0; k < ns[ax]; k++, o++)
            t[o] = make_double2(std::cos(-pi * k / ns[ax]), std::sin(-pi * k / ns[ax]));
    if ((e = cudaMemcpyAsync(tw, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, st)) ||
        (e = green_build_octant64(ni, nj, nl, kd, g, st)) || (e = cudaStreamSynchronize(st))) {
        release();
        return e;
    }
    return cudaSuccess;
}

namespace {

struct Fp64Run {
    Fp64Buffers &B;
    cudaStream_t st;
    F64 f;
    Mv64 m;
    int nact;
    long long *launches;
    int matvecs = 0;

    static size_t smem(int M, int lines) { return (size_t)lines * (M + 1) * sizeof(double2); }

    // out = sv v - alpha_m conv(src) on active cells (0 elsewhere); conj: the conjugate
    // operator with conj(alpha) (Convolution_conj)
    cudaError_t matvec(const double2 *src, double2 *out, double sv, const double2 *v, int conj)
    {
        Mv64 a = m;
        a.conj = conj;
        Ep64 ep{1, sv, v, f.occ, f.mv, f.alpha, conj};
        const int ni = a.ni, nj = a.nj, nl = a.nl, tz = 2 * nl < kTZ ? 2 * nl : kTZ;
        z_fwd<<<dim3(nb(nj, kLJ), ni, 3), kT, smem(2 * nl, kLJ), st>>>(a, src);
        y_pass<<<dim3(2 * nl / tz, ni, 3), kT, smem(2 * nj, tz), st>>>(a, 0, tz);
        x_pass<<<dim3(2 * nl / tz, 2 * nj), kT, smem(2 * ni, 3 * tz), st>>>(a, tz);
        y_pass<<<dim3(2 * nl / tz, ni, 3), kT, smem(2 * nj, tz), st>>>(a, 1, tz);
        z_inv<<<dim3(nb(nj, kLJ), ni, 3), kT, smem(2 * nl, kLJ), st>>>(a, ep, out);
        *launches += 5;
        matvecs++;
        return cudaGetLastError();
    }

    cudaError_t reduce(int kind, const double2 *a, const double2 *b, double out[2])
    {
        cudaError_t e = cudaMemsetAsync(B.acc, 0, 2 * sizeof(double), st);
        if (e) return e;
        reduce64<<<4 * 148, kT, 0, st>>>(f, kind, a, b, B.acc);
        *launches += 1;
        if ((e = cudaMemcpyAsync(out, B.acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st))) return e;
        return cudaStreamSynchronize(st);
    }
    cudaError_t bil(const double2 *a, const double2 *b, std::complex<double> &z)
    {
        double o[2];
        cudaError_t e = reduce(0, a, b, o);
        z = {o[0], o[1]};
        return e;
    }
    cudaError_t herm(const double2 *a, const double2 *b, double &x)
    {
        double o[2];
        cudaError_t e = reduce(1, a, b, o);
        x = o[0];
        return e;
    }
    cudaError_t err(const double2 *r, double &x)
    {
        double o[2];
        cudaError_t e = reduce(2, r, nullptr, o);
        x = o[0] / nact;
        return e;
    }
    cudaError_t lin3(const double2 *x, std::complex<double> c1, const double2 *y, std::complex<double> c2,
                     const double2 *z, double2 *o, int mask_zero)
    {
        lin3_64<<<nb(f.N, kT), kT, 0, st>>>(f, x, make_double2(c1.real(), c1.imag()), y,
                                             make_double2(c2.real(), c2.imag()), z, o, mask_zero);
        *launches += 1;
        return cudaGetLastError();
    }
    cudaError_t copy(double2 *dst, const double2 *src)
    {
        return cudaMemcpyAsync(dst, src, 3 * f.N * sizeof(double2), cudaMemcpyDeviceToDevice, st);
    }
};

}  // namespace

#define CKE(x)                                                                               \
    do {                                                                                     \
        cudaError_t _e = (x);                                                                \
        if (_e != cudaSuccess) return _e;                                                    \
    } while (0)

cudaError_t solve_fp64(Fp64Buffers &B, const Fp64Problem &P, cudaStream_t st, Fp64Result &R,
                       long long *launches)
{
    typedef std::complex<double> cd;
    const int ni = B.ni, nj = B.nj, nl = B.nl;
    const size_t N = (size_t)ni * nj * nl;
    // the passes hold up to 3 kTZ lines of 2n + 1 points in shared memory
    const int big = (int)Fp64Run::smem(2 * ni, 3 * kTZ);
    CKE(raise_smem_limit((const void *)x_pass, big));
    CKE(raise_smem_limit((const void *)y_pass, (int)Fp64Run::smem(2 * nj, kTZ)));
    CKE(raise_smem_limit((const void *)z_fwd, (int)Fp64Run::smem(2 * nl, kLJ)));
    CKE(raise_smem_limit((const void *)z_inv, (int)Fp64Run::smem(2 * nl, kLJ)));
    CKE(cudaMemcpyAsync(B.alpha, P.alpha, P.nmat1 * sizeof(double2), cudaMemcpyHostToDevice, st));
    F64 f{N, ni, nj, nl, P.occ, P.mv, B.alpha};
    Mv64 m{ni, nj, nl, N, B.tw, B.tw + ni, B.tw + ni + nj, B.g, B.work, 0};
    Fp64Run X{B, st, f, m, P.nact, launches};
    double2 *p = B.p, *pmin = B.pmin, *r = B.r, *s = B.s, *g = B.gg, *h = B.h, *w = B.w, *b = B.b;
    const size_t bytes = 3 * N * sizeof(double2);
    const int solver = P.solver;

    // right-hand side b (p_inc or the caller's), start p = x0 or b (dda_func.cpp:1102-1104)
    if (P.rhs) CKE(cudaMemcpyAsync(w, P.rhs, bytes, cudaMemcpyHostToDevice, st));
    first_approx64<<<nb(N, kT), kT, 0, st>>>(f, P.d0, P.kinc[0], P.kinc[1], P.kinc[2],
                                             make_double2(P.einc[0], P.einc[1]),
                                             make_double2(P.einc[2], P.einc[3]),
                                             make_double2(P.einc[4], P.einc[5]), P.rhs ? w : nullptr, b);
    *launches += 1;
    if (P.x0) {
        CKE(cudaMemcpyAsync(w, P.x0, bytes, cudaMemcpyHostToDevice, st));
        CKE(X.lin3(w, 0.0, nullptr, 0.0, nullptr, p, 1));          // p = x0 on active cells
        CKE(X.matvec(p, w, 1.0, p, 0));                              // w = A p
        CKE(X.lin3(w, -1.0, b, 0.0, nullptr, r, 1));                // r = A p - b
    } else {
        CKE(X.copy(p, b));
        CKE(X.matvec(p, r, 0.0, nullptr, 0));                        // r = -alpha conv(p)
    }

    cd ldA = 0, ldW = 0, rho1 = 0, z;
    double RR1 = 0;
    if (solver == 0) CKE(X.copy(s, r));
    if (solver == 1) {
        CKE(X.herm(r, r, RR1));
        CKE(X.matvec(r, s, 1.0, r, 1));
    }
    if (solver == 2) {
        CKE(X.copy(g, r));
        CKE(X.copy(s, r));
        CKE(X.bil(r, g, rho1));
        CKE(X.matvec(s, h, 1.0, s, 0));
        CKE(X.bil(g, h, z));
        ldA = rho1 / z;
        CKE(X.lin3(r, -ldA, h, 0.0, nullptr, r, 0));
        CKE(X.matvec(r, w, 1.0, r, 0));
        cd wr, ww;
        CKE(X.bil(w, r, wr));
        CKE(X.bil(w, w, ww));
        ldW = wr / ww;
        CKE(X.lin3(p, -ldA, s, -ldW, r, p, 1));
        CKE(X.lin3(r, -ldW, w, 0.0, nullptr, r, 0));
    }
    if (solver == 3) {
        CKE(X.copy(s, p));
        CKE(X.lin3(s, -1.0, r, 0.0, nullptr, p, 0));   // p = s - r (r vanishes off the target)
    }
    double err = 0;
    CKE(X.err(r, err));
    double err_min = err;
    int step_min = 0, nt = 0;
    if (R.trace && nt < R.trace_len) R.trace[nt] = err;
    nt++;
    CKE(X.copy(pmin, p));
    for (int o = 1; o <= P.max_step; o++) {   // dda_func.cpp:1301-1535
        if (err <= P.err_max) break;
        if (err < err_min) {
            err_min = err;
            step_min = o - 1;
            CKE(X.copy(pmin, p));
        }
        if (solver == 2) {
            cd rho;
            CKE(X.bil(r, g, rho));
            const cd ldB = (rho * ldA) / (rho1 * ldW);
            CKE(X.lin3(r, ldB, s, -(ldB * ldW), h, s, 1));
            rho1 = rho;
            CKE(X.matvec(s, h, 1.0, s, 0));
            CKE(X.bil(g, h, z));
            ldA = rho / z;
            CKE(X.lin3(r, -ldA, h, 0.0, nullptr, r, 0));
            CKE(X.matvec(r, w, 1.0, r, 0));
            cd wr, ww;
            CKE(X.bil(w, r, wr));
            CKE(X.bil(w, w, ww));
            ldW = wr / ww;
            CKE(X.lin3(p, -ldA, s, -ldW, r, p, 1));
            CKE(X.lin3(r, -ldW, w, 0.0, nullptr, r, 0));
        } else if (solver == 0) {
            CKE(X.matvec(s, w, 1.0, s, 0));
            cd den, rs, rw;
            CKE(X.bil(s, w, den));
            CKE(X.bil(r, s, rs));
            const cd a = rs / den;
            CKE(X.lin3(p, -a, s, 0.0, nullptr, p, 0));
            CKE(X.lin3(r, -a, w, 0.0, nullptr, r, 0));
            CKE(X.bil(r, w, rw));
            const cd bb = rw / den;
            CKE(X.lin3(r, -bb, s, 0.0, nullptr, s, 0));
        } else if (solver == 1) {
            CKE(X.matvec(s, w, 1.0, s, 0));
            double SS, RR;
            CKE(X.herm(s, s, SS));
            const double rA = -RR1 / SS;
            CKE(X.lin3(r, rA, w, 0.0, nullptr, r, 0));
            CKE(X.lin3(p, rA, s, 0.0, nullptr, p, 0));
            CKE(X.herm(r, r, RR));
            const double rB = RR / RR1;
            RR1 = RR;
            CKE(X.matvec(r, w, 1.0, r, 1));
            CKE(X.lin3(w, rB, s, 0.0, nullptr, s, 0));
        } else {
            CKE(X.matvec(p, w, 1.0, p, 0));
            simple64<<<nb(N, kT), kT, 0, st>>>(f, w, s, r, p, P.tau);
            *launches += 1;
        }
        CKE(X.err(r, err));
        if (R.trace && nt < R.trace_len) R.trace[nt] = err;
        nt++;
    }
    R.steps = nt - 1;
    R.err = err;
    R.err_min = err < err_min ? err : err_min;
    R.step_min = -1;
    if (err > err_min) {   // best-iterate rollback, dda_func.cpp:1537-1548
        CKE(X.copy(p, pmin));
        R.step_min = step_min;
    }
    R.rolled_back = R.step_min >= 0;
    R.matvecs = X.matvecs;
    // CabsCext and the far field of the final dipoles
    CKE(cudaMemsetAsync(B.acc, 0, 2 * sizeof(double), st));
    cabscext64<<<4 * 148, kT, 0, st>>>(f, P.nmat1, P.d0, P.kinc[0], P.kinc[1], P.kinc[2],
                                       make_double2(P.einc[0], P.einc[1]), make_double2(P.einc[2], P.einc[3]),
                                       make_double2(P.einc[4], P.einc[5]), p, B.acc);
    *launches += 1;
    double cc[2];
    CKE(cudaMemcpyAsync(cc, B.acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (P.ndir > 0) {
        double *kd = nullptr, *ed = nullptr;
        CKE(cudaMallocAsync((void **)&kd, (size_t)P.ndir * 3 * sizeof(double), st));
        CKE(cudaMallocAsync((void **)&ed, (size_t)P.ndir * 6 * sizeof(double), st));
        CKE(cudaMemcpyAsync(kd, P.ksc, (size_t)P.ndir * 3 * sizeof(double), cudaMemcpyHostToDevice, st));
        CKE(cudaMemsetAsync(ed, 0, (size_t)P.ndir * 6 * sizeof(double), st));
        farfield64<<<dim3(2 * 148, P.ndir), kT, 0, st>>>(f, P.d0, kd, p, ed);
        *launches += 1;
        CKE(cudaMemcpyAsync(R.esc, ed, (size_t)P.ndir * 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
        cudaFreeAsync(kd, st);
        cudaFreeAsync(ed, st);
    }
    CKE(cudaStreamSynchronize(st));
    double e2 = 0;
    for (int c = 0; c < 6; c++) e2 += P.einc[c] * P.einc[c];
    const double pi = 3.14159265358979323846264338327950288;
    R.cext = 4.0 * pi / e2 * cc[0];
    R.cabs = 4.0 * pi / e2 * cc[1];
    if (R.p) CKE(cudaMemcpyAsync(R.p, p, bytes, cudaMemcpyDeviceToHost, st));
    return cudaStreamSynchronize(st);
}

// ------------------------------------------------------------------ mixed precision (host)

MixedCgBuffers::~MixedCgBuffers() { release(); }

void MixedCgBuffers::release()
{
    void *ptrs[] = {x, r, s, w, b, best, alpha, acc};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    x = r = s = w = b = best = alpha = nullptr;
    acc = nullptr;
    n3 = 0;
}

cudaError_t MixedCgBuffers::ensure(size_t n)
{
    if (x && n3 == n) return cudaSuccess;
    release();
    cudaError_t e = cudaSuccess;
    auto A = [&](double2 **q, size_t k) {
        if (e == cudaSuccess) e = cudaMalloc((void **)q, k * sizeof(double2));
    };
    A(&x, n);
    A(&r, n);
    A(&s, n);
    A(&w, n);
    A(&b, n);
    A(&best, n);
    A(&alpha, 256);
    if (e == cudaSuccess) e = cudaMalloc((void **)&acc, 8 * sizeof(double));
    if (e != cudaSuccess) {
        release();
        return e;
    }
    n3 = n;
    return cudaSuccess;
}

cudaError_t f64_right_hand_side(const Field64View &f, double d0, const double *kinc,
                                const double *einc, const float2 *from_f32, double2 *out,
                                cudaStream_t st)
{
    if (from_f32) {
        from_f32_masked<<<nb(f.N, kT), kT, 0, st>>>(f, from_f32, out);
    } else {
        first_approx64<<<nb(f.N, kT), kT, 0, st>>>(f, d0, kinc[0], kinc[1], kinc[2],
                                                   make_double2(einc[0], einc[1]),
                                                   make_double2(einc[2], einc[3]),
                                                   make_double2(einc[4], einc[5]), nullptr, out);
    }
    return cudaGetLastError();
}

cudaError_t mixed_cg(MixedCgBuffers &B, const Field64View &f, const double2 *alpha_host, int nmat1,
                     int nact, double err_max, int max_outer, double inner_rel, int inner_max_step,
                     const ConvFn &conv, float2 *s32, float2 *conv32, float2 *x32, float2 *p32,
                     cudaStream_t st, MixedCgResult &R, long long *launches)
{
    typedef std::complex<double> cd;
    const size_t N = f.N, n3 = 3 * N, bytes = n3 * sizeof(double2);
    const unsigned red = 4 * 148;
    double h[4];
    auto sums = [&](int k) -> cudaError_t {
        CKE(cudaMemcpyAsync(h, B.acc, k * sizeof(double), cudaMemcpyDeviceToHost, st));
        return cudaStreamSynchronize(st);
    };
    auto zero = [&]() { return cudaMemsetAsync(B.acc, 0, 4 * sizeof(double), st); };
    // true residual r = x - alpha G*x - b and its discrepancy (ldError of it)
    auto true_residual = [&](double &err) -> cudaError_t {
        to_f32<<<red, kT, 0, st>>>(B.x, x32, n3);
        CKE(conv(x32, conv32));
        CKE(zero());
        mixed_apply<<<red, kT, 0, st>>>(f, B.x, conv32, B.b, B.r, B.acc);
        *launches += 2;
        R.matvecs++;
        CKE(sums(1));
        err = h[0] / nact;
        return cudaSuccess;
    };
    CKE(cudaMemcpyAsync(B.alpha, alpha_host, nmat1 * sizeof(double2), cudaMemcpyHostToDevice, st));
    CKE(cudaMemcpyAsync(B.x, B.b, bytes, cudaMemcpyDeviceToDevice, st));   // x = b (p_inc)
    R = MixedCgResult();
    double err = 0;
    CKE(true_residual(err));
    R.history[0] = err;
    double err_best = err, anchor = err;
    CKE(cudaMemcpyAsync(B.best, B.x, bytes, cudaMemcpyDeviceToDevice, st));
    if (err > err_max) {
        CKE(cudaMemcpyAsync(B.s, B.r, bytes, cudaMemcpyDeviceToDevice, st));
        to_f32<<<red, kT, 0, st>>>(B.s, s32, n3);
        *launches += 1;
        int since = 0;
        const long long cap = (long long)(max_outer + 1) * inner_max_step;
        for (long long it = 0; it < cap; it++) {
            // w = A s (dda_func.cpp:1325-1357)
            CKE(conv(s32, conv32));
            mixed_apply<<<red, kT, 0, st>>>(f, B.s, conv32, nullptr, B.w, nullptr);
            CKE(zero());
            cg_dots<<<red, kT, 0, st>>>(f, B.s, B.w, B.r, B.acc);
            *launches += 2;
            R.matvecs++;
            CKE(sums(4));
            const cd den(h[0], h[1]), rs(h[2], h[3]);
            const cd a = rs / den;   // dda_func.cpp:1359-1371, without the float casts
            CKE(zero());
            cg_update<<<red, kT, 0, st>>>(f, make_double2(a.real(), a.imag()), B.x, B.r, B.s, B.w, B.acc);
            CKE(sums(3));
            const cd bb = cd(h[0], h[1]) / den;
            const double err_rec = h[2] / nact;
            cg_dir<<<nb(N, kT), kT, 0, st>>>(f, make_double2(bb.real(), bb.imag()), B.r, B.s, s32);
            *launches += 2;
            R.iterations++;
            since++;
            if (err_rec <= err_max || err_rec <= inner_rel * anchor || since >= inner_max_step) {
                CKE(true_residual(err));
                R.outer++;
                if (R.outer < 64) R.history[R.outer] = err;
                if (err < err_best) {
                    err_best = err;
                    CKE(cudaMemcpyAsync(B.best, B.x, bytes, cudaMemcpyDeviceToDevice, st));
                }
                if (err <= err_max || R.outer >= max_outer) break;
                // restart from the current solution: fresh direction s = r (true residual)
                CKE(cudaMemcpyAsync(B.s, B.r, bytes, cudaMemcpyDeviceToDevice, st));
                to_f32<<<red, kT, 0, st>>>(B.s, s32, n3);
                *launches += 1;
                anchor = err;
                since = 0;
            }
        }
    }
    if (err > err_best) CKE(cudaMemcpyAsync(B.x, B.best, bytes, cudaMemcpyDeviceToDevice, st));
    R.err = err < err_best ? err : err_best;
    to_f32<<<red, kT, 0, st>>>(B.x, p32, n3);
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace ddagpu
