// Post-processing of the solved dipoles: extinction and absorption cross sections
// (CabsCext, dda_func.cpp:1679-1727), the far-field amplitude sums (FarField,
// dda_func.cpp:1576-1625), and the Jones -> Mueller conversion averaged over scattering
// planes (BuildMatrixJones and JonesToMuller, mmuller.cpp:175-314; averaging
// main.cpp:943-954).
//
// The far field is computed as S(k) = sum_d exp(i k.(r_d - c)) P_d followed by one
// projection S - k (k.S), equal by linearity to the reference's per-dipole projection.
// The phase is separable, exp(i kx x) exp(i ky y) exp(i kz z), so each CTA builds small
// tables and the inner loop is three complex multiply-adds per dipole and direction.
#include <mutex>

#include "common.cuh"
#include "internal.h"
#include "post.h"

namespace ddagpu {

namespace {

// Far-field tiling: a CTA takes FF_PLANES lattice planes i of one right-hand side and up
// to FF_DMAX directions (the phase tables, one per axis, are built once for them); a
// thread accumulates FF_DPT directions x 3 components for the rows rg, rg + RG, ... of
// each staged group and the columns of its column group lg, so every staged dipole value
// and phase factor it loads from shared memory feeds 4 to 12 complex multiply-adds.
constexpr int FF_DMAX = 32;
constexpr int FF_DPT = 4;
constexpr int FF_CELLS = 2048;   // lattice cells staged per round
constexpr int FF_PLANES = 8;     // lattice planes per CTA

struct FFShape {
    int D, DG, rows, RG, LG, threads;
};

FFShape ff_shape(int ndir, int nj, int nl)
{
    FFShape s;
    s.D = ndir >= FF_DMAX ? FF_DMAX : ((ndir + FF_DPT - 1) / FF_DPT) * FF_DPT;
    if (s.D < FF_DPT) s.D = FF_DPT;
    s.DG = s.D / FF_DPT;
    s.rows = FF_CELLS / nl < nj ? FF_CELLS / nl : nj;
    if (s.rows < 1) s.rows = 1;
    s.RG = 256 / s.DG < s.rows ? 256 / s.DG : s.rows;
    // column groups: a power of two (it divides nl), at least 8 columns each
    s.LG = 1;
    while (2 * s.LG * s.DG * s.RG <= 256 && 2 * s.LG * 8 <= nl) s.LG *= 2;
    s.threads = s.DG * s.RG * s.LG;
    return s;
}

size_t ff_smem(const FFShape &s, int nj, int nl)
{
    const size_t tables = (size_t)(nl + nj + FF_PLANES) * s.D;
    const size_t staged = (size_t)s.rows * (3 * nl + 1);
    const size_t red = (size_t)s.threads * FF_DPT * 3;
    return (tables + (staged > red ? staged : red)) * sizeof(float2);
}

// grid (direction chunks of D, plane groups of FF_PLANES, nrhs)
__global__ void __launch_bounds__(256) farfield_sum(PostArgs a, FFShape s)
{
    extern __shared__ float2 sm[];
    const int nj = a.nj, nl = a.nl, D = s.D;
    const int dbase = blockIdx.x * D, i0 = blockIdx.y * FF_PLANES, rhs = blockIdx.z;
    const int np = a.ni - i0 < FF_PLANES ? a.ni - i0 : FF_PLANES;
    const int dg = threadIdx.x % s.DG, rest = threadIdx.x / s.DG;
    const int lg = rest % s.LG, rg = rest / s.LG;
    const int PSR = 3 * nl + 1;            // staged row stride (odd: rows fall on other banks)
    float2 *ez = sm;                       // [nl][D]
    float2 *ey = ez + (size_t)nl * D;      // [nj][D]
    float2 *ex = ey + (size_t)nj * D;      // [FF_PLANES][D]
    float2 *P = ex + FF_PLANES * D;        // [rows][PSR], later the reduction buffer
    __shared__ int span[2 * FF_CELLS / 8]; // first and last dipole column of each staged row
    const double cx = (a.ni - 1) * a.d0 / 2, cy = (nj - 1) * a.d0 / 2, cz = (nl - 1) * a.d0 / 2;
    const double *K = a.ksc + (size_t)rhs * a.ndir * 3;
    for (int e = threadIdx.x; e < (nl + nj + np) * D; e += blockDim.x) {
        const int dl = e % D, pos = e / D, dd = dbase + dl;
        float2 val = czero();
        if (dd < a.ndir) {
            double ph;
            if (pos < nl) ph = K[3 * dd + 2] * (pos * a.d0 - cz);
            else if (pos < nl + nj) ph = K[3 * dd + 1] * ((pos - nl) * a.d0 - cy);
            else ph = K[3 * dd + 0] * ((i0 + pos - nl - nj) * a.d0 - cx);
            val = expi_reduced(ph);
        }
        ez[e] = val;   // ez, ey, ex are consecutive [pos][D] blocks
    }
    __syncthreads();   // the tables are read below before the first staging barrier
    const size_t N = a.N;
    const int lcnt = nl / s.LG, l0 = lg * lcnt;
    float2 acc[FF_DPT][3];
#pragma unroll
    for (int u = 0; u < FF_DPT; u++)
#pragma unroll
        for (int c = 0; c < 3; c++) acc[u][c] = czero();
#pragma unroll 1
    for (int ip = 0; ip < np; ip++) {
    const int i = i0 + ip;
    const float2 *p = a.p + (size_t)rhs * 3 * N + (size_t)i * nj * nl;
    const signed char *occ = a.occ + (size_t)rhs * a.occ_stride + (size_t)i * nj * nl;
    // x phase of this plane folded into the row factors
    float2 exv[FF_DPT];
#pragma unroll
    for (int u = 0; u < FF_DPT; u++) exv[u] = ex[ip * D + FF_DPT * dg + u];
    for (int j0 = 0; j0 < nj; j0 += s.rows) {
        const int rows = nj - j0 < s.rows ? nj - j0 : s.rows;
        __syncthreads();
        for (int rr = threadIdx.x; rr < rows; rr += blockDim.x) {
            span[2 * rr] = nl;
            span[2 * rr + 1] = -1;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < rows * nl; e += blockDim.x) {
            const int rr = e / nl, l = e - rr * nl;
            const size_t q = (size_t)j0 * nl + e;
            const bool act = a.mv[(int)occ[q]] != 0;
#pragma unroll
            for (int c = 0; c < 3; c++) P[rr * PSR + 3 * l + c] = act ? p[c * N + q] : czero();
            if (act) {
                atomicMin(&span[2 * rr], l);
                atomicMax(&span[2 * rr + 1], l);
            }
        }
        __syncthreads();
        for (int rr = rg; rr < rows; rr += s.RG) {
            // only the columns between the row's first and last dipole contribute (the
            // others are zeros; skipping them changes no sum)
            const int lb = span[2 * rr] > l0 ? span[2 * rr] : l0;
            const int le = span[2 * rr + 1] + 1 < l0 + lcnt ? span[2 * rr + 1] + 1 : l0 + lcnt;
            if (lb >= le) continue;
            float2 t[FF_DPT][3];
#pragma unroll
            for (int u = 0; u < FF_DPT; u++)
#pragma unroll
                for (int c = 0; c < 3; c++) t[u][c] = czero();
            const float2 *row = P + rr * PSR;
#pragma unroll 2
            for (int l = lb; l < le; l++) {
                const float4 e01 = *reinterpret_cast<const float4 *>(ez + (size_t)l * D + FF_DPT * dg);
                const float4 e23 = *reinterpret_cast<const float4 *>(ez + (size_t)l * D + FF_DPT * dg + 2);
                const float2 ev[FF_DPT] = {make_float2(e01.x, e01.y), make_float2(e01.z, e01.w),
                                           make_float2(e23.x, e23.y), make_float2(e23.z, e23.w)};
                const float2 pv[3] = {row[3 * l], row[3 * l + 1], row[3 * l + 2]};
#pragma unroll
                for (int u = 0; u < FF_DPT; u++)
#pragma unroll
                    for (int c = 0; c < 3; c++) t[u][c] = cfma(ev[u], pv[c], t[u][c]);
            }
            const float2 *eyr = ey + (size_t)(j0 + rr) * D + FF_DPT * dg;
#pragma unroll
            for (int u = 0; u < FF_DPT; u++) {
                const float2 f = cmul(eyr[u], exv[u]);
#pragma unroll
                for (int c = 0; c < 3; c++) acc[u][c] = cfma(f, t[u][c], acc[u][c]);
            }
        }
    }
    }   // planes of this CTA
    // the sum over row and column groups in FP64
    __syncthreads();
    float2 *red = P;   // [threads][FF_DPT][3]
#pragma unroll
    for (int u = 0; u < FF_DPT; u++)
#pragma unroll
        for (int c = 0; c < 3; c++) red[((size_t)threadIdx.x * FF_DPT + u) * 3 + c] = acc[u][c];
    __syncthreads();
    for (int o = threadIdx.x; o < D * 6; o += blockDim.x) {
        const int dl = o / 6, k = o % 6, u = dl % FF_DPT, g = dl / FF_DPT, c = k >> 1;
        const int dd = dbase + dl;
        if (dd >= a.ndir) continue;
        double sum = 0.0;
        for (int r = 0; r < s.RG * s.LG; r++) {
            const float2 v = red[((size_t)(g + s.DG * r) * FF_DPT + u) * 3 + c];
            sum += (k & 1) ? v.y : v.x;
        }
        if (sum != 0.0) atomicAdd(a.esc_acc + ((size_t)rhs * a.ndir + dd) * 6 + k, sum);
    }
}

// Cext and Cabs sums (before the 4 pi / |E|^2 factor), grid (ni, nrhs)
__global__ void __launch_bounds__(256) cabs_cext_sum(PostArgs a)
{
    extern __shared__ float2 tab[];   // [nj] then [nl]
    __shared__ double scratch[8 * 2];
    const int i = blockIdx.x, rhs = blockIdx.y, nj = a.nj, nl = a.nl;
    const double *k = a.kinc + 3 * rhs, *E = a.einc + 6 * rhs;
    // centre n d0 / 2 (dda_func.cpp:1685), phase -k.(r - c')
    const double cx = a.ni * a.d0 / 2, cy = nj * a.d0 / 2, cz = nl * a.d0 / 2;
    for (int e = threadIdx.x; e < nj + nl; e += blockDim.x) {
        const double ph = e < nj ? -k[1] * (e * a.d0 - cy) : -k[2] * ((e - nj) * a.d0 - cz);
        tab[e] = expi_reduced(ph);
    }
    __syncthreads();
    const float2 exv = expi_reduced(-k[0] * (i * a.d0 - cx));
    const size_t N = a.N;
    const float2 *p = a.p + (size_t)rhs * 3 * N;
    const float2 *al = a.alpha + (size_t)rhs * a.nmat1;
    const signed char *occ = a.occ + (size_t)rhs * a.occ_stride;
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < nj * nl; e += blockDim.x) {
        const size_t q = (size_t)i * nj * nl + e;
        const int m = occ[q];
        const float2 alpha = al[m];
        if (alpha.x == 0.f && alpha.y == 0.f) continue;
        const int j = e / nl, l = e - j * nl;
        double per = 0.0, pei = 0.0, pp = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float2 P = p[c * N + q];
            const double er = E[2 * c], ei = -E[2 * c + 1];   // conj(E)
            per += P.x * er - P.y * ei;
            pei += P.x * ei + P.y * er;
            pp += (double)P.x * P.x + (double)P.y * P.y;
        }
        const float2 ph = cmul(cmul(exv, tab[j]), tab[nj + l]);
        v[0] += (double)ph.x * pei + (double)ph.y * per;   // Im(ph * (P . conj E))
        const double ar = alpha.x, ai = alpha.y;
        v[1] += pp * ai / (ar * ar + ai * ai) - (2.0 / 3.0) * pp;   // Im(pp / conj(alpha)) - 2/3 pp
    }
    block_sum_atomic<2>(v, scratch, a.cc_acc + 2 * rhs);
}

// Esc = S - k (k.S); Cext, Cabs = 4 pi / |E|^2 * sums
__global__ void post_finalize(PostArgs a, float2 *esc, float *cabs, float *cext)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t nd = (size_t)a.nrhs * a.ndir;
    if (q < nd) {
        const double *K = a.ksc + 3 * q, *S = a.esc_acc + 6 * q;
        const double kr = K[0] * S[0] + K[1] * S[2] + K[2] * S[4];
        const double ki = K[0] * S[1] + K[1] * S[3] + K[2] * S[5];
        for (int c = 0; c < 3; c++)
            esc[3 * q + c] = make_float2((float)(S[2 * c] - K[c] * kr), (float)(S[2 * c + 1] - K[c] * ki));
    }
    if (q < (size_t)a.nrhs && cabs && cext) {
        const double *E = a.einc + 6 * q;
        double e2 = 0.0;
        for (int c = 0; c < 6; c++) e2 += E[c] * E[c];
        const double r0 = 4.0 * 3.14159265358979323846 / e2;
        cext[q] = (float)(r0 * a.cc_acc[2 * q]);
        cabs[q] = (float)(r0 * a.cc_acc[2 * q + 1]);
    }
}

struct dc {
    double r, i;
};
__device__ inline dc dcm(dc a, dc b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ inline dc dcs(dc a, dc b) { return {a.r - b.r, a.i - b.i}; }
__device__ inline dc dca(dc a, dc b) { return {a.r + b.r, a.i + b.i}; }
__device__ inline dc dcc(dc a) { return {a.r, -a.i}; }
__device__ inline dc dcdiv(dc a, dc b)
{
    const double d = b.r * b.r + b.i * b.i;
    return {(a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d};
}
__device__ inline dc rdotc(const double *v, const dc *e)
{
    return {v[0] * e[0].r + v[1] * e[1].r + v[2] * e[2].r, v[0] * e[0].i + v[1] * e[1].i + v[2] * e[2].i};
}

// One Mueller matrix per (orientation, angle), averaged over the scattering planes.
// The two polarisations of orientation o are right-hand sides 2o and 2o+1.
__global__ void mueller_avg(MuellerArgs m)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m.norient * m.nangles) return;
    const int o = q / m.nangles, ang = q % m.nangles;
    const double *ki = m.kinc + 6 * o;      // rhs 2o
    double M[16];
    for (int k = 0; k < 16; k++) M[k] = 0.0;
    dc E0[3], E1[3];
    for (int c = 0; c < 3; c++) {
        E0[c] = {m.einc[12 * o + 2 * c], m.einc[12 * o + 2 * c + 1]};
        E1[c] = {m.einc[12 * o + 6 + 2 * c], m.einc[12 * o + 6 + 2 * c + 1]};
    }
    for (int pl = 0; pl < m.nplanes; pl++) {
        const size_t dir = (size_t)pl * m.nangles + ang;
        const double *ks = m.ksc + ((size_t)(2 * o) * m.ndir + dir) * 3;
        const double *nv = m.normals + ((size_t)o * m.nplanes + pl) * 3;
        const float2 *s0 = m.esc + ((size_t)(2 * o) * m.ndir + dir) * 3;
        const float2 *s1 = m.esc + ((size_t)(2 * o + 1) * m.ndir + dir) * 3;
        dc S0[3], S1[3];
        for (int c = 0; c < 3; c++) {
            S0[c] = {s0[c].x, s0[c].y};
            S1[c] = {s1[c].x, s1[c].y};
        }
        // plane basis: across = normal, along = (k x n)/|k x n| for the incident beam and
        // -(k_sc x n)/|k_sc x n| for the scattered one (mmuller.cpp:181-182)
        double pin[3] = {ki[1] * nv[2] - ki[2] * nv[1], ki[2] * nv[0] - ki[0] * nv[2],
                         ki[0] * nv[1] - ki[1] * nv[0]};
        double psc[3] = {ks[1] * nv[2] - ks[2] * nv[1], ks[2] * nv[0] - ks[0] * nv[2],
                         ks[0] * nv[1] - ks[1] * nv[0]};
        const double a1 = sqrt(pin[0] * pin[0] + pin[1] * pin[1] + pin[2] * pin[2]);
        const double a2 = sqrt(psc[0] * psc[0] + psc[1] * psc[1] + psc[2] * psc[2]);
        for (int c = 0; c < 3; c++) {
            pin[c] /= a1;
            psc[c] = -psc[c] / a2;
        }
        const dc i0n = rdotc(nv, E0), i1n = rdotc(nv, E1), i0p = rdotc(pin, E0), i1p = rdotc(pin, E1);
        const dc det = dcs(dcm(i0n, i1p), dcm(i1n, i0p));
        const dc den = {-det.i, det.r};   // i * det
        const dc s0n = rdotc(nv, S0), s1n = rdotc(nv, S1), s0p = rdotc(psc, S0), s1p = rdotc(psc, S1);
        const dc A = dcdiv(dcs(dcm(s1p, i0n), dcm(s0p, i1n)), den);
        const dc B = dcdiv(dcs(dcm(s0p, i1p), dcm(s1p, i0p)), den);
        const dc C = dcdiv(dcs(dcm(s1n, i0n), dcm(s0n, i1n)), den);
        const dc D = dcdiv(dcs(dcm(s0n, i1p), dcm(s1n, i0p)), den);
        const double aa = A.r * A.r + A.i * A.i, bb = B.r * B.r + B.i * B.i,
                     cc = C.r * C.r + C.i * C.i, dd = D.r * D.r + D.i * D.i;
        const dc ab = dcm(A, dcc(B)), dc_ = dcm(D, dcc(C)), ac = dcm(A, dcc(C)),
                 db = dcm(D, dcc(B)), da = dcm(D, dcc(A)), bc = dcm(B, dcc(C)),
                 ad = dcm(A, dcc(D)), cb = dcm(C, dcc(B)), ca = dcm(C, dcc(A));
        // JonesToMuller, mmuller.cpp:254-314
        M[0] += 0.5 * (aa + bb + cc + dd);
        M[1] += 0.5 * (aa - bb + cc - dd);
        M[2] += dca(ab, dc_).r;
        M[3] += dcs(ab, dc_).i;
        M[4] += 0.5 * (aa + bb - cc - dd);
        M[5] += 0.5 * (aa - bb - cc + dd);
        M[6] += dcs(ab, dc_).r;
        M[7] += dca(ab, dc_).i;
        M[8] += dca(ac, db).r;
        M[9] += dcs(ac, db).r;
        M[10] += dca(da, bc).r;
        M[11] += dca(ad, cb).i;
        M[12] += dca(ca, db).i;
        M[13] += dcs(ca, db).i;
        M[14] += dcs(da, bc).i;
        M[15] += dcs(da, bc).r;
    }
    for (int k = 0; k < 16; k++) m.out[(size_t)q * 16 + k] = M[k] / m.nplanes;
}

inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

size_t farfield_smem(int nj, int nl)
{
    // the largest shape any direction count gives on this lattice
    size_t m = 0;
    for (int nd = FF_DPT; nd <= FF_DMAX; nd += FF_DPT) {
        const size_t b = ff_smem(ff_shape(nd, nj, nl), nj, nl);
        m = b > m ? b : m;
    }
    return m;
}

cudaError_t post_prepare(int nj, int nl)
{
    return cudaFuncSetAttribute(farfield_sum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)farfield_smem(nj, nl));
}

cudaError_t launch_post(const PostArgs &a, float2 *esc, float *cabs, float *cext, cudaStream_t st)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(a.esc_acc, 0, (size_t)a.nrhs * a.ndir * 6 * sizeof(double), st))) return e;
    if ((e = cudaMemsetAsync(a.cc_acc, 0, (size_t)a.nrhs * 2 * sizeof(double), st))) return e;
    if (a.ndir > 0)
    {
        const FFShape s = ff_shape(a.ndir, a.nj, a.nl);
        farfield_sum<<<dim3(nblk(a.ndir, s.D), nblk(a.ni, FF_PLANES), a.nrhs), s.threads,
                       ff_smem(s, a.nj, a.nl), st>>>(a, s);
    }
    cabs_cext_sum<<<dim3(a.ni, a.nrhs), 256, (a.nj + a.nl) * sizeof(float2), st>>>(a);
    const size_t nd = (size_t)a.nrhs * a.ndir;
    const size_t nt = nd > (size_t)a.nrhs ? nd : (size_t)a.nrhs;
    post_finalize<<<nblk(nt, 256), 256, 0, st>>>(a, esc, cabs, cext);
    return cudaGetLastError();
}

cudaError_t launch_mueller(const MuellerArgs &m, cudaStream_t st)
{
    const size_t n = (size_t)m.norient * m.nangles;
    if (n == 0) return cudaSuccess;
    mueller_avg<<<nblk(n, 128), 128, 0, st>>>(m);
    return cudaGetLastError();
}

}  // namespace ddagpu

// ---------------------------------------------------------------------------------------
// Far field with no allocation, for callers that must not allocate device memory: code
// running inside a CUDA graph capture, a real-time loop that forbids allocator calls, or
// a host that hands this library only pre-allocated buffers.  The FP64 accumulators and
// the double copy of the directions live in this file-scope device array instead of in a
// context; every call on a device shares it.
namespace ddagpu {

namespace {

constexpr int kNoAllocMaxDirs = 8192;   // 8192 x 9 doubles = 576 KiB per device
__device__ __align__(256) double g_farfield_scratch[kNoAllocMaxDirs * 9];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kNoAllocMaxDevices] = {};

__global__ void ksc_to_double(const float *ksc, double *out, int n3)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n3) out[q] = (double)ksc[q];
}

}  // namespace

int farfield_noalloc_max_dirs() { return kNoAllocMaxDirs; }

// Device address of the scratch array on the current device, looked up once per device.
cudaError_t farfield_noalloc_scratch(int device, double **ptr)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_farfield_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = (double *)p;
    }
    *ptr = g_noalloc_ptr[device];
    return cudaSuccess;
}

cudaError_t farfield_noalloc(const PostArgs &in, const float *ksc_dev, float2 *esc_dev,
                             double *scratch, cudaStream_t st)
{
    PostArgs a = in;
    a.nrhs = 1;
    a.esc_acc = scratch;                       // [ndir][6]
    double *kscd = scratch + (size_t)kNoAllocMaxDirs * 6;   // [ndir][3]
    a.ksc = kscd;
    cudaError_t e;
    if ((e = post_prepare(a.nj, a.nl)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.esc_acc, 0, (size_t)a.ndir * 6 * sizeof(double), st))) return e;
    const int n3 = 3 * a.ndir;
    ksc_to_double<<<nblk((size_t)n3, 256), 256, 0, st>>>(ksc_dev, kscd, n3);
    const FFShape s = ff_shape(a.ndir, a.nj, a.nl);
    farfield_sum<<<dim3(nblk(a.ndir, s.D), nblk(a.ni, FF_PLANES), 1), s.threads, ff_smem(s, a.nj, a.nl),
                   st>>>(a, s);
    post_finalize<<<nblk((size_t)a.ndir, 256), 256, 0, st>>>(a, esc_dev, nullptr, nullptr);
    return cudaGetLastError();
}

}  // namespace ddagpu
