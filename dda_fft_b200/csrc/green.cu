// The FFT of the lattice Green tensor, Ahat = DFT_2n(G) / (8 ni nj nl)
// (CreateAMatrix, dda_func.cpp:85-148, and FFT_3D(cmatrix), fft_func.cpp:317-416).
//
// G(r) = e^{i|r|}/|r|^3 [ (|r|^2 - 1 + i|r|) I + (3 - |r|^2 - 3i|r|) r r^T / |r|^2 ], G(0) = 0,
// with r = (i or i - 2n) kd per axis.  Every component is even or odd along each axis,
// except on the index-n planes, whose values reach only the discarded half of the
// convolution output.  With those planes set to zero the transform is exactly even/odd in
// each frequency axis and only the octant k in [0, n]^3 is stored:
//   even axis:  sum_x f(x) e^{-i pi k x / n} = f(0) + 2 sum_{0<x<n} f(x) cos(pi k x / n)
//   odd axis:                                  -2i sum_{0<x<n} f(x) sin(pi k x / n)
// The three axis sums run in FP64 here; the octant is stored in float as
// Ahat[kx][ky][zmap(kz)][comp], z in parity order (even kz first, then odd kz), so the six
// components of one frequency form one 48-byte entry.
#include "common.cuh"
#include "internal.h"

namespace ddagpu {

namespace {

// odd-parity masks of the components e00,e01,e02,e11,e12,e22 along x, y, z
__host__ __device__ inline bool odd_x(int c) { return c == 1 || c == 2; }
__host__ __device__ inline bool odd_y(int c) { return c == 1 || c == 4; }
__host__ __device__ inline bool odd_z(int c) { return c == 2 || c == 4; }

__global__ void trig_table(int n, double *ct, double *st)
{
    // ct[k][x] = cos(pi k x / n), st[k][x] = sin(pi k x / n), k in [0, n], x in [0, n)
    const int k = blockIdx.x, x = threadIdx.x;
    if (k > n || x >= n) return;
    double s, c;
    sincospi((double)((k * x) % (2 * n)) / (double)n, &s, &c);
    ct[k * n + x] = c;
    st[k * n + x] = s;
}

__global__ void g_real(int ni, int nj, int nl, double kd, double2 *out)
{
    // out[comp][x][y][z], x < ni, y < nj, z < nl: G * w(x) w(y) w(z) / (8 N)
    const size_t N = (size_t)ni * nj * nl;
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= N) return;
    const int z = (int)(q % nl), y = (int)((q / nl) % nj), x = (int)(q / ((size_t)nl * nj));
    const double rx = x * kd, ry = y * kd, rz = z * kd;
    const double r2 = rx * rx + ry * ry + rz * rz;
    double2 e[6];
    for (int c = 0; c < 6; c++) e[c] = make_double2(0.0, 0.0);
    if (r2 >= 1e-10) {
        const double r1 = sqrt(r2);
        double s, co;
        sincos(r1, &s, &co);
        const double inv = 1.0 / (r1 * r2);
        const double c2r = co * inv, c2i = s * inv;                      // e^{ir}/r^3
        const double dr = c2r * (r2 - 1.0) - c2i * r1, di = c2r * r1 + c2i * (r2 - 1.0);
        const double ar = (3.0 - r2), ai = -3.0 * r1;                    // 3 - r^2 - 3ir
        const double orr = (c2r * ar - c2i * ai) / r2, ori = (c2r * ai + c2i * ar) / r2;
        const double rr[6] = {rx * rx, rx * ry, rx * rz, ry * ry, ry * rz, rz * rz};
        for (int c = 0; c < 6; c++) e[c] = make_double2(orr * rr[c], ori * rr[c]);
        e[0].x += dr; e[0].y += di;
        e[3].x += dr; e[3].y += di;
        e[5].x += dr; e[5].y += di;
    }
    const double w = (x ? 2.0 : 1.0) * (y ? 2.0 : 1.0) * (z ? 2.0 : 1.0) / (8.0 * (double)N);
    for (int c = 0; c < 6; c++) out[c * N + q] = make_double2(e[c].x * w, e[c].y * w);
}

// out[a][k][b] = sum_t in[a][t][b] T(k, t), T = cos (even) or -i sin (odd) along this axis;
// in extent nt, out extent nt + 1; `a` runs over comp * A6 (A6 = A / 6).
__global__ void axis_sum(const double2 *in, double2 *out, int A6, int nt, int B, const double *ct,
                         const double *st, int axis)
{
    const size_t total = (size_t)6 * A6 * (nt + 1) * B;
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= total) return;
    const int b = (int)(q % B);
    const int k = (int)((q / B) % (nt + 1));
    const size_t a = q / ((size_t)B * (nt + 1));
    const int comp = (int)(a / A6);
    const bool odd = axis == 0 ? odd_x(comp) : axis == 1 ? odd_y(comp) : odd_z(comp);
    const double2 *src = in + a * (size_t)nt * B + b;
    const double *T = (odd ? st : ct) + (size_t)k * nt;
    double sr = 0.0, si = 0.0;
    for (int t = 0; t < nt; t++) {
        const double2 v = src[(size_t)t * B];
        sr = fma(v.x, T[t], sr);
        si = fma(v.y, T[t], si);
    }
    // odd: multiply by -i
    out[q] = odd ? make_double2(si, -sr) : make_double2(sr, si);
}

__device__ inline int zmapd(int oz, int nl) { return (oz & 1) ? (nl / 2 + 1 + (oz >> 1)) : (oz >> 1); }

__global__ void to_octant(const double2 *in, float2 *ahat, int ni, int nj, int nl)
{
    // in[comp][kx][ky][kz] -> ahat[kx][ky][zmap(kz)][comp]
    const size_t per = (size_t)(ni + 1) * (nj + 1) * (nl + 1);
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= 6 * per) return;
    const int oz = (int)(q % (nl + 1));
    const size_t xy = (q / (nl + 1)) % ((size_t)(ni + 1) * (nj + 1));
    const int comp = (int)(q / per);
    const double2 v = in[q];
    ahat[((xy * (nl + 1)) + zmapd(oz, nl)) * 6 + comp] = make_float2((float)v.x, (float)v.y);
}

// Octant from a dense float Ahat [2ni][2nj][2nl][6] (the reference's cmA layout): the
// average of the 8 mirror images with the parity signs, which removes the index-n plane
// contributions and keeps everything else.
__global__ void project_dense(const float2 *dense, float2 *ahat, int ni, int nj, int nl)
{
    const size_t per = (size_t)(ni + 1) * (nj + 1) * (nl + 1);
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= 6 * per) return;
    const int oz = (int)(q % (nl + 1));
    const int oy = (int)((q / (nl + 1)) % (nj + 1));
    const int ox = (int)((q / ((size_t)(nl + 1) * (nj + 1))) % (ni + 1));
    const int c = (int)(q / per);
    double sr = 0.0, si = 0.0;
    for (int m = 0; m < 8; m++) {
        const int bx = m & 1, by = (m >> 1) & 1, bz = (m >> 2) & 1;
        const int kx = bx ? (2 * ni - ox) % (2 * ni) : ox;
        const int ky = by ? (2 * nj - oy) % (2 * nj) : oy;
        const int kz = bz ? (2 * nl - oz) % (2 * nl) : oz;
        double s = 1.0;
        if (bx && odd_x(c)) s = -s;
        if (by && odd_y(c)) s = -s;
        if (bz && odd_z(c)) s = -s;
        const float2 v = dense[(((size_t)kx * (2 * nj) + ky) * (2 * nl) + kz) * 6 + c];
        sr += s * v.x;
        si += s * v.y;
    }
    ahat[((((size_t)ox * (nj + 1) + oy) * (nl + 1)) + zmapd(oz, nl)) * 6 + c] =
        make_float2((float)(sr / 8.0), (float)(si / 8.0));
}

inline unsigned blocks(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

size_t ahat_elems(int ni, int nj, int nl) { return (size_t)6 * (ni + 1) * (nj + 1) * (nl + 1); }

namespace {

// The octant in FP64 into b1 as [comp][kx][ky][kz] (natural kz order); b0 and tab are
// scratch of ahat_elems and 6 (nmax + 1) nmax doubles.
void octant_fp64(int ni, int nj, int nl, double kd, double2 *b0, double2 *b1, double *tab,
                 size_t tabn, cudaStream_t st)
{
    const size_t big = ahat_elems(ni, nj, nl);
    double *ct[3], *stb[3];
    const int ns[3] = {ni, nj, nl};
    for (int a = 0; a < 3; a++) {
        ct[a] = tab + 2 * a * tabn;
        stb[a] = tab + (2 * a + 1) * tabn;
        trig_table<<<ns[a] + 1, ns[a], 0, st>>>(ns[a], ct[a], stb[a]);
    }
    const size_t N = (size_t)ni * nj * nl;
    g_real<<<blocks(N, 256), 256, 0, st>>>(ni, nj, nl, kd, b0);
    // z: a = comp*ni*nj, nt = nl, B = 1
    axis_sum<<<blocks((size_t)6 * ni * nj * (nl + 1), 256), 256, 0, st>>>(b0, b1, ni * nj, nl, 1,
                                                                         ct[2], stb[2], 2);
    // y: a = comp*ni, nt = nj, B = nl+1
    axis_sum<<<blocks((size_t)6 * ni * (nj + 1) * (nl + 1), 256), 256, 0, st>>>(
        b1, b0, ni, nj, nl + 1, ct[1], stb[1], 1);
    // x: a = comp, nt = ni, B = (nj+1)(nl+1)
    axis_sum<<<blocks(big, 256), 256, 0, st>>>(b0, b1, 1, ni, (nj + 1) * (nl + 1), ct[0], stb[0], 0);
}

size_t trig_elems(int ni, int nj, int nl)
{
    const int nmax = ni > nj ? (ni > nl ? ni : nl) : (nj > nl ? nj : nl);
    return (size_t)(nmax + 1) * nmax;
}

}  // namespace

cudaError_t green_build_octant(int ni, int nj, int nl, double kd, float2 *ahat, cudaStream_t st)
{
    const size_t big = ahat_elems(ni, nj, nl), tabn = trig_elems(ni, nj, nl);
    double2 *b0 = nullptr, *b1 = nullptr;
    double *tab = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync(&b0, big * sizeof(double2), st))) return e;
    if ((e = cudaMallocAsync(&b1, big * sizeof(double2), st))) return e;
    if ((e = cudaMallocAsync(&tab, 6 * tabn * sizeof(double), st))) return e;
    octant_fp64(ni, nj, nl, kd, b0, b1, tab, tabn, st);
    to_octant<<<blocks(big, 256), 256, 0, st>>>(b1, ahat, ni, nj, nl);
    cudaFreeAsync(b0, st);
    cudaFreeAsync(b1, st);
    cudaFreeAsync(tab, st);
    return cudaGetLastError();
}

cudaError_t green_build_octant64(int ni, int nj, int nl, double kd, double2 *out, cudaStream_t st)
{
    const size_t big = ahat_elems(ni, nj, nl), tabn = trig_elems(ni, nj, nl);
    double2 *b0 = nullptr;
    double *tab = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync(&b0, big * sizeof(double2), st))) return e;
    if ((e = cudaMallocAsync(&tab, 6 * tabn * sizeof(double), st))) return e;
    octant_fp64(ni, nj, nl, kd, b0, out, tab, tabn, st);
    cudaFreeAsync(b0, st);
    cudaFreeAsync(tab, st);
    return cudaGetLastError();
}

cudaError_t green_project_dense(int ni, int nj, int nl, const float2 *dense_dev, float2 *ahat,
                                cudaStream_t st)
{
    const size_t big = ahat_elems(ni, nj, nl);
    project_dense<<<blocks(big, 256), 256, 0, st>>>(dense_dev, ahat, ni, nj, nl);
    return cudaGetLastError();
}

}  // namespace ddagpu
