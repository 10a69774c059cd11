// The dipole-interaction matvec G * p on the zero-padded 2ni x 2nj x 2nl grid
// (Convolution, dda_func.cpp:150-187; FFT_3D / iFFT_3D, fft_func.cpp:418-653).
//
// Three kernels per matvec, every FFT an n-point transform:
//   K1  forward y then z, one CTA per (i < ni, component, j-parity half)
//   K2  forward x, symmetric 3x3 product with the Green tensor, inverse x, in place,
//       one CTA per (j spectral row, tile of l spectral columns), all 3 components
//   K3  inverse z then y, a 2-CTA cluster per (i, component) that combines the two
//       j-halves through distributed shared memory, then the solver epilogue
//
// The zero padding is never materialised: a 2n-point DFT of a line whose upper half is
// zero splits into even bins DFT_n(x) and odd bins DFT_n(x * W_2n^j) (the reference's own
// composite, fft_func.cpp:442-463), and the inverse, of which only the first n outputs
// are kept, is IDFT_n(even) + W_2n^-j IDFT_n(odd).  The spectral axes y and z are stored
// in that split order: index s = h * n + k holds frequency 2k + h.
#include <cooperative_groups.h>

#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace ddagpu {

namespace {

DDA_DEV int zmap(int oz, int nl) { return (oz & 1) ? (nl / 2 + 1 + (oz >> 1)) : (oz >> 1); }

// ------------------------------------------------------------------------------ K1
// src plane (nj x nl, component c, lattice plane i) -> work rows j_s = h nj + kj, each
// 2nl long in split order.
__global__ void __launch_bounds__(512) k1_forward_yz(MatvecArgs a)
{
    extern __shared__ float2 sm[];
    const int h = blockIdx.x & 1, i = blockIdx.x >> 1, c = blockIdx.y, rhs = blockIdx.z;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    const int ni = a.L.ni, nj = a.L.nj, nl = a.L.nl, PS = nl + 1, G = a.rows_g;
    float2 *P = sm;               // [nj][PS]
    float2 *S = sm + nj * PS;     // [2G][PS]
    const float2 *src = a.src + (size_t)rhs * a.fstride + ((size_t)c * ni + i) * nj * nl;
    const float2 *hwj = a.L.tw_j + nj, *hwl = a.L.tw_l + nl;

    for (int e = threadIdx.x; e < nj * nl; e += blockDim.x) {
        const int j = e / nl, l = e - j * nl;
        float2 x = src[e];
        if (h) x = cmul(x, __ldg(&hwj[j]));
        P[j * PS + l] = x;
    }
    __syncthreads();
    fft_lines_rt<false>(nj, P, PS, 1, nl, a.L.tw_j);   // along j, nl columns

    float2 *dst = a.work + (size_t)rhs * a.wstride +
                  (((size_t)c * ni + i) * (2 * nj) + (size_t)h * nj) * (2 * nl);
    for (int r0 = 0; r0 < nj; r0 += G) {
        for (int e = threadIdx.x; e < G * nl; e += blockDim.x) {
            const int g = e / nl, l = e - g * nl;
            const float2 x = P[(r0 + g) * PS + l];
            S[(2 * g) * PS + l] = x;
            S[(2 * g + 1) * PS + l] = cmul(x, __ldg(&hwl[l]));
        }
        __syncthreads();
        fft_lines_rt<false>(nl, S, 1, PS, 2 * G, a.L.tw_l);   // along l, 2G rows
        for (int e = threadIdx.x; e < G * 2 * nl; e += blockDim.x) {
            const int g = e / (2 * nl), ls = e - g * 2 * nl;
            const int half = ls >= nl, k = ls - half * nl;
            dst[(size_t)(r0 + g) * (2 * nl) + ls] = S[(2 * g + half) * PS + k];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------ K2
// Lines along i for one spectral row j_s and TW spectral columns, all 3 components.
// Shared layout B[i][b][t], b = 2 c + parity half, so the 6 TW lines are affine.
__global__ void __launch_bounds__(512) k2_x_product(MatvecArgs a)
{
    extern __shared__ float2 sm[];
    const int js = blockIdx.x, rhs = blockIdx.z;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    const int ni = a.L.ni, nj = a.L.nj, nl = a.L.nl, TW = a.tile_x;
    const int l0 = blockIdx.y * TW;
    const int LW = 6 * TW;   // element stride
    const size_t plane = (size_t)(2 * nj) * (2 * nl);
    const size_t cstr = (size_t)ni * plane;
    float2 *base = a.work + (size_t)rhs * a.wstride + (size_t)js * (2 * nl) + l0;
    const float2 *hwi = a.L.tw_i + ni;

    for (int e = threadIdx.x; e < 3 * ni * TW; e += blockDim.x) {
        const int c = e / (ni * TW), r = e - c * ni * TW, i = r / TW, t = r - i * TW;
        const float2 x = base[c * cstr + i * plane + t];
        sm[i * LW + (2 * c) * TW + t] = x;
        sm[i * LW + (2 * c + 1) * TW + t] = cmul(x, __ldg(&hwi[i]));
    }
    __syncthreads();
    fft_lines_rt<false>(ni, sm, LW, 1, LW, a.L.tw_i);

    // Symmetric 3x3 product with the Green tensor at frequency (kx, j', l').
    const int hj = js >= nj, kj = js - hj * nj, jp = 2 * kj + hj;
    const int my = jp > nj, oy = my ? 2 * nj - jp : jp;
    // Ahat[ox][oy][zmap(oz)][6]
    const size_t sz = 6, sy = (size_t)(nl + 1) * 6, sxo = (size_t)(nj + 1) * sy;
    for (int e = threadIdx.x; e < 2 * ni * TW; e += blockDim.x) {
        const int t = e % TW, kh = e / TW, k = kh >> 1, hx = kh & 1;
        const int kx = 2 * k + hx, mx = kx > ni, ox = mx ? 2 * ni - kx : kx;
        const int ls = l0 + t, hl = ls >= nl, kl = ls - hl * nl, lp = 2 * kl + hl;
        const int mz = lp > nl, oz = mz ? 2 * nl - lp : lp;
        const float2 *A = a.ahat + (size_t)ox * sxo + (size_t)oy * sy + (size_t)zmap(oz, nl) * sz;
        float2 g0 = __ldg(A), g1 = __ldg(A + 1), g2 = __ldg(A + 2), g3 = __ldg(A + 3),
               g4 = __ldg(A + 4), g5 = __ldg(A + 5);
        if (mx ^ my) g1 = cscale(g1, -1.f);
        if (mx ^ mz) g2 = cscale(g2, -1.f);
        if (my ^ mz) g4 = cscale(g4, -1.f);
        if (a.conj) {
            g0 = cconj(g0); g1 = cconj(g1); g2 = cconj(g2);
            g3 = cconj(g3); g4 = cconj(g4); g5 = cconj(g5);
        }
        float2 *b = sm + k * LW + hx * TW + t;
        const float2 vx = b[0], vy = b[2 * TW], vz = b[4 * TW];
        b[0] = cadd(cadd(cmul(g0, vx), cmul(g1, vy)), cmul(g2, vz));
        b[2 * TW] = cadd(cadd(cmul(g1, vx), cmul(g3, vy)), cmul(g4, vz));
        b[4 * TW] = cadd(cadd(cmul(g2, vx), cmul(g4, vy)), cmul(g5, vz));
    }
    __syncthreads();
    fft_lines_rt<true>(ni, sm, LW, 1, LW, a.L.tw_i);

    for (int e = threadIdx.x; e < 3 * ni * TW; e += blockDim.x) {
        const int c = e / (ni * TW), r = e - c * ni * TW, i = r / TW, t = r - i * TW;
        const float2 ev = sm[i * LW + (2 * c) * TW + t], od = sm[i * LW + (2 * c + 1) * TW + t];
        base[c * cstr + i * plane + t] = cadd(ev, cmulc(od, __ldg(&hwi[i])));
    }
}

// ------------------------------------------------------------------------------ K3
// Cluster rank h holds work rows j_s in [h nj, (h+1) nj) of plane (i, c): inverse along l
// (keep l < nl), inverse along j of its half, then the two halves are summed through
// distributed shared memory and the epilogue writes the output rows of this rank.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(512) k3_inverse_zy(MatvecArgs a)
{
    extern __shared__ float2 sm[];
    cg::cluster_group cl = cg::this_cluster();
    const int h = (int)cl.block_rank();
    const int i = blockIdx.x >> 1, c = blockIdx.y, rhs = blockIdx.z;
    if (a.rhs_active && !a.rhs_active[rhs]) return;   // uniform over the cluster
    const int ni = a.L.ni, nj = a.L.nj, nl = a.L.nl, PS = nl + 1, G = a.rows_g;
    float2 *Q = sm;               // [nj][PS]
    float2 *S = sm + nj * PS;     // [2G][PS]
    const float2 *src = a.work + (size_t)rhs * a.wstride +
                        (((size_t)c * ni + i) * (2 * nj) + (size_t)h * nj) * (2 * nl);
    const float2 *hwj = a.L.tw_j + nj, *hwl = a.L.tw_l + nl;

    for (int r0 = 0; r0 < nj; r0 += G) {
        for (int e = threadIdx.x; e < G * 2 * nl; e += blockDim.x) {
            const int g = e / (2 * nl), ls = e - g * 2 * nl;
            const int half = ls >= nl, k = ls - half * nl;
            S[(2 * g + half) * PS + k] = src[(size_t)(r0 + g) * (2 * nl) + ls];
        }
        __syncthreads();
        fft_lines_rt<true>(nl, S, 1, PS, 2 * G, a.L.tw_l);
        for (int e = threadIdx.x; e < G * nl; e += blockDim.x) {
            const int g = e / nl, l = e - g * nl;
            Q[(r0 + g) * PS + l] =
                cadd(S[(2 * g) * PS + l], cmulc(S[(2 * g + 1) * PS + l], __ldg(&hwl[l])));
        }
        __syncthreads();
    }
    fft_lines_rt<true>(nj, Q, PS, 1, nl, a.L.tw_j);
    if (h == 1) {
        for (int e = threadIdx.x; e < nj * nl; e += blockDim.x) {
            const int j = e / nl, l = e - j * nl;
            Q[j * PS + l] = cmulc(Q[j * PS + l], __ldg(&hwj[j]));
        }
    }
    cl.sync();
    const float2 *R = cl.map_shared_rank(sm, h ^ 1);
    const int half_rows = nj / 2, j0 = h * half_rows;
    const size_t N = a.L.N;
    const size_t obase = (size_t)rhs * a.fstride + (size_t)c * N + (size_t)i * nj * nl;
    const Epilogue &ep = a.ep;
    for (int e = threadIdx.x; e < half_rows * nl; e += blockDim.x) {
        const int jj = e / nl, l = e - jj * nl, j = j0 + jj;
        const float2 conv = cadd(Q[j * PS + l], R[j * PS + l]);
        const size_t o = obase + (size_t)j * nl + l;
        float2 res = conv;
        if (ep.mode == 1) {
            const int m = ep.occ[(size_t)rhs * ep.occ_stride + (size_t)i * nj * nl + (size_t)j * nl + l];
            if (!ep.mv[m]) {
                res = czero();
            } else {
                float2 al = ep.alpha[(size_t)rhs * ep.nmat1 + m];
                if (ep.conj) al = cconj(al);
                res = csub(ep.sv != 0.f ? cscale(ep.v[o], ep.sv) : czero(), cmul(al, conv));
            }
        }
        a.out[o] = res;
    }
    cl.sync();
}

}  // namespace

size_t matvec_smem_yz(const Lat &L, int rows_g)
{
    return (size_t)(L.nj + 2 * rows_g) * (L.nl + 1) * sizeof(float2);
}

size_t matvec_smem_x(const Lat &L, int tile_x) { return (size_t)6 * tile_x * L.ni * sizeof(float2); }

cudaError_t raise_smem_limit(const void *kernel, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> set;   // (device, kernel) -> limit
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    int &cur = set[{dev, kernel}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

cudaError_t kernel_binary_version(int *version)
{
    cudaFuncAttributes fa{};
    const cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)k2_x_product);
    if (e == cudaSuccess) *version = fa.binaryVersion;
    return e;
}

cudaError_t matvec_prepare(const Lat &L, int tile_x, int rows_g)
{
    cudaError_t e;
    const int syz = (int)matvec_smem_yz(L, rows_g), sx = (int)matvec_smem_x(L, tile_x);
    if ((e = raise_smem_limit((const void *)k1_forward_yz, syz))) return e;
    if ((e = raise_smem_limit((const void *)k3_inverse_zy, syz))) return e;
    return raise_smem_limit((const void *)k2_x_product, sx);
}

cudaError_t launch_matvec(const MatvecArgs &a, cudaStream_t st)
{
    if (a.fast) return launch_matvec_fast(a, st);
    if (a.inc) return cudaErrorInvalidValue;   // the incident-field input needs the sized passes
    const Lat &L = a.L;
    const size_t syz = matvec_smem_yz(L, a.rows_g), sx = matvec_smem_x(L, a.tile_x);
    k1_forward_yz<<<dim3(2 * L.ni, 3, a.nrhs), 512, syz, st>>>(a);
    k2_x_product<<<dim3(2 * L.nj, (2 * L.nl) / a.tile_x, a.nrhs), 512, sx, st>>>(a);
    k3_inverse_zy<<<dim3(2 * L.ni, 3, a.nrhs), 512, syz, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ddagpu
