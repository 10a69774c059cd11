// Shared device helpers for the B200 DDA-FFT kernels: complex arithmetic on float2,
// in-register DFTs of 2..16 points and the two-step (R1 x R2) line FFT over tiles held
// in shared memory.
//
// FFT conventions follow the reference (fft_kernel.hpp:1-30, fft_func.cpp:556-653):
// forward  X[k] = sum_j x[j] exp(-2 pi i j k / N), natural order in and out;
// inverse  = conj(DFT(conj(x))) = sum_j x[j] exp(+2 pi i j k / N), no 1/N.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DDA_DEV __device__ __forceinline__

DDA_DEV float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
DDA_DEV float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
DDA_DEV float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// acc + a * b as four fused multiply-adds
DDA_DEV float2 cfma(float2 a, float2 b, float2 acc)
{
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}

DDA_DEV float2 cmulc(float2 a, float2 b) // a * conj(b)
{
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
DDA_DEV float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
DDA_DEV float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
DDA_DEV float2 czero() { return make_float2(0.f, 0.f); }

// exp(i ph) for a phase given in FP64: the reduction to [-pi, pi] is done in FP64 (phases
// reach tens of radians), the sine and cosine of the reduced angle in float.
DDA_DEV float2 expi_reduced(double ph)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double r = fma(-two_pi, rint(ph * (1.0 / two_pi)), ph);
    float s, c;
    sincosf((float)r, &s, &c);
    return make_float2(c, s);
}

// W_16^m = exp(-2 pi i m / 16) for m = 0..7 (the values of cos and sin at multiples of
// pi/8: 1, cos(pi/8) = 0.9238795..., sqrt(1/2), sin(pi/8) = 0.3826834...).
DDA_DEV float2 w16(int m)
{
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f,
                h = 0.70710678118654752440f;
    switch (m) {
    case 0: return make_float2(1.f, 0.f);
    case 1: return make_float2(c1, -s1);
    case 2: return make_float2(h, -h);
    case 3: return make_float2(s1, -c1);
    case 4: return make_float2(0.f, -1.f);
    case 5: return make_float2(-s1, -c1);
    case 6: return make_float2(-h, -h);
    default: return make_float2(-c1, -s1);
    }
}

template <int R>
struct ilog2c {
    static constexpr int v = (R <= 1) ? 0 : 1 + ilog2c<(R > 1 ? R / 2 : 1)>::v;
};
template <>
struct ilog2c<1> {
    static constexpr int v = 0;
};

__host__ __device__ constexpr int bitrev_c(int k, int bits)
{
    int r = 0;
    for (int b = 0; b < bits; b++) r |= ((k >> b) & 1) << (bits - 1 - b);
    return r;
}

// In-register DFT of R (power of two, <= 16) points: radix-2 decimation in frequency,
// then a compile-time bit-reversal.  INV conjugates the twiddles.
template <int R, bool INV>
DDA_DEV void dft_reg(float2 (&v)[R])
{
    if (R == 1) return;
#pragma unroll
    for (int len = R; len >= 2; len >>= 1) {
#pragma unroll
        for (int s = 0; s < R; s += len) {
#pragma unroll
            for (int j = 0; j < len / 2; j++) {
                float2 a = v[s + j], b = v[s + j + len / 2];
                v[s + j] = cadd(a, b);
                float2 d = csub(a, b);
                if (j == 0) {
                    v[s + j + len / 2] = d;
                } else if (4 * j == len) { // times -i (forward) or +i (inverse)
                    v[s + j + len / 2] = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
                } else {
                    float2 w = w16(j * (16 / len));
                    if (INV) w.y = -w.y;
                    v[s + j + len / 2] = cmul(d, w);
                }
            }
        }
    }
    float2 t[R];
#pragma unroll
    for (int k = 0; k < R; k++) t[k] = v[bitrev_c(k, ilog2c<R>::v)];
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = t[k];
}

// N = R1 * R2 factorisation of the line FFT (R1 >= R2).
template <int N>
struct fft_split;
template <> struct fft_split<2>   { static constexpr int R1 = 2,  R2 = 1; };
template <> struct fft_split<4>   { static constexpr int R1 = 4,  R2 = 1; };
template <> struct fft_split<8>   { static constexpr int R1 = 8,  R2 = 1; };
template <> struct fft_split<16>  { static constexpr int R1 = 4,  R2 = 4; };
template <> struct fft_split<32>  { static constexpr int R1 = 8,  R2 = 4; };
template <> struct fft_split<64>  { static constexpr int R1 = 8,  R2 = 8; };
template <> struct fft_split<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct fft_split<256> { static constexpr int R1 = 16, R2 = 16; };

// N-point DFT of `nlines` lines held in shared memory: element m of line t sits at
// buf[m * ES + t * LS].  All threads of the block must call it (it synchronises); the
// caller synchronises before the call, the routine synchronises before returning.
// tw[k] = W_N^k for k < N (forward sign; INV conjugates).
//
// Two steps (the "four-step" factorisation N = R1 R2, m = t2 + R2 r1, k = k1 + R1 k2):
//   A: per (line, t2): R1-point DFT over r1, times W_N^(t2 k1), written back in place;
//   B: per (line, k1): R2-point DFT over t2 of the block R2 k1 .. R2 k1 + R2 - 1, written
//      to natural positions k1 + R1 k2 after a barrier.
template <int N, bool INV>
__device__ void fft_lines(float2 *buf, int ES, int LS, int nlines, const float2 *__restrict__ tw)
{
    constexpr int R1 = fft_split<N>::R1, R2 = fft_split<N>::R2;
    constexpr int RM = R1 > R2 ? R1 : R2;
    const int per_group = blockDim.x / RM;
    const int lt = threadIdx.x % per_group, sub = threadIdx.x / per_group;
    for (int l0 = 0; l0 < nlines; l0 += per_group) {
        const int line = l0 + lt;
        const bool ok = (line < nlines) && (sub < RM);
        float2 *b = buf + (size_t)line * LS;
        if (R2 == 1) {
            if (ok && sub == 0) {
                float2 v[R1];
#pragma unroll
                for (int r = 0; r < R1; r++) v[r] = b[r * ES];
                dft_reg<R1, INV>(v);
#pragma unroll
                for (int r = 0; r < R1; r++) b[r * ES] = v[r];
            }
            __syncthreads();
            continue;
        }
        if (ok && sub < R2) {
            const int t2 = sub;
            float2 v[R1];
#pragma unroll
            for (int r = 0; r < R1; r++) v[r] = b[(t2 + R2 * r) * ES];
            dft_reg<R1, INV>(v);
#pragma unroll
            for (int k1 = 1; k1 < R1; k1++) {
                float2 w = __ldg(&tw[t2 * k1]);
                if (INV) w.y = -w.y;
                v[k1] = cmul(v[k1], w);
            }
#pragma unroll
            for (int r = 0; r < R1; r++) b[(t2 + R2 * r) * ES] = v[r];
        }
        __syncthreads();
        float2 u[R2];
        if (ok && sub < R1) {
            const int k1 = sub;
#pragma unroll
            for (int t = 0; t < R2; t++) u[t] = b[(R2 * k1 + t) * ES];
            dft_reg<R2, INV>(u);
        }
        __syncthreads();
        if (ok && sub < R1) {
            const int k1 = sub;
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) b[(k1 + R1 * k2) * ES] = u[k2];
        }
        __syncthreads();
    }
}

// Runtime dispatch of fft_lines over the supported sizes.
template <bool INV>
__device__ void fft_lines_rt(int N, float2 *buf, int ES, int LS, int nlines,
                             const float2 *__restrict__ tw)
{
    switch (N) {
    case 2: fft_lines<2, INV>(buf, ES, LS, nlines, tw); break;
    case 4: fft_lines<4, INV>(buf, ES, LS, nlines, tw); break;
    case 8: fft_lines<8, INV>(buf, ES, LS, nlines, tw); break;
    case 16: fft_lines<16, INV>(buf, ES, LS, nlines, tw); break;
    case 32: fft_lines<32, INV>(buf, ES, LS, nlines, tw); break;
    case 64: fft_lines<64, INV>(buf, ES, LS, nlines, tw); break;
    case 128: fft_lines<128, INV>(buf, ES, LS, nlines, tw); break;
    default: fft_lines<256, INV>(buf, ES, LS, nlines, tw); break;
    }
}

// FP64 block reduction of NV values per thread; thread 0 of the block gets the totals
// in out[] (out must be in shared memory with NV * 32 doubles of scratch in `scratch`).
template <int NV>
DDA_DEV void warp_sum(double (&v)[NV])
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
}

template <int NV>
__device__ void block_sum_atomic(double (&v)[NV], double *scratch, double *dst)
{
    warp_sum<NV>(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) scratch[warp * NV + q] = v[q];
    __syncthreads();
    if (warp == 0) {
        double t[NV];
#pragma unroll
        for (int q = 0; q < NV; q++) t[q] = lane < nw ? scratch[lane * NV + q] : 0.0;
        warp_sum<NV>(t);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < NV; q++)
                if (t[q] != 0.0) atomicAdd(dst + q, t[q]);
    }
    __syncthreads();
}
