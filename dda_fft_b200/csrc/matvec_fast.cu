// Fast matvec passes for lattice edges in {16, 32, 64, 128}: the same three passes and the
// same split-order spectral layout as matvec.cu, with every size a compile-time constant.
//
// Every n-point FFT uses the factorisation n = R1 R2 (fft_split): a thread holds R1
// elements of a line for step A and R2 elements for step B, and the steps exchange data
// through shared memory.  Two thread roles occur:
//   row role    -- the RM = max(R1,R2) lanes of one warp-aligned group own one line whose
//                  elements are contiguous in shared memory (z lines); the exchange is
//                  warp-local (__syncwarp);
//   column role -- thread (sub, col) with consecutive lanes on consecutive lines; the
//                  exchange needs the block (__syncthreads) but every access is a
//                  contiguous run of the warp.
// Shared planes use the swizzled row layout pos(p) = p ^ ((p >> 3) & 7), a permutation
// inside each aligned block of 8 elements, with a row stride PS = N + 8 or N + 4 float2
// (PS = RM mod 16, or 8 mod 16 where two rows share a half-warp).  A warp reading 32
// consecutive columns of one row, a row group reading positions t2 + R2 r (step A) and a
// row group reading positions R2 k1 + t (step B) all touch distinct banks.
#include <cooperative_groups.h>
#include <cuda.h>   // CUtensorMap (the type only; maps are encoded in ddagpu.cu)

#include <type_traits>

#include "common.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace ddagpu {

namespace {

template <int N>
struct Sp {
    static constexpr int R1 = fft_split<N>::R1, R2 = fft_split<N>::R2;
    static constexpr int RM = R1 > R2 ? R1 : R2;
    // row stride = RM (mod 16) float2: the rows of one half-warp land in disjoint banks; 8
    // (mod 16) when R1 = 2 R2, where a half-warp holds two rows in step A (row_fft2_from_regs)
    static constexpr int PS = N + (((R1 == 2 * R2 ? 8 : RM % 16) - (N % 16) + 16) % 16);
};

// The x pass's line factorisation N = R1 R2: ALT 0 is fft_split<N>; ALT 1 the second
// schedule the autotuner may pick -- the two factors swapped, or for a square split
// 2 R1 x R2 / 2 (16: 8 x 2, 32: 4 x 8, 64: 16 x 4, 128: 8 x 16).  The reference chooses
// among radix-8/4/2 stage sequences per length the same way (fft_kernel.hpp:210-263).
template <int N, int ALT>
struct Sx {
    static constexpr int A1 = fft_split<N>::R1, A2 = fft_split<N>::R2;
    static constexpr int R1 = ALT == 0 ? A1 : (A1 == A2 ? 2 * A1 : A2);
    static constexpr int R2 = ALT == 0 ? A2 : (A1 == A2 ? A2 / 2 : A1);
    static constexpr int RM = R1 > R2 ? R1 : R2;
    static_assert(R1 * R2 == N && R1 <= 16 && R2 <= 16, "bad line factorisation");
};

DDA_DEV int spos(int p) { return p ^ ((p >> 3) & 7); }

DDA_DEV int zmapf(int oz, int nl) { return (oz & 1) ? (nl / 2 + 1 + (oz >> 1)) : (oz >> 1); }

template <bool INV>
DDA_DEV float2 twid(const float2 *__restrict__ tw, int k)
{
    float2 w = __ldg(&tw[k]);
    if (INV) w.y = -w.y;
    return w;
}

// Row role, one line of N elements at `row` (swizzled), in place, natural order out.
// lane_sub in [0, RM).  v: the R1 step-A inputs of this lane (positions t2 + R2 r), loaded
// by the caller for lane_sub < R2.  Every lane of the warp calls this (it synchronises the
// warp); `valid` guards the shared-memory accesses of lanes without a line.
template <int N, bool INV>
DDA_DEV void row_fft_from_regs(float2 *row, int lane_sub, bool valid, float2 (&v)[Sp<N>::R1],
                               const float2 *__restrict__ tw)
{
    constexpr int R1 = Sp<N>::R1, R2 = Sp<N>::R2;
    static_assert(R2 > 1, "single-step sizes are not on the fast path");
    if (valid && lane_sub < R2) {
        const int t2 = lane_sub;
        dft_reg<R1, INV>(v);
#pragma unroll
        for (int k1 = 1; k1 < R1; k1++) v[k1] = cmul(v[k1], twid<INV>(tw, t2 * k1));
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) row[spos(t2 + R2 * k1)] = v[k1];
    }
    __syncwarp();
    float2 u[R2];
    if (valid && lane_sub < R1) {
        const int k1 = lane_sub;
#pragma unroll
        for (int t = 0; t < R2; t++) u[t] = row[spos(R2 * k1 + t)];
        dft_reg<R2, INV>(u);
    }
    __syncwarp();
    if (valid && lane_sub < R1) {
        const int k1 = lane_sub;
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) row[spos(k1 + R1 * k2)] = u[k2];
    }
    __syncwarp();
}

// Row role for two lines at once when N = R1 R2 with R1 = 2 R2 (32 = 8 x 4, 128 = 16 x 8):
// lanes [0, R2) of the group hold line A's step-A inputs and lanes [R2, R1) line B's (the
// positions t2 + R2 r with t2 = lane_sub mod R2), so every lane works in step A, where the
// single-line form idles half of them; step B takes both lines on all R1 lanes.
template <int N, bool INV>
DDA_DEV void row_fft2_from_regs(float2 *rowA, float2 *rowB, int lane_sub, bool validA, bool validB,
                                float2 (&v)[Sp<N>::R1], const float2 *__restrict__ tw)
{
    constexpr int R1 = Sp<N>::R1, R2 = Sp<N>::R2;
    static_assert(R1 == 2 * R2, "two lines per lane group need R1 = 2 R2");
    const int h = lane_sub >= R2, t2 = lane_sub - h * R2;
    float2 *row = h ? rowB : rowA;
    if (h ? validB : validA) {
        dft_reg<R1, INV>(v);
#pragma unroll
        for (int k1 = 1; k1 < R1; k1++) v[k1] = cmul(v[k1], twid<INV>(tw, t2 * k1));
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) row[spos(t2 + R2 * k1)] = v[k1];
    }
    __syncwarp();
    // step B, line A then line B (one line's R2 values live at a time)
    const int k1 = lane_sub;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        float2 *ln = q ? rowB : rowA;
        const bool ok = q ? validB : validA;
        float2 u[R2];
        if (ok) {
#pragma unroll
            for (int t = 0; t < R2; t++) u[t] = ln[spos(R2 * k1 + t)];
            dft_reg<R2, INV>(u);
        }
        __syncwarp();
        if (ok) {
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) ln[spos(k1 + R1 * k2)] = u[k2];
        }
    }
    __syncwarp();
}

// Two lines per lane group in the row role of a yz pass of NT threads: R1 = 2 R2 and the
// rows fill at least two passes of one line per group.
template <int NJ, int NL, int NT>
__host__ __device__ constexpr bool rows_paired()
{
    return Sp<NL>::R1 == 2 * Sp<NL>::R2 && NJ >= 2 * (NT / Sp<NL>::RM);
}

// Both y halves' step A at once in the column role (R1 = 2 R2 on the y lines): the
// sub-lines [0, R2) take half 0 in place and [R2, R1) half 1 into a scratch block of NJ x
// (NT / RM) elements after the plane.
template <int NJ>
__host__ __device__ constexpr bool halves_paired()
{
    return Sp<NJ>::R1 == 2 * Sp<NJ>::R2;
}

// ------------------------------------------------------------------------------ K1
// CTA (i, component, z half hl): z-forward of the NJ rows of plane i (half hl only), then
// y-forward of the NL columns for both y halves; writes work rows in split order.
// IM 1: the input is the incident field, computed here (and written by the hl = 0 CTAs).
// IM 2: incident field of a polarisation pair (MatvecArgs::pair): CTA (i, hl, pair k)
// transforms phi = alpha_m exp(i k.(r - c)) into component slot 0 of right-hand side 2k
// and writes p = phi E_q of both polarisations.
template <int NJ, int NL, int NT, int IM>
__global__ void __launch_bounds__(NT) k1f(MatvecArgs a)
{
    using SJ = Sp<NJ>;
    using SL = Sp<NL>;
    constexpr int PS = SL::PS;
    constexpr bool INC = IM != 0, PAIR = IM == 2;
    extern __shared__ float2 Z[];   // [NJ][PS]
    const int hl = blockIdx.x & 1, i = blockIdx.x >> 1, c = blockIdx.y;
    const int rhs = PAIR ? 2 * (int)blockIdx.z : (int)blockIdx.z;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    const int ni = a.L.ni;
    const float2 *src = a.src + (size_t)rhs * a.fstride + ((size_t)c * ni + i) * (NJ * NL);
    const float2 *twl = a.L.tw_l, *hwl = a.L.tw_l + NL, *twj = a.L.tw_j, *hwj = a.L.tw_j + NJ;

    // ---- z: rows, row role
    if constexpr (INC) {
        // incident dipoles of this plane and component (FirstApproximation,
        // dda_func.cpp:654-689) with the products of the separate pass, in its order:
        // ((x phase * y phase) * z phase) * alpha_m * E_c
        constexpr int RM = SL::RM, RPP = NT / RM, R1 = SL::R1, R2 = SL::R2;
        // PR: two rows per lane group (lane half h, step-A index t2); else one row
        constexpr bool PR = rows_paired<NJ, NL, NT>();
        constexpr int ROWS = PR ? 2 * RPP : RPP;
        const int sub = threadIdx.x % RM, rr = threadIdx.x / RM;
        const int h = PR ? (sub >= R2) : 0, t2 = sub - h * R2, rbase = PR ? 2 * rr : rr;
        const bool lane_a = PR || sub < R2;   // holds step-A inputs
        const Epilogue &ep = a.ep;
        const float2 *tab = a.inc_tab + (size_t)rhs * (NJ + NL + ni);
        const float2 tx = tab[NJ + NL + i];
        // this lane's z phases: held in registers up to 64-point rows; at 128 points they
        // are re-read from the (L1-resident) table, which keeps the pass from spilling
        constexpr bool tz_reg = NL <= 64;
        float2 tz[tz_reg ? R1 : 1];
#pragma unroll
        for (int r = 0; r < (tz_reg ? R1 : 1); r++) tz[r] = lane_a ? tab[NJ + t2 + R2 * r] : czero();
        const double *E = a.einc + 6 * rhs;
        const float2 Ef = make_float2((float)E[2 * c], (float)E[2 * c + 1]);
        float2 Ep[2][3];   // pair: the incident fields of both polarisations
        if constexpr (PAIR) {
#pragma unroll
            for (int q = 0; q < 2; q++)
#pragma unroll
                for (int k = 0; k < 3; k++)
                    Ep[q][k] = make_float2((float)E[6 * q + 2 * k], (float)E[6 * q + 2 * k + 1]);
        }
        const signed char *ob = ep.occ + (size_t)rhs * ep.occ_stride + (size_t)i * NJ * NL;
        const float2 *al = ep.alpha + (size_t)rhs * ep.nmat1;
        // up to two materials from registers
        const bool rt = ep.nmat1 <= 2;
        const bool mv0 = ep.mv[0] != 0, mv1 = ep.nmat1 > 1 && ep.mv[1] != 0;
        const float2 al0 = al[0], al1 = ep.nmat1 > 1 ? al[1] : czero();
        float2 *pout = a.inc_out + (size_t)rhs * a.fstride + ((size_t)c * ni + i) * (NJ * NL);
        // the occupancy of the next pass's row is loaded while this pass's row is transformed
        auto load = [&](int row, int (&o)[R1], float2 &ty) {
            if (row < NJ && lane_a) {
#pragma unroll
                for (int r = 0; r < R1; r++) o[r] = ob[row * NL + t2 + R2 * r];
                ty = tab[row];
            }
        };
        int o[R1], on[R1];
        float2 ty = czero(), tyn = czero();
        load(rbase + h, o, ty);
#pragma unroll 1
        for (int r0 = 0; r0 < NJ; r0 += ROWS) {
            const int row0 = r0 + rbase, row = row0 + h;
            if (r0 + ROWS < NJ) load(row + ROWS, on, tyn);
            float2 v[R1];
            if (row < NJ && lane_a) {
                const float2 txy = cmul(tx, ty);
#pragma unroll
                for (int r = 0; r < R1; r++) {
                    const int m = o[r];
                    const bool act = rt ? ((m & 1) ? mv1 : mv0) : ep.mv[m] != 0;
                    float2 val = czero();
                    const float2 tzr = tz_reg ? tz[tz_reg ? r : 0] : __ldg(&tab[NJ + t2 + R2 * r]);
                    if constexpr (PAIR) {
                        // val = phi; the dipoles phi E_q of both polarisations, the same
                        // float operations as the single form's ((phi) E_c)
                        if (act) val = cmul(cmul(txy, tzr), rt ? ((m & 1) ? al1 : al0) : al[m]);
                        if (hl == 0) {
                            const size_t o = (size_t)row * NL + t2 + R2 * r;
#pragma unroll
                            for (int q = 0; q < 2; q++)
#pragma unroll
                                for (int k = 0; k < 3; k++)
                                    pout[q * a.fstride + (size_t)k * ni * (NJ * NL) + o] = cmul(val, Ep[q][k]);
                        }
                    } else {
                        if (act) val = cmul(cmul(cmul(txy, tzr), rt ? ((m & 1) ? al1 : al0) : al[m]), Ef);
                        if (hl == 0) pout[row * NL + t2 + R2 * r] = val;
                    }
                    v[r] = hl ? cmul(val, __ldg(&hwl[t2 + R2 * r])) : val;
                }
            }
            if constexpr (PR)
                row_fft2_from_regs<NL, false>(Z + (row0 < NJ ? row0 : 0) * PS, Z + (row0 + 1 < NJ ? row0 + 1 : 0) * PS,
                                              sub, row0 < NJ, row0 + 1 < NJ, v, twl);
            else
                row_fft_from_regs<NL, false>(Z + (row < NJ ? row : 0) * PS, sub, row < NJ, v, twl);
#pragma unroll
            for (int r = 0; r < R1; r++) o[r] = on[r];
            ty = tyn;
        }
    } else {
        constexpr int RM = SL::RM, RPP = NT / RM, R1 = SL::R1, R2 = SL::R2;
        constexpr bool PR = rows_paired<NJ, NL, NT>();
        constexpr int ROWS = PR ? 2 * RPP : RPP;   // rows per pass
        const int sub = threadIdx.x % RM, rr = threadIdx.x / RM;
        const int h = PR ? (sub >= R2) : 0, t2 = sub - h * R2, rbase = PR ? 2 * rr : rr;
        const bool lane_a = PR || sub < R2;
        // the next pass's row is loaded while this pass's row is transformed
        auto load = [&](int row, float2 (&v)[R1]) {
            if (row < NJ && lane_a) {
#pragma unroll
                for (int r = 0; r < R1; r++) v[r] = src[row * NL + t2 + R2 * r];
            }
        };
        float2 v[R1], vn[R1];
        load(rbase + h, v);
#pragma unroll 1
        for (int r0 = 0; r0 < NJ; r0 += ROWS) {
            const int row0 = r0 + rbase, row = row0 + h;
            if (r0 + ROWS < NJ) load(row + ROWS, vn);
            if (hl && row < NJ && lane_a) {
#pragma unroll
                for (int r = 0; r < R1; r++) v[r] = cmul(v[r], __ldg(&hwl[t2 + R2 * r]));
            }
            if constexpr (PR)
                row_fft2_from_regs<NL, false>(Z + (row0 < NJ ? row0 : 0) * PS, Z + (row0 + 1 < NJ ? row0 + 1 : 0) * PS,
                                              sub, row0 < NJ, row0 + 1 < NJ, v, twl);
            else
                row_fft_from_regs<NL, false>(Z + (row < NJ ? row : 0) * PS, sub, row < NJ, v, twl);
#pragma unroll
            for (int r = 0; r < R1; r++) v[r] = vn[r];
        }
    }
    __syncthreads();

    // ---- y: columns, column role, both halves from the same registers
    {
        constexpr int R1 = SJ::R1, R2 = SJ::R2, RM = SJ::RM;
        constexpr int CPP = NT / RM;   // columns per pass
        static_assert(CPP >= 1, "block too small");
        const int col0 = threadIdx.x % CPP, sub = threadIdx.x / CPP;
        float2 *dst = a.work + (size_t)rhs * a.wstride + ((size_t)c * ni + i) * (2 * NJ) * (2 * NL);
        if constexpr (halves_paired<NJ>()) {
            // sub-lines [0, R2) transform half 0 in place, [R2, R1) half 1 into the scratch
            // block S [NJ][CPP]; then every sub-line finishes both halves (step B)
            float2 *S = Z + NJ * PS;
            const int hy = sub >= R2, t2 = sub - hy * R2;
#pragma unroll 1
            for (int cbase = 0; cbase < NL; cbase += CPP) {
                const int col = cbase + col0;
                const bool ok = col < NL;
                float2 v[R1];
                if (ok) {
#pragma unroll
                    for (int r = 0; r < R1; r++) v[r] = Z[(t2 + R2 * r) * PS + spos(col)];
                }
                __syncthreads();
                if (ok) {
                    if (hy) {
#pragma unroll
                        for (int r = 0; r < R1; r++) v[r] = cmul(v[r], __ldg(&hwj[t2 + R2 * r]));
                    }
                    dft_reg<R1, false>(v);
#pragma unroll
                    for (int k1 = 1; k1 < R1; k1++) v[k1] = cmul(v[k1], twid<false>(twj, t2 * k1));
                    if (hy) {
#pragma unroll
                        for (int k1 = 0; k1 < R1; k1++) S[(t2 + R2 * k1) * CPP + col0] = v[k1];
                    } else {
#pragma unroll
                        for (int k1 = 0; k1 < R1; k1++) Z[(t2 + R2 * k1) * PS + spos(col)] = v[k1];
                    }
                }
                __syncthreads();
                if (ok) {
#pragma unroll
                    for (int h2 = 0; h2 < 2; h2++) {
                        float2 u[R2];
#pragma unroll
                        for (int t = 0; t < R2; t++)
                            u[t] = h2 ? S[(R2 * sub + t) * CPP + col0] : Z[(R2 * sub + t) * PS + spos(col)];
                        dft_reg<R2, false>(u);
                        float2 *d = dst + (size_t)(h2 * NJ) * (2 * NL) + hl * NL + col;
#pragma unroll
                        for (int k2 = 0; k2 < R2; k2++) d[(size_t)(sub + R1 * k2) * (2 * NL)] = u[k2];
                    }
                }
                __syncthreads();
            }
        } else {
#pragma unroll 1
        for (int cbase = 0; cbase < NL; cbase += CPP) {
            const int col = cbase + col0;
            const bool ok = col < NL;
            float2 orig[R1];
            if (ok && sub < R2) {
#pragma unroll
                for (int r = 0; r < R1; r++) orig[r] = Z[(sub + R2 * r) * PS + spos(col)];
            }
            __syncthreads();
#pragma unroll 1
            for (int hy = 0; hy < 2; hy++) {
                if (ok && sub < R2) {
                    float2 v[R1];
#pragma unroll
                    for (int r = 0; r < R1; r++)
                        v[r] = hy ? cmul(orig[r], __ldg(&hwj[sub + R2 * r])) : orig[r];
                    dft_reg<R1, false>(v);
#pragma unroll
                    for (int k1 = 1; k1 < R1; k1++) v[k1] = cmul(v[k1], twid<false>(twj, sub * k1));
#pragma unroll
                    for (int k1 = 0; k1 < R1; k1++) Z[(sub + R2 * k1) * PS + spos(col)] = v[k1];
                }
                __syncthreads();
                if (ok && sub < R1) {
                    float2 u[R2];
#pragma unroll
                    for (int t = 0; t < R2; t++) u[t] = Z[(R2 * sub + t) * PS + spos(col)];
                    dft_reg<R2, false>(u);
                    float2 *d = dst + (size_t)(hy * NJ) * (2 * NL) + hl * NL + col;
#pragma unroll
                    for (int k2 = 0; k2 < R2; k2++) d[(size_t)(sub + R1 * k2) * (2 * NL)] = u[k2];
                }
                __syncthreads();
            }
        }
        }
    }
}

// ------------------------------------------------------------------------------ K2
// CTA (spectral row js, TL spectral columns): forward x (both halves), 3x3 product,
// inverse x, in place.  Shared B[c][h][pos][t].
// grid order of the x pass: right-hand side fastest where the Green octant outgrows L2
__host__ __device__ constexpr bool k2_rhs_fastest(int NI) { return NI >= 128; }

// at least this many CTAs per SM: about 128 registers a thread (80 for the 16-point lines)
constexpr int k2_min_blocks(int NI, int threads)
{
    return NI == 16 ? (6 * 128) / threads : (512 / threads > 0 ? 512 / threads : 1);
}

// ---- bulk asynchronous copies (the copy engine moves global rows into shared memory and
// signals an mbarrier; no multicast)
DDA_DEV unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

DDA_DEV void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

DDA_DEV void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

DDA_DEV void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
                     "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// One tile of a 5-D tensor map (TMA, no multicast): the box at coordinates (x0 .. x4)
// into shared memory, completing on the mbarrier.  x0 is the innermost coordinate; its
// byte offset (x0 x 8) must be a multiple of 16, which the callers' column tiles keep.
DDA_DEV void tma_load_5d(void *dst, const CUtensorMap *map, int x0, int x1, int x2, int x3, int x4,
                         unsigned long long *bar)
{
    asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<unsigned long long>(map)), "r"(x0), "r"(x1), "r"(x2), "r"(x3), "r"(x4),
                 "r"(smem_addr(bar))
                 : "memory");
}

// Waits for the barrier's phase `parity` to complete, at most `polls` polls; false if it did
// not (the caller reports it through the error flag instead of hanging).
DDA_DEV bool mbar_wait(unsigned long long *bar, unsigned parity, int polls = 1 << 22)
{
    const unsigned a = smem_addr(bar);
    for (int it = 0; it < polls; it++) {
        unsigned done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// LD: how the input columns reach the CTA -- 0 register loads, 1 one bulk copy per row,
// 2 one TMA tensor tile per component (tmap: the work buffer as [rhs][c][i][js][ls] with
// the box TL x 1 x NI; unused otherwise)
template <int NI, int TL, int LD, int ALT>
__global__ void __launch_bounds__(Sx<NI, ALT>::RM * TL, k2_min_blocks(NI, Sx<NI, ALT>::RM * TL))
k2f(MatvecArgs a, const __grid_constant__ CUtensorMap tmap)
{
    using S = Sx<NI, ALT>;
    constexpr bool BULK = LD != 0;
    static_assert(!BULK || ALT == 0, "bulk copies with the default factorisation only");
    constexpr int R1 = S::R1, R2 = S::R2, RM = S::RM;
    extern __shared__ __align__(128) float2 B[];   // [6][NI][TL]
    // at edge 128 the right-hand side is the fastest grid index: CTAs that run together
    // read the same Green-tensor columns, which then come from L2 (that octant, 103 MB,
    // does not stay resident while a whole right-hand side streams through; 18.8 -> 18.4 ms
    // per 42-RHS matvec).  Smaller octants stay in L2, and there the spectral row first
    // is faster (64^3, 128 RHS: 2.42 vs 2.63 ms for this pass)
    constexpr bool rhs_fast = k2_rhs_fastest(NI);
    const int js = rhs_fast ? blockIdx.z : blockIdx.x, rhs = rhs_fast ? blockIdx.x : blockIdx.z;
    if (a.rhs_active && !a.rhs_active[rhs]) return;
    const int nj = a.L.nj, nl = a.L.nl;
    const int l0 = blockIdx.y * TL;
    const int t = threadIdx.x % TL, sub = threadIdx.x / TL;
    const size_t plane = (size_t)(2 * nj) * (2 * nl), cstr = (size_t)NI * plane;
    float2 *base = a.work + (size_t)rhs * a.wstride + (size_t)js * (2 * nl) + l0 + t;
    const float2 *tw = a.L.tw_i, *hw = a.L.tw_i + NI;
    auto Bat = [&](int c, int h, int pos) -> float2 & { return B[((c * 2 + h) * NI + pos) * TL + t]; };

    // ---- bulk variant: the 3 x NI input rows of TL columns arrive in the half-0 planes of B
    // by asynchronous bulk copies (one per row, 16-byte aligned: l0 and TL are multiples
    // of 4 float2); step A then reads them from shared memory and works in place
    if constexpr (BULK && R2 > 1) {
        __shared__ __align__(8) unsigned long long bar;
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_expect_tx(&bar, 3u * NI * TL * (unsigned)sizeof(float2));
        }
        __syncthreads();
        if constexpr (LD == 2) {
            // three tensor tiles: component c's NI x TL columns land as [i][t] in half 0
            if (threadIdx.x == 0)
#pragma unroll
                for (int c = 0; c < 3; c++) tma_load_5d(&B[(c * 2) * NI * TL], &tmap, l0, js, 0, c, rhs, &bar);
        } else {
            const float2 *row0 = a.work + (size_t)rhs * a.wstride + (size_t)js * (2 * nl) + l0;
            for (int q = threadIdx.x; q < 3 * NI; q += blockDim.x) {
                const int c = q / NI, i = q - c * NI;
                bulk_g2s(&B[((c * 2) * NI + i) * TL], row0 + c * cstr + (size_t)i * plane,
                         TL * (unsigned)sizeof(float2), &bar);
            }
        }
        // (self-test: after the copies, wait briefly for the next phase, which nothing completes)
        bool got = mbar_wait(&bar, 0);
        if (got && a.wait_selftest) got = mbar_wait(&bar, 1, 1 << 10);
        if (!__syncthreads_and(got)) {   // the same decision for every thread
            if (threadIdx.x == 0 && a.err) atomicExch(a.err, 1);
            mbar_wait(&bar, 0);           // one more bounded wait for the copies in flight
            return;
        }
        if constexpr (R1 == 2 * R2) {
            // R1 = 2 R2 (edges 32, 128): every lane works -- lane (t2, hb) transforms half hb
            // (hb = 1: the input times W_2NI^m) of the lines t2 + R2 r
            const int t2 = sub % R2, hb = sub / R2;
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                float2 v[R1];
#pragma unroll
                for (int r = 0; r < R1; r++) {
                    v[r] = Bat(c, 0, t2 + R2 * r);
                    if (hb) v[r] = cmul(v[r], __ldg(&hw[t2 + R2 * r]));
                }
                __syncthreads();   // half 0 of component c is read by both lane halves before it is rewritten
                dft_reg<R1, false>(v);
#pragma unroll
                for (int k1 = 0; k1 < R1; k1++) {
                    const float2 tk = k1 ? twid<false>(tw, t2 * k1) : make_float2(1.f, 0.f);
                    Bat(c, hb, t2 + R2 * k1) = k1 ? cmul(v[k1], tk) : v[k1];
                }
            }
        } else if (sub < R2) {
            auto step_a_smem = [&](int c) {
                float2 v[R1], w[R1];
#pragma unroll
                for (int r = 0; r < R1; r++) {
                    v[r] = Bat(c, 0, sub + R2 * r);
                    w[r] = cmul(v[r], __ldg(&hw[sub + R2 * r]));
                }
                dft_reg<R1, false>(v);
                dft_reg<R1, false>(w);
#pragma unroll
                for (int k1 = 0; k1 < R1; k1++) {
                    const float2 tk = k1 ? twid<false>(tw, sub * k1) : make_float2(1.f, 0.f);
                    Bat(c, 0, sub + R2 * k1) = k1 ? cmul(v[k1], tk) : v[k1];
                    Bat(c, 1, sub + R2 * k1) = k1 ? cmul(w[k1], tk) : w[k1];
                }
            };
#pragma unroll 1
            for (int c = 0; c < 3; c++) step_a_smem(c);
        }
    } else
    // ---- forward step A (both halves from one load)
    if (R2 == 1) {
        if (sub == 0) {
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                float2 v[R1], w[R1];
#pragma unroll
                for (int r = 0; r < R1; r++) {
                    v[r] = base[c * cstr + r * plane];
                    w[r] = cmul(v[r], __ldg(&hw[r]));
                }
                dft_reg<R1, false>(v);
                dft_reg<R1, false>(w);
#pragma unroll
                for (int k = 0; k < R1; k++) {
                    Bat(c, 0, k) = v[k];
                    Bat(c, 1, k) = w[k];
                }
            }
        }
    } else if (sub < R2) {
        // step A of one component from its R1 loaded values
        auto step_a = [&](int c, float2 (&v)[R1]) {
            float2 w[R1];
#pragma unroll
            for (int r = 0; r < R1; r++) w[r] = cmul(v[r], __ldg(&hw[sub + R2 * r]));
            dft_reg<R1, false>(v);
            dft_reg<R1, false>(w);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) {
                const float2 tk = k1 ? twid<false>(tw, sub * k1) : make_float2(1.f, 0.f);
                Bat(c, 0, sub + R2 * k1) = k1 ? cmul(v[k1], tk) : v[k1];
                Bat(c, 1, sub + R2 * k1) = k1 ? cmul(w[k1], tk) : w[k1];
            }
        };
        if constexpr (BULK) {
            // unreachable: the bulk variant loads below, before this branch
        } else if constexpr (3 * R1 <= 24) {
            // all three components' loads in flight before any arithmetic
            float2 v0[R1], v1[R1], v2[R1];
#pragma unroll
            for (int r = 0; r < R1; r++) {
                const size_t o = (size_t)(sub + R2 * r) * plane;
                v0[r] = base[o];
                v1[r] = base[cstr + o];
                v2[r] = base[2 * cstr + o];
            }
            step_a(0, v0);
            step_a(1, v1);
            step_a(2, v2);
        } else {
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                float2 v[R1];
#pragma unroll
                for (int r = 0; r < R1; r++) v[r] = base[c * cstr + (size_t)(sub + R2 * r) * plane];
                step_a(c, v);
            }
        }
    }
    __syncthreads();

    // ---- forward step B, product with the Green tensor, inverse step A
    const int hj = js >= nj, kj = js - hj * nj, jp = 2 * kj + hj;
    const int my = jp > nj, oy = my ? 2 * nj - jp : jp;
    const int ls = l0 + t, hl = ls >= nl, kl = ls - hl * nl, lp = 2 * kl + hl;
    const int mz = lp > nl, oz = mz ? 2 * nl - lp : lp;
    // Ahat[ox][oy][zmap(oz)][6]: the 6 components of one frequency are one 48-byte entry
    const size_t sz = 6, sy = (size_t)(nl + 1) * 6, sxo = (size_t)(nj + 1) * sy;
    const float2 *Ayz = a.ahat + (size_t)oy * sy + (size_t)zmapf(oz, nl) * sz;
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
        float2 X[3][R2];
        const bool act = (R2 == 1) ? (sub == 0) : (sub < R1);
        const int k1 = sub;
        if (act) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (R2 == 1) {
                    X[c][0] = czero();
                } else {
#pragma unroll
                    for (int q = 0; q < R2; q++) X[c][q] = Bat(c, h, R2 * k1 + q);
                    dft_reg<R2, false>(X[c]);
                }
            }
        }
        __syncthreads();
        if (act) {
            if (R2 == 1) {
                // single-step sizes: the whole line is in shared memory; this lane does all
#pragma unroll 1
                for (int k = 0; k < R1; k++) {
                    const int kx = 2 * k + h, mx = kx > NI, ox = mx ? 2 * NI - kx : kx;
                    const float4 *A = reinterpret_cast<const float4 *>(Ayz + (size_t)ox * sxo);
                    const float4 a01 = __ldg(A), a23 = __ldg(A + 1), a45 = __ldg(A + 2);
                    float2 g0 = make_float2(a01.x, a01.y), g1 = make_float2(a01.z, a01.w),
                           g2 = make_float2(a23.x, a23.y), g3 = make_float2(a23.z, a23.w),
                           g4 = make_float2(a45.x, a45.y), g5 = make_float2(a45.z, a45.w);
                    if (mx ^ my) g1 = cscale(g1, -1.f);
                    if (mx ^ mz) g2 = cscale(g2, -1.f);
                    if (my ^ mz) g4 = cscale(g4, -1.f);
                    if (a.conj) {
                        g0 = cconj(g0); g1 = cconj(g1); g2 = cconj(g2);
                        g3 = cconj(g3); g4 = cconj(g4); g5 = cconj(g5);
                    }
                    const float2 vx = Bat(0, h, k), vy = Bat(1, h, k), vz = Bat(2, h, k);
                    Bat(0, h, k) = cadd(cadd(cmul(g0, vx), cmul(g1, vy)), cmul(g2, vz));
                    Bat(1, h, k) = cadd(cadd(cmul(g1, vx), cmul(g3, vy)), cmul(g4, vz));
                    Bat(2, h, k) = cadd(cadd(cmul(g2, vx), cmul(g4, vy)), cmul(g5, vz));
                }
            } else {
#pragma unroll
                for (int q = 0; q < R2; q++) {
                    const int kx = 2 * (k1 + R1 * q) + h, mx = kx > NI, ox = mx ? 2 * NI - kx : kx;
                    const float4 *A = reinterpret_cast<const float4 *>(Ayz + (size_t)ox * sxo);
                    const float4 a01 = __ldg(A), a23 = __ldg(A + 1), a45 = __ldg(A + 2);
                    float2 g0 = make_float2(a01.x, a01.y), g1 = make_float2(a01.z, a01.w),
                           g2 = make_float2(a23.x, a23.y), g3 = make_float2(a23.z, a23.w),
                           g4 = make_float2(a45.x, a45.y), g5 = make_float2(a45.z, a45.w);
                    if (mx ^ my) g1 = cscale(g1, -1.f);
                    if (mx ^ mz) g2 = cscale(g2, -1.f);
                    if (my ^ mz) g4 = cscale(g4, -1.f);
                    if (a.conj) {
                        g0 = cconj(g0); g1 = cconj(g1); g2 = cconj(g2);
                        g3 = cconj(g3); g4 = cconj(g4); g5 = cconj(g5);
                    }
                    const float2 vx = X[0][q], vy = X[1][q], vz = X[2][q];
                    X[0][q] = cadd(cadd(cmul(g0, vx), cmul(g1, vy)), cmul(g2, vz));
                    X[1][q] = cadd(cadd(cmul(g1, vx), cmul(g3, vy)), cmul(g4, vz));
                    X[2][q] = cadd(cadd(cmul(g2, vx), cmul(g4, vy)), cmul(g5, vz));
                }
                // inverse step A with the transposed split: lane k1 owns positions k1 + R1 q
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    dft_reg<R2, true>(X[c]);
#pragma unroll
                    for (int u = 0; u < R2; u++) {
                        const float2 y = u ? cmul(X[c][u], twid<true>(tw, k1 * u)) : X[c][u];
                        Bat(c, h, k1 + R1 * u) = y;
                    }
                }
            }
        }
        __syncthreads();
    }

    // ---- inverse step B (transposed split: R2 lanes of R1 elements), combine, store
    if (R2 == 1) {
        if (sub == 0) {
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                float2 e[R1], o[R1];
#pragma unroll
                for (int k = 0; k < R1; k++) {
                    e[k] = Bat(c, 0, k);
                    o[k] = Bat(c, 1, k);
                }
                dft_reg<R1, true>(e);
                dft_reg<R1, true>(o);
#pragma unroll
                for (int k = 0; k < R1; k++)
                    base[c * cstr + k * plane] = cadd(e[k], cmulc(o[k], __ldg(&hw[k])));
            }
        }
    } else if constexpr (R1 == 2 * R2) {
        // every lane works: lane (k1p, hb) produces the outputs k2 = 2 m + hb of its lines,
        // an R1/2-point inverse DFT of y[n] = (x[n] + (-1)^hb x[n + R1/2]) exp(2 pi i n hb / R1)
        const int k1p = sub % R2, hb = sub / R2;
        constexpr int H = R1 / 2;
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
            float2 e[H], o[H];
#pragma unroll
            for (int n = 0; n < H; n++) {
                const float2 e0 = Bat(c, 0, R1 * k1p + n), e1 = Bat(c, 0, R1 * k1p + n + H);
                const float2 o0 = Bat(c, 1, R1 * k1p + n), o1 = Bat(c, 1, R1 * k1p + n + H);
                if (hb) {
                    const float2 wn = cconj(w16(n * (16 / R1)));
                    e[n] = n ? cmul(csub(e0, e1), wn) : csub(e0, e1);
                    o[n] = n ? cmul(csub(o0, o1), wn) : csub(o0, o1);
                } else {
                    e[n] = cadd(e0, e1);
                    o[n] = cadd(o0, o1);
                }
            }
            dft_reg<H, true>(e);
            dft_reg<H, true>(o);
#pragma unroll
            for (int m = 0; m < H; m++) {
                const int i = k1p + R2 * (2 * m + hb);
                base[c * cstr + i * plane] = cadd(e[m], cmulc(o[m], __ldg(&hw[i])));
            }
        }
    } else if (sub < R2) {
        const int k1p = sub;
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
            float2 e[R1], o[R1];
#pragma unroll
            for (int q = 0; q < R1; q++) {
                e[q] = Bat(c, 0, R1 * k1p + q);
                o[q] = Bat(c, 1, R1 * k1p + q);
            }
            dft_reg<R1, true>(e);
            dft_reg<R1, true>(o);
#pragma unroll
            for (int k2 = 0; k2 < R1; k2++) {
                const int i = k1p + R2 * k2;
                base[c * cstr + i * plane] = cadd(e[k2], cmulc(o[k2], __ldg(&hw[i])));
            }
        }
    }
}

// Pair form of the x pass (MatvecArgs::pair, step 0): CTA (spectral row js, TL spectral
// columns, polarisation pair k).  The forward transform of phi (component slot 0 of
// right-hand side 2k) is done once; then for each polarisation q the spectrum G (E_q phi)
// is formed -- the product of the single form with v = E_q phi -- inverse-transformed and
// written to the three component slots of right-hand side 2k + q.  Shared B[c][h][pos][t]
// with c = 0..2 the output components and c = 3 the spectrum of phi.
template <int NI, int TL>
__global__ void __launch_bounds__(Sp<NI>::RM * TL, k2_min_blocks(NI, Sp<NI>::RM * TL)) k2p(MatvecArgs a)
{
    using S = Sp<NI>;
    constexpr int R1 = S::R1, R2 = S::R2;
    static_assert(R2 > 1, "the pair form needs a two-step line FFT");
    extern __shared__ __align__(128) float2 B[];   // [4][2][NI][TL]
    constexpr bool rhs_fast = k2_rhs_fastest(NI);
    const int js = rhs_fast ? blockIdx.z : blockIdx.x, pr = rhs_fast ? blockIdx.x : blockIdx.z;
    const int rhs0 = 2 * pr;
    if (a.rhs_active && !a.rhs_active[rhs0]) return;
    const int nj = a.L.nj, nl = a.L.nl;
    const int l0 = blockIdx.y * TL;
    const int t = threadIdx.x % TL, sub = threadIdx.x / TL;
    const size_t plane = (size_t)(2 * nj) * (2 * nl), cstr = (size_t)NI * plane;
    const size_t col = (size_t)js * (2 * nl) + l0 + t;
    const float2 *tw = a.L.tw_i, *hw = a.L.tw_i + NI;
    auto Bat = [&](int c, int h, int pos) -> float2 & { return B[((c * 2 + h) * NI + pos) * TL + t]; };

    // ---- forward step A of phi, both halves from one load
    if (sub < R2) {
        const float2 *src = a.work + (size_t)rhs0 * a.wstride + col;
        float2 v[R1], w[R1];
#pragma unroll
        for (int r = 0; r < R1; r++) v[r] = src[(size_t)(sub + R2 * r) * plane];
#pragma unroll
        for (int r = 0; r < R1; r++) w[r] = cmul(v[r], __ldg(&hw[sub + R2 * r]));
        dft_reg<R1, false>(v);
        dft_reg<R1, false>(w);
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) {
            const float2 tk = k1 ? twid<false>(tw, sub * k1) : make_float2(1.f, 0.f);
            Bat(3, 0, sub + R2 * k1) = k1 ? cmul(v[k1], tk) : v[k1];
            Bat(3, 1, sub + R2 * k1) = k1 ? cmul(w[k1], tk) : w[k1];
        }
    }
    __syncthreads();
    // ---- forward step B of phi, in place: lane k1 keeps frequencies k1 + R1 q at R2 k1 + q
    if (sub < R1) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float2 X[R2];
#pragma unroll
            for (int q = 0; q < R2; q++) X[q] = Bat(3, h, R2 * sub + q);
            dft_reg<R2, false>(X);
#pragma unroll
            for (int q = 0; q < R2; q++) Bat(3, h, R2 * sub + q) = X[q];
        }
    }
    __syncthreads();

    const int hj = js >= nj, kj = js - hj * nj, jp = 2 * kj + hj;
    const int my = jp > nj, oy = my ? 2 * nj - jp : jp;
    const int ls = l0 + t, hl = ls >= nl, kl = ls - hl * nl, lp = 2 * kl + hl;
    const int mz = lp > nl, oz = mz ? 2 * nl - lp : lp;
    const size_t sz = 6, sy = (size_t)(nl + 1) * 6, sxo = (size_t)(nj + 1) * sy;
    const float2 *Ayz = a.ahat + (size_t)oy * sy + (size_t)zmapf(oz, nl) * sz;
#pragma unroll 1
    for (int pol = 0; pol < 2; pol++) {
        const double *E = a.einc + 6 * (rhs0 + pol);
        const float2 Ex = make_float2((float)E[0], (float)E[1]), Ey = make_float2((float)E[2], (float)E[3]),
                     Ez = make_float2((float)E[4], (float)E[5]);
        // a real incident field (every rotated x or y polarisation): u = G E with real
        // weights (fused multiply-adds on the components), then u psi -- 30 instead of 54
        // floating-point instructions per frequency
        const bool Ereal = Ex.y == 0.f && Ey.y == 0.f && Ez.y == 0.f;
        // ---- product with the Green tensor, inverse step A (transposed split); the branch
        // on a real field is taken once per polarisation, outside the unrolled loops
        auto product = [&](auto real_tag) {
            constexpr bool REAL = decltype(real_tag)::value;
            const int k1 = sub;
#pragma unroll 1
            for (int h = 0; h < 2; h++) {
                float2 X[3][R2];
#pragma unroll
                for (int q = 0; q < R2; q++) {
                    const int kx = 2 * (k1 + R1 * q) + h, mx = kx > NI, ox = mx ? 2 * NI - kx : kx;
                    const float4 *A = reinterpret_cast<const float4 *>(Ayz + (size_t)ox * sxo);
                    const float4 a01 = __ldg(A), a23 = __ldg(A + 1), a45 = __ldg(A + 2);
                    float2 g0 = make_float2(a01.x, a01.y), g1 = make_float2(a01.z, a01.w),
                           g2 = make_float2(a23.x, a23.y), g3 = make_float2(a23.z, a23.w),
                           g4 = make_float2(a45.x, a45.y), g5 = make_float2(a45.z, a45.w);
                    if (mx ^ my) g1 = cscale(g1, -1.f);
                    if (mx ^ mz) g2 = cscale(g2, -1.f);
                    if (my ^ mz) g4 = cscale(g4, -1.f);
                    const float2 ps = Bat(3, h, R2 * k1 + q);
                    if constexpr (REAL) {
                        const float ex = Ex.x, ey = Ey.x, ez = Ez.x;
                        auto dot = [&](float2 ga, float2 gb, float2 gc) {
                            return make_float2(fmaf(ga.x, ex, fmaf(gb.x, ey, gc.x * ez)),
                                               fmaf(ga.y, ex, fmaf(gb.y, ey, gc.y * ez)));
                        };
                        X[0][q] = cmul(dot(g0, g1, g2), ps);
                        X[1][q] = cmul(dot(g1, g3, g4), ps);
                        X[2][q] = cmul(dot(g2, g4, g5), ps);
                    } else {
                        const float2 vx = cmul(Ex, ps), vy = cmul(Ey, ps), vz = cmul(Ez, ps);
                        X[0][q] = cadd(cadd(cmul(g0, vx), cmul(g1, vy)), cmul(g2, vz));
                        X[1][q] = cadd(cadd(cmul(g1, vx), cmul(g3, vy)), cmul(g4, vz));
                        X[2][q] = cadd(cadd(cmul(g2, vx), cmul(g4, vy)), cmul(g5, vz));
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    dft_reg<R2, true>(X[c]);
#pragma unroll
                    for (int u = 0; u < R2; u++) {
                        const float2 y = u ? cmul(X[c][u], twid<true>(tw, k1 * u)) : X[c][u];
                        Bat(c, h, k1 + R1 * u) = y;
                    }
                }
            }
        };
        if (sub < R1) {
            if (Ereal) product(std::true_type{});
            else product(std::false_type{});
        }
        __syncthreads();
        // ---- inverse step B, combine the halves, store to right-hand side 2k + pol
        float2 *base = a.work + (size_t)(rhs0 + pol) * a.wstride + col;
        if constexpr (R1 == 2 * R2) {
            const int k1p = sub % R2, hb = sub / R2;
            constexpr int H = R1 / 2;
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                float2 e[H], o[H];
#pragma unroll
                for (int n = 0; n < H; n++) {
                    const float2 e0 = Bat(c, 0, R1 * k1p + n), e1 = Bat(c, 0, R1 * k1p + n + H);
                    const float2 o0 = Bat(c, 1, R1 * k1p + n), o1 = Bat(c, 1, R1 * k1p + n + H);
                    if (hb) {
                        const float2 wn = cconj(w16(n * (16 / R1)));
                        e[n] = n ? cmul(csub(e0, e1), wn) : csub(e0, e1);
                        o[n] = n ? cmul(csub(o0, o1), wn) : csub(o0, o1);
                    } else {
                        e[n] = cadd(e0, e1);
                        o[n] = cadd(o0, o1);
                    }
                }
                dft_reg<H, true>(e);
                dft_reg<H, true>(o);
#pragma unroll
                for (int m = 0; m < H; m++) {
                    const int i = k1p + R2 * (2 * m + hb);
                    base[c * cstr + i * plane] = cadd(e[m], cmulc(o[m], __ldg(&hw[i])));
                }
            }
        } else if (sub < R2) {
            const int k1p = sub;
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                float2 e[R1], o[R1];
#pragma unroll
                for (int q = 0; q < R1; q++) {
                    e[q] = Bat(c, 0, R1 * k1p + q);
                    o[q] = Bat(c, 1, R1 * k1p + q);
                }
                dft_reg<R1, true>(e);
                dft_reg<R1, true>(o);
#pragma unroll
                for (int k2 = 0; k2 < R1; k2++) {
                    const int i = k1p + R2 * k2;
                    base[c * cstr + i * plane] = cadd(e[k2], cmulc(o[k2], __ldg(&hw[i])));
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------ K3
// Cluster pair (rank = z half hl) per (i, component): y-inverse of this half's NL
// columns (both y halves), z-inverse of the NJ rows restricted to this half, then the two
// halves are summed through distributed shared memory and the epilogue writes the rows of
// this rank.
template <int NJ, int NL, int NT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NT) k3f(MatvecArgs a)
{
    using SJ = Sp<NJ>;
    using SL = Sp<NL>;
    constexpr int PS = SL::PS;
    extern __shared__ float2 Q[];   // [NJ][PS]
    cg::cluster_group cl = cg::this_cluster();
    const int hl = (int)cl.block_rank();
    const int i = blockIdx.x >> 1, c = blockIdx.y, rhs = blockIdx.z;
    if (a.rhs_active && !a.rhs_active[rhs]) return;   // uniform over the cluster
    const int ni = a.L.ni;
    const float2 *src = a.work + (size_t)rhs * a.wstride + ((size_t)c * ni + i) * (2 * NJ) * (2 * NL) + hl * NL;
    const float2 *twl = a.L.tw_l, *hwl = a.L.tw_l + NL, *twj = a.L.tw_j, *hwj = a.L.tw_j + NJ;

    // ---- y inverse on this half's columns: x[j] = IDFT(even)[j] + W^-j IDFT(odd)[j]
    if constexpr (halves_paired<NJ>()) {
        // sub-lines [0, R2) take the even half (step A in place), [R2, R1) the odd half
        // (into the scratch block S [NJ][CPP]); every sub-line then finishes both and sums
        constexpr int R1 = SJ::R1, R2 = SJ::R2, RM = SJ::RM;
        constexpr int CPP = NT / RM;
        const int col0 = threadIdx.x % CPP, sub = threadIdx.x / CPP;
        const int hy = sub >= R2, t2 = sub - hy * R2;
        float2 *S = Q + NJ * PS;
#pragma unroll 1
        for (int cbase = 0; cbase < NL; cbase += CPP) {
            const int col = cbase + col0;
            const bool ok = col < NL;
            if (ok) {
                float2 v[R1];
#pragma unroll
                for (int r = 0; r < R1; r++) v[r] = src[(size_t)(hy * NJ + t2 + R2 * r) * (2 * NL) + col];
                dft_reg<R1, true>(v);
#pragma unroll
                for (int k1 = 1; k1 < R1; k1++) v[k1] = cmul(v[k1], twid<true>(twj, t2 * k1));
                if (hy) {
#pragma unroll
                    for (int k1 = 0; k1 < R1; k1++) S[(t2 + R2 * k1) * CPP + col0] = v[k1];
                } else {
#pragma unroll
                    for (int k1 = 0; k1 < R1; k1++) Q[(t2 + R2 * k1) * PS + spos(col)] = v[k1];
                }
            }
            __syncthreads();
            float2 y[R2];
            if (ok) {
                float2 u0[R2], u1[R2];
#pragma unroll
                for (int t = 0; t < R2; t++) {
                    u0[t] = Q[(R2 * sub + t) * PS + spos(col)];
                    u1[t] = S[(R2 * sub + t) * CPP + col0];
                }
                dft_reg<R2, true>(u0);
                dft_reg<R2, true>(u1);
#pragma unroll
                for (int k2 = 0; k2 < R2; k2++) y[k2] = cadd(u0[k2], cmulc(u1[k2], __ldg(&hwj[sub + R1 * k2])));
            }
            __syncthreads();
            if (ok) {
#pragma unroll
                for (int k2 = 0; k2 < R2; k2++) Q[(sub + R1 * k2) * PS + spos(col)] = y[k2];
            }
        }
    } else {
        constexpr int R1 = SJ::R1, R2 = SJ::R2, RM = SJ::RM;
        constexpr int CPP = NT / RM;
        const int col0 = threadIdx.x % CPP, sub = threadIdx.x / CPP;
#pragma unroll 1
        for (int cbase = 0; cbase < NL; cbase += CPP) {
            const int col = cbase + col0;
            const bool ok = col < NL;
            float2 y0[R2];
            // both y halves' loads in flight before the first transform
            float2 vh[2][R1];
            if (ok && sub < R2) {
#pragma unroll
                for (int hy = 0; hy < 2; hy++)
#pragma unroll
                    for (int r = 0; r < R1; r++)
                        vh[hy][r] = src[(size_t)(hy * NJ + sub + R2 * r) * (2 * NL) + col];
            }
#pragma unroll
            for (int hy = 0; hy < 2; hy++) {
                if (ok && sub < R2) {
                    float2 (&v)[R1] = vh[hy];
                    dft_reg<R1, true>(v);
#pragma unroll
                    for (int k1 = 1; k1 < R1; k1++) v[k1] = cmul(v[k1], twid<true>(twj, sub * k1));
#pragma unroll
                    for (int k1 = 0; k1 < R1; k1++) Q[(sub + R2 * k1) * PS + spos(col)] = v[k1];
                }
                __syncthreads();
                float2 u[R2];
                if (ok && sub < R1) {
#pragma unroll
                    for (int t = 0; t < R2; t++) u[t] = Q[(R2 * sub + t) * PS + spos(col)];
                    dft_reg<R2, true>(u);
                    if (hy == 0) {
#pragma unroll
                        for (int k2 = 0; k2 < R2; k2++) y0[k2] = u[k2];
                    } else {
#pragma unroll
                        for (int k2 = 0; k2 < R2; k2++) {
                            const int j = sub + R1 * k2;
                            y0[k2] = cadd(y0[k2], cmulc(u[k2], __ldg(&hwj[j])));
                        }
                    }
                }
                __syncthreads();
            }
            if (ok && sub < R1) {
#pragma unroll
                for (int k2 = 0; k2 < R2; k2++) Q[(sub + R1 * k2) * PS + spos(col)] = y0[k2];
            }
        }
    }
    __syncthreads();

    // ---- z inverse of the rows (this half's spectral columns), row role
    {
        constexpr int RM = SL::RM, RPP = NT / RM, R1 = SL::R1, R2 = SL::R2;
        // PR: two rows per lane group (lane half h, step-A index t2); else one row
        constexpr bool PR = rows_paired<NJ, NL, NT>();
        constexpr int ROWS = PR ? 2 * RPP : RPP;
        const int sub = threadIdx.x % RM, rr = threadIdx.x / RM;
        const int h = PR ? (sub >= R2) : 0, t2 = sub - h * R2, rbase = PR ? 2 * rr : rr;
        const bool lane_a = PR || sub < R2;
#pragma unroll 1
        for (int r0 = 0; r0 < NJ; r0 += ROWS) {
            const int row0 = r0 + rbase, row = row0 + h;
            float2 v[R1];
            if (row < NJ && lane_a) {
#pragma unroll
                for (int r = 0; r < R1; r++) v[r] = Q[row * PS + spos(t2 + R2 * r)];
            }
            __syncwarp();
            if constexpr (PR)
                row_fft2_from_regs<NL, true>(Q + (row0 < NJ ? row0 : 0) * PS, Q + (row0 + 1 < NJ ? row0 + 1 : 0) * PS,
                                             sub, row0 < NJ, row0 + 1 < NJ, v, twl);
            else
                row_fft_from_regs<NL, true>(Q + (row < NJ ? row : 0) * PS, sub, row < NJ, v, twl);
            if (hl == 1) {
                // odd half: times W_2NL^-l
#pragma unroll
                for (int q = 0; q < (PR ? 2 : 1); q++) {
                    const int rw = row0 + q;
                    if (rw < NJ)
                        for (int l = sub; l < NL; l += RM) Q[rw * PS + spos(l)] = cmulc(Q[rw * PS + spos(l)], __ldg(&hwl[l]));
                }
            }
        }
    }
    cl.sync();

    // ---- sum of the two halves, epilogue, rows of this rank
    const float2 *R = cl.map_shared_rank(Q, hl ^ 1);
    constexpr int HR = NJ / 2, EPK = (HR * NL + NT - 1) / NT;   // output cells per thread
    const size_t N = a.L.N;
    const size_t obase = (size_t)rhs * a.fstride + (size_t)c * N + (size_t)i * NJ * NL;
    const Epilogue &ep = a.ep;
    // the solver form's materials: all of this thread's occupancy bytes are loaded before
    // the first is used (one latency instead of one per cell), and with at most two
    // materials the activity flags and polarisabilities come from registers
    int mk[EPK];
    bool act0 = false, act1 = false;
    float2 al0 = czero(), al1 = czero();
    const bool regtab = ep.mode == 1 && ep.nmat1 <= 2;
    if (ep.mode == 1) {
        const signed char *ob = ep.occ + (size_t)rhs * ep.occ_stride + ((size_t)i * NJ + (size_t)hl * HR) * NL;
#pragma unroll
        for (int k = 0; k < EPK; k++) {
            const int e = threadIdx.x + NT * k;
            mk[k] = e < HR * NL ? (int)ob[e] : 0;
        }
        if (regtab) {
            act0 = ep.mv[0] != 0;
            al0 = ep.alpha[(size_t)rhs * ep.nmat1];
            if (ep.nmat1 > 1) {
                act1 = ep.mv[1] != 0;
                al1 = ep.alpha[(size_t)rhs * ep.nmat1 + 1];
            }
            if (ep.conj) {
                al0 = cconj(al0);
                al1 = cconj(al1);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < EPK; k++) {
        const int e = threadIdx.x + NT * k;
        if (e >= HR * NL) break;
        const int jj = e / NL, l = e % NL, j = hl * HR + jj;
        const int q = j * PS + spos(l);
        const float2 conv = cadd(Q[q], R[q]);
        const size_t o = obase + (size_t)j * NL + l;
        float2 res = conv;
        if (ep.mode == 1) {
            const int m = mk[k];
            const bool act = regtab ? ((m & 1) ? act1 : act0) : ep.mv[m] != 0;
            if (!act) {
                res = czero();
            } else {
                float2 al;
                if (regtab) {
                    al = (m & 1) ? al1 : al0;
                } else {
                    al = ep.alpha[(size_t)rhs * ep.nmat1 + m];
                    if (ep.conj) al = cconj(al);
                }
                res = csub(ep.sv != 0.f ? cscale(ep.v[o], ep.sv) : czero(), cmul(al, conv));
            }
        }
        a.out[o] = res;
    }
    cl.sync();
}

// Launch variants the autotuner chooses between (variant 0 is the default): block size of
// the y/z passes, columns per CTA of the x pass.
template <int NJ, int NL>
constexpr int yz_threads(int v)
{
    // variant 0: enough threads for the column role on all NL columns and the row role on
    // all rows; variant 1: the other of 256 / 512; variant 2: 128
    const int t0 = (Sp<NJ>::RM * NL) > 256 ? 512 : 256;
    return v == 0 ? t0 : v == 1 ? (t0 == 512 ? 256 : 512) : 128;
}

template <int NJ, int NL, int NT>
constexpr size_t yz_smem()
{
    // one plane (128 KB at 128 x 128), and the odd y half's scratch when the halves pair
    return (size_t)NJ * Sp<NL>::PS * sizeof(float2) +
           (halves_paired<NJ>() ? (size_t)NJ * (NT / Sp<NJ>::RM) * sizeof(float2) : 0);
}

template <int NJ, int NL, int V>
void launch_yz_v(const MatvecArgs &a, int fwd, cudaStream_t st)
{
    constexpr int NT = yz_threads<NJ, NL>(V);
    constexpr size_t S = yz_smem<NJ, NL, NT>();
    if (fwd && a.inc && a.pair) k1f<NJ, NL, NT, 2><<<dim3(2 * a.L.ni, 1, a.nrhs / 2), NT, S, st>>>(a);
    else if (fwd && a.inc) k1f<NJ, NL, NT, 1><<<dim3(2 * a.L.ni, 3, a.nrhs), NT, S, st>>>(a);
    else if (fwd) k1f<NJ, NL, NT, 0><<<dim3(2 * a.L.ni, 3, a.nrhs), NT, S, st>>>(a);
    else k3f<NJ, NL, NT><<<dim3(2 * a.L.ni, 3, a.nrhs), NT, S, st>>>(a);
}

template <int NJ, int NL>
void launch_yz(const MatvecArgs &a, int fwd, cudaStream_t st)
{
    if (a.fyz == 2) launch_yz_v<NJ, NL, 2>(a, fwd, st);
    else if (a.fyz == 1) launch_yz_v<NJ, NL, 1>(a, fwd, st);
    else launch_yz_v<NJ, NL, 0>(a, fwd, st);
}

template <int NJ, int NL, int V>
cudaError_t prep_yz_v()
{
    constexpr int NT = yz_threads<NJ, NL>(V);
    constexpr int S = (int)yz_smem<NJ, NL, NT>();
    cudaError_t e = cudaFuncSetAttribute(k1f<NJ, NL, NT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, S);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k1f<NJ, NL, NT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, S);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k1f<NJ, NL, NT, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, S);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k3f<NJ, NL, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S);
    return e;
}

template <int NJ, int NL>
cudaError_t prep_yz()
{
    cudaError_t e = prep_yz_v<NJ, NL, 0>();
    if (e == cudaSuccess) e = prep_yz_v<NJ, NL, 1>();
    return e == cudaSuccess ? prep_yz_v<NJ, NL, 2>() : e;
}

template <int NI>
constexpr int x_tile(int v)
{
    // variant 0: 32 columns per CTA (16 at NI = 128); variants 1, 2: a half, a quarter
    const int t0 = NI <= 64 ? 32 : 16;
    return t0 >> v;
}

// x variants 0..2: register loads with 32 / 16 / 8 columns (16 / 8 / 4 at edge 128);
// 3..5: the same tiles fed by bulk asynchronous copies; 6..8: register loads with the
// second line factorisation (Sx<N, 1>)
// 9..11: the same tiles as 0..2 fed by one TMA tensor tile per component
template <int V>
constexpr int x_load(int) { return (V >= 3 && V < 6) ? 1 : (V >= 9 ? 2 : 0); }

template <int NI, int V>
void launch_x_v(const MatvecArgs &a, cudaStream_t st)
{
    constexpr int TL = x_tile<NI>(V % 3), ALT = (V >= 6 && V < 9) ? 1 : 0, LD = x_load<V>(0);
    const int ncol = 2 * a.L.nl;
    const size_t smem = (size_t)6 * NI * TL * sizeof(float2);
    const dim3 grid = k2_rhs_fastest(NI) ? dim3(a.nrhs, ncol / TL, 2 * a.L.nj)
                                         : dim3(2 * a.L.nj, ncol / TL, a.nrhs);
    static const CUtensorMap none{};
    const CUtensorMap &map = LD == 2 ? static_cast<const CUtensorMap *>(a.tmaps)[V % 3] : none;
    k2f<NI, TL, LD, ALT><<<grid, Sx<NI, ALT>::RM * TL, smem, st>>>(a, map);
}

// the pair form of the x pass (step 0 of polarisation pairs), same column tiles
template <int NI, int V>
void launch_x_pair_v(const MatvecArgs &a, cudaStream_t st)
{
    constexpr int TL = x_tile<NI>(V);
    const int ncol = 2 * a.L.nl, np = a.nrhs / 2;
    const size_t smem = (size_t)8 * NI * TL * sizeof(float2);
    const dim3 grid = k2_rhs_fastest(NI) ? dim3(np, ncol / TL, 2 * a.L.nj) : dim3(2 * a.L.nj, ncol / TL, np);
    k2p<NI, TL><<<grid, Sp<NI>::RM * TL, smem, st>>>(a);
}

template <int NI>
void launch_x(const MatvecArgs &a, cudaStream_t st)
{
    if (a.inc && a.pair) {
        switch (a.fx % 3) {
        case 2: launch_x_pair_v<NI, 2>(a, st); break;
        case 1: launch_x_pair_v<NI, 1>(a, st); break;
        default: launch_x_pair_v<NI, 0>(a, st); break;
        }
        return;
    }
    switch (a.fx) {
    case 11: launch_x_v<NI, 11>(a, st); break;
    case 10: launch_x_v<NI, 10>(a, st); break;
    case 9: launch_x_v<NI, 9>(a, st); break;
    case 8: launch_x_v<NI, 8>(a, st); break;
    case 7: launch_x_v<NI, 7>(a, st); break;
    case 6: launch_x_v<NI, 6>(a, st); break;
    case 5: launch_x_v<NI, 5>(a, st); break;
    case 4: launch_x_v<NI, 4>(a, st); break;
    case 3: launch_x_v<NI, 3>(a, st); break;
    case 2: launch_x_v<NI, 2>(a, st); break;
    case 1: launch_x_v<NI, 1>(a, st); break;
    default: launch_x_v<NI, 0>(a, st); break;
    }
}

template <int NI, int V>
cudaError_t prep_x_v()
{
    constexpr int TL = x_tile<NI>(V % 3), ALT = (V >= 6 && V < 9) ? 1 : 0, LD = x_load<V>(0);
    cudaError_t e = cudaFuncSetAttribute(k2f<NI, TL, LD, ALT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(6 * NI * TL * sizeof(float2)));
    if (e == cudaSuccess && V < 3)
        e = cudaFuncSetAttribute(k2p<NI, TL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(8 * NI * TL * sizeof(float2)));
    return e;
}

template <int NI>
cudaError_t prep_x()
{
    cudaError_t e = prep_x_v<NI, 0>();
    if (e == cudaSuccess) e = prep_x_v<NI, 1>();
    if (e == cudaSuccess) e = prep_x_v<NI, 2>();
    if (e == cudaSuccess) e = prep_x_v<NI, 3>();
    if (e == cudaSuccess) e = prep_x_v<NI, 4>();
    if (e == cudaSuccess) e = prep_x_v<NI, 5>();
    if (e == cudaSuccess) e = prep_x_v<NI, 6>();
    if (e == cudaSuccess) e = prep_x_v<NI, 7>();
    if (e == cudaSuccess) e = prep_x_v<NI, 8>();
    if (e == cudaSuccess) e = prep_x_v<NI, 9>();
    if (e == cudaSuccess) e = prep_x_v<NI, 10>();
    return e == cudaSuccess ? prep_x_v<NI, 11>() : e;
}

bool fast_edge(int n) { return n == 16 || n == 32 || n == 64 || n == 128; }

}  // namespace

int matvec_fast_x_tile(int ni, int v)
{
    switch (ni) {
    case 16: return x_tile<16>(v % 3);
    case 32: return x_tile<32>(v % 3);
    case 64: return x_tile<64>(v % 3);
    case 128: return x_tile<128>(v % 3);
    }
    return 0;
}

bool matvec_fast_supported(const Lat &L)
{
    return fast_edge(L.ni) && fast_edge(L.nj) && fast_edge(L.nl) && 2 * L.nl >= 32;
}

#define DISPATCH_YZ(NJv, CALL)                                                               \
    case NJv:                                                                                \
        switch (nl) {                                                                        \
        case 16: CALL(NJv, 16); break;                                                       \
        case 32: CALL(NJv, 32); break;                                                       \
        case 64: CALL(NJv, 64); break;                                                       \
        case 128: CALL(NJv, 128); break;                                                     \
        }                                                                                    \
        break;
#define YZ_SWITCH(CALL)                                                                      \
    switch (nj) {                                                                            \
        DISPATCH_YZ(16, CALL)                                                                \
        DISPATCH_YZ(32, CALL)                                                                \
        DISPATCH_YZ(64, CALL)                                                                \
        DISPATCH_YZ(128, CALL)                                                               \
    }

cudaError_t matvec_fast_prepare(const Lat &L)
{
    cudaError_t e = cudaErrorInvalidValue;
    const int nj = L.nj, nl = L.nl;
#define PREP(J, K) e = prep_yz<J, K>()
    YZ_SWITCH(PREP)
#undef PREP
    if (e != cudaSuccess) return e;
    switch (L.ni) {
    case 16: return prep_x<16>();
    case 32: return prep_x<32>();
    case 64: return prep_x<64>();
    case 128: return prep_x<128>();
    }
    return cudaErrorInvalidValue;
}

static void yz(const MatvecArgs &a, int fwd, cudaStream_t st)
{
    const int nj = a.L.nj, nl = a.L.nl;
#define LAUNCH(J, K) launch_yz<J, K>(a, fwd, st)
    YZ_SWITCH(LAUNCH)
#undef LAUNCH
}

cudaError_t launch_matvec_fast(const MatvecArgs &a, cudaStream_t st)
{
    if (a.fx >= 9 && !a.tmaps) return cudaErrorInvalidValue;   // no tensor maps for the TMA variants
    yz(a, 1, st);
    switch (a.L.ni) {
    case 16: launch_x<16>(a, st); break;
    case 32: launch_x<32>(a, st); break;
    case 64: launch_x<64>(a, st); break;
    case 128: launch_x<128>(a, st); break;
    }
    yz(a, 0, st);
    return cudaGetLastError();
}

}  // namespace ddagpu
