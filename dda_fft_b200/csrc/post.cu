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
#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "internal.h"
#include "post.h"

namespace ddagpu {

namespace {

// Far-field tiling.  A CTA takes s.planes (<= FF_PLANES) lattice planes i of one right-hand side and up to
// FF_DMAX directions, whose phase tables (one per axis) it builds once.  Thread (dg, w)
// accumulates DPT directions x 3 components; the RW threads w of one direction group are
// workers that split the plane's dipoles evenly:
//   1. the plane's occupancy is staged in shared memory and each row's active cells
//      counted with warp ballots; a prefix sum over the rows gives every active cell a
//      position in one list (row by row, columns in order), so a porous target's holes
//      cost nothing;
//   2. the list is taken in chunks of ff_cap cells: the dipoles of a chunk are copied into
//      shared memory (cp.async) with their row, column and material packed in one word,
//      and worker w sums positions [w len / RW, (w + 1) len / RW) of the chunk:
//      t += exp(i kz z) P along a row, and at each row end acc += exp(i (kx x + ky y)) t.
// So every lane does the same number of cells whatever the target's shape.  With NR = 2 a
// CTA takes the two right-hand sides of one orientation (both incident polarisations: the
// same scattering directions and occupancy), so each phase factor it loads feeds both and
// the occupancy, spans and list are built once for the pair; a thread then takes DPT = 2
// directions, which keeps its accumulators in registers.  With CC set, the CTAs of the
// first direction chunk also sum Cext and Cabs over the staged cells, so the dipoles are
// read from HBM once for both.
constexpr int FF_DMAX = 32;
constexpr int FF_DQ = 4;         // directions per CTA are padded to a multiple of this
constexpr int FF_PLANES = 8;     // lattice planes per CTA at most

// list cells per chunk
__host__ __device__ constexpr int ff_cap(int nr) { return nr == 2 ? 512 : 1024; }

struct FFShape {
    int D, dpt, DG, RW, threads, planes;
};

// blocks: right-hand-side blocks of the grid (nrhs / NR); the planes per CTA are the most
// that still give the grid eight CTAs per SM (148 SMs), two at least, so that the plane
// groups' unequal work (a target's middle planes hold more dipoles) is spread
FFShape ff_shape(int ndir, int dpt, int ni = 1, int blocks = 1)
{
    FFShape s;
    const int chunks = (ndir + FF_DMAX - 1) / FF_DMAX;
    s.planes = FF_PLANES;
    while (s.planes > 2 && (long long)((ni + s.planes - 1) / s.planes) * chunks * blocks < 8 * 148) s.planes /= 2;
    s.D = ndir >= FF_DMAX ? FF_DMAX : ((ndir + FF_DQ - 1) / FF_DQ) * FF_DQ;
    if (s.D < FF_DQ) s.D = FF_DQ;
    s.dpt = dpt;
    s.DG = s.D / dpt;
    // the block is a whole number of warps, at most 256 threads
    if (s.DG <= 8) {
        const int k = 8 / s.DG;
        s.RW = 32 * (k > 1 ? k : 1);
    } else {
        s.RW = 16;   // DG even (D is a multiple of 4 and dpt 2), so 16 DG is a whole number of warps
    }
    s.threads = s.DG * s.RW;
    return s;
}

template <int DPT>
DDA_DEV void ld_dirs(const float2 *p, float2 (&v)[DPT])
{
#pragma unroll
    for (int k = 0; k < DPT; k += 2) {
        const float4 q = *reinterpret_cast<const float4 *>(p + k);
        v[k] = make_float2(q.x, q.y);
        v[k + 1] = make_float2(q.z, q.w);
    }
}

// Shared-memory layout (byte offsets, 16-byte aligned blocks).
struct FFLayout {
    size_t tab, eyx, P, cc, idx, ints, occ, total;
};

__host__ __device__ inline size_t ff_al16(size_t b) { return (b + 15) & ~(size_t)15; }

__host__ __device__ inline FFLayout ff_layout(FFShape s, int nj, int nl, int nmat1, bool cc, int nr)
{
    const size_t f2 = sizeof(float2);
    size_t pz = (size_t)ff_cap(nr) * 3 * nr;
    const size_t red = (size_t)s.threads * s.dpt * 3 * nr;   // the reduction reuses the dipole buffer
    if (red > pz) pz = red;
    FFLayout L;
    L.tab = 0;                                                          // ez [nl][D], ey [nj][D], ex [8][D]
    L.eyx = ff_al16(L.tab + (size_t)(nl + nj + FF_PLANES) * s.D * f2);  // [nj][D] row factors of a plane
    L.P = ff_al16(L.eyx + (size_t)nj * s.D * f2);                       // [cap][nr][3]
    L.cc = ff_al16(L.P + pz * f2);                                      // CC: cy [nj], cz [nl], cx [8], weights
    L.idx = ff_al16(L.cc + (cc ? (size_t)(nj + nl + FF_PLANES) * f2 + (size_t)nr * nmat1 * sizeof(double) : 0));
    L.ints = ff_al16(L.idx + (size_t)ff_cap(nr) * sizeof(unsigned));    // count [nj], off [nj+1], mv, modes, misc
    L.occ = ff_al16(L.ints + (size_t)(2 * nj + 1 + (1 + nr) * nmat1 + 4) * sizeof(int));
    L.total = ff_al16(L.occ + (size_t)nj * nl);
    return L;
}

DDA_DEV void cp_async8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
DDA_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
DDA_DEV void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// grid (direction chunks of D, plane groups of s.planes, nrhs / NR); the lattice has
// nj, nl < 4096
template <bool CC, int NR, int DPT>
__global__ void __launch_bounds__(256) farfield_sum(PostArgs a, FFShape s)
{
    constexpr int CAP = ff_cap(NR);
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nj = a.nj, nl = a.nl, D = s.D, T = blockDim.x, nmat1 = a.nmat1;
    const int dbase = blockIdx.x * D, i0 = blockIdx.y * s.planes, rhs = NR * blockIdx.z;
    const int np = a.ni - i0 < s.planes ? a.ni - i0 : s.planes;
    const bool cc = CC && blockIdx.x == 0;
    const int dg = threadIdx.x % s.DG, w = threadIdx.x / s.DG;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = T >> 5;
    const FFLayout L = ff_layout(s, nj, nl, nmat1, CC, NR);
    float2 *ez = reinterpret_cast<float2 *>(smraw + L.tab);   // [nl][D]
    float2 *ey = ez + (size_t)nl * D;                          // [nj][D]
    float2 *ex = ey + (size_t)nj * D;                          // [FF_PLANES][D]
    float2 *eyx = reinterpret_cast<float2 *>(smraw + L.eyx);   // [nj][D]
    float2 *P = reinterpret_cast<float2 *>(smraw + L.P);       // [CAP][NR][3], later the reduction
    float2 *cy = reinterpret_cast<float2 *>(smraw + L.cc);     // CC: [nj], [nl], [FF_PLANES]
    float2 *cz = cy + nj, *cx = cz + nl;
    double *cwt = reinterpret_cast<double *>(cx + FF_PLANES);  // CC: [NR][nmat1]
    unsigned *idx = reinterpret_cast<unsigned *>(smraw + L.idx);   // [CAP] l | row << 12 | m << 24
    int *ln = reinterpret_cast<int *>(smraw + L.ints);         // [nj] active cells of each row
    int *off = ln + nj;                                        // [nj + 1] list position of each row
    int *mvs = off + nj + 1;                                   // [nmat1]
    int *ccm = mvs + nmat1;                                    // [NR][nmat1]
    int *misc = ccm + NR * nmat1;                              // [0]: some material in mode 2
    signed char *occs = reinterpret_cast<signed char *>(smraw + L.occ);   // [nj][nl] one plane

    const double cxf = (a.ni - 1) * a.d0 / 2, cyf = (nj - 1) * a.d0 / 2, czf = (nl - 1) * a.d0 / 2;
    const double *K = a.ksc + (size_t)rhs * a.ndir * 3;
    for (int e = threadIdx.x; e < (nl + nj + np) * D; e += T) {
        const int dl = e % D, pos = e / D, dd = dbase + dl;
        float2 val = czero();
        if (dd < a.ndir) {
            double ph;
            if (pos < nl) ph = K[3 * dd + 2] * (pos * a.d0 - czf);
            else if (pos < nl + nj) ph = K[3 * dd + 1] * ((pos - nl) * a.d0 - cyf);
            else ph = K[3 * dd + 0] * ((i0 + pos - nl - nj) * a.d0 - cxf);
            val = expi_reduced(ph);
        }
        ez[e] = val;   // ez, ey, ex are consecutive [pos][D] blocks
    }
    if (threadIdx.x == 0) misc[0] = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < nmat1; e += T) {
        const int mv = a.mv[e];
        mvs[e] = mv;
        if (CC) {
            // cross-section mode of a material: 0 no polarisability (skipped), 1 dipoles
            // staged, 2 a polarisability but switched off in the activity list (its dipoles
            // are read from global memory); weight Im(1 / conj(alpha))
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const float2 al = a.alpha[(size_t)(rhs + r) * nmat1 + e];
                const bool nz = !(al.x == 0.f && al.y == 0.f);
                const int mode = nz ? (mv ? 1 : 2) : 0;
                ccm[r * nmat1 + e] = mode;
                if (mode == 2) misc[0] = 1;
                const double ar = al.x, ai = al.y;
                cwt[r * nmat1 + e] = nz ? ai / (ar * ar + ai * ai) : 0.0;
            }
        }
    }
    // the incident direction is the pair's (both polarisations of one orientation)
    const double *ki = a.kinc + 3 * rhs;
    if (cc) {
        // CabsCext's phase -k.(r - c') with the centre c' = n d0 / 2 (dda_func.cpp:1685)
        const double ccx = a.ni * a.d0 / 2, ccy = nj * a.d0 / 2, ccz = nl * a.d0 / 2;
        for (int e = threadIdx.x; e < nj + nl + np; e += T) {
            const double ph = e < nj ? -ki[1] * (e * a.d0 - ccy)
                            : e < nj + nl ? -ki[2] * ((e - nj) * a.d0 - ccz)
                                          : -ki[0] * ((i0 + e - nj - nl) * a.d0 - ccx);
            cy[e] = expi_reduced(ph);   // cy, cz, cx are consecutive
        }
    }
    double Ec[NR][6];   // CC: conj(E_inc) of each right-hand side
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const double e = CC ? a.einc[6 * (rhs + r) + k] : 0.0;
            Ec[r][k] = (k & 1) ? -e : e;
        }
    __syncthreads();
    const bool slow_cc = cc && misc[0] != 0;

    const size_t N = a.N, plane = (size_t)nj * nl;
    const float2 *pr = a.p + (size_t)rhs * 3 * N;   // the NR right-hand sides follow each other
    const signed char *occr = a.occ + (size_t)rhs * a.occ_stride;
    const bool vec_occ = plane % 16 == 0 && (reinterpret_cast<size_t>(occr) & 15) == 0;
    float2 acc[NR][DPT][3];
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int u = 0; u < DPT; u++)
#pragma unroll
            for (int c = 0; c < 3; c++) acc[r][u][c] = czero();
    double v[NR][2];   // CC: Cext and Cabs sums
#pragma unroll
    for (int r = 0; r < NR; r++) v[r][0] = v[r][1] = 0.0;

#pragma unroll 1
    for (int ip = 0; ip < np; ip++) {
        const size_t q0 = (size_t)(i0 + ip) * plane;
        // ---- occupancy of the plane into shared memory
        if (vec_occ) {
            const int4 *src = reinterpret_cast<const int4 *>(occr + q0);
            int4 *dst = reinterpret_cast<int4 *>(occs);
            for (int e = threadIdx.x; e < (int)(plane / 16); e += T) dst[e] = src[e];
        } else {
            for (int e = threadIdx.x; e < (int)plane; e += T) occs[e] = occr[q0 + e];
        }
        // row factors exp(i (kx x + ky y)) of this plane
        for (int e = threadIdx.x; e < nj * D; e += T) eyx[e] = cmul(ey[e], ex[ip * D + e % D]);
        __syncthreads();
        // activity of a staged cell; nmat1 == 0: the activity list's length is not known
        // (allocation-free entry point), so it is read from global memory at the
        // occupancy's indices
        auto active = [&](int m) {
            return nmat1 ? ((unsigned)m < (unsigned)nmat1 && mvs[m] != 0) : (m >= 0 && a.mv[m] != 0);
        };
        // ---- active cells of every row (warp per row)
        for (int r = warp; r < nj; r += nwarps) {
            int cnt = 0;
            for (int c0 = 0; c0 < nl; c0 += 32) {
                const int l = c0 + lane;
                const bool act = l < nl && active(occs[r * nl + l]);
                cnt += __popc(__ballot_sync(0xffffffffu, act));
            }
            if (lane == 0) ln[r] = cnt;
        }
        __syncthreads();
        // ---- list positions of the rows (exclusive prefix sum, warp 0)
        if (warp == 0) {
            int carry = 0;
            for (int r0 = 0; r0 < nj; r0 += 32) {
                const int r = r0 + lane;
                const int x = r < nj ? ln[r] : 0;
                int inc = x;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += y;
                }
                if (r < nj) off[r] = carry + inc - x;
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
            if (lane == 0) off[nj] = carry;
        }
        __syncthreads();
        const int total = off[nj];
        // ---- chunks of the list
#pragma unroll 1
        for (int v0 = 0; v0 < total; v0 += CAP) {
            const int v1 = v0 + CAP < total ? v0 + CAP : total, len = v1 - v0;
            // copies: warp per row, the row's active cells that fall in [v0, v1), each at
            // its row's list position plus the active cells before it (ballot ranks)
            for (int r = warp; r < nj; r += nwarps) {
                const int o = off[r], n = ln[r];
                if (o + n <= v0 || o >= v1) continue;   // uniform over the warp
                int base = o;
                for (int c0 = 0; c0 < nl && base < v1; c0 += 32) {   // uniform over the warp
                    const int l = c0 + lane;
                    const int m = l < nl ? (int)occs[r * nl + l] : 0;
                    const bool act = l < nl && active(m);
                    const unsigned bal = __ballot_sync(0xffffffffu, act);
                    const int vv = base + __popc(bal & ((1u << lane) - 1u));
                    if (act && vv >= v0 && vv < v1) {
                        float2 *dst = P + 3 * NR * (size_t)(vv - v0);
#pragma unroll
                        for (int k = 0; k < NR; k++) {
                            const float2 *src = pr + (size_t)k * 3 * N + q0 + (size_t)r * nl + l;
                            cp_async8(dst + 3 * k, src);
                            cp_async8(dst + 3 * k + 1, src + N);
                            cp_async8(dst + 3 * k + 2, src + 2 * N);
                        }
                        idx[vv - v0] = (unsigned)l | ((unsigned)r << 12) | ((unsigned)(m & 0xff) << 24);
                    }
                    base += __popc(bal);
                }
            }
            cp_async_commit();
            cp_async_wait_all();
            __syncthreads();
            // far field: worker w's share of the chunk
            const int p0 = (int)(((long long)w * len) / s.RW), p1 = (int)(((long long)(w + 1) * len) / s.RW);
            if (p0 < p1) {
                float2 tt[NR][DPT][3];
#pragma unroll
                for (int r = 0; r < NR; r++)
#pragma unroll
                    for (int u = 0; u < DPT; u++)
#pragma unroll
                        for (int c = 0; c < 3; c++) tt[r][u][c] = czero();
                int cur = (int)((idx[p0] >> 12) & 0xfff);
#pragma unroll 2
                for (int p = p0; p < p1; p++) {
                    const unsigned id = idx[p];
                    const int row = (int)((id >> 12) & 0xfff), l = (int)(id & 0xfff);
                    if (row != cur) {
                        // row end: acc += exp(i (kx x + ky y)) t
                        float2 f[DPT];
                        ld_dirs<DPT>(eyx + (size_t)cur * D + DPT * dg, f);
#pragma unroll
                        for (int r = 0; r < NR; r++)
#pragma unroll
                            for (int u = 0; u < DPT; u++)
#pragma unroll
                                for (int c = 0; c < 3; c++) {
                                    acc[r][u][c] = cfma(f[u], tt[r][u][c], acc[r][u][c]);
                                    tt[r][u][c] = czero();
                                }
                        cur = row;
                    }
                    float2 ev[DPT];
                    ld_dirs<DPT>(ez + (size_t)l * D + DPT * dg, ev);
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        const float2 *pp = P + 3 * (NR * p + r);
                        const float2 pv[3] = {pp[0], pp[1], pp[2]};
#pragma unroll
                        for (int u = 0; u < DPT; u++)
#pragma unroll
                            for (int c = 0; c < 3; c++) tt[r][u][c] = cfma(ev[u], pv[c], tt[r][u][c]);
                    }
                }
                float2 f[DPT];
                ld_dirs<DPT>(eyx + (size_t)cur * D + DPT * dg, f);
#pragma unroll
                for (int r = 0; r < NR; r++)
#pragma unroll
                    for (int u = 0; u < DPT; u++)
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[r][u][c] = cfma(f[u], tt[r][u][c], acc[r][u][c]);
            }
            if (cc) {
                // CabsCext (dda_func.cpp:1688-1723) over the staged cells whose material has a
                // nonzero polarisability and is active (mode 1)
                for (int p = threadIdx.x; p < len; p += T) {
                    const unsigned id = idx[p];
                    const int m = (int)(id >> 24);
                    if (m >= nmat1) continue;
                    const int row = (int)((id >> 12) & 0xfff), l = (int)(id & 0xfff);
                    const float2 ph = cmul(cmul(cx[ip], cy[row]), cz[l]);
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        if (ccm[r * nmat1 + m] != 1) continue;
                        double per = 0.0, pei = 0.0, pp = 0.0;
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const float2 Pc = P[3 * (NR * p + r) + c];
                            const double er = Ec[r][2 * c], ei = Ec[r][2 * c + 1];   // conj(E)
                            per += Pc.x * er - Pc.y * ei;
                            pei += Pc.x * ei + Pc.y * er;
                            pp += (double)Pc.x * Pc.x + (double)Pc.y * Pc.y;
                        }
                        v[r][0] += (double)ph.x * pei + (double)ph.y * per;   // Im(ph * (P . conj E))
                        v[r][1] += pp * cwt[r * nmat1 + m] - (2.0 / 3.0) * pp;   // Im(pp / conj(alpha)) - 2/3 pp
                    }
                }
            }
            __syncthreads();   // the chunk buffers are refilled next
        }
        if (slow_cc) {
            // materials with a polarisability but switched off in the activity list: their
            // dipoles were not staged and are read from global memory
            for (int e = threadIdx.x; e < (int)plane; e += T) {
                const int m = occs[e];
                if ((unsigned)m >= (unsigned)nmat1) continue;
                const int row = e / nl, l = e - row * nl;
                const float2 ph = cmul(cmul(cx[ip], cy[row]), cz[l]);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    if (ccm[r * nmat1 + m] != 2) continue;
                    double per = 0.0, pei = 0.0, pp = 0.0;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const float2 Pc = pr[(size_t)r * 3 * N + c * N + q0 + e];
                        const double er = Ec[r][2 * c], ei = Ec[r][2 * c + 1];
                        per += Pc.x * er - Pc.y * ei;
                        pei += Pc.x * ei + Pc.y * er;
                        pp += (double)Pc.x * Pc.x + (double)Pc.y * Pc.y;
                    }
                    v[r][0] += (double)ph.x * pei + (double)ph.y * per;
                    v[r][1] += pp * cwt[r * nmat1 + m] - (2.0 / 3.0) * pp;
                }
            }
        }
        __syncthreads();   // the plane's occupancy and spans are replaced next
    }
    // the sum over workers in FP64
    float2 *red = P;   // [threads][NR][DPT][3]
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int u = 0; u < DPT; u++)
#pragma unroll
            for (int c = 0; c < 3; c++)
                red[(((size_t)threadIdx.x * NR + r) * DPT + u) * 3 + c] = acc[r][u][c];
    __syncthreads();
    for (int o = threadIdx.x; o < NR * D * 6; o += T) {
        const int r = o / (D * 6), dl = (o / 6) % D, k = o % 6, u = dl % DPT, g = dl / DPT, c = k >> 1;
        const int dd = dbase + dl;
        if (dd >= a.ndir) continue;
        double sum = 0.0;
        for (int q = 0; q < s.RW; q++) {
            const float2 x = red[(((size_t)(g + s.DG * q) * NR + r) * DPT + u) * 3 + c];
            sum += (k & 1) ? x.y : x.x;
        }
        if (sum != 0.0) atomicAdd(a.esc_acc + ((size_t)(rhs + r) * a.ndir + dd) * 6 + k, sum);
    }
    if (cc) {
#pragma unroll
        for (int r = 0; r < NR; r++) {
            __syncthreads();   // the reduction buffer is read above; block_sum_atomic reuses it
            block_sum_atomic<2>(v[r], reinterpret_cast<double *>(red), a.cc_acc + 2 * (rhs + r));
        }
    }
}

// Cext and Cabs sums (before the 4 pi / |E|^2 factor), grid (ni x parts, nrhs): CTA
// (i, part) sums the part-th of plane i's cells
__global__ void __launch_bounds__(256) cabs_cext_sum(PostArgs a, int parts)
{
    extern __shared__ float2 tab[];   // [nj] then [nl]
    __shared__ double scratch[8 * 2];
    const int i = blockIdx.x / parts, part = blockIdx.x - i * parts, rhs = blockIdx.y, nj = a.nj, nl = a.nl;
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
    const int e0 = (int)((long long)part * nj * nl / parts), e1 = (int)((long long)(part + 1) * nj * nl / parts);
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
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

// ---- Far field by kz groups
//
// The scattering planes of a fixed orientation turn about the incident direction, the
// lattice z axis (main.cpp:376-387 rotates each plane's directions about z), so the
// directions at one scattering angle share kz.  When a block's directions take few
// distinct kz, the z sum of the separable phase is done once per distinct value:
//   T_g(i, j) = sum_l exp(i kz_g (z_l - cz)) P(i, j, l)                        (ff_zsum)
//   S(k) = sum_{i,j} exp(i ky (y_j - cy)) exp(i kx (x_i - cx)) T_{g(k)}(i, j)  (ff_xysum)
// -- farfield_sum's sum (dda_func.cpp:1576-1625 by linearity) in another order, with the
// same phase arguments.  ff_zsum is a complex product (groups x z) . (z x rows) per
// plane: a thread holds 4 groups x 3 NR components of one row, the plane's dipoles go
// through shared memory masked by the activity list, 32 z at a time.
constexpr int ZG = 32;   // kz groups per CTA (8 warps x 4)
constexpr int ZR = 32;   // rows per row block (one per lane)
constexpr int ZL = 32;   // z positions per staged chunk

__host__ __device__ inline int kz_dirs_at(int G) { return 3 + G; }
__host__ __device__ inline int kz_items_at(int G, int ndir) { return 3 + G + ndir; }

__host__ __device__ inline size_t zsum_smem(int nl, int nr)
{
    return (size_t)nl * ZG * sizeof(float2) + (size_t)ZL * (3 * nr * ZR + 1) * sizeof(float2) + 256 * sizeof(int);
}

// grid (ni, group tiles of ZG, blocks), 256 threads
template <int NR>
__global__ void __launch_bounds__(256, 3) ff_zsum(PostArgs a)
{
    constexpr int Q = 3 * NR, ZS = Q * ZR + 1;   // ZS: z stride of the staged chunk (float2)
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nj = a.nj, nl = a.nl, G = a.kz_groups, nmat1 = a.nmat1;
    const int i = blockIdx.x, g0 = blockIdx.y * ZG, b = blockIdx.z, rhs = NR * b;
    const int *tab = a.kz_tab + (size_t)b * a.kz_stride;
    const int gb = tab[0];
    if (g0 >= gb) return;   // uniform over the block
    float2 *ez = reinterpret_cast<float2 *>(smraw);              // [nl][ZG]
    float2 *ps = ez + (size_t)nl * ZG;                           // [ZL][ZS]: [z][q][row]
    int *mvs = reinterpret_cast<int *>(ps + (size_t)ZL * ZS);    // [nmat1]
    const double czf = (nl - 1) * a.d0 / 2;
    const double *kz = a.kz_val + (size_t)b * G;
    for (int e = threadIdx.x; e < nl * ZG; e += blockDim.x) {
        const int l = e / ZG, g = g0 + e % ZG;
        ez[e] = g < gb ? expi_reduced(kz[g] * (l * a.d0 - czf)) : czero();
    }
    for (int e = threadIdx.x; e < nmat1; e += blockDim.x) mvs[e] = a.mv[e];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t N = a.N, q0 = (size_t)i * nj * nl;
    const float2 *pr = a.p + (size_t)rhs * 3 * N;
    const signed char *occr = a.occ + (size_t)rhs * a.occ_stride;
    const size_t gstride = (size_t)a.ni * nj * Q;
    float2 *out = a.kz_sum + (size_t)b * G * gstride + (size_t)i * nj * Q;
#pragma unroll 1
    for (int j0 = 0; j0 < nj; j0 += ZR) {
        float2 acc[4][Q];
#pragma unroll
        for (int g = 0; g < 4; g++)
#pragma unroll
            for (int q = 0; q < Q; q++) acc[g][q] = czero();
#pragma unroll 1
        for (int l0 = 0; l0 < nl; l0 += ZL) {
            __syncthreads();   // the tables are written / the previous chunk is consumed
            for (int e = threadIdx.x; e < ZL * ZR; e += blockDim.x) {
                const int l = e % ZL, r = e / ZL, j = j0 + r, ll = l0 + l;
                bool act = false;
                size_t cell = 0;
                if (j < nj && ll < nl) {
                    cell = q0 + (size_t)j * nl + ll;
                    const int m = occr[cell];
                    act = (unsigned)m < (unsigned)nmat1 && mvs[m] != 0;
                }
#pragma unroll
                for (int q = 0; q < Q; q++)
                    ps[l * ZS + q * ZR + r] = act ? pr[(size_t)(q / 3) * 3 * N + (size_t)(q % 3) * N + cell] : czero();
            }
            __syncthreads();
            const int lc = nl - l0 < ZL ? nl - l0 : ZL;
#pragma unroll 4
            for (int l = 0; l < lc; l++) {
                const float4 e01 = *reinterpret_cast<const float4 *>(ez + (size_t)(l0 + l) * ZG + 4 * warp);
                const float4 e23 = *reinterpret_cast<const float4 *>(ez + (size_t)(l0 + l) * ZG + 4 * warp + 2);
                const float2 ev[4] = {make_float2(e01.x, e01.y), make_float2(e01.z, e01.w),
                                      make_float2(e23.x, e23.y), make_float2(e23.z, e23.w)};
#pragma unroll
                for (int q = 0; q < Q; q++) {
                    const float2 pv = ps[l * ZS + q * ZR + lane];
#pragma unroll
                    for (int g = 0; g < 4; g++) acc[g][q] = cfma(ev[g], pv, acc[g][q]);
                }
            }
        }
        const int j = j0 + lane;
        if (j < nj) {
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const int gg = g0 + 4 * warp + g;
                if (gg < gb) {
#pragma unroll
                    for (int q = 0; q < Q; q++) out[gg * gstride + (size_t)j * Q + q] = acc[g][q];
                }
            }
        }
    }
}

__host__ __device__ inline size_t xysum_smem(int nj, int slice, int nr)
{
    return ((size_t)slice * nj * 3 * nr + (size_t)kKzItem * (slice + nj)) * sizeof(float2);
}

// grid (items, plane slices of a.kz_slice, blocks), 256 threads: an item's directions
// (one kz group), two per warp, over the group sums of the slice's planes
template <int NR>
__global__ void __launch_bounds__(256) ff_xysum(PostArgs a)
{
    constexpr int Q = 3 * NR;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nj = a.nj, G = a.kz_groups, b = blockIdx.z, rhs = NR * b, slice = a.kz_slice;
    const int *tab = a.kz_tab + (size_t)b * a.kz_stride;
    if ((int)blockIdx.x >= tab[1]) return;   // uniform over the block
    const int *dirs = tab + kz_dirs_at(G);
    const int *item = tab + kz_items_at(G, a.ndir) + 2 * blockIdx.x;
    const int g = item[0], s0 = item[1], send = tab[2 + g + 1];
    const int nd = send - s0 < kKzItem ? send - s0 : kKzItem;
    const int i0 = blockIdx.y * slice, np = a.ni - i0 < slice ? a.ni - i0 : slice;
    float2 *ts = reinterpret_cast<float2 *>(smraw);     // [np][nj][Q]
    float2 *ex = ts + (size_t)slice * nj * Q;           // [kKzItem][slice]
    float2 *ey = ex + (size_t)kKzItem * slice;          // [kKzItem][nj]
    const float2 *src = a.kz_sum + (((size_t)b * G + g) * a.ni + i0) * nj * Q;
    const int cnt = np * nj * Q;   // even: nj is
    for (int e = threadIdx.x; e < cnt / 2; e += blockDim.x)
        reinterpret_cast<float4 *>(ts)[e] = reinterpret_cast<const float4 *>(src)[e];
    if ((cnt & 1) && threadIdx.x == 0) ts[cnt - 1] = src[cnt - 1];
    const double cxf = (a.ni - 1) * a.d0 / 2, cyf = (nj - 1) * a.d0 / 2;
    const double *K = a.ksc + (size_t)rhs * a.ndir * 3;
    const int w = slice + nj;
    for (int e = threadIdx.x; e < kKzItem * w; e += blockDim.x) {
        const int d = e / w, pos = e - d * w;
        float2 v = czero();
        if (d < nd) {
            const int dd = dirs[s0 + d];
            if (pos < slice) {
                if (pos < np) v = expi_reduced(K[3 * dd + 0] * ((i0 + pos) * a.d0 - cxf));
            } else {
                v = expi_reduced(K[3 * dd + 1] * ((pos - slice) * a.d0 - cyf));
            }
        }
        if (pos < slice) ex[d * slice + pos] = v;
        else ey[d * nj + pos - slice] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, d0 = 2 * warp;
    if (d0 >= nd) return;   // uniform over the warp; no barrier follows
    float2 acc[2][Q];
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
        for (int q = 0; q < Q; q++) acc[u][q] = czero();
    for (int e = lane; e < np * nj; e += 32) {
        const int ii = e / nj, j = e - ii * nj;
        float2 tv[Q];
#pragma unroll
        for (int q = 0; q < Q; q++) tv[q] = ts[(size_t)e * Q + q];
        const float2 f0 = cmul(ey[d0 * nj + j], ex[d0 * slice + ii]);
        const float2 f1 = cmul(ey[(d0 + 1) * nj + j], ex[(d0 + 1) * slice + ii]);
#pragma unroll
        for (int q = 0; q < Q; q++) {
            acc[0][q] = cfma(f0, tv[q], acc[0][q]);
            acc[1][q] = cfma(f1, tv[q], acc[1][q]);
        }
    }
    // the warp's sum in FP64, added by lane 0
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const bool have = d0 + u < nd;
        const int dd = have ? dirs[s0 + d0 + u] : 0;
#pragma unroll
        for (int q = 0; q < Q; q++)
#pragma unroll
            for (int part = 0; part < 2; part++) {
                double v = part ? acc[u][q].y : acc[u][q].x;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0 && have && v != 0.0)
                    atomicAdd(a.esc_acc + ((size_t)(rhs + q / 3) * a.ndir + dd) * 6 + 2 * (q % 3) + part, v);
            }
    }
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
// The two polarisations of orientation o are right-hand sides 2o and 2o+1.  Block of
// MU_T threads: ppb (orientation, angle) pairs, a thread per (pair, plane) -- planes
// pl, pl + npl, ... when there are more than MU_T -- then the planes' matrices are summed
// in plane order (the order of the single-thread loop, so the same bits).
constexpr int MU_T = 128;
__global__ void __launch_bounds__(MU_T) mueller_avg(MuellerArgs m, int npl, int ppb)
{
    __shared__ double part[MU_T][17];
    const int t = threadIdx.x, pr = t / npl, pl0 = t - pr * npl;
    const int q = blockIdx.x * ppb + pr;
    double M[16];
    for (int k = 0; k < 16; k++) M[k] = 0.0;
    if (pr < ppb && q < m.norient * m.nangles) {
        const int o = q / m.nangles, ang = q % m.nangles;
        const double *ki = m.kinc + 6 * o;      // rhs 2o
        dc E0[3], E1[3];
        for (int c = 0; c < 3; c++) {
            E0[c] = {m.einc[12 * o + 2 * c], m.einc[12 * o + 2 * c + 1]};
            E1[c] = {m.einc[12 * o + 6 + 2 * c], m.einc[12 * o + 6 + 2 * c + 1]};
        }
        for (int pl = pl0; pl < m.nplanes; pl += npl) {
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
    }
    for (int k = 0; k < 16; k++) part[t][k] = M[k];
    __syncthreads();
    for (int e = t; e < ppb * 16; e += MU_T) {
        const int p = e >> 4, k = e & 15, qq = blockIdx.x * ppb + p;
        if (qq >= m.norient * m.nangles) continue;
        double v = 0.0;
        for (int u = 0; u < npl; u++) v += part[p * npl + u][k];
        m.out[(size_t)qq * 16 + k] = v / m.nplanes;
    }
}

inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

size_t farfield_smem(int nj, int nl)
{
    // the largest shape any direction count gives on this lattice, cross sections fused,
    // every material slot in use
    size_t m = 0;
    for (int nd = FF_DQ; nd <= FF_DMAX; nd += FF_DQ) {
        const size_t b1 = ff_layout(ff_shape(nd, 4), nj, nl, kMaxMaterials + 1, true, 1).total;
        const size_t b2 = ff_layout(ff_shape(nd, 2), nj, nl, kMaxMaterials + 1, true, 2).total;
        m = b1 > m ? b1 : m;
        m = b2 > m ? b2 : m;
    }
    return m;
}

cudaError_t post_prepare(int nj, int nl)
{
    // raised only: a context or call on a smaller lattice keeps what a larger one needs
    const int bytes = (int)farfield_smem(nj, nl);
    cudaError_t e = raise_smem_limit((const void *)farfield_sum<true, 1, 4>, bytes);
    if (e == cudaSuccess) e = raise_smem_limit((const void *)farfield_sum<true, 2, 2>, bytes);
    if (e == cudaSuccess) e = raise_smem_limit((const void *)farfield_sum<false, 1, 4>, bytes);
    if (e == cudaSuccess) e = raise_smem_limit((const void *)ff_zsum<1>, (int)zsum_smem(nl, 1));
    if (e == cudaSuccess) e = raise_smem_limit((const void *)ff_zsum<2>, (int)zsum_smem(nl, 2));
    // three group-sum CTAs per SM want the largest shared-memory carveout
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute((const void *)ff_zsum<1>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute((const void *)ff_zsum<2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return e;
}

// plane slice of ff_xysum: about 32 KB of group sums, 64 planes at most
static int kz_slice_for(int ni, int nj, int nr)
{
    int sl = 32768 / (nj * 3 * nr * (int)sizeof(float2));
    if (sl < 1) sl = 1;
    if (sl > 64) sl = 64;
    return sl < ni ? sl : ni;
}

void plan_kz_groups(const double *ks, int nrhs, int ndir, bool pairs, int ni, int nj, int nl,
                    double nact, int mode, KzPlan &P)
{
    P.groups = 0;
    P.tab.clear();
    P.kz.clear();
    if (mode == 1 || ndir <= 0 || nrhs <= 0 || !ks) return;
    const int NR = pairs && nrhs % 2 == 0 ? 2 : 1, nb = nrhs / NR;
    // a direction that is not finite keeps the direct form (and the sort its strict order)
    for (size_t q = 0; q < (size_t)nrhs * ndir * 3; q++)
        if (!std::isfinite(ks[q])) return;
    // per block: direction indices sorted by kz (ties in index order), groups of equal kz
    std::vector<std::vector<int>> order((size_t)nb);
    std::vector<std::vector<int>> offs((size_t)nb);
    int G = 0, items = 0;
    for (int b = 0; b < nb; b++) {
        const double *K = ks + (size_t)b * NR * ndir * 3;
        std::vector<int> &o = order[(size_t)b];
        o.resize((size_t)ndir);
        for (int d = 0; d < ndir; d++) o[(size_t)d] = d;
        std::stable_sort(o.begin(), o.end(), [&](int x, int y) { return K[3 * x + 2] < K[3 * y + 2]; });
        std::vector<int> &f = offs[(size_t)b];
        int it = 0;
        for (int d = 0; d < ndir; d++)
            if (d == 0 || K[3 * o[(size_t)d] + 2] != K[3 * o[(size_t)d - 1] + 2]) f.push_back(d);
        f.push_back(ndir);
        const int gb = (int)f.size() - 1;
        for (int g = 0; g < gb; g++) it += (f[(size_t)g + 1] - f[(size_t)g] + kKzItem - 1) / kKzItem;
        G = std::max(G, gb);
        items = std::max(items, it);
    }
    const double plane = (double)nj * nl, cells = (double)ni * plane;
    const size_t elems = (size_t)nb * G * ni * nj * 3 * NR;
    if (elems * sizeof(float2) > ((size_t)1 << 30)) return;   // group sums above 1 GiB: direct
    if (zsum_smem(nl, NR) > 200 * 1024 || xysum_smem(nj, kz_slice_for(ni, nj, NR), NR) > 48 * 1024) return;
    // work: a complex multiply-add per (group, cell) and per (direction, row) against one
    // per (direction, active cell)
    if (mode == 0 && 2.0 * (G * cells + 2.0 * ndir * ni * nj) > (double)ndir * nact) return;
    P.groups = G;
    P.items = items;
    P.blocks = nb;
    P.slice = kz_slice_for(ni, nj, NR);
    P.stride = kz_items_at(G, ndir) + 2 * items;
    P.sum_elems = elems;
    P.tab.assign((size_t)nb * P.stride, 0);
    P.kz.assign((size_t)nb * G, 0.0);
    for (int b = 0; b < nb; b++) {
        const double *K = ks + (size_t)b * NR * ndir * 3;
        int *t = P.tab.data() + (size_t)b * P.stride;
        const std::vector<int> &o = order[(size_t)b], &f = offs[(size_t)b];
        const int gb = (int)f.size() - 1;
        t[0] = gb;
        for (int g = 0; g <= G; g++) t[2 + g] = g <= gb ? f[(size_t)g] : ndir;
        for (int d = 0; d < ndir; d++) t[kz_dirs_at(G) + d] = o[(size_t)d];
        int it = 0;
        for (int g = 0; g < gb; g++) {
            P.kz[(size_t)b * G + g] = K[3 * o[(size_t)f[(size_t)g]] + 2];
            for (int s0 = f[(size_t)g]; s0 < f[(size_t)g + 1]; s0 += kKzItem, it++) {
                t[kz_items_at(G, ndir) + 2 * it] = g;
                t[kz_items_at(G, ndir) + 2 * it + 1] = s0;
            }
        }
        t[1] = it;
    }
}

// parts of a plane per cross-section CTA: about four CTAs per SM, 256 cells per CTA at least
static int cc_parts(const PostArgs &a)
{
    int parts = 1;
    while (parts < 16 && (long long)a.ni * a.nrhs * parts < 4 * 148 && (long long)a.nj * a.nl / (2 * parts) >= 256)
        parts *= 2;
    return parts;
}

cudaError_t launch_post(const PostArgs &a, float2 *esc, float *cabs, float *cext, cudaStream_t st, int *kernels)
{
    cudaError_t e;
    int nk = 1;
    if ((e = cudaMemsetAsync(a.esc_acc, 0, (size_t)a.nrhs * a.ndir * 6 * sizeof(double), st))) return e;
    if ((e = cudaMemsetAsync(a.cc_acc, 0, (size_t)a.nrhs * 2 * sizeof(double), st))) return e;
    if (a.ndir > 0 && a.kz_groups > 0) {
        // far field by kz groups, then the cross sections
        const int NR = a.pairs && a.nrhs % 2 == 0 ? 2 : 1, nb = a.nrhs / NR;
        const dim3 gz(a.ni, nblk(a.kz_groups, ZG), nb), gx(a.kz_items, nblk(a.ni, a.kz_slice), nb);
        if (NR == 2) {
            ff_zsum<2><<<gz, 256, zsum_smem(a.nl, 2), st>>>(a);
            ff_xysum<2><<<gx, 256, xysum_smem(a.nj, a.kz_slice, 2), st>>>(a);
        } else {
            ff_zsum<1><<<gz, 256, zsum_smem(a.nl, 1), st>>>(a);
            ff_xysum<1><<<gx, 256, xysum_smem(a.nj, a.kz_slice, 1), st>>>(a);
        }
        const int parts = cc_parts(a);
        cabs_cext_sum<<<dim3(a.ni * parts, a.nrhs), 256, (a.nj + a.nl) * sizeof(float2), st>>>(a, parts);
        nk += 3;
    } else if (a.ndir > 0) {
        // far field with the cross sections summed by the first direction chunk
        if (a.nj >= 4096 || a.nl >= 4096) return cudaErrorInvalidValue;   // packed list words
        if (a.pairs && a.nrhs % 2 == 0) {
            const FFShape s = ff_shape(a.ndir, 2, a.ni, a.nrhs / 2);
            farfield_sum<true, 2, 2><<<dim3(nblk(a.ndir, s.D), nblk(a.ni, s.planes), a.nrhs / 2), s.threads,
                                       ff_layout(s, a.nj, a.nl, a.nmat1, true, 2).total, st>>>(a, s);
        } else {
            const FFShape s = ff_shape(a.ndir, 4, a.ni, a.nrhs);
            farfield_sum<true, 1, 4><<<dim3(nblk(a.ndir, s.D), nblk(a.ni, s.planes), a.nrhs), s.threads,
                                       ff_layout(s, a.nj, a.nl, a.nmat1, true, 1).total, st>>>(a, s);
        }
        nk += 1;
    } else {
        const int parts = cc_parts(a);
        cabs_cext_sum<<<dim3(a.ni * parts, a.nrhs), 256, (a.nj + a.nl) * sizeof(float2), st>>>(a, parts);
        nk += 1;
    }
    const size_t nd = (size_t)a.nrhs * a.ndir;
    const size_t nt = nd > (size_t)a.nrhs ? nd : (size_t)a.nrhs;
    post_finalize<<<nblk(nt, 256), 256, 0, st>>>(a, esc, cabs, cext);
    if (kernels) *kernels = nk;
    return cudaGetLastError();
}

cudaError_t launch_mueller(const MuellerArgs &m, cudaStream_t st)
{
    const size_t n = (size_t)m.norient * m.nangles;
    if (n == 0) return cudaSuccess;
    const int npl = m.nplanes < MU_T ? m.nplanes : MU_T, ppb = MU_T / npl;
    mueller_avg<<<nblk(n, ppb), MU_T, 0, st>>>(m, npl, ppb);
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
    if (a.nj >= 4096 || a.nl >= 4096) return cudaErrorInvalidValue;   // packed list words
    const FFShape s = ff_shape(a.ndir, 4, a.ni, 1);
    farfield_sum<false, 1, 4><<<dim3(nblk(a.ndir, s.D), nblk(a.ni, s.planes), 1), s.threads,
                                ff_layout(s, a.nj, a.nl, a.nmat1, false, 1).total, st>>>(a, s);
    post_finalize<<<nblk((size_t)a.ndir, 256), 256, 0, st>>>(a, esc_dev, nullptr, nullptr);
    return cudaGetLastError();
}

}  // namespace ddagpu
