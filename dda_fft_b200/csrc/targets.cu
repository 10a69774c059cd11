// Random targets of libddagpu: placement on the host from the reference's random stream,
// rasterisation into the lattice on the GPU.
//
// Agglomerates of capsule monomers (the anthrax-like target, iGenerateAnthrax,
// particle.cpp:21-85).
// Placement consumes the reference's random stream (xorshift64*, randomize.cpp:44-58) and
// accepts or rejects monomers with the reference's float geometry (worm,
// particle.cpp:302-344; CrossTwoWorms, 233-300; PointToWorm, 379-400), so it is written
// with the same float operations in the same order: a realisation drawn here is the
// reference's realisation.  Rasterisation -- every cell inside the sphere of radius n/2
// tested against every monomer (SeedToWorm, particle.cpp:346-377) -- is the O(cells x
// monomers) part (about a minute per sample at 128^3 on one core); it runs one thread per
// cell with the monomers staged through shared memory, in explicitly rounded float
// arithmetic (no fused multiply-add) so that boundary cells fall on the same side as in the
// reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "targets.h"

namespace ddagpu {

namespace {

struct V3 {
    float x, y, z;
};

// host float vector algebra of cvector.cpp (left-to-right evaluation, no contraction)
inline V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 vscale(float r, V3 a) { return {r * a.x, r * a.y, r * a.z}; }
inline float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 vcross(V3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float vabs(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

struct Worm {
    float r, l;
    V3 b, e, n;
};

int rng_draw(unsigned long long &s)
{
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return (int)((s * 2685821657736338717ULL) >> 33);
}

const double kPi = 3.1415926535897932384626433832795;   // PI of complex.hpp
const float kRandMax = 2147483647.f;

// worm(), particle.cpp:302-344
Worm make_worm(float r1, float th1, float ph1, float r2, float th2, float ph2, float length,
               float radius, float R2)
{
    const float ct1 = std::cos(th1), st1 = std::sin(th1), cp1 = std::cos(ph1), sp1 = std::sin(ph1);
    V3 begin = {r1, ph1, th1}, end = {r2, ph2, th2};
    const V3 dir0 = vsub(end, begin);
    Worm w;
    w.r = -1.f;
    begin.x = r1 * st1 * cp1;
    begin.y = r1 * st1 * sp1;
    begin.z = r1 * ct1;
    if (vdot(begin, begin) > R2) return w;
    V3 v0;
    v0.x = st1 * cp1 * dir0.x - sp1 * dir0.y + ct1 * cp1 * dir0.z;
    v0.y = st1 * sp1 * dir0.x + cp1 * dir0.y + ct1 * sp1 * dir0.z;
    v0.z = ct1 * dir0.x - st1 * dir0.z;
    const float inv = (float)(1. / (double)vabs(v0));
    const V3 dir = vscale(inv, v0);
    end = vadd(begin, vscale(length, dir));
    if (vdot(end, end) > R2) return w;
    w.r = radius;
    w.l = length;
    w.b = begin;
    w.e = end;
    w.n = dir;
    return w;
}

// PointToWorm, particle.cpp:379-400
int point_to_worm(const Worm &w, V3 p, float radius)
{
    const float t = vdot(vsub(p, w.b), w.n), max_d = w.r + radius;
    float d = vabs(vadd(vsub(w.b, p), vscale(t, w.n)));
    if (d > max_d) return 0;
    if (t >= 0.f && t <= w.l) return 1;
    if (t < 0) {
        d = vabs(vsub(w.b, p));
        return d > max_d ? 0 : 1;
    }
    d = vabs(vsub(w.e, p));
    return d > max_d ? 0 : 1;
}

// CrossTwoWorms, particle.cpp:233-300, up to its first decision that needs no point test:
// 1 / 0 for the parallel-axes rule, the line-distance exit and the "nearest points inside
// both segments" rule (its 2x2 system, signs included); -1 otherwise, with the two line
// parameters in r0_out / r1_out.
int cross_head(const Worm &a, const Worm &b, float &r0_out, float &r1_out)
{
    const V3 v0 = vcross(a.n, b.n);
    float r0 = vabs(v0);
    if (r0 <= 1.e-20) return 1;
    const V3 v1 = vsub(b.b, a.b);
    const float d = std::fabs(vdot(v1, v0) / r0);
    float r2 = a.r + b.r;
    if (d > r2) return 0;
    const float b1 = vdot(v1, a.n), b2 = vdot(v1, b.n);
    const float a11 = 1.f, a12 = vdot(b.n, a.n), a21 = -a12, a22 = -a11;
    r2 = a11 * a22 - a12 * a21;
    r0 = (b1 * a22 - b2 * a12) / r2;
    const float r1 = (b2 * a11 - b1 * a21) / r2;
    if (r0 >= 0.f && r0 <= a.l && r1 >= 0.f && r1 <= b.l) return 1;
    r0_out = r0;
    r1_out = r1;
    return -1;
}

// CrossTwoWorms, particle.cpp:233-300 (including its reuse of the nearest point)
int cross_two_worms(const Worm &a, const Worm &b)
{
    float r0 = 0.f, r1 = 0.f;
    const int h = cross_head(a, b, r0, r1);
    if (h >= 0) return h;
    V3 near = {0.f, 0.f, 0.f};
    int i0 = 0, i1 = 0;
    if (r0 >= 0.f && r0 <= a.l) {
        near = vadd(a.b, vscale(r0, a.n));
        i0 = 1;
    }
    if (r1 >= 0.f && r1 <= b.l) {
        near = vadd(b.b, vscale(r1, b.n));
        i1 = 1;
    }
    if (point_to_worm(a, b.b, b.r) == 1) return 1;
    if (point_to_worm(a, b.e, b.r) == 1) return 1;
    if (point_to_worm(b, a.b, a.r) == 1) return 1;
    if (point_to_worm(b, a.e, a.r) == 1) return 1;
    if (i0 == 1 && point_to_worm(b, near, a.r) == 1) return 1;
    if (i1 == 1 && point_to_worm(a, near, b.r) == 1) return 1;
    return 0;
}

// ---- device rasterisation (SeedToWorm, particle.cpp:346-377)
struct DW {
    float r, l, bx, by, bz, ex, ey, ez, nx, ny, nz;
};

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz)
{
    return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

__device__ bool seed_to_worm(const DW &w, float px, float py, float pz)
{
    const float t = dot3(fs(px, w.bx), fs(py, w.by), fs(pz, w.bz), w.nx, w.ny, w.nz);
    const float rr = fm(w.r, w.r);
    if (t >= 0.f && t <= w.l) {
        const float vx = fa(fs(w.bx, px), fm(w.nx, t)), vy = fa(fs(w.by, py), fm(w.ny, t)),
                    vz = fa(fs(w.bz, pz), fm(w.nz, t));
        return dot3(vx, vy, vz, vx, vy, vz) <= rr;
    }
    if (t > -w.r && t < 0.f) {
        const float vx = fs(w.bx, px), vy = fs(w.by, py), vz = fs(w.bz, pz);
        return dot3(vx, vy, vz, vx, vy, vz) <= rr;
    }
    if (t > w.l && t < fa(w.l, w.r)) {
        const float vx = fs(w.ex, px), vy = fs(w.ey, py), vz = fs(w.ez, pz);
        return dot3(vx, vy, vz, vx, vy, vz) <= rr;
    }
    return false;
}

constexpr int kChunk = 256;
constexpr int kTile = 8;   // rasterisation tile: 8 x 8 x 8 cells per CTA, two cells per thread

// One CTA per lattice tile.  The monomers pass through shared memory in chunks; a monomer
// is tested against the tile's cells only if its box, widened by its radius and one cell,
// meets the tile's box (SeedToWorm can only accept points within the radius of the axis
// segment, so the skipped tests are all rejections).  A cell is filled if any monomer
// accepts it, as in the reference's loop (particle.cpp:65-80), so the test order is free.
__global__ void __launch_bounds__(256) rasterize(const DW *worms, int count, int ni, int nj, int nl,
                                                 float cx, float cy, float cz, float R2,
                                                 signed char *occ, int *ndip)
{
    __shared__ DW sw[kChunk];
    __shared__ short surv[kChunk];
    __shared__ int nsurv, block_hits;
    const int tiles_l = (nl + kTile - 1) / kTile, tiles_j = (nj + kTile - 1) / kTile;
    const int t = blockIdx.x;
    const int i0 = (t / (tiles_l * tiles_j)) * kTile, j0 = ((t / tiles_l) % tiles_j) * kTile,
              l0 = (t % tiles_l) * kTile;
    if (threadIdx.x == 0) block_hits = 0;
    // this thread's cells: tile-local indices threadIdx.x and threadIdx.x + 256
    float px[2], py[2], pz[2];
    bool valid[2], inside[2], hit[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int e = threadIdx.x + 256 * u;
        const int i = i0 + e / (kTile * kTile), j = j0 + (e / kTile) % kTile, l = l0 + e % kTile;
        valid[u] = i < ni && j < nj && l < nl;
        px[u] = fs((float)i, cx);
        py[u] = fs((float)j, cy);
        pz[u] = fs((float)l, cz);
        inside[u] = valid[u] && fa(fa(fm(px[u], px[u]), fm(py[u], py[u])), fm(pz[u], pz[u])) <= R2;
        hit[u] = false;
    }
    // the tile's box in point coordinates
    const float xlo = fs((float)i0, cx), ylo = fs((float)j0, cy), zlo = fs((float)l0, cz);
    const float xhi = fs((float)min(i0 + kTile - 1, ni - 1), cx), yhi = fs((float)min(j0 + kTile - 1, nj - 1), cy),
                zhi = fs((float)min(l0 + kTile - 1, nl - 1), cz);
    for (int c0 = 0; c0 < count; c0 += kChunk) {
        __syncthreads();
        if (threadIdx.x == 0) nsurv = 0;
        const int m = count - c0 < kChunk ? count - c0 : kChunk;
        for (int k = threadIdx.x; k < m; k += blockDim.x) sw[k] = worms[c0 + k];
        __syncthreads();
        if (threadIdx.x < m) {
            const DW &w = sw[threadIdx.x];
            const float g = w.r + 1.f;
            const bool meet = fminf(w.bx, w.ex) - g <= xhi && fmaxf(w.bx, w.ex) + g >= xlo &&
                              fminf(w.by, w.ey) - g <= yhi && fmaxf(w.by, w.ey) + g >= ylo &&
                              fminf(w.bz, w.ez) - g <= zhi && fmaxf(w.bz, w.ez) + g >= zlo;
            if (meet) surv[atomicAdd(&nsurv, 1)] = (short)threadIdx.x;
        }
        __syncthreads();
        const int ns = nsurv;
#pragma unroll
        for (int u = 0; u < 2; u++)
            if (inside[u] && !hit[u])
                for (int s = 0; s < ns; s++)
                    if (seed_to_worm(sw[surv[s]], px[u], py[u], pz[u])) {
                        hit[u] = true;
                        break;
                    }
    }
    int mine = 0;
#pragma unroll
    for (int u = 0; u < 2; u++) {
        if (!valid[u]) continue;
        const int e = threadIdx.x + 256 * u;
        const int i = i0 + e / (kTile * kTile), j = j0 + (e / kTile) % kTile, l = l0 + e % kTile;
        occ[((size_t)i * nj + j) * nl + l] = hit[u] ? 1 : 0;
        mine += hit[u] ? 1 : 0;
    }
    if (mine) atomicAdd(&block_hits, mine);
    __syncthreads();
    if (threadIdx.x == 0 && block_hits) atomicAdd(ndip, block_hits);
}

// ---- random (Voronoi) ellipsoid, iGenerateRandomEllipsoid, particle.cpp:531-614
struct EllGeom {
    float cx, cy, cz;      // centre n / 2 - 0.5 per axis
    float a2, b2, c2;      // squared semi-axes
};

EllGeom ellipsoid_geom(int ni, int nj, int nl, float b_a, float c_a)
{
    EllGeom g;
    g.cx = (float)((double)(float)ni / 2. - .5);
    g.cy = (float)((double)(float)nj / 2. - .5);
    g.cz = (float)((double)(float)nl / 2. - .5);
    float a = (float)ni, b = a * b_a, c = a * c_a;
    a = (float)((double)a / 2.);
    b = (float)((double)b / 2.);
    c = (float)((double)c / 2.);
    g.a2 = a * a;
    g.b2 = b * b;
    g.c2 = c * c;
    return g;
}

// rounding(), complex.cpp:213-223, for the non-negative arguments used here
int rounding_pos(float r0)
{
    double ip;
    const double fr = std::modf((double)r0, &ip);
    return fr > 0.5 ? (int)ip + 1 : (int)ip;
}

__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

constexpr int kSeedChunk = 512;

__global__ void __launch_bounds__(256) voronoi_fill(const float *seeds, int nseeds, const int *sort_end,
                                                    int nsorts, int ni, int nj, int nl, EllGeom g,
                                                    float dist0, signed char *occ, int *ndip)
{
    __shared__ float s[3 * kSeedChunk];
    __shared__ int block_hits;
    const size_t N = (size_t)ni * nj * nl;
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (threadIdx.x == 0) block_hits = 0;
    float px = 0.f, py = 0.f, pz = 0.f;
    bool inside = false;
    if (q < N) {
        const int l = (int)(q % nl), j = (int)((q / nl) % nj), i = (int)(q / ((size_t)nl * nj));
        px = (float)i;
        py = (float)j;
        pz = (float)l;
        const float vx = fs(px, g.cx), vy = fs(py, g.cy), vz = fs(pz, g.cz);
        inside = fa(fa(fd(fm(vx, vx), g.a2), fd(fm(vy, vy), g.b2)), fd(fm(vz, vz), g.c2)) <= 1.f;
    }
    int best = 0;
    float dmin = dist0;
    for (int c0 = 0; c0 < nseeds; c0 += kSeedChunk) {
        __syncthreads();
        const int m = nseeds - c0 < kSeedChunk ? nseeds - c0 : kSeedChunk;
        for (int k = threadIdx.x; k < 3 * m; k += blockDim.x) s[k] = seeds[3 * (size_t)c0 + k];
        __syncthreads();
        if (inside)
            for (int k = 0; k < m; k++) {
                const float dx = fs(px, s[3 * k]), dy = fs(py, s[3 * k + 1]), dz = fs(pz, s[3 * k + 2]);
                const float dist = __fsqrt_rn(dot3(dx, dy, dz, dx, dy, dz));
                if (dist < dmin) {
                    best = c0 + k;
                    dmin = dist;
                }
            }
    }
    int mat = 0;
    if (inside) {
        // material m + 1 for seeds [sort_end[m-1], sort_end[m]) (first seed range: material 1)
        for (int m = 0; m < nsorts; m++)
            if (best < sort_end[m]) {
                mat = m + 1;
                break;
            }
    }
    if (q < N) occ[q] = (signed char)mat;
    if (mat == 1) atomicAdd(&block_hits, 1);   // the reference counts material-1 cells only
    __syncthreads();
    if (threadIdx.x == 0 && block_hits) atomicAdd(ndip, block_hits);
}

}  // namespace

int random_ellipsoid_seeds(unsigned long long *state, int ni, int nj, int nl, float b_a, float c_a,
                           int nseeds, float *seeds3)
{
    // iGenerateRandomEllipsoid, particle.cpp:538-573 (fits check, then seed draws)
    const float a = (float)ni, b = a * b_a, c = a * c_a;
    if (b > (float)nj || c > (float)nl) return -1;
    const EllGeom g = ellipsoid_geom(ni, nj, nl, b_a, c_a);
    unsigned long long s = *state;
    for (int m = 0; m < nseeds; m++) {
        V3 v0, v1;
        int dup;
        do {
            dup = 0;
            // (real)rand / (real)RAND_MAX in float, times ((real)n - 1.) in double, to float
            v0.x = (float)rounding_pos((float)((double)((float)rng_draw(s) / kRandMax) * ((double)(float)ni - 1.)));
            v0.y = (float)rounding_pos((float)((double)((float)rng_draw(s) / kRandMax) * ((double)(float)nj - 1.)));
            v0.z = (float)rounding_pos((float)((double)((float)rng_draw(s) / kRandMax) * ((double)(float)nl - 1.)));
            for (int i = 0; i < m; i++) {
                const V3 d = vsub({seeds3[3 * i], seeds3[3 * i + 1], seeds3[3 * i + 2]}, v0);
                if ((double)vabs(d) < 0.0000000001) {
                    dup = 1;
                    break;
                }
            }
            v1 = vsub(v0, {g.cx, g.cy, g.cz});
        } while (((v1.x * v1.x) / g.a2 + (v1.y * v1.y) / g.b2 + (v1.z * v1.z) / g.c2 > 1.f) && dup == 1);
        seeds3[3 * m] = v0.x;
        seeds3[3 * m + 1] = v0.y;
        seeds3[3 * m + 2] = v0.z;
    }
    *state = s;
    return 0;
}

cudaError_t random_ellipsoid_fill(const float *seeds3, const int *counts, int nsorts, int ni, int nj,
                                  int nl, float b_a, float c_a, signed char *occ_dev, int *ndip_dev,
                                  cudaStream_t st)
{
    // iGenerateRandomEllipsoid, particle.cpp:575-610: nearest seed (first on ties) inside
    int nseeds = 0;
    std::vector<int> ends((size_t)nsorts);
    for (int m = 0; m < nsorts; m++) ends[(size_t)m] = (nseeds += counts[m]);
    const EllGeom g = ellipsoid_geom(ni, nj, nl, b_a, c_a);
    const float dist0 = std::sqrt((float)(ni * ni + nj * nj + nl * nl));
    float *ds = nullptr;
    int *de = nullptr;
    cudaError_t e = cudaMallocAsync(&ds, (size_t)3 * (nseeds ? nseeds : 1) * sizeof(float), st);
    if (!e) e = cudaMallocAsync(&de, (size_t)(nsorts ? nsorts : 1) * sizeof(int), st);
    if (!e && nseeds) e = cudaMemcpyAsync(ds, seeds3, (size_t)3 * nseeds * sizeof(float), cudaMemcpyHostToDevice, st);
    if (!e && nsorts) e = cudaMemcpyAsync(de, ends.data(), nsorts * sizeof(int), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(ndip_dev, 0, sizeof(int), st);
    if (!e) {
        const size_t N = (size_t)ni * nj * nl;
        voronoi_fill<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(ds, nseeds, de, nsorts, ni, nj, nl, g,
                                                                 dist0, occ_dev, ndip_dev);
        e = cudaGetLastError();
    }
    if (ds) cudaFreeAsync(ds, st);
    if (de) cudaFreeAsync(de, st);
    return e;
}

long long anthrax_count(int ni, int nj, int nl, float packing, float radius, float ratio)
{
    // iWormsNumber, main.cpp:585
    const double v = (double)(packing * (float)(ni * nj * nl)) /
                     (8. * (double)(radius * radius * radius) * (0.75 * (double)ratio + 1));
    return (long long)v + 1;
}

// CrossTwoWorms (particle.cpp:233-300) of a candidate c against n placed monomers, up to its
// point tests, as one branch-free loop over distinct arrays that the compiler vectorises:
// flag 1 -- crossing (parallel axes, or the "nearest points inside both segments" rule
// with the reference's signs), 0 -- no crossing (line distance beyond r_a + r_b, or the
// point tests cannot accept: the segments lie farther apart than r_a + r_b + 1 cell, so
// each point test measures a distance beyond its threshold by more than a cell), 2 -- the
// point tests decide.  Every lane performs cross_head's float operations in its order
// (correctly rounded vector square root and division, no contraction), so the flags are
// those of the scalar test.
__attribute__((target_clones("avx2", "default"))) void cross_flags(const float *__restrict__ nx, const float *__restrict__ ny, const float *__restrict__ nz,
                 const float *__restrict__ bx, const float *__restrict__ by, const float *__restrict__ bz,
                 const float *__restrict__ r, const float *__restrict__ len, const double *__restrict__ mx,
                 const double *__restrict__ my, const double *__restrict__ mz,
                 const double *__restrict__ reach, unsigned char *__restrict__ flag, int n, const Worm &c,
                 double cmx, double cmy, double cmz, double creach)
{
    const float cnx = c.n.x, cny = c.n.y, cnz = c.n.z, cbx = c.b.x, cby = c.b.y, cbz = c.b.z, cr = c.r,
                cl = c.l;
    for (int j = 0; j < n; j++) {
        // v0 = a.n x b.n, v1 = b.b - a.b with a = the candidate
        const float vx = cny * nz[j] - cnz * ny[j], vy = cnz * nx[j] - cnx * nz[j], vz = cnx * ny[j] - cny * nx[j];
        const float r0 = std::sqrt(vx * vx + vy * vy + vz * vz);
        const float ux = bx[j] - cbx, uy = by[j] - cby, uz = bz[j] - cbz;
        const float dd = std::fabs((ux * vx + uy * vy + uz * vz) / r0);
        // decisions as 0 / 1 integers combined without branches
        const int par = r0 <= 1.e-20f;   // (double)r0 <= 1e-20 for every float r0
        const int near = !(dd > cr + r[j]);
        const float b1 = ux * cnx + uy * cny + uz * cnz, b2 = ux * nx[j] + uy * ny[j] + uz * nz[j];
        const float a11 = 1.f, a12 = nx[j] * cnx + ny[j] * cny + nz[j] * cnz, a21 = -a12, a22 = -a11;
        const float det = a11 * a22 - a12 * a21;
        const float q0 = (b1 * a22 - b2 * a12) / det, q1 = (b2 * a11 - b1 * a21) / det;
        const int inside = (q0 >= 0.f) & (q0 <= cl) & (q1 >= 0.f) & (q1 <= len[j]);
        const double dx = cmx - mx[j], dy = cmy - my[j], dz = cmz - mz[j], rr = creach + reach[j];
        const int reachable = dx * dx + dy * dy + dz * dz <= rr * rr;
        const int one = par | (near & inside), two = (par ^ 1) & near & (inside ^ 1) & reachable;
        flag[j] = (unsigned char)(one | (two << 1));
    }
}

int anthrax_place(unsigned long long *state, int ni, float radius, float length, int count,
                  float *cyl13, long long max_tries)
{
    // iGenerateAnthrax placement, particle.cpp:21-60
    const float R = (float)((double)(float)ni / 2.), R2 = (R - radius) * (R - radius);
    std::vector<Worm> w;
    w.reserve((size_t)count);
    // placed monomers' axes, starts, radii, midpoints and reach (half length + radius)
    std::vector<float> nx_, ny_, nz_, bx_, by_, bz_, r_, l_;
    std::vector<double> mx_, my_, mz_, reach_;
    std::vector<unsigned char> cand_;
    // placed monomers bucketed by midpoint on a grid whose cell G exceeds every reach sum,
    // so that a pair within reach of the point tests lies in neighbouring buckets
    const double G = (double)length + 2.0 * (double)radius + 2.0, org = -(double)R - G;
    const int nb = (int)std::ceil((2.0 * (double)R + 2.0 * G) / G) + 1;
    std::vector<std::vector<int>> bucket((size_t)nb * nb * nb);
    auto bidx = [&](double x) {
        const int b = (int)std::floor((x - org) / G);
        return b < 0 ? 0 : b >= nb ? nb - 1 : b;
    };
    unsigned long long s = *state;
    long long tries = 0;
    int l = 0;
    while ((int)w.size() < count) {
        Worm c;
        c.r = -1.f;
        while (c.r < 0.f) {
            if (++tries > max_tries) return -1;
            const float r1 = R * (float)rng_draw(s) / kRandMax;
            const float r2 = r1;
            const float ph1 = (float)(2. * kPi * (double)(float)rng_draw(s) / (double)kRandMax);
            const float ph2 = (float)(2. * kPi * (double)(float)rng_draw(s) / (double)kRandMax);
            float r0 = (float)(2. * (double)(float)rng_draw(s) / (double)kRandMax - 1.);
            const float th1 = std::acos(r0);
            r0 = (float)(2. * (double)(float)rng_draw(s) / (double)kRandMax - 1.);
            const float th2 = std::acos(r0);
            c = make_worm(r1, th1, ph1, r2, th2, ph2, length, radius, R2);
        }
        // The reference tests the candidate against every placed monomer with
        // CrossTwoWorms and rejects it on the first crossing; only that yes / no matters.
        // The monomers in the candidate's and the neighbouring buckets are tested first
        // (most rejections come from them); if none crosses, all pairs are decided chunk by
        // chunk of placed monomers: cross_flags for the whole chunk, then the point tests
        // only for the pairs it leaves to them.
        const double mx = 0.5 * ((double)c.b.x + c.e.x), my = 0.5 * ((double)c.b.y + c.e.y),
                     mz = 0.5 * ((double)c.b.z + c.e.z);
        const int bi = bidx(mx), bj = bidx(my), bk = bidx(mz);
        l = 0;
        // the candidate's own bucket first (s = 0), then the 26 around it
        for (int s = 0; s < 27 && !l; s++) {
            const int o = s == 0 ? 13 : (s <= 13 ? s - 1 : s);   // offsets 0..26, 13 = (0, 0, 0)
            const int a = bi + o / 9 - 1, b = bj + (o / 3) % 3 - 1, q = bk + o % 3 - 1;
            if (a < 0 || b < 0 || q < 0 || a >= nb || b >= nb || q >= nb) continue;
            for (const int j : bucket[((size_t)a * nb + b) * nb + q])
                if (cross_two_worms(c, w[(size_t)j])) {
                    l = 1;
                    break;
                }
        }
        if (!l && !w.empty()) {
            const size_t nw = w.size();
            const double reach = 0.5 * (double)c.l + c.r + 1.0;
            for (size_t j0 = 0; j0 < nw && !l; j0 += 256) {
                const size_t j1 = std::min(nw, j0 + 256);
                cross_flags(nx_.data() + j0, ny_.data() + j0, nz_.data() + j0, bx_.data() + j0, by_.data() + j0,
                            bz_.data() + j0, r_.data() + j0, l_.data() + j0, mx_.data() + j0, my_.data() + j0,
                            mz_.data() + j0, reach_.data() + j0, cand_.data() + j0, (int)(j1 - j0), c, mx, my,
                            mz, reach);
                for (size_t j = j0; j < j1 && !l; j++) {
                    if (cand_[j] == 1) l = 1;
                    else if (cand_[j] == 2) l = cross_two_worms(c, w[j]);
                }
            }
        }
        if (l == 0) {
            w.push_back(c);
            nx_.push_back(c.n.x);
            ny_.push_back(c.n.y);
            nz_.push_back(c.n.z);
            bx_.push_back(c.b.x);
            by_.push_back(c.b.y);
            bz_.push_back(c.b.z);
            r_.push_back(c.r);
            l_.push_back(c.l);
            mx_.push_back(0.5 * ((double)c.b.x + c.e.x));
            my_.push_back(0.5 * ((double)c.b.y + c.e.y));
            mz_.push_back(0.5 * ((double)c.b.z + c.e.z));
            reach_.push_back(0.5 * (double)c.l + c.r);
            cand_.push_back(0);
            bucket[((size_t)bidx(mx) * nb + bidx(my)) * nb + bidx(mz)].push_back((int)w.size() - 1);
        }
    }
    *state = s;
    for (int k = 0; k < count; k++) {
        float *o = cyl13 + 13 * (size_t)k;
        const Worm &m = w[(size_t)k];
        const float v[13] = {m.r, m.l, m.b.x, m.b.y, m.b.z, m.e.x, m.e.y, m.e.z, m.n.x, m.n.y, m.n.z, 0.f, 0.f};
        for (int q = 0; q < 13; q++) o[q] = v[q];
    }
    return 0;
}

size_t anthrax_scratch_bytes(int count) { return (size_t)(count ? count : 1) * sizeof(DW); }

cudaError_t anthrax_rasterize(const float *cyl13, int count, int ni, int nj, int nl,
                              signed char *occ_dev, int *ndip_dev, cudaStream_t st, void *scratch,
                              size_t scratch_bytes)
{
    // iGenerateAnthrax rasterisation, particle.cpp:62-83: centre n/2 - 0.5, radius n/2
    std::vector<DW> h((size_t)count);
    for (int k = 0; k < count; k++) {
        const float *c = cyl13 + 13 * (size_t)k;
        h[(size_t)k] = DW{c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9], c[10]};
    }
    // the caller's device scratch when it is large enough, else a stream-ordered allocation
    const bool own = !scratch || scratch_bytes < anthrax_scratch_bytes(count);
    DW *d = own ? nullptr : static_cast<DW *>(scratch);
    cudaError_t e = own ? cudaMallocAsync(&d, anthrax_scratch_bytes(count), st) : cudaSuccess;
    if (e) return e;
    // pageable source: the copy has taken the host data when the call returns
    if (count) e = cudaMemcpyAsync(d, h.data(), count * sizeof(DW), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(ndip_dev, 0, sizeof(int), st);
    if (!e) {
        const float R = (float)((double)(float)ni / 2.);
        const float cx = (float)((double)(float)ni / 2. - .5),
                    cy = (float)((double)(float)nj / 2. - .5),
                    cz = (float)((double)(float)nl / 2. - .5);
        const unsigned tiles = (unsigned)(((ni + kTile - 1) / kTile) * ((nj + kTile - 1) / kTile) *
                                          ((nl + kTile - 1) / kTile));
        rasterize<<<tiles, 256, 0, st>>>(d, count, ni, nj, nl, cx, cy, cz, R * R, occ_dev, ndip_dev);
        e = cudaGetLastError();
    }
    if (own) cudaFreeAsync(d, st);
    return e;
}

}  // namespace ddagpu
