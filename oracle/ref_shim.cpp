/*
 * ref_shim.cpp -- test infrastructure, NOT part of the product.
 *
 * A thin extern "C" layer over the reference DDA-FFT sources (physicist2018/dda-fft
 * v7.2), compiled from the reference tree where it lies by oracle/Makefile into
 * oracle/_ref/libddaref.so.  Nothing here re-implements the reference's arithmetic:
 * every number comes out of the reference's own functions (Convolution, DDA_FFT,
 * FarField, CabsCext, BuildMatrixJones, JonesToMuller, the polarisability models, the
 * FFT kernels, iGenerateEllipsoid, dda_rand).  The shim only converts between dense
 * arrays and the reference's pointer-of-pointer fields, and drives them the way
 * main.cpp does.
 *
 * Dense layouts used at this boundary (and by the GPU library's C-ABI):
 *   field  : [ni][nj][nl] cvector  = 6 floats per cell (x.re,x.im,y.re,y.im,z.re,z.im)
 *   Green  : [2ni][2nj][2nl] cmatrix = 12 floats per cell (e00,e01,e02,e11,e12,e22)
 *   occ    : [ni][nj][nl] signed char material index (0 = empty)
 *
 * Used only by tests/golden/make_golden.py (fixture generation), by the CPU parity
 * tests and by bench.py's reference arm.
 */
#include "function.hpp"
#include "mmuller.hpp"
#include "randomize.hpp"
#include "fft_kernel.hpp"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <unistd.h>

typedef real ioreal; /* array element type at this boundary: float, or double in the FP64 build */

namespace {

/* pointer-of-pointer views onto dense blocks (the reference indexes a[i][j][l]) */
template <class T>
struct view3 {
    std::vector<T **> p;
    std::vector<T *> rows;
    T ***get() { return p.data(); }
    view3(T *blk, int ni, int nj, int nl) : p((size_t)ni), rows((size_t)ni * nj)
    {
        for (int i = 0; i < ni; i++) {
            p[(size_t)i] = rows.data() + (size_t)i * nj;
            for (int j = 0; j < nj; j++)
                rows[(size_t)i * nj + j] = blk + ((size_t)i * nj + j) * nl;
        }
    }
};

/* CT twiddle tables, as main.cpp:411-419,466-475 builds them for --fft 0 */
struct ct_tables {
    std::vector<cplx> w2i, w2j, w2l, wi, wj, wl;
    ct_tables(int ni, int nj, int nl)
        : w2i(ni / 2 > 0 ? ni / 2 : 1), w2j(nj / 2 > 0 ? nj / 2 : 1), w2l(nl / 2 > 0 ? nl / 2 : 1),
          wi(ni), wj(nj), wl(nl)
    {
        FourierPhase(ni / 2, w2i.data());
        FourierPhase(nj / 2, w2j.data());
        FourierPhase(nl / 2, w2l.data());
        FourierPhase(ni, wi.data());
        FourierPhase(nj, wj.data());
        FourierPhase(nl, wl.data());
    }
};

/* RB (Rader-Brenner) tables, main.cpp:421-464,477-485 for --fft 1 */
struct rb_tables {
    int ni, nj, nl;
    std::vector<std::vector<real>> imi, imj, iml;
    std::vector<std::vector<cplx>> c2i, c2j, c2l;
    std::vector<real *> pimi, pimj, piml;
    std::vector<cplx *> pc2i, pc2j, pc2l;
    static void mk(int n, std::vector<std::vector<real>> &im, std::vector<std::vector<cplx>> &c2,
                   std::vector<real *> &pim, std::vector<cplx *> &pc2)
    {
        im.assign((size_t)n, std::vector<real>((size_t)n));
        c2.assign((size_t)n, std::vector<cplx>((size_t)n));
        pim.resize((size_t)n);
        pc2.resize((size_t)n);
        for (int i = 0; i < n; i++) {
            pim[(size_t)i] = im[(size_t)i].data();
            pc2[(size_t)i] = c2[(size_t)i].data();
        }
    }
    rb_tables(int ni_, int nj_, int nl_) : ni(ni_), nj(nj_), nl(nl_)
    {
        mk(ni, imi, c2i, pimi, pc2i);
        mk(nj, imj, c2j, pimj, pc2j);
        mk(nl, iml, c2l, piml, pc2l);
        FourierPhase(2 * ni, pimi.data(), pc2i.data());
        FourierPhase(2 * nj, pimj.data(), pc2j.data());
        FourierPhase(2 * nl, piml.data(), pc2l.data());
    }
};

struct green_holder {
    std::vector<cmatrix> blk;
    view3<cmatrix> v;
    green_holder(const ioreal *dense, int ni, int nj, int nl)
        : blk((size_t)8 * ni * nj * nl), v(blk.data(), 2 * ni, 2 * nj, 2 * nl)
    {
        std::memcpy(blk.data(), dense, blk.size() * sizeof(cmatrix));
    }
};

/* Capture what a reference call prints on stdout (the per-step discrepancies) in an
 * anonymous temporary file. */
struct stdout_capture {
    int saved = -1;
    FILE *tmp = nullptr;
    void begin()
    {
        std::fflush(stdout);
        tmp = std::tmpfile();
        if (!tmp) return;
        saved = dup(1);
        dup2(fileno(tmp), 1);
    }
    std::string end()
    {
        if (!tmp) return std::string();
        std::fflush(stdout);
        dup2(saved, 1);
        close(saved);
        std::string s;
        std::rewind(tmp);
        char buf[4096];
        size_t k;
        while ((k = std::fread(buf, 1, sizeof buf, tmp)) > 0) s.append(buf, k);
        std::fclose(tmp);
        tmp = nullptr;
        return s;
    }
};

} // namespace

extern "C" {

int dref_sizeof_real(void) { return (int)sizeof(real); }

/* cmA exactly as main.cpp:466-486 builds it: CreateAMatrix then FFT_3D(cmatrix). */
int dref_green(int ni, int nj, int nl, double kd, int fft_mode, ioreal *out)
{
    std::vector<cmatrix> blk((size_t)8 * ni * nj * nl);
    view3<cmatrix> a(blk.data(), 2 * ni, 2 * nj, 2 * nl);
    CreateAMatrix(ni, nj, nl, (real)kd, a.get());
    if (fft_mode == 0) {
        ct_tables t(ni, nj, nl);
        FFT_3D(2 * ni, 2 * nj, 2 * nl, t.wi.data(), t.wj.data(), t.wl.data(), a.get());
    } else {
        rb_tables t(ni, nj, nl);
        FFT_3D(2 * ni, 2 * nj, 2 * nl, t.pimi.data(), t.pimj.data(), t.piml.data(), t.pc2i.data(),
               t.pc2j.data(), t.pc2l.data(), a.get());
    }
    std::memcpy(out, blk.data(), blk.size() * sizeof(cmatrix));
    return 0;
}

/* The real-space Green tensor only (CreateAMatrix, dda_func.cpp:85-148). */
int dref_green_realspace(int ni, int nj, int nl, double kd, ioreal *out)
{
    std::vector<cmatrix> blk((size_t)8 * ni * nj * nl);
    view3<cmatrix> a(blk.data(), 2 * ni, 2 * nj, 2 * nl);
    CreateAMatrix(ni, nj, nl, (real)kd, a.get());
    std::memcpy(out, blk.data(), blk.size() * sizeof(cmatrix));
    return 0;
}

/* CopyingBack + Convolution(_conj) + read back the valid n-block (dda_func.cpp:1105-1112). */
int dref_convolution(int ni, int nj, int nl, int fft_mode, int conj, const ioreal *cmA,
                     const ioreal *p, ioreal *out)
{
    green_holder g(cmA, ni, nj, nl);
    std::vector<cvector> fld((size_t)ni * nj * nl), work((size_t)8 * ni * nj * nl);
    std::memcpy(fld.data(), p, fld.size() * sizeof(cvector));
    view3<cvector> vf(fld.data(), ni, nj, nl), vw(work.data(), 2 * ni, 2 * nj, 2 * nl);
    CopyingBack(ni, nj, nl, vf.get(), vw.get());
    if (fft_mode == 0) {
        ct_tables t(ni, nj, nl);
        if (conj)
            Convolution_conj(2 * ni, 2 * nj, 2 * nl, t.w2i.data(), t.w2j.data(), t.w2l.data(),
                             t.wi.data(), t.wj.data(), t.wl.data(), g.v.get(), vw.get());
        else
            Convolution(2 * ni, 2 * nj, 2 * nl, t.w2i.data(), t.w2j.data(), t.w2l.data(), t.wi.data(),
                        t.wj.data(), t.wl.data(), g.v.get(), vw.get());
    } else {
        rb_tables t(ni, nj, nl);
        if (conj)
            Convolution_conj(2 * ni, 2 * nj, 2 * nl, t.pimi.data(), t.pimj.data(), t.piml.data(),
                             t.pc2i.data(), t.pc2j.data(), t.pc2l.data(), g.v.get(), vw.get());
        else
            Convolution(2 * ni, 2 * nj, 2 * nl, t.pimi.data(), t.pimj.data(), t.piml.data(),
                        t.pc2i.data(), t.pc2j.data(), t.pc2l.data(), g.v.get(), vw.get());
    }
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++)
            std::memcpy(out + 6 * (((size_t)i * nj + j) * nl), &vw.get()[i][j][0],
                        (size_t)nl * sizeof(cvector));
    return 0;
}

/* The reference's complete solver for one polarisation (DDA_FFT, dda_func.cpp:1075-1570).
   trace[k] receives the printed step discrepancies (%9.7Lf, main's verbose output);
   *step_min_out is the rolled-back step or -1 when no rollback happened. */
int dref_dda_fft(int ni, int nj, int nl, int solver, double tau, int nmat, const ioreal *alpha,
                 const int *listmv, const signed char *occ, int max_step, double err_max, double d0,
                 const ioreal *kinc3, const ioreal *einc6, int fft_mode, const ioreal *cmA, int nplanes,
                 int nangles, const ioreal *ksc, ioreal *esc, ioreal *cabs, ioreal *cext, ioreal *p_out,
                 double *trace, int *ntrace, int *step_min_out)
{
    green_holder g(cmA, ni, nj, nl);
    std::vector<char> occb((size_t)ni * nj * nl);
    std::memcpy(occb.data(), occ, occb.size());
    view3<char> vo(occb.data(), ni, nj, nl);
    std::vector<cplx> mats((size_t)nmat + 1);
    std::vector<int> mv((size_t)nmat + 1);
    for (int m = 0; m <= nmat; m++) {
        mats[(size_t)m].r = alpha[2 * m];
        mats[(size_t)m].i = alpha[2 * m + 1];
        mv[(size_t)m] = listmv[m];
    }
    vector kinc = {kinc3[0], kinc3[1], kinc3[2]};
    cvector einc = {{einc6[0], einc6[1]}, {einc6[2], einc6[3]}, {einc6[4], einc6[5]}};
    std::vector<vector> kscb((size_t)nplanes * nangles);
    std::vector<vector *> kscp((size_t)nplanes);
    std::vector<cvector> escb((size_t)nplanes * nangles);
    std::vector<cvector *> escp((size_t)nplanes);
    for (int pl = 0; pl < nplanes; pl++) {
        kscp[(size_t)pl] = kscb.data() + (size_t)pl * nangles;
        escp[(size_t)pl] = escb.data() + (size_t)pl * nangles;
        for (int a = 0; a < nangles; a++) {
            const ioreal *k = ksc + 3 * ((size_t)pl * nangles + a);
            kscb[(size_t)pl * nangles + a] = vector{k[0], k[1], k[2]};
        }
    }
    dda_workspace ws;
    dda_workspace_create(&ws, ni, nj, nl, solver);
    ws.iVerbose = 1;
    real rcabs = 0, rcext = 0;
    stdout_capture cap;
    cap.begin();
    if (fft_mode == 0) {
        ct_tables t(ni, nj, nl);
        DDA_FFT(0, solver, (real)tau, ni, nj, nl, mats.data(), mv.data(), vo.get(), max_step,
                (real)err_max, (real)d0, kinc, einc, t.w2i.data(), t.w2j.data(), t.w2l.data(),
                t.wi.data(), t.wj.data(), t.wl.data(), NULL, NULL, NULL, NULL, NULL, NULL, 0,
                g.v.get(), nplanes, nangles, kscp.data(), escp.data(), &rcabs, &rcext, &ws);
    } else {
        rb_tables t(ni, nj, nl);
        DDA_FFT(0, solver, (real)tau, ni, nj, nl, mats.data(), mv.data(), vo.get(), max_step,
                (real)err_max, (real)d0, kinc, einc, NULL, NULL, NULL, NULL, NULL, NULL,
                t.pimi.data(), t.pimj.data(), t.piml.data(), t.pc2i.data(), t.pc2j.data(),
                t.pc2l.data(), 1, g.v.get(), nplanes, nangles, kscp.data(), escp.data(), &rcabs,
                &rcext, &ws);
    }
    std::string txt = cap.end();
    *cabs = rcabs;
    *cext = rcext;
    for (size_t k = 0; k < escb.size(); k++) std::memcpy(esc + 6 * k, &escb[k], sizeof(cvector));
    if (p_out)
        for (int i = 0; i < ni; i++)
            for (int j = 0; j < nj; j++)
                std::memcpy(p_out + 6 * (((size_t)i * nj + j) * nl), &ws.cvP[i][j][0],
                            (size_t)nl * sizeof(cvector));
    /* parse "Step %4d    discrepancy=%9.7Lf" lines; the rollback message is followed by
       "Step %3d    discrepancy=" of the best iterate */
    int nt = 0, smin = -1;
    size_t pos = 0;
    bool after_rollback = false;
    const std::string key = "discrepancy=";
    const std::string rb = "replaced with the most optimal";
    size_t rbpos = txt.find(rb);
    while ((pos = txt.find(key, pos)) != std::string::npos) {
        double v = std::strtod(txt.c_str() + pos + key.size(), NULL);
        if (rbpos != std::string::npos && pos > rbpos) {
            /* the step number precedes "discrepancy=" on the same line */
            size_t ls = txt.rfind("Step", pos);
            smin = std::atoi(txt.c_str() + ls + 4);
            after_rollback = true;
        } else if (trace && nt < max_step + 1) {
            trace[nt++] = v;
        }
        pos += key.size();
    }
    (void)after_rollback;
    if (ntrace) *ntrace = nt;
    if (step_min_out) *step_min_out = smin;
    dda_workspace_free(&ws);
    return 0;
}

/* FarField for one direction (dda_func.cpp:1576-1625). */
int dref_farfield(int ni, int nj, int nl, int nmat, const int *listmv, const signed char *occ,
                  double d0, const ioreal *p, const ioreal *ksc3, ioreal *out6)
{
    std::vector<char> occb((size_t)ni * nj * nl);
    std::memcpy(occb.data(), occ, occb.size());
    view3<char> vo(occb.data(), ni, nj, nl);
    std::vector<cvector> fld((size_t)ni * nj * nl);
    std::memcpy(fld.data(), p, fld.size() * sizeof(cvector));
    view3<cvector> vf(fld.data(), ni, nj, nl);
    std::vector<int> mv(listmv, listmv + nmat + 1);
    vector k = {ksc3[0], ksc3[1], ksc3[2]};
    cvector r = FarField(ni, nj, nl, mv.data(), vo.get(), (real)d0, vf.get(), k);
    std::memcpy(out6, &r, sizeof r);
    return 0;
}

/* CabsCext (dda_func.cpp:1679-1727). */
int dref_cabscext(int ni, int nj, int nl, int nmat, const ioreal *alpha, const signed char *occ,
                  double d0, const ioreal *kinc3, const ioreal *einc6, const ioreal *p, ioreal *cabs,
                  ioreal *cext)
{
    std::vector<char> occb((size_t)ni * nj * nl);
    std::memcpy(occb.data(), occ, occb.size());
    view3<char> vo(occb.data(), ni, nj, nl);
    std::vector<cvector> fld((size_t)ni * nj * nl);
    std::memcpy(fld.data(), p, fld.size() * sizeof(cvector));
    view3<cvector> vf(fld.data(), ni, nj, nl);
    std::vector<cplx> mats((size_t)nmat + 1);
    for (int m = 0; m <= nmat; m++) {
        mats[(size_t)m].r = alpha[2 * m];
        mats[(size_t)m].i = alpha[2 * m + 1];
    }
    vector kinc = {kinc3[0], kinc3[1], kinc3[2]};
    cvector einc = {{einc6[0], einc6[1]}, {einc6[2], einc6[3]}, {einc6[4], einc6[5]}};
    real a = 0, b = 0;
    CabsCext((real)d0, kinc, einc, ni, nj, nl, mats.data(), vo.get(), vf.get(), &a, &b);
    *cabs = a;
    *cext = b;
    return 0;
}

/* BuildMatrixJones + JonesToMuller (mmuller.cpp:175-314); out16 row-major. */
int dref_jones_mueller(const ioreal *kinc3, const ioreal *ksc3, const ioreal *normal3,
                       const ioreal *einc0, const ioreal *einc1, const ioreal *esc0, const ioreal *esc1,
                       ioreal *jones8, ioreal *out16)
{
    vector ki = {kinc3[0], kinc3[1], kinc3[2]}, ks = {ksc3[0], ksc3[1], ksc3[2]},
           nv = {normal3[0], normal3[1], normal3[2]};
    cvector e[4];
    const ioreal *src[4] = {einc0, einc1, esc0, esc1};
    for (int q = 0; q < 4; q++) std::memcpy(&e[q], src[q], sizeof(cvector));
    mjones mj = BuildMatrixJones(ki, ks, nv, e[0], e[1], e[2], e[3]);
    mmuller mm = JonesToMuller(mj);
    if (jones8) std::memcpy(jones8, &mj, sizeof mj);
    std::memcpy(out16, &mm, sizeof mm);
    return 0;
}

/* Polarisability of one material as main.cpp:599-642 (and 926-931 for LDR) selects it.
   model: 1 CM, 2 CMRR, 3 CMNR, 4 ILDR, 5 LDR. */
int dref_polarizability(int model, double d0, double m_re, double m_im, const ioreal *kinc3,
                        const ioreal *einc6, ioreal *out2)
{
    cplx m = {(real)m_re, (real)m_im};
    cplx a = Polarizability_CM((real)d0, m);
    if (model == 2) a = Polarizability_CMRR(a);
    if (model == 3) a = Polarizability_CMNR((real)d0, a);
    if (model == 4) a = Polarizability_ILDR((real)d0, m, a);
    if (model == 5) {
        vector k = {kinc3[0], kinc3[1], kinc3[2]};
        cvector e = {{einc6[0], einc6[1]}, {einc6[2], einc6[3]}, {einc6[4], einc6[5]}};
        a = Polarizability_LDR((real)d0, m, a, k, e);
    }
    out2[0] = a.r;
    out2[1] = a.i;
    return 0;
}

/* The reference's 1-D line kernels: kind 0 = mixed-radix ddafft::fft_line,
   1 = ddafft::ifft_line, 2 = legacy FFT (fft_func.cpp:229), 3 = legacy iFFT. */
int dref_fft_line(int N, int kind, const ioreal *in, ioreal *out)
{
    std::vector<cvector> a((size_t)N), b((size_t)N);
    std::memcpy(a.data(), in, a.size() * sizeof(cvector));
    if (kind <= 1) {
        const ddafft::plan *pl = ddafft::get_plan(N);
        if (!pl) return -1;
        if (kind == 0) ddafft::fft_line(pl, b.data(), a.data());
        else ddafft::ifft_line(pl, b.data(), a.data());
    } else {
        std::vector<cplx> w((size_t)(N / 2 > 0 ? N / 2 : 1));
        FourierPhase(N / 2, w.data());
        int bits = 0;
        Get_number_bits(N - 1, &bits);
        if (kind == 2) FFT(bits, N, w.data(), a.data(), b.data());
        else iFFT(bits, N, w.data(), a.data(), b.data());
    }
    std::memcpy(out, b.data(), b.size() * sizeof(cvector));
    return 0;
}

int dref_gen_ellipsoid(int ni, int nj, int nl, double b_a, double c_a, signed char *occ)
{
    std::vector<char> occb((size_t)ni * nj * nl);
    view3<char> vo(occb.data(), ni, nj, nl);
    int n = iGenerateEllipsoid(ni, nj, nl, (real)b_a, (real)c_a, vo.get());
    std::memcpy(occ, occb.data(), occb.size());
    return n;
}

/* iGenerateAnthrax (particle.cpp:21-85) after dda_srand(seed): occupancy, the monomers
   (13 reals each: r, l, b[3], e[3], n[3]) and the next draw of the stream. */
int dref_gen_anthrax(unsigned long long seed, int ni, int nj, int nl, double radius,
                     double length, int count, signed char *occ, ioreal *cyl, int *next_draw)
{
    std::vector<char> occb((size_t)ni * nj * nl);
    view3<char> vo(occb.data(), ni, nj, nl);
    std::vector<cylinder> w((size_t)count);
    dda_srand(seed);
    int n = iGenerateAnthrax(ni, nj, nl, (real)radius, (real)length, count, w.data(), vo.get());
    std::memcpy(occ, occb.data(), occb.size());
    for (int k = 0; k < count; k++) {
        ioreal *o = cyl + 13 * (size_t)k;
        o[0] = w[(size_t)k].r;
        o[1] = w[(size_t)k].l;
        o[2] = w[(size_t)k].b.x; o[3] = w[(size_t)k].b.y; o[4] = w[(size_t)k].b.z;
        o[5] = w[(size_t)k].e.x; o[6] = w[(size_t)k].e.y; o[7] = w[(size_t)k].e.z;
        o[8] = w[(size_t)k].n.x; o[9] = w[(size_t)k].n.y; o[10] = w[(size_t)k].n.z;
        o[11] = o[12] = 0;
    }
    if (next_draw) *next_draw = dda_rand();
    return n;
}

/* iGenerateRandomEllipsoid (particle.cpp:531-614) after dda_srand(seed): occupancy, the
   count the reference returns (material-1 cells) and the next draw of the stream. */
int dref_gen_random_ellipsoid(unsigned long long seed, int ni, int nj, int nl, double b_a,
                              double c_a, int nsorts, int *seeds_per_sort, signed char *occ,
                              int *next_draw)
{
    std::vector<char> occb((size_t)ni * nj * nl);
    view3<char> vo(occb.data(), ni, nj, nl);
    dda_srand(seed);
    int n = iGenerateRandomEllipsoid(ni, nj, nl, (real)b_a, (real)c_a, nsorts, seeds_per_sort, vo.get());
    std::memcpy(occ, occb.data(), occb.size());
    if (next_draw) *next_draw = dda_rand();
    return n;
}

/* count draws of the reference generator after dda_srand(seed) (randomize.cpp:44-58). */
int dref_rng(unsigned long long seed, int count, int *out)
{
    dda_srand(seed);
    for (int k = 0; k < count; k++) out[k] = dda_rand();
    return 0;
}

/* ---------------------------------------------------------------------------------
 * The sample loop of main.cpp:774-995 for targets whose geometry does not depend on
 * the RNG (1 sphere, 2 ellipsoid, 11 = caller-supplied occupancy), driving the
 * reference's DDA_FFT / BuildMatrixJones / JonesToMuller from a pool of std::threads
 * with one workspace each, like main.cpp.  Setup (Green tensor, tables, scattering
 * geometry) runs before the clock starts; *seconds is the wall time of the pool.
 * ------------------------------------------------------------------------------- */
struct dref_run_cfg {
    int ni, nj, nl;
    int target;             /* 1 sphere, 2 ellipsoid, 6 agglomerate, 11 occ_in       */
    double b_a, c_a;
    double x;               /* size parameter                                        */
    int nmat;               /* materials                                             */
    double m[2 * 16];       /* refractive indices (re, im)                           */
    int polarizability;     /* 1..5                                                  */
    int solver;             /* 0..3                                                  */
    double tau;
    double err_max;
    int max_step;
    int fft_mode;
    int orientation;        /* 0 fixed, 1 Monte-Carlo                                */
    double psi, iota, kappa; /* degrees, fixed mode                                  */
    int nplanes;
    double theta_min, theta_max, theta_step;
    unsigned long long seed;
    double monomer_radius, monomer_ratio, packing;   /* target 6 (main.cpp:300, 585-586) */
};

/* Per-sample results of the next dref_run_samples call (null: none): sample k writes
 * Cabs, Cext and its plane-averaged Mueller matrices, 2 + 16 n_angles reals, at
 * each + k (2 + 16 n_angles).  Cleared by the call. */
static ioreal *g_each = nullptr;
int dref_set_per_sample(ioreal *each)
{
    g_each = each;
    return 0;
}

int dref_run_samples(const dref_run_cfg *c, const signed char *occ_in, int nthreads, int nsamples,
                     int verbose, double *seconds, ioreal *cabs_sum, ioreal *cext_sum,
                     ioreal *mueller_sum, int *nangles_out)
{
    ioreal *each = g_each;
    g_each = nullptr;
    const int ni = c->ni, nj = c->nj, nl = c->nl;
    const real xr = (real)c->x, tmin = (real)c->theta_min, tmax = (real)c->theta_max,
               tstep = (real)c->theta_step;
    const real kd = 2. * xr / (real)ni; /* main.cpp:318 */
    const int nA = rounding(((tmax - tmin) / tstep) + 1.);
    const int nP = c->nplanes;
    if (nangles_out) *nangles_out = nA;
    random_init_seed(c->seed);

    /* scattering geometry in the particle frame before rotation (main.cpp:336-387) */
    std::vector<vector> nrm0((size_t)nP), ksc0((size_t)nP * nA);
    nrm0[0] = vector{0., 1., 0.};
    for (int a = 0; a < nA; a++) {
        real th = tmin + tstep * a;
        SphCart_d(1., 0., th, ksc0[(size_t)a]);
    }
    {
        real step = 180. / ((real)nP), acc = 0.;
        for (int pl = 1; pl < nP; pl++) {
            acc += step;
            real cp = cos(acc * (PI / 180.)), sp = sin(acc * (PI / 180.));
            nrm0[(size_t)pl] = Rotation_z(cp, sp, nrm0[0]);
            for (int a = 0; a < nA; a++)
                ksc0[(size_t)pl * nA + a] = Rotation_z(cp, sp, ksc0[(size_t)a]);
        }
    }
    /* Green tensor and tables (main.cpp:466-486) */
    std::vector<cmatrix> gblk((size_t)8 * ni * nj * nl);
    view3<cmatrix> ga(gblk.data(), 2 * ni, 2 * nj, 2 * nl);
    CreateAMatrix(ni, nj, nl, kd, ga.get());
    ct_tables ct(ni, nj, nl);
    rb_tables *rb = nullptr;
    if (c->fft_mode == 0)
        FFT_3D(2 * ni, 2 * nj, 2 * nl, ct.wi.data(), ct.wj.data(), ct.wl.data(), ga.get());
    else {
        rb = new rb_tables(ni, nj, nl);
        FFT_3D(2 * ni, 2 * nj, 2 * nl, rb->pimi.data(), rb->pimj.data(), rb->piml.data(),
               rb->pc2i.data(), rb->pc2j.data(), rb->pc2l.data(), ga.get());
    }
    /* materials (main.cpp:599-643) */
    std::vector<cplx> mats0((size_t)c->nmat + 1);
    std::vector<int> mv((size_t)c->nmat + 1);
    mats0[0] = zero();
    mv[0] = 0;
    for (int k = 0; k < c->nmat; k++) {
        cplx m = {(real)c->m[2 * k], (real)c->m[2 * k + 1]};
        cplx a = Polarizability_CM(kd, m);
        mv[(size_t)k + 1] = (m.r == 1. && m.i == 0.) ? 0 : 1;
        if (c->polarizability == 2) a = Polarizability_CMRR(a);
        if (c->polarizability == 3) a = Polarizability_CMNR(kd, a);
        if (c->polarizability == 4 || c->polarizability == 5) a = Polarizability_ILDR(kd, m, a);
        mats0[(size_t)k + 1] = a;
    }
    /* fixed orientation (main.cpp:516-542) */
    vector kinc_ini = {0., 0., 1.};
    cvector einc_ini[2] = {{{1., 0.}, {0., 0.}, {0., 0.}}, {{0., 0.}, {1., 0.}, {0., 0.}}};
    std::vector<vector> nrmF((size_t)nP), kscF((size_t)nP * nA);
    vector kincF;
    cvector eincF[2];
    {
        real psi = (real)c->psi * PI / 180., iota = (real)c->iota * PI / 180.,
             kap = (real)c->kappa * PI / 180.;
        real cps = cos(-psi), sps = sin(-psi), cio = cos(-iota), sio = sin(-iota), cka = cos(-kap),
             ska = sin(-kap);
        for (int pl = 0; pl < nP; pl++) {
            vector v = Rotation_z(cps, sps, nrm0[(size_t)pl]);
            v = Rotation_y(cio, sio, v);
            nrmF[(size_t)pl] = Rotation_x(cka, ska, v);
            for (int a = 0; a < nA; a++) {
                vector k = Rotation_z(cps, sps, ksc0[(size_t)pl * nA + a]);
                k = Rotation_y(cio, sio, k);
                kscF[(size_t)pl * nA + a] = Rotation_x(cka, ska, k);
            }
        }
        vector k = Rotation_z(cps, sps, kinc_ini);
        k = Rotation_y(cio, sio, k);
        kincF = Rotation_x(cka, ska, k);
        for (int q = 0; q < 2; q++) {
            cvector e = Rotation_z(cps, sps, einc_ini[q]);
            e = Rotation_y(cio, sio, e);
            eincF[q] = Rotation_x(cka, ska, e);
        }
    }

    std::mutex mtx;
    std::atomic<int> next(0);
    double sum_cabs = 0., sum_cext = 0.;
    std::vector<mmuller> acc((size_t)nA, mmNull());
    real fcabs = 0., fcext = 0.;

    auto worker = [&](int wid) {
        std::vector<char> occb((size_t)ni * nj * nl);
        view3<char> vo(occb.data(), ni, nj, nl);
        if (c->target == 11) std::memcpy(occb.data(), occ_in, occb.size());
        std::vector<cplx> mats(mats0);
        std::vector<vector> kscb((size_t)nP * nA), nrm(nrmF);
        std::vector<vector *> kscp((size_t)nP);
        std::vector<cvector> escb[2];
        std::vector<cvector *> escp[2];
        for (int q = 0; q < 2; q++) {
            escb[q].resize((size_t)nP * nA);
            escp[q].resize((size_t)nP);
        }
        for (int pl = 0; pl < nP; pl++) {
            kscp[(size_t)pl] = kscb.data() + (size_t)pl * nA;
            for (int q = 0; q < 2; q++) escp[q][(size_t)pl] = escb[q].data() + (size_t)pl * nA;
        }
        kscb = kscF;
        vector kinc = kincF;
        cvector einc[2] = {eincF[0], eincF[1]};
        std::vector<mmuller> mm((size_t)nA);
        const real rw = (real)c->monomer_radius, lrw = (real)c->monomer_ratio, rho = (real)c->packing;
        const int nworms = c->target == 6
            ? (int)(rho * (real)(ni * nj * nl) / (8. * (rw * rw * rw) * (0.75 * lrw + 1))) + 1 : 0;
        std::vector<cylinder> worms((size_t)(nworms > 0 ? nworms : 1));
        dda_workspace ws;
        dda_workspace_create(&ws, ni, nj, nl, c->solver);
        ws.iVerbose = verbose;
        dda_srand(random_base_seed() + 0x9E3779B97F4A7C15ULL * (unsigned long long)(wid + 1));
        for (;;) {
            int task = next.fetch_add(1);
            if (task >= nsamples) break;
            if (c->target == 1) iGenerateEllipsoid(ni, nj, nl, 1., 1., vo.get());
            if (c->target == 2) iGenerateEllipsoid(ni, nj, nl, (real)c->b_a, (real)c->c_a, vo.get());
            if (c->target == 6)
                iGenerateAnthrax(ni, nj, nl, rw, rw * lrw, nworms, worms.data(), vo.get());
            if (c->orientation == 1) {
                /* Euler-angle draw and rotation matrix of main.cpp:875-917 */
                real cps = (real)dda_rand() * 2. / (real)DDA_RAND_MAX - 1.;
                real psi = acos(cps), sps = sin(psi);
                real iota = (real)dda_rand() * 2. * PI / (real)DDA_RAND_MAX;
                real cio = cos(iota), sio = sin(iota);
                real kap = (real)dda_rand() * 2. * PI / (real)DDA_RAND_MAX;
                real cka = cos(kap), ska = sin(kap);
                real T[3][3];
                T[0][0] = cio * cka - cps * sio * ska;
                T[0][1] = sio * cka + cps * cio * ska;
                T[0][2] = sps * ska;
                T[1][0] = -cio * ska - cps * sio * cka;
                T[1][1] = -sio * ska + cps * cio * cka;
                T[1][2] = sps * cka;
                T[2][0] = sps * sio;
                T[2][1] = -sps * cio;
                T[2][2] = cps;
                auto rot = [&](vector v) {
                    vector r;
                    r.x = T[0][0] * v.x + T[0][1] * v.y + T[0][2] * v.z;
                    r.y = T[1][0] * v.x + T[1][1] * v.y + T[1][2] * v.z;
                    r.z = T[2][0] * v.x + T[2][1] * v.y + T[2][2] * v.z;
                    return r;
                };
                for (int pl = 0; pl < nP; pl++) {
                    for (int a = 0; a < nA; a++)
                        kscb[(size_t)pl * nA + a] = rot(ksc0[(size_t)pl * nA + a]);
                    nrm[(size_t)pl] = rot(nrm0[(size_t)pl]);
                }
                kinc = rot(kinc_ini);
                for (int q = 0; q < 2; q++) {
                    cvector e0 = einc_ini[q];
                    einc[q].x = T[0][0] * e0.x + T[0][1] * e0.y + T[0][2] * e0.z;
                    einc[q].y = T[1][0] * e0.x + T[1][1] * e0.y + T[1][2] * e0.z;
                    einc[q].z = T[2][0] * e0.x + T[2][1] * e0.y + T[2][2] * e0.z;
                }
            }
            real scabs = 0., scext = 0.;
            for (int q = 0; q < 2; q++) {
                if (c->polarizability == 5)
                    for (int k = 0; k < c->nmat; k++) {
                        cplx m = {(real)c->m[2 * k], (real)c->m[2 * k + 1]};
                        cplx a = Polarizability_CM(kd, m);
                        mats[(size_t)k + 1] = Polarizability_LDR(kd, m, a, kinc, einc[q]);
                    }
                real rc = 0., re = 0.;
                if (c->fft_mode == 0)
                    DDA_FFT(q, c->solver, (real)c->tau, ni, nj, nl, mats.data(), mv.data(), vo.get(),
                            c->max_step, (real)c->err_max, kd, kinc, einc[q], ct.w2i.data(),
                            ct.w2j.data(), ct.w2l.data(), ct.wi.data(), ct.wj.data(), ct.wl.data(),
                            NULL, NULL, NULL, NULL, NULL, NULL, 0, ga.get(), nP, nA, kscp.data(),
                            escp[q].data(), &rc, &re, &ws);
                else
                    DDA_FFT(q, c->solver, (real)c->tau, ni, nj, nl, mats.data(), mv.data(), vo.get(),
                            c->max_step, (real)c->err_max, kd, kinc, einc[q], NULL, NULL, NULL, NULL,
                            NULL, NULL, rb->pimi.data(), rb->pimj.data(), rb->piml.data(),
                            rb->pc2i.data(), rb->pc2j.data(), rb->pc2l.data(), 1, ga.get(), nP, nA,
                            kscp.data(), escp[q].data(), &rc, &re, &ws);
                scabs += .5 * rc;
                scext += .5 * re;
            }
            for (int a = 0; a < nA; a++) {
                mm[(size_t)a] = mmNull();
                for (int pl = 0; pl < nP; pl++) {
                    mjones mj = BuildMatrixJones(kinc, kscb[(size_t)pl * nA + a], nrm[(size_t)pl],
                                                 einc[0], einc[1], escb[0][(size_t)pl * nA + a],
                                                 escb[1][(size_t)pl * nA + a]);
                    mm[(size_t)a] = mm[(size_t)a] + JonesToMuller(mj);
                }
                mm[(size_t)a] = mm[(size_t)a] / (real)nP;
            }
            if (each) {
                ioreal *o = each + (size_t)task * (2 + 16 * (size_t)nA);
                o[0] = scabs;
                o[1] = scext;
                for (int a = 0; a < nA; a++) std::memcpy(o + 2 + 16 * a, &mm[(size_t)a], sizeof(mmuller));
            }
            std::lock_guard<std::mutex> lk(mtx);
            fcabs += scabs;
            fcext += scext;
            for (int a = 0; a < nA; a++) acc[(size_t)a] = acc[(size_t)a] + mm[(size_t)a];
        }
        dda_workspace_free(&ws);
    };

    auto t0 = std::chrono::steady_clock::now();
    if (nthreads <= 1) worker(0);
    else {
        std::vector<std::thread> th;
        for (int w = 0; w < nthreads; w++) th.emplace_back(worker, w);
        for (auto &t : th) t.join();
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    (void)sum_cabs;
    (void)sum_cext;
    *cabs_sum = fcabs;
    *cext_sum = fcext;
    for (int a = 0; a < nA; a++) std::memcpy(mueller_sum + 16 * a, &acc[(size_t)a], sizeof(mmuller));
    delete rb;
    return 0;
}

} /* extern "C" */
