// Post-processing kernels of libddagpu (far field, cross sections, Mueller matrices).
#pragma once
#include "internal.h"

namespace ddagpu {

struct PostArgs {
    size_t N;
    int nrhs, ni, nj, nl;
    const signed char *occ;   // [N], or [nrhs][N] with occ_stride = N
    size_t occ_stride;        // 0: one occupancy shared by every right-hand side
    const int *mv;            // [nmat1]
    const float2 *alpha;      // [nrhs][nmat1]
    int nmat1;
    const float2 *p;          // [nrhs][3][N] dipole moments
    const double *kinc;       // [nrhs][3]
    const double *einc;       // [nrhs][6]
    double d0;
    int ndir;                 // scattering directions per right-hand side
    const double *ksc;        // [nrhs][ndir][3]
    double *esc_acc;          // [nrhs][ndir][6] scratch
    double *cc_acc;           // [nrhs][2] scratch (Cext sum, Cabs sum)
    int pairs;                // right-hand sides 2k, 2k+1 share directions, incident
                              // direction and occupancy (both polarisations of one orientation)
};

struct MuellerArgs {
    int norient, nplanes, nangles, ndir;   // ndir = nplanes * nangles
    const double *kinc;       // [2 norient][3]
    const double *einc;       // [2 norient][6]
    const double *ksc;        // [2 norient][ndir][3]
    const double *normals;    // [norient][nplanes][3]
    const float2 *esc;        // [2 norient][ndir][3]
    double *out;              // [norient][nangles][16]
};

size_t farfield_smem(int nj, int nl);
cudaError_t post_prepare(int nj, int nl);
cudaError_t launch_post(const PostArgs &a, float2 *esc, float *cabs, float *cext, cudaStream_t st);
cudaError_t launch_mueller(const MuellerArgs &m, cudaStream_t st);

// allocation-free far field (scratch in a file-scope device array of post.cu)
int farfield_noalloc_max_dirs();
cudaError_t farfield_noalloc_scratch(int device, double **ptr);
cudaError_t farfield_noalloc(const PostArgs &a, const float *ksc_dev, float2 *esc_dev,
                             double *scratch, cudaStream_t st);

}  // namespace ddagpu
