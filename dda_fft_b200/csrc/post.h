// Post-processing kernels of libddagpu (far field, cross sections, Mueller matrices).
#pragma once
#include <vector>

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
    // far field by kz groups (KzPlan; kz_groups 0: one sum per direction)
    int kz_groups, kz_items, kz_slice, kz_stride;
    const int *kz_tab;        // [blocks][kz_stride]
    const double *kz_val;     // [blocks][kz_groups]
    float2 *kz_sum;           // [blocks][kz_groups][ni][nj][3 NR]
};

// Directions of a right-hand side (or of a pair) grouped by their z component.  A block is
// one right-hand side, or one pair when PostArgs::pairs and the count is even.  Per block,
// kz_stride ints: [0] groups, [1] items, [2 .. 2 + G] the groups' offsets into the sorted
// list, [3 + G ..) the directions sorted by kz, then items of (group, first position), each
// at most kKzItem directions of one group.
constexpr int kKzItem = 16;
struct KzPlan {
    int groups = 0;           // the most groups of a block; 0: the direct far field
    int items = 0, slice = 0, stride = 0, blocks = 0;
    size_t sum_elems = 0;     // float2 elements of the group sums
    std::vector<int> tab;
    std::vector<double> kz;
};
// ks: [nrhs][ndir][3] directions; nact: active cells per right-hand side (for the choice);
// mode 0: the grouped form when it saves at least half the work, 1: never, 2: always
void plan_kz_groups(const double *ks, int nrhs, int ndir, bool pairs, int ni, int nj, int nl,
                    double nact, int mode, KzPlan &P);

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
// *kernels (may be null) receives the number of kernels launched
cudaError_t launch_post(const PostArgs &a, float2 *esc, float *cabs, float *cext, cudaStream_t st,
                        int *kernels = nullptr);
cudaError_t launch_mueller(const MuellerArgs &m, cudaStream_t st);

// allocation-free far field (scratch in a file-scope device array of post.cu)
int farfield_noalloc_max_dirs();
cudaError_t farfield_noalloc_scratch(int device, double **ptr);
cudaError_t farfield_noalloc(const PostArgs &a, const float *ksc_dev, float2 *esc_dev,
                             double *scratch, cudaStream_t st);

}  // namespace ddagpu
