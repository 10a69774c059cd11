// Random targets of libddagpu (agglomerates, random ellipsoids): host placement, GPU rasterisation.
#pragma once
#include <cuda_runtime.h>

namespace ddagpu {

long long anthrax_count(int ni, int nj, int nl, float packing, float radius, float ratio);
int anthrax_place(unsigned long long *state, int ni, float radius, float length, int count,
                  float *cyl13, long long max_tries);
cudaError_t anthrax_rasterize(const float *cyl13, int count, int ni, int nj, int nl,
                              signed char *occ_dev, int *ndip_dev, cudaStream_t st);

int random_ellipsoid_seeds(unsigned long long *state, int ni, int nj, int nl, float b_a, float c_a,
                           int nseeds, float *seeds3);
cudaError_t random_ellipsoid_fill(const float *seeds3, const int *counts, int nsorts, int ni, int nj,
                                  int nl, float b_a, float c_a, signed char *occ_dev, int *ndip_dev,
                                  cudaStream_t st);

}  // namespace ddagpu
