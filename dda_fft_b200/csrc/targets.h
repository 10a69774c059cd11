// Random targets of libddagpu (agglomerates, random ellipsoids): host placement, GPU rasterisation.
#pragma once
#include <cuda_runtime.h>

namespace ddagpu {

long long anthrax_count(int ni, int nj, int nl, float packing, float radius, float ratio);
int anthrax_place(unsigned long long *state, int ni, float radius, float length, int count,
                  float *cyl13, long long max_tries);
// scratch (may be null): device memory for the monomers, used when it holds
// anthrax_scratch_bytes(count); otherwise the call allocates stream-ordered memory
size_t anthrax_scratch_bytes(int count);
cudaError_t anthrax_rasterize(const float *cyl13, int count, int ni, int nj, int nl,
                              signed char *occ_dev, int *ndip_dev, cudaStream_t st,
                              void *scratch = nullptr, size_t scratch_bytes = 0);

int random_ellipsoid_seeds(unsigned long long *state, int ni, int nj, int nl, float b_a, float c_a,
                           int nseeds, float *seeds3);
cudaError_t random_ellipsoid_fill(const float *seeds3, const int *counts, int nsorts, int ni, int nj,
                                  int nl, float b_a, float c_a, signed char *occ_dev, int *ndip_dev,
                                  cudaStream_t st);

}  // namespace ddagpu
