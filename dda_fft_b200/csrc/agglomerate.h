// Agglomerate (anthrax-like) targets of libddagpu: host placement, GPU rasterisation.
#pragma once
#include <cuda_runtime.h>

namespace ddagpu {

long long anthrax_count(int ni, int nj, int nl, float packing, float radius, float ratio);
int anthrax_place(unsigned long long *state, int ni, float radius, float length, int count,
                  float *cyl13, long long max_tries);
cudaError_t anthrax_rasterize(const float *cyl13, int count, int ni, int nj, int nl,
                              signed char *occ_dev, int *ndip_dev, cudaStream_t st);

}  // namespace ddagpu
