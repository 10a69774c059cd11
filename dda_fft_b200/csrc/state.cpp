// State (.dst) and result (.dat) files of the sample loop, in the layout of the reference's
// float build, so that runs resume from and compare against the reference's own files.
//
// .dst (main.cpp:214-274 read/create, 966-981 refresh): int sample counter, float Cabs sum,
// float Cext sum, then n_angles Mueller sums of 16 floats (mmuller, mmuller.hpp:12-15), all
// native-endian with no padding.  .dat (main.cpp:1085-1118): the sums divided by the
// counter, printed with the reference's formats.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ddagpu.h"

namespace ddagpu {
int set_error(int code, const std::string &msg);   // ddagpu.cu
}

namespace {

int io_fail(const std::string &what, const char *path)
{
    return ddagpu::set_error(DDAGPU_EINVAL, what + " '" + std::string(path ? path : "") + "': " +
                                                std::strerror(errno));
}

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

int ddagpu_state_write(const char *path, int counter, float cabs, float cext, int n_angles,
                       const float *mueller)
{
    if (!path || n_angles < 0 || (n_angles && !mueller))
        return ddagpu::set_error(DDAGPU_EINVAL, "bad state-file arguments");
    File f;
    // rewrite in place like the reference (fseek to 0, fwrite, fflush); create if missing
    f.f = std::fopen(path, "rb+");
    if (!f.f) f.f = std::fopen(path, "wb+");
    if (!f.f) return io_fail("cannot create the dst-file", path);
    bool ok = std::fwrite(&counter, sizeof counter, 1, f.f) == 1 &&
              std::fwrite(&cabs, sizeof cabs, 1, f.f) == 1 &&
              std::fwrite(&cext, sizeof cext, 1, f.f) == 1;
    if (ok && n_angles)
        ok = std::fwrite(mueller, sizeof(float) * 16, (size_t)n_angles, f.f) == (size_t)n_angles;
    if (!ok || std::fflush(f.f) != 0) return io_fail("cannot write the dst-file", path);
    return DDAGPU_OK;
}

int ddagpu_state_read(const char *path, int n_angles, int restart, int *counter, float *cabs,
                      float *cext, float *mueller)
{
    if (!path || n_angles < 0 || !counter || !cabs || !cext || (n_angles && !mueller))
        return ddagpu::set_error(DDAGPU_EINVAL, "bad state-file arguments");
    if (restart) std::remove(path);
    {
        File probe;
        probe.f = std::fopen(path, "rb");
        if (!probe.f) {
            // a fresh state: zero counter and sums (main.cpp:218-238)
            std::vector<float> zero((size_t)n_angles * 16, 0.f);
            const int rc = ddagpu_state_write(path, 0, 0.f, 0.f, n_angles, zero.data());
            if (rc) return rc;
        }
    }
    File f;
    f.f = std::fopen(path, "rb");
    if (!f.f) return io_fail("cannot open the dst-file", path);
    bool ok = std::fread(counter, sizeof *counter, 1, f.f) == 1 &&
              std::fread(cabs, sizeof *cabs, 1, f.f) == 1 && std::fread(cext, sizeof *cext, 1, f.f) == 1;
    if (ok && n_angles)
        ok = std::fread(mueller, sizeof(float) * 16, (size_t)n_angles, f.f) == (size_t)n_angles;
    if (!ok)
        return ddagpu::set_error(DDAGPU_EINVAL, std::string("cannot read data from the dst-file '") +
                                                    path + "' (too short for the angle count?)");
    return DDAGPU_OK;
}

int ddagpu_state_accumulate(int n, const double *cabs, const double *cext, int n_angles,
                            const double *mueller, int *counter, float *cabs_sum,
                            float *cext_sum, float *mueller_sum)
{
    if (n < 0 || n_angles < 0 || !counter || !cabs_sum || !cext_sum ||
        (n && (!cabs || !cext)) || (n && n_angles && (!mueller || !mueller_sum)))
        return ddagpu::set_error(DDAGPU_EINVAL, "bad accumulation arguments");
    // per sample, in order, in float (main.cpp:961-966)
    for (int s = 0; s < n; s++) {
        *cabs_sum += (float)cabs[s];
        *cext_sum += (float)cext[s];
        for (int k = 0; k < 16 * n_angles; k++)
            mueller_sum[k] += (float)mueller[(size_t)s * 16 * n_angles + k];
        *counter += 1;
    }
    return DDAGPU_OK;
}

int ddagpu_write_dat(const char *path, int counter, float cabs, float cext, int n_angles,
                     float theta_min, float theta_step, const float *mueller)
{
    if (!path || counter < 1 || n_angles < 0 || (n_angles && !mueller))
        return ddagpu::set_error(DDAGPU_EINVAL, "bad result-file arguments");
    File f;
    f.f = std::fopen(path, "w");
    if (!f.f) return io_fail("cannot write the output data file", path);
    const float w = (float)(1. / (double)(float)counter);   // kd = 1./(real)count
    std::fprintf(f.f, "Cabs=%.8f\t\tCext=%.8f", (double)(w * cabs), (double)(w * cext));
    for (int m = 0; m < n_angles; m++) {
        const float theta = theta_min + theta_step * (float)m;
        std::fprintf(f.f, "\n%7.3f\t", (double)theta);
        for (int k = 0; k < 16; k++) std::fprintf(f.f, "\t%+10.8e", (double)(w * mueller[16 * m + k]));
    }
    if (std::fclose(f.f) != 0) {
        f.f = nullptr;
        return io_fail("cannot close the output data file", path);
    }
    f.f = nullptr;
    return DDAGPU_OK;
}

}  // extern "C"
