// Shared device-side definitions for the barotropic-step kernels.
//
// Device arrays keep the Fortran layout of the host arrays (x fastest,
// element (m,n) at row n-bnd_y1, column m-bnd_x1+xoff) with a padded row
// pitch: every row starts on a 256-byte boundary, xoff columns of padding
// precede bnd_x1 (so that the streaming kernel's column pairs and its TMA
// row segments are both 16-byte aligned) and padding follows bnd_x2 (so the
// segments, which may run past bnd_x2, stay inside the allocation).  Padding
// columns are zero and never written.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace inmsom {

struct Dom {
    int nx_start, nx_end, ny_start, ny_end;
    int bnd_x1, bnd_x2, bnd_y1, bnd_y2;
    int mmm, mm, nnn, nn;
    int px, py;            // periodicity_x, periodicity_y
    long long pitch;       // elements per device row
    int xoff;              // padding columns before bnd_x1
    int nxa() const { return bnd_x2 - bnd_x1 + 1; }
    int nya() const { return bnd_y2 - bnd_y1 + 1; }
};

__host__ __device__ inline long long ix(const Dom &d, int m, int n)
{
    return (long long)(n - d.bnd_y1) * d.pitch + (long long)(m - d.bnd_x1 + d.xoff);
}

// Static grid of the basin_grid module (Modules/mod_basin_grid.f90:6-37).
struct GridDev {
    const float *lu, *luu, *luh, *lcu, *lcv, *llu, *llv;
    const double *dx, *dy, *dxt, *dyt, *dxh, *dyh, *dxb, *dyb;
    const double *rlh, *hrest;
};

struct Consts {
    double ts;     // time_smooth
    double g;      // FreeFallAcc
    double rho;    // RefDen
    int ffs;       // full_free_surface
};

}  // namespace inmsom
