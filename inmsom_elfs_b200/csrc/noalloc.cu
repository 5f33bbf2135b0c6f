// inmsom_diag_noalloc: the volume/energy reduction of inmsom_gpu_diag for
// callers that cannot allocate GPU memory.
//
// A host ocean model often owns the whole device: it hands the GPU's memory
// to its own pool at start-up, or it must not call cudaMalloc/cudaFree in
// the middle of a time step because those calls synchronise the device and
// stall its streams.  Such a caller can still pass its own device arrays for
// the inputs and the two-double output, but it cannot give this library room
// for the reduction's scratch.  The scratch -- one volume and one energy
// partial per interior row -- therefore lives in a fixed array that is part
// of this file's device image: the CUDA runtime reserves it on each GPU that
// loads the image and keeps it until the process exits.
//
// The array is shared by every call on a device and keeps whatever the last
// call left in it.  The row kernel writes every partial that the final
// kernel reads, so no part of it has to start at zero; two calls whose
// kernels overlap on the GPU would interleave their partials, so callers
// order their calls (one stream, or events).
#include "inmsom_gpu.h"

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "general.h"

namespace inmsom {
int record_error(int code, const char *msg);
}

using namespace inmsom;

// Row partials: volume of interior row k at [k], energy at [nrows + k].
static __device__ __align__(256) double g_diag_rows[2 * INMSOM_DIAG_NOALLOC_MAX_ROWS];

namespace {

constexpr int kMaxDevices = 64;

std::mutex g_setup_mutex;
double *g_rows_on_device[kMaxDevices] = {};

int fail(int code, const char *fmt, ...)
{
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return record_error(code, buf);
}

// Device address of g_diag_rows on the current device.  In host code the
// name g_diag_rows only stands for the array; its address on a given GPU
// comes from cudaGetSymbolAddress with that GPU current, looked up once per
// device on its first call here and cached.
int rows_scratch(double **rows)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(INMSOM_ECUDA, "inmsom_diag_noalloc: cudaGetDevice failed: %s",
                    cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(INMSOM_EUNSUPPORTED, "inmsom_diag_noalloc: device %d beyond %d", dev,
                    kMaxDevices);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_rows_on_device[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_diag_rows);
        if (e != cudaSuccess || !p)
            return fail(INMSOM_ECUDA,
                        "inmsom_diag_noalloc: cudaGetSymbolAddress of the scratch array on "
                        "device %d failed: %s",
                        dev, cudaGetErrorString(e));
        g_rows_on_device[dev] = static_cast<double *>(p);
    }
    *rows = g_rows_on_device[dev];
    return INMSOM_OK;
}

}  // namespace

extern "C" int inmsom_diag_noalloc(const inmsom_bounds *b, const inmsom_consts *c, long long ld,
                                   const float *lu, const float *lcu, const float *lcv,
                                   const double *dx, const double *dy, const double *dxt,
                                   const double *dyt, const double *dxh, const double *dyh,
                                   const double *hhq_rest, const double *ssh, const double *u,
                                   const double *v, const double *hu, const double *hv,
                                   double *out, void *stream)
{
    // every argument check comes before the first CUDA call
    if (!b || !c) return fail(INMSOM_EARG, "inmsom_diag_noalloc: bounds or consts is NULL");
    if (!lu || !lcu || !lcv || !dx || !dy || !dxt || !dyt || !dxh || !dyh || !hhq_rest || !ssh ||
        !u || !v || !hu || !hv || !out)
        return fail(INMSOM_EARG, "inmsom_diag_noalloc: NULL array argument");
    const long long nxa = (long long)b->bnd_x2 - b->bnd_x1 + 1;
    const long long nya = (long long)b->bnd_y2 - b->bnd_y1 + 1;
    if (nxa < 1 || nya < 1)
        return fail(INMSOM_EARG, "inmsom_diag_noalloc: empty arrays %d..%d x %d..%d", b->bnd_x1,
                    b->bnd_x2, b->bnd_y1, b->bnd_y2);
    if (ld < nxa)
        return fail(INMSOM_EARG, "inmsom_diag_noalloc: ld = %lld is below the row length %lld",
                    ld, nxa);
    const bool empty = b->nx_start > b->nx_end || b->ny_start > b->ny_end;
    if (!empty && (b->nx_start < b->bnd_x1 || b->nx_end > b->bnd_x2 || b->ny_start < b->bnd_y1 ||
                   b->ny_end > b->bnd_y2))
        return fail(INMSOM_EARG, "inmsom_diag_noalloc: interior %d..%d x %d..%d outside the arrays",
                    b->nx_start, b->nx_end, b->ny_start, b->ny_end);
    const long long nrows = empty ? 0 : (long long)b->ny_end - b->ny_start + 1;
    if (nrows > INMSOM_DIAG_NOALLOC_MAX_ROWS)
        return fail(INMSOM_EARG,
                    "inmsom_diag_noalloc: %lld interior rows exceed INMSOM_DIAG_NOALLOC_MAX_ROWS "
                    "(%d); use inmsom_gpu_diag",
                    nrows, INMSOM_DIAG_NOALLOC_MAX_ROWS);

    double *rows = nullptr;
    int rc = rows_scratch(&rows);
    if (rc != INMSOM_OK) return rc;

    Dom d{};
    d.nx_start = b->nx_start; d.nx_end = b->nx_end; d.ny_start = b->ny_start; d.ny_end = b->ny_end;
    d.bnd_x1 = b->bnd_x1; d.bnd_x2 = b->bnd_x2; d.bnd_y1 = b->bnd_y1; d.bnd_y2 = b->bnd_y2;
    d.mmm = b->mmm; d.mm = b->mm; d.nnn = b->nnn; d.nn = b->nn;
    d.px = b->periodicity_x; d.py = b->periodicity_y;
    d.pitch = ld;
    d.xoff = 0;
    if (empty) { d.ny_end = d.ny_start - 1; d.nx_end = d.nx_start - 1; }

    GridDev g{};
    g.lu = lu; g.lcu = lcu; g.lcv = lcv;
    g.dx = dx; g.dy = dy; g.dxt = dxt; g.dyt = dyt; g.dxh = dxh; g.dyh = dyh;
    g.hrest = hhq_rest;
    Consts k{};
    k.ts = c->time_smooth; k.g = c->free_fall_acc; k.rho = c->ref_den; k.ffs = c->full_free_surface;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    general::diag_rows(d, g, k, ssh, u, v, hu, hv, rows, s);
    general::diag_final((int)nrows, rows, out, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(INMSOM_ECUDA, "inmsom_diag_noalloc: kernel launch failed: %s",
                    cudaGetErrorString(e));
    return INMSOM_OK;
}
