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
// of this file's device image: the CUDA driver reserves it on each GPU when
// it loads the image there and keeps it until the process exits.  CUDA 12
// loads device images lazily by default, so on each device that happens at
// the first call here (the address look-up below), together with the
// reduction kernels' code -- not when the library is loaded.  A caller whose
// pool is about to claim the device's memory therefore makes one call (or
// runs with CUDA_MODULE_LOADING=EAGER) before the pool does.
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

// cuCtxGetCurrent from the driver, reached through the runtime (the library
// does not link libcuda): the address of the array belongs to one CUDA
// context, so the cache below keys on the context as well as the device.
typedef int (*CtxGetCurrentFn)(void **ctx);

std::mutex g_setup_mutex;
struct Resolved {
    void *ctx = nullptr;
    double *rows = nullptr;
};
Resolved g_rows_on_device[kMaxDevices];
CtxGetCurrentFn g_ctx_get_current = nullptr;

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
// comes from cudaGetSymbolAddress with that GPU current.  It is looked up
// once per device, on the first call there, and cached together with the
// CUDA context that was current; a call under another context of that
// device (after cudaDeviceReset, or with a context the caller made current
// through the driver) looks it up again for that context.
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
    if (!g_ctx_get_current) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult qr{};
        e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &qr);
        if (e != cudaSuccess || qr != cudaDriverEntryPointSuccess || !fn)
            return fail(INMSOM_ECUDA, "inmsom_diag_noalloc: cuCtxGetCurrent not found: %s",
                        cudaGetErrorString(e));
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    Resolved &r = g_rows_on_device[dev];
    void *ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0) ctx = nullptr;
    if (!ctx || r.ctx != ctx) {
        // first call on this device (or under a new context): the look-up
        // also makes the runtime's context current when none is yet
        void *addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_diag_rows);
        if (e != cudaSuccess || !addr)
            return fail(INMSOM_ECUDA,
                        "inmsom_diag_noalloc: cudaGetSymbolAddress of the scratch array on "
                        "device %d failed: %s",
                        dev, cudaGetErrorString(e));
        if (g_ctx_get_current(&ctx) != 0 || !ctx)
            return fail(INMSOM_ECUDA, "inmsom_diag_noalloc: no current CUDA context on device %d",
                        dev);
        r.ctx = ctx;
        r.rows = static_cast<double *>(addr);
    }
    *rows = r.rows;
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
    // an error left pending by an earlier, unrelated runtime call stays
    // pending for its owner: only an error these launches raise is taken
    // (and cleared) as this call's failure
    const cudaError_t before = cudaPeekAtLastError();
    general::diag_rows(d, g, k, ssh, u, v, hu, hv, rows, s);
    general::diag_final((int)nrows, rows, out, s);
    const cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess && e != before) {
        cudaGetLastError();
        return fail(INMSOM_ECUDA, "inmsom_diag_noalloc: kernel launch failed: %s",
                    cudaGetErrorString(e));
    }
    return INMSOM_OK;
}
