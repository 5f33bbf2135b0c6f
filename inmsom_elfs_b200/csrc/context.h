// Internal to the library: the context behind inmsom_ctx and the helpers
// its source files share (capi.cu, capi_column.cu, capi_io.cu).  Not part
// of the C ABI.
#pragma once

#include "inmsom_gpu.h"

#include <cstdarg>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "closure.h"
#include "fused.h"
#include "general.h"

namespace inmsom {
namespace capi {

// sets the message of inmsom_gpu_last_error() and returns code
int set_err(int code, const char *fmt, ...);

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            return set_err(INMSOM_ECUDA, "%s failed: %s (%s:%d)", #call,             \
                           cudaGetErrorString(e_), __FILE__, __LINE__);              \
    } while (0)

#define CKR(expr)                  \
    do {                           \
        int r_ = (expr);           \
        if (r_ != INMSOM_OK) return r_; \
    } while (0)

enum { M_LU, M_LUU, M_LUH, M_LCU, M_LCV, M_LLU, M_LLV, NMASK };
enum { G_DX, G_DY, G_DXT, G_DYT, G_DXH, G_DYH, G_DXB, G_DYB, G_RLH, G_HREST, NMET };
// external depths, in the argument order of hh_init/hh_shift
enum { H_Q, H_QP, H_QN, H_U, H_UP, H_UN, H_V, H_VP, H_VN, H_H, H_HP, H_HN, NDEPTH };
// saved state *_e, in barotropic_dynamics argument order
enum { S_U, S_UP, S_V, S_VP, S_SSH, S_SSHP, NSTATE };
enum { W_U, W_V, W_SSH, W_UP, W_VP, W_SSHP, W_UN, W_VN, W_SSHN, NWORK };
enum { A_UI, A_VI, A_GX, A_GY, NACC };
enum { F_RHSX, F_RHSY, F_WFLUX, F_MU, F_MU4, F_RDIS, NFORC };
enum { C_VORT, C_STRT, C_STRS, C_FX, C_FY, C_ADVX, C_ADVY, C_DIFX, C_DIFY, NSCR };
enum { I_SSH, I_SSHP, I_U, I_V, I_WFLUX, I_NEW, I_HQN, I_HUN, I_HVN, I_HHN, NINT };

}  // namespace capi
}  // namespace inmsom

using namespace inmsom;
using namespace inmsom::capi;

struct inmsom_ctx {
    Dom dom{};
    Consts c{};
    unsigned flags = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ph[4] = {};          // barotropic_dynamics phases: start, uploaded, computed, downloaded
    bool ph_valid = false;
    size_t nbytes = 0;  // one double field on the device

    float *mask[NMASK] = {};
    double *met[NMET] = {};
    double *depth[NDEPTH] = {};
    double *state[NSTATE] = {};
    double *work[NWORK] = {};
    double *acc[NACC] = {};
    double *forc[NFORC] = {};
    double *scr[NSCR] = {};
    double *intl[NINT] = {};
    double *tmp[4] = {};
    double *r2d[7] = {};             // inmsom_rhs2d: RHSx, RHSy, four inputs, a zero field (one block)
    double *v2d[9] = {};             // inmsom_velocity2d: its nine arrays (one block)
    // inmsom_baroclinic_dynamics / inmsom_vertical_velocity: fields of col_nz
    // levels in one block (col3, colw, col2) and dz, hzt
    double *col = nullptr, *col_lev = nullptr;
    int col_nz = 0;
    // inmsom_baroclinic_dynamics' copy pipeline: upload and download streams,
    // events per row band, and the phase times of a pipelined call
    cudaStream_t s_up = nullptr, s_dn = nullptr;
    cudaEvent_t bev[4 * 8 + 4] = {};
    float ph_ms[3] = {};
    bool ph_direct = false;
    // inmsom_tracer_tran_diff: fields of trc_nz levels in one block and dz, hzt
    double *trc = nullptr, *trc_lev = nullptr;
    int trc_nz = 0;
    std::vector<float> h_lu;          // the registered lu (argument checks)
    unsigned long long *d_nbad = nullptr;
    double *d_rows = nullptr, *d_out = nullptr;

    // host arrays registered / last passed
    double *h_depth[NDEPTH] = {};
    double *h_state[NSTATE] = {};
    double *h_scr[NSCR] = {};

    bool grid_ok = false;
    bool state_on_device = false;   // resident state has been uploaded
    bool depths_current = false;    // depth[] == hh_init(state) or evolved faithfully
    bool scratch_on_device = false;
    bool coef_on_device[NFORC] = {};   // INMSOM_STATIC_COEFFS: field copied in and current
    unsigned forc_gen = 1;           // changes whenever forc[] is written (the fused path's staging key)
    double *h_rs = nullptr;          // pinned staging of the per-substep RHS scales
    size_t h_rs_cap = 0;

    fused::Plan plan{};              // fused-path layout and eligibility
    // run_substeps as replays of a graph of rs_len (even, <= RS_GROUP) substeps
    cudaGraphExec_t rs_exec = nullptr;
    unsigned rs_gen = 0;
    const double *rs_src = nullptr;  // state set the graph reads first (an odd run moves the state)
    double rs_dt = 0.0;
    int rs_len = 0;
    // the forcing mode the graph's launches were captured with
    int rs_pgen = -1;
    double rs_mu0 = 0.0, rs_rd0 = 0.0, rs_wq0 = 0.0;
    double *d_rs = nullptr;          // RHS scale per substep of the run
    size_t rs_cap = 0;
    int *d_base = nullptr;           // first substep of the next replay
    // inmsom_run_closure: per-point tendency factors and the replayed graph
    double *cl_fac[2] = {};
    double *cl_tmp[3] = {};          // inmsom_closure_tendency: out u, out v, zero base
    cudaGraphExec_t cl_exec = nullptr;
    closure::Args cl_args{};         // the arguments the graph was captured with
    unsigned cl_gen = 0;
    double cl_dt = 0.0;
    int cl_every = 0, cl_groups = 0;
    bool fused_ok = false;
    const char *fused_reason = "grid not registered";

    GridDev gdev() const
    {
        GridDev g;
        g.lu = mask[M_LU]; g.luu = mask[M_LUU]; g.luh = mask[M_LUH];
        g.lcu = mask[M_LCU]; g.lcv = mask[M_LCV]; g.llu = mask[M_LLU]; g.llv = mask[M_LLV];
        g.dx = met[G_DX]; g.dy = met[G_DY]; g.dxt = met[G_DXT]; g.dyt = met[G_DYT];
        g.dxh = met[G_DXH]; g.dyh = met[G_DYH]; g.dxb = met[G_DXB]; g.dyb = met[G_DYB];
        g.rlh = met[G_RLH]; g.hrest = met[G_HREST];
        return g;
    }
};

namespace inmsom {
namespace capi {

template <typename T>
int dalloc(inmsom_ctx *c, T **p, size_t elem)
{
    size_t bytes = (size_t)c->dom.pitch * (size_t)c->dom.nya() * elem;
    CK(cudaMalloc((void **)p, bytes));
    CK(cudaMemsetAsync(*p, 0, bytes, c->stream));
    return INMSOM_OK;
}

template <typename T>
int h2d(inmsom_ctx *c, T *dev, const T *host)
{
    if (!host) return set_err(INMSOM_EARG, "NULL host array");
    const size_t w = (size_t)c->dom.nxa() * sizeof(T);
    CK(cudaMemcpy2DAsync(dev + c->dom.xoff, (size_t)c->dom.pitch * sizeof(T), host, w, w,
                         (size_t)c->dom.nya(), cudaMemcpyHostToDevice, c->stream));
    return INMSOM_OK;
}

template <typename T>
int d2h(inmsom_ctx *c, T *host, const T *dev)
{
    if (!host) return set_err(INMSOM_EARG, "NULL host array");
    const size_t w = (size_t)c->dom.nxa() * sizeof(T);
    CK(cudaMemcpy2DAsync(host, w, dev + c->dom.xoff, (size_t)c->dom.pitch * sizeof(T), w,
                         (size_t)c->dom.nya(), cudaMemcpyDeviceToHost, c->stream));
    return INMSOM_OK;
}

int check_bounds(const inmsom_bounds *b);
int sync_stream(inmsom_ctx *c);
int alloc_block(inmsom_ctx *c, double **arr, int n);
int alloc_set(inmsom_ctx *c, double **arr, int n);
void depths_from_state(inmsom_ctx *c);
int ensure_grid(inmsom_ctx *c);
int fused_flag_error(const inmsom_ctx *c, const char *who);
int run_guard(inmsom_ctx *c, long *nbad);

}  // namespace capi
}  // namespace inmsom
