// C ABI of the barotropic checkpoint and restart (include/inmsom_gpu.h;
// the file formats are in dstd.cu).
#include "context.h"

namespace inmsom {
// Service/input_output_data.f90:4-115 fulfname (csrc/dstd.cu)
std::string full_file_name(const char *path, const char *fname);
}  // namespace inmsom

extern "C" {

namespace {

// one field pair of the checkpoint: the FP64 file, the FP32 file, the
// descriptor's name, its box and mask (Control/output.f90:1736-1847)
struct CpField {
    const char *f8, *f4, *ctl;
    int s0, s1;          // the two state fields
    int mask;            // M_LU, M_LLU, M_LLV
    int dx, dy;          // box starts at mmm - dx, nnn - dy
    const char *title, *var;
};
const CpField CP_FIELDS[3] = {
    {"cpsshe8.dat", "cpsshe.dat", "cpsshe.dat", S_SSH, S_SSHP, M_LU, 0, 0, "External SSH, m", "ssh"},
    {"cpube8.dat", "cpubi.dat", "cpube.dat", S_U, S_UP, M_LLU, 1, 0, "External UB, m/s", "ub"},
    {"cpvbe8.dat", "cpvbe.dat", "cpvbe.dat", S_V, S_VP, M_LLV, 0, 1, "External VB, m/s", "vb"},
};

}  // namespace

int inmsom_write_checkpoint(inmsom_ctx *c, const char *path, const inmsom_ctl_axes *ax)
{
    CKR(ensure_grid(c));
    if (!path || !ax || !ax->xt || !ax->xu || !ax->yt || !ax->yv)
        return set_err(INMSOM_EARG, "inmsom_write_checkpoint: NULL argument");
    if (!c->state_on_device) return set_err(INMSOM_EARG, "inmsom_write_checkpoint: no resident state");
    const Dom &d = c->dom;
    const int nx = d.nxa(), ny = d.nya();
    const size_t n = (size_t)nx * ny;
    std::vector<double> st(NSTATE * n);
    std::vector<float> mk(3 * n);
    for (int k = 0; k < NSTATE; k++) CKR(d2h(c, st.data() + k * n, c->state[k]));
    const int mids[3] = {M_LU, M_LLU, M_LLV};
    for (int k = 0; k < 3; k++) CKR(d2h(c, mk.data() + k * n, c->mask[mids[k]]));
    CKR(sync_stream(c));
    // 1-based positions in the (bnd_x1:bnd_x2, bnd_y1:bnd_y2) arrays
    const int i0 = d.mmm - d.bnd_x1 + 1, i1 = d.mm - d.bnd_x1 + 1;
    const int j0 = d.nnn - d.bnd_y1 + 1, j1 = d.nn - d.bnd_y1 + 1;
    const int nx_glob = d.mm - d.mmm + 1, ny_glob = d.nn - d.nnn + 1;
    const double zero = 0.0;
    std::vector<float> f4(n);
    for (const CpField &f : CP_FIELDS) {
        const float *lu = mk.data() + (f.mask == M_LU ? 0 : f.mask == M_LLU ? 1 : 2) * n;
        const int b[2] = {f.s0, f.s1};
        for (int t = 0; t < 2; t++) {
            double *fld = st.data() + b[t] * n;
            // the FP32 copy first: wdstd8 leaves the land points of its field at 0
            for (size_t q = 0; q < n; q++) f4[q] = (float)fld[q];
            CKR(inmsom_wdstd8(path, f.f8, t + 1, fld, lu, nx, ny, 1, i0 - f.dx, i1, j0 - f.dy, j1, 1, 1));
            CKR(inmsom_wdstd(path, f.f4, t + 1, f4.data(), lu, nx, ny, 1, i0 - f.dx, i1, j0 - f.dy, j1, 1, 1));
        }
        const std::string name = inmsom::full_file_name(path, f.ctl);   // fulfname, as the reference
        CKR(inmsom_ctl_file_write(name.c_str(), -1.0e32f, nx_glob + f.dx, ny_glob + f.dy, 1, 2, ax->xgr_type,
                                  f.dx ? ax->xu : ax->xt, ax->dxst, ax->ygr_type, f.dy ? ax->yv : ax->yt, ax->dyst,
                                  0, &zero, 1.0, ax->calendar, ax->year, ax->month, ax->day, ax->hour, ax->minute,
                                  ax->tstep, f.title, f.var));
    }
    return INMSOM_OK;
}

int inmsom_read_checkpoint(inmsom_ctx *c, const char *path, double *ubrtr_e, double *ubrtrp_e, double *vbrtr_e,
                           double *vbrtrp_e, double *ssh_e, double *sshp_e)
{
    CKR(ensure_grid(c));
    if (!path) return set_err(INMSOM_EARG, "inmsom_read_checkpoint: NULL path");
    const Dom &d = c->dom;
    const int nx = d.nxa(), ny = d.nya();
    const size_t n = (size_t)nx * ny;
    double *user[NSTATE] = {ubrtr_e, ubrtrp_e, vbrtr_e, vbrtrp_e, ssh_e, sshp_e};
    std::vector<double> st(NSTATE * n, 0.0);
    for (int k = 0; k < NSTATE; k++)
        if (user[k]) std::memcpy(st.data() + k * n, user[k], n * sizeof(double));
    std::vector<float> mk(3 * n);
    const int mids[3] = {M_LU, M_LLU, M_LLV};
    for (int k = 0; k < 3; k++) CKR(d2h(c, mk.data() + k * n, c->mask[mids[k]]));
    CKR(sync_stream(c));
    const int i0 = d.mmm - d.bnd_x1 + 1, i1 = d.mm - d.bnd_x1 + 1;
    const int j0 = d.nnn - d.bnd_y1 + 1, j1 = d.nn - d.bnd_y1 + 1;
    for (const CpField &f : CP_FIELDS) {
        const float *lu = mk.data() + (f.mask == M_LU ? 0 : f.mask == M_LLU ? 1 : 2) * n;
        const int b[2] = {f.s0, f.s1};
        for (int t = 0; t < 2; t++)
            CKR(inmsom_rdstd8(path, f.f8, t + 1, st.data() + b[t] * n, lu, nx, ny, 1, i0 - f.dx, i1, j0 - f.dy, j1,
                              1, 1));
    }
    for (int k = 0; k < NSTATE; k++) {
        CKR(h2d(c, c->state[k], (const double *)(st.data() + k * n)));
        general::halo(d, c->state[k], c->stream);           // cyclize8_x/_y when periodic
        CK(cudaGetLastError());
    }
    c->state_on_device = true;
    fused::mark_state_changed(c->plan);
    depths_from_state(c);
    for (int k = 0; k < NSTATE; k++)
        if (user[k]) CKR(d2h(c, user[k], c->state[k]));
    return sync_stream(c);
}

}  // extern "C"
