// Fused streaming kernel of the barotropic step ("fused path").
//
// One kernel launch performs one whole leap-frog substep of
// Function/vel_ssh.f90:484-612 (continuity, depth update, stress,
// advection, viscosity, Coriolis, pressure gradient, drag, momentum,
// time-mean accumulation and Robert-Asselin filter with time shift) for the
// whole basin.  Each CTA owns a strip of columns and marches down a chunk of
// rows; input rows arrive through a ring of shared-memory slots filled by
// 3-D tiled TMA copies (cp.async.bulk.tensor, each copy for one CTA) of field-blocked
// arrays, tracked by mbarriers.
//
// Device layout of the fused path: a state set is ONE allocation holding the
// six *_e fields back to back (field stride = pitch * rows), so that one
// tensor-map box {36 columns, 1 row, 6 fields} brings a row segment of all
// of them; the static block holds the rest depth and the forcing the same
// way.  The caller's state must be such a block (state[k] = state[0] + k *
// pitch * rows).
//
// The fused path derives the external depths from SSH each substep
// (hq = H + ssh and its mask-weighted averages, which is what hh_init,
// hh_update and hh_shift produce up to rounding) and the derived masks from
// a 1-bit T mask, so per cell and substep it reads u, v, ssh at two levels,
// H and the forcing, and writes the six new state values: the 120 bytes of
// the algorithmic minimum plus one bit of mask.
//
// It is used when the grid allows (make_plan/check_eligible say why not):
// one domain whose halo is land, metrics and Coriolis constant along rows
// (every Cartesian or spherical INMSOM grid), no periodic wrap, full free
// surface, no biharmonic term.
#pragma once

#include <cuda.h>

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "inmsom_gpu.h"

namespace inmsom {
namespace fused {

constexpr int XOFF = 1;   // device padding columns before bnd_x1 (see common.cuh)

// fields of a state set, in memory order (the *_e argument order)
enum { S_U, S_UP, S_V, S_VP, S_SSH, S_SSHP, NSET };
// fields of the static block: rest depth, RHSx, RHSy (the uniform
// variant's ring holds these three), mu, rdis, wflux (the general variant's
// holds all six)
enum { T_H, T_RX, T_RY, T_MU, T_RD, T_WF, NSTAT };

// per-row coefficients, row index = device row (n - bnd_y1); 38 doubles so
// that a row is a whole number of 16-byte units for the bulk copies
struct RowCoef {
    double ku, ku2;           // hu: area(n)/(dxt*dyh)(n), and half of it
    double wv0, wv1;          // hv: area(n)/(dxh*dyt)(n), area(n+1)/(dxh*dyt)(n)
    double wh0, wh1;          // hh: area(n)/(dxb*dyb)(n), area(n+1)/(dxb*dyb)(n)
    double c_u, c_v0, c_v1;   // continuity: dyh(n)/area(n), dxh(n)/area(n), dxh(n-1)/area(n)
    double fx, fy;            // advection: dyh(n)/4, dxh(n)/4
    double gx0, gx1;          // GX_h: dyh(n)/4, dyh(n+1)/4
    double gy0, gy1;          // GY_T: dxh(n-1)/4, dxh(n)/4
    double cor;               // rlh_s(n)*dxb(n)*dyb(n)
    double vt0, vt1, vt2;     // vorticity metric terms: dyt-dyb, dxt(n+1)-dxb, dxt-dxb
    double t1, t2, t3;        // tension: dy/(dx*dyh), dx/(dy*dxh(n)), dx/(dy*dxh(n-1))
    double s1, s2, s3;        // shear: dxb/(dyb*dxt(n+1)), dxb/(dyb*dxt(n)), dyb/(dxb*dyt)
    double dux, dus0, dus1;   // u viscosity: dy^2/dyh, dxb^2/dxt, dxb(n-1)^2/dxt
    double dvt0, dvt1, dvs;   // v viscosity: dx^2/dxh, dx(n+1)^2/dxh, dyb^2/dyt
    double gdyh, gdxh;        // g*dyh, g*dxh
    double au, av;            // dxt*dyh, dyt*dxh
    double rau, rav;          // 1/(dxt*dyh), 1/(dyt*dxh)
    double pad;
};
static_assert(sizeof(RowCoef) % 16 == 0, "RowCoef must be a multiple of 16 bytes");

struct Plan {
    int ncol = 32;            // columns per CTA (one warp, one column per lane)
    int outw = 30;            // output columns per CTA
    int nstrips = 0;
    // work-item tables (item_table): uniform and general variant, plain and
    // time-mean substeps, and the FP32-velocity substep (their kernels hold
    // different numbers of CTAs per SM)
    int nitems[5] = {0, 0, 0, 0, 0};
    int4 *items[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // {g0, first row, end row, 0} per item
    bool uni = false;         // metrics all equal one spacing d (square uniform grid)
    double d = 0.0;           // that spacing
    long long min_pitch = 0;  // device row pitch the strips need
    // device data
    RowCoef *rows = nullptr;        // per-row coefficients (general variant)
    double *cor = nullptr;          // per-row rlh_s*d*d (uniform variant)
    uint32_t *bits = nullptr;       // 1-bit T mask, bm_words per row
    int bm_words = 0;
    double *buf[2][6] = {};         // the two ping-pong sets (field views)
    double *set[3] = {};            // base of each state set (field 0)
    double *stat = nullptr;         // static block, NSTAT fields
    long long fstride = 0;          // doubles between the fields of a block
    CUtensorMap tm_set[3];          // box {36, 1, 6} over each state set
    CUtensorMap tm_stat[2];         // box {36, 1, 3 | 6} over the static block
    int occ[5] = {0, 0, 0, 0, 0};   // resident CTAs per SM, per item table
    std::vector<uint8_t> ocean;     // per strip and interior row: any written column is ocean
    int rows_per_item[2] = {0, 0};  // 0: one wave of items by cost; else rows per item
    int min_rows = 4;               // no work item is shorter (an ensemble member: 16)
    // plain-substep items over rows extended into the halo (a row strip
    // that advances several substeps per exchange): per variant and number
    // of rows computed south / north of the interior, built on first use
    struct ExtTable {
        int gen, s, n, nitems;
        int4 *items;
    };
    std::vector<ExtTable> ext;
    unsigned generation = 0;        // bumped whenever buffers or work items change
    // prepare_steps: classification of the forcing for launch_steps
    bool prepared = false;
    unsigned staged_key = 0;        // key of the preparation the staged forcing belongs to (0: none)
    int prep_gen = 0;
    double prep_mu0 = 0.0, prep_rd0 = 0.0, prep_wq0 = 0.0;
    // FP32 velocity storage for run_substeps (uniform variant): per state
    // set, u up v vp in FP32 (same field stride), SSH stays in the FP64 set
    bool f32 = false;
    float *vset[3] = {};
    float *stat32 = nullptr;        // RHSx, RHSy in FP32
    CUtensorMap tm_vel[3];          // box {40, 1, 4} FP32 over each velocity set
    CUtensorMap tm_ssh[3];          // box {36, 1, 2} over the SSH fields of each state set
    CUtensorMap tm_stat_f32;        // box {36, 1, 1}: H alone, for the FP32-velocity ring
    CUtensorMap tm_rhs32;           // box {40, 1, 2} FP32 over stat32: RHSx, RHSy
    bool f32_land[3] = {false, false, false};   // vset[b] holds set b's values where the kernel does not write
    unsigned f32_rhs_key = 0;       // forcing key stat32 was converted for (0: stale)
    int stat_box[2] = {0, 0};       // static fields in tm_stat[v], checked against the ring layout
    int stat_box_f32 = 0;
    double *d_uniform = nullptr;    // per-block min/max of mu, rdis, wflux
    unsigned *d_flags = nullptr;    // [0] status bits (guard / timeout)
    const float *lu = nullptr;      // borrowed
    int nsm = 148;
    bool vort_zero = false;
    bool buffers_synced = false;    // buf[][] hold the state's land/halo values
    unsigned last_flags = 0;        // status bits of the last run
    // bounded waits: polls before giving up (0: the built-in 2^20); test
    // hook: item hold_item withholds the copies of its hold_row-th ring row
    unsigned wait_limit = 0;
    int hold_item = -1, hold_row = -1;
    int last_variant = -1;          // 0 uniform, 1 general, 2 uniform with FP32 velocities (last launch)
};

// status bits the fused kernel sets: a bounded wait gave up; the dynamic
// shared memory did not start on a 128-byte boundary (the ring's TMA slots
// need it; the kernel then does nothing).  The range/NaN guard is the
// separate k_guard pass (INMSOM_GUARD).
enum : unsigned { FLAG_TIMEOUT = 1u, FLAG_SMEM = 4u };

constexpr int NTABLE = 5;
constexpr int TABLE_F32 = 4;   // the FP32-velocity substep's items
// item table of an FP64 launch: variant (0 uniform, 1 general) + 2 for the
// substeps that accumulate time means (mode % 3 != 0)
inline int item_table(bool gen, int mode) { return (gen ? 1 : 0) + (mode % 3 != 0 ? 2 : 0); }

// The fused path writes only ocean points; land and halo points of the
// ping-pong sets must equal those of the state.  Call after the state was
// replaced from the host.
inline void mark_state_changed(Plan &p) { p.buffers_synced = false; }

Plan make_plan(const inmsom_bounds &b);
// nullptr if the fused path can run this grid, else the reason
const char *check_eligible(const Plan &p, const Dom &d, const Consts &c,
                           const float *const masks[7], const double *const grid[10]);
// build the row table and the bit mask, allocate the ping-pong sets and the
// static block, encode the tensor maps; state[] is the caller's state set
int setup(Plan &p, const Dom &d, const Consts &c, const float *const masks[7],
          const double *const grid[10], const double *d_hrest, const float *d_lu,
          double *state[NSET], cudaStream_t s);
// barotropic_dynamics(tau, nstep) on state[6] (in/out) with acc[4] out
int dynamics(Plan &p, const Dom &d, const Consts &c, double tau, int nstep,
             double *state[6], double *acc[4], double *forc[6], cudaStream_t s);
// nsub advancing substeps (the first substep of barotropic_dynamics(dt,1));
// returns 2 if FP32 velocity storage is asked for a grid that needs the
// general variant
int run_substeps(Plan &p, const Dom &d, const Consts &c, int nsub, double dt,
                 const double *rhs_scale, double *state[6], double *forc[6],
                 cudaStream_t s);
// Capture-friendly form of run_substeps for CUDA graphs (FP64): prepare_steps
// classifies the forcing and stages it (it synchronises the stream) -- or,
// given the nonzero key of its last preparation (the caller changes the key
// whenever it writes the forcing fields), keeps what it found then;
// launch_steps then only enqueues nsteps kernels, the RHS scale of launch k
// being rs_dev[*rs_base + k] read on the device, or rs_host when rs_dev is
// NULL (an even nsteps leaves the
// state in the same set, so the launches can be replayed); finish_steps
// reads the status bits.
int prepare_steps(Plan &p, const Dom &d, const Consts &c, double *state[6], double *forc[6],
                  cudaStream_t s, unsigned key = 0);
int launch_steps(Plan &p, const Dom &d, const Consts &c, double dt, int nsteps, const double *rs_dev,
                 const int *rs_base, double *state[6], cudaStream_t s, double rs_host = 1.0);
int finish_steps(Plan &p, cudaStream_t s);
// One plain substep (prepared by prepare_steps) over the interior rows and
// ext_s rows south / ext_n rows north of them, in the halo of a row strip
// whose halo is at least 2 rows wider than that on each side: a strip that
// advances k substeps per halo exchange of 2k rows computes 2(k-i) rows
// into its halo in substep i, which its neighbour computes alike.
int launch_step_ext(Plan &p, const Dom &d, const Consts &c, double dt, int ext_s, int ext_n, double *state[6],
                    cudaStream_t s, double rs_host);
// The FP32-velocity run in the same parts: prepare_steps_f32 also converts
// the state, the other ping-pong set and RHSx/RHSy to FP32 (returns 2 if the
// grid needs the general variant); launch_steps_f32 enqueues nsteps
// substeps, the RHS scale of launch k being rs_dev[*rs_base + k] or
// rs_host[k] (or 1); finish_steps_f32 writes the velocities back to the
// FP64 state and reads the status bits.
int prepare_steps_f32(Plan &p, const Dom &d, const Consts &c, double *state[6], double *forc[6],
                      cudaStream_t s, unsigned key = 0);
int launch_steps_f32(Plan &p, const Dom &d, const Consts &c, double dt, int nsteps, const double *rs_dev,
                     const int *rs_base, const double *rs_host, double *state[6], cudaStream_t s);
int finish_steps_f32(Plan &p, const Dom &d, double *state[6], cudaStream_t s);
// re-cut the work items: rows_per_item = 0 for one wave of items by cost
int repartition(Plan &p, const Dom &d, int rows_per_item, cudaStream_t s);
// Persistent ensemble launch: one cooperative launch of one wave of CTAs
// advances every member by `group` plain substeps (prepared by
// prepare_steps, RHS scale of substep k read at rs_dev[*rs_base + k]); its
// CTAs claim the members' work items in the order (substep, member, item),
// an item of a member waiting (bounded) until that member's items of the
// previous substep are done.  ens_table builds the device tables (the
// members' source/destination sets of both parities and item tables);
// ens_launch enqueues the counter resets and the launch (capturable).
struct EnsMemberIn {
    Plan *p;
    const Dom *d;
    const Consts *c;
    double dt;
    double *const *state;
};
struct EnsTable {
    void *d_mem = nullptr;
    int2 *d_order = nullptr;   // {member, item} per claim within a substep
    unsigned *d_ctr = nullptr, *d_done = nullptr;
    int nmem = 0, total = 0, group = 0, grid = 0;
    bool anygen = false;   // some member takes the general variant (fewer CTAs per SM)
    size_t smem = 0;
};
int ens_table(const std::vector<EnsMemberIn> &mem, int group, const double *rs_dev, const int *rs_base, EnsTable &t,
              cudaStream_t s);
int ens_launch(const EnsTable &t, cudaStream_t s);
void ens_free(EnsTable &t);
void free_plan(Plan &p);

}  // namespace fused
}  // namespace inmsom
