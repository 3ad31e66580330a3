// stages.hpp -- host-side launchers of the stage kernels and of the fused
// step, shared between the translation units of the library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "hcl_device.cuh"

namespace hcl {

// Count of kernel launches issued by this library (reported by
// hcl_kernel_launch_count()).
extern std::atomic<int64_t> g_launches;

namespace stage {

void conv_prim_to_cons(const GridDev& g, int ng_eff, const double* rho, const double* u, const double* P,
                       double* rhou, double* E, cudaStream_t s);
void conv_cons_to_prim(const GridDev& g, int ng_eff, const double* rho, const double* rhou, const double* E,
                       double* u, double* P, cudaStream_t s);
// analysis/temperature.hpp:18-25 on the range with ng_eff ghost layers
void temperature(const GridDev& g, int ng_eff, const double* rho, const double* P, double* T, cudaStream_t s);
void face_reconstruction(const GridDev& g, int ng_eff, const double* var, double* var_rec, cudaStream_t s);
void hydro_reconstruction(const GridDev& g, int ng_eff, double dt, const double* rho, const double* u,
                          const double* P, const double* fx, double* rho_rec, double* rhou_rec, double* E_rec,
                          double* fx_rec, double* u_rec, double* P_rec, double* fx_rec_old, cudaStream_t s);
void godunov(const GridDev& g, int ng_eff, double dt, const double* rho, const double* rhou, const double* E,
             const double* fx, const double* rho_rec, const double* rhou_rec, const double* E_rec,
             const double* fx_rec, double* rho_new, double* rhou_new, double* E_new, double* fx_new,
             cudaStream_t s);
void boundaries(const GridDev& g, double* rho, double* rhou, double* E, double* fx, cudaStream_t s);
// InternalMassGravity (gravity.cpp:59-128): the radial table g_r (n0 doubles)
// from rho, whose rows are `pitch` doubles apart (n0 for the reference
// layout, StateDev::pitch for the fused state); shell: nx0 + ng doubles
void internal_mass_gravity(const GridDev& g, const double* rho, int pitch, double central_mass, double* shell,
                           double* g_r, cudaStream_t s);
// pressure_fix.hpp:19-172 on no_ghosts: updates E_new in place
void pressure_fix(const GridDev& g, double dt, double eps, const double* rho, const double* rhou, const double* E,
                  const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* rho_new,
                  const double* rhou_new, double* E_new, cudaStream_t s);
// writes the bits of max_cells(sum_d (|u_d|+c)/dx_d) into *inv_bits (device),
// which must hold 0 before the call
void time_step_inv(const GridDev& g, int ng_eff, const double* rho, const double* u, const double* P,
                   unsigned long long* inv_bits, cudaStream_t s);
// min over interior cells of E - ek; *key must hold ~0ull, *nan_flag 0
void min_internal_energy(const GridDev& g, const double* rho, const double* rhou, const double* E,
                         unsigned long long* key, int* nan_flag, cudaStream_t s);
double decode_min_key(unsigned long long key);
// compensated sum of var*dv over the interior: partials must hold
// 2*integrate_blocks() doubles; result (sum, compensation) in out[0..1]
int integrate_blocks();
void integrate(const GridDev& g, const double* var, double* partials, double* out, cudaStream_t s);

} // namespace stage

namespace fused {

// Output columns of one warp strip of the 2-D mixed kernel (32 lanes less a
// 2-cell halo on each side).
constexpr int kStripLanesOut = 28;
// State buffers of the fused path: nvar planes, each n2*n1*pitch doubles with
// the x0 row padded to `pitch` (a multiple of 16 doubles).
struct StateDev {
    double* q;        // base of plane 0
    int64_t plane;    // doubles per plane
    int pitch;        // doubles per x0 row
};

// Computes 1/dt of the current state into ctl->inv_dt_bits[0], clears the
// other slots, sets t, iteration counters and flags for step 0.
void prologue(const GridDev& g, const StateDev& st, StepCtl* ctl, double t_ini, int iter0, cudaStream_t s);

// One fused step.  `slot` is the step counter modulo 6 (selects the control
// slots); out_buf is the index of the output state buffer.
void step_exact(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                int slot, int out_buf, cudaStream_t s);
void step_mixed(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                int slot, int out_buf, int shape, cudaStream_t s);
// fast FP64 (HCL_FP64_FAST): the FP64 tile kernels with the fast perfect-gas
// forms, built with FMA contraction
void step_fast64(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                 int slot, int out_buf, cudaStream_t s);
void configure_fast64();
int mixed_shape_count(int ndim);
bool mixed_shape_valid(const GridDev& g, int shape);
// Dynamic shared memory of the fused tile kernels for g (g.nfx passive
// scalars included), and the device's opt-in limit per block.
size_t mixed_smem_bytes(const GridDev& g, int shape);
size_t exact_smem_bytes(const GridDev& g);
int smem_optin();
// room left in the opt-in limit for the tile kernels' static shared memory
constexpr size_t kFusedStaticSmemMargin = 1024;
bool strip2d_eligible(const GridDev& g);
// 4-warp strips (schedules 3-6) with one passive scalar.
bool strip2d_fx_eligible(const GridDev& g);
// 3-D column march (uniform Cartesian grids, uniform gravity); L <= 0 fits
// the plane count per CTA to the resident CTAs.
bool strip3d_eligible(const GridDev& g);
// the column march with one passive scalar
bool strip3d_fx_eligible(const GridDev& g);
void step_strip3d(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                  int slot, int out_buf, int L, cudaStream_t s);
// sync: 16-warp CTAs marching in step; tma: their rows staged by the Tensor
// Memory Accelerator where strip2d_tma_eligible (per-lane cp.async otherwise)
void step_strip2d(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                  int slot, int out_buf, int L, bool sync, bool tma, cudaStream_t s);
bool strip2d_tma_eligible(const GridDev& g);
// Tiled tensor map of a state's first nv planes for the fused tile kernels'
// TMA staging: dims n0 x n1 (x n2) x nv, box {box[0], box[1], (box[2]), nv}
// (2-D and 3-D).  False where the driver offers no encoder, or the base or a
// stride is not a multiple of 16 bytes.
bool encode_tile_map(const GridDev& g, const StateDev& st, int nv, const int box[3], CUtensorMap* map);
void configure_exact();
void configure_mixed();
int conservation_partials_doubles(int ndim);

// Copies between the reference layout (contiguous LayoutLeft) and StateDev.
void pack_state(const GridDev& g, const StateDev& st, const double* rho, const double* rhou, const double* E,
                cudaMemcpyKind kind, cudaStream_t s);
void unpack_state(const GridDev& g, const StateDev& st, double* rho, double* rhou, double* E, cudaMemcpyKind kind,
                  cudaStream_t s);
// The g.nfx passive-scalar planes (after the ndim + 2 hydro planes); a null
// fx packs zeros.
void pack_fx(const GridDev& g, const StateDev& st, const double* fx, cudaMemcpyKind kind, cudaStream_t s);
void unpack_fx(const GridDev& g, const StateDev& st, double* fx, cudaMemcpyKind kind, cudaStream_t s);

// Compensated conservation sums of the fused state: out[0..ndim+1].
void conservation_sums(const GridDev& g, const StateDev& st, double* partials, double* out_dev, cudaStream_t s);

} // namespace fused

namespace ensemble {

// One problem of the batch: its grid, its two state buffers, its control
// block, dt log and its range of work items (warp strips).
struct Prob {
    GridDev g;
    double* q[2];
    int64_t plane;
    int pitch;
    int ncolw, nstrip;
    int item0;
    StepCtl* ctl;
    double* dt_log;
    int dt_cap;
    int64_t seg_stride; // segment mode: state s at q[0] + s * seg_stride
};

// polls of the ensemble's step barrier before it records HCL_ERR_TIMEOUT
// (each poll sleeps ~64 ns: a few seconds in all)
constexpr long long kSpinLimit = 1ll << 26;

struct Params {
    double cfl;
    int nsteps;
    int step0;   // global step index of the first step (slots and buffers)
    int L;       // strip rows
    int nitems;
    int nprob;
    int fixed_dt;
    const double* dts; // [nprob][dts_stride], indexed by iteration
    int dts_stride;
    int seg_mode;      // 1: step s reads state s and writes state s+1 of each segment buffer
    long long spin_limit;         // polls of the step barrier before HCL_ERR_TIMEOUT (> 0)
    unsigned int extra_arrivals;  // arrivals the step barrier waits for beyond the CTAs (tests only)
};

// Reverse pass of a batch: one problem's segment states, adjoint buffers,
// checkpoints and dts.
struct AdjProb {
    GridDev g;
    fused::StateDev seg0;  // segment state 0; state j at seg0.q + j * sz
    int64_t sz;            // doubles per state buffer
    fused::StateDev lam[3];  // rotating adjoint buffers (see reverse())
    const double* ckpt;    // checkpoints, sz apart
    StepCtl* ctl;          // control block of the recomputation
    const double* dts;     // dts of the forward run
    int tile0;             // first work item of this problem
};

struct AdjParams {
    int nprob;
    int ntiles;  // work items (16x16 tiles) over all problems
    int first;   // step index of the segment's first state
    int len;     // steps in the segment
    int cur;     // lam[cur] holds the adjoint of the segment's last output state;
                 // lam[(cur + 1) % 3] is zero on the interior
};

int reverse_blocks_per_sm(bool fp64);
// adjoint-tile size (16x16) of the batched reverse kernel
constexpr int kRevTile = 16;
void seg_init(const AdjProb* probs, int nprob, int sg, int first, cudaStream_t s);
cudaError_t reverse(bool fp64, int grid, const AdjProb* probs, const int* tile_prob, const AdjParams& ap,
                    unsigned int* barrier, int* status, cudaStream_t s);

int max_blocks_per_sm(int lim, int rs, int nw);
cudaError_t launch(int lim, int rs, int nw, int grid, const Prob* probs, const int* item_prob, const Params& ep,
                   unsigned int* barrier, int* status, cudaStream_t s);

} // namespace ensemble

namespace adjoint {

void configure();
// Whether the reverse sweep's tile with nfx passive scalars fits the current
// device's shared memory: *need bytes against the opt-in *avail.
int scalar_sweep_fits(int ndim, bool fp64, int nfx, size_t* need, size_t* avail);
// One adjoint step: lam_in (zero on entry) += (dU^{n+1}/dU^n)^T lam_out, with
// U = U^n and lam_out on interior cells (ghost entries zero); the
// contributions to ghost cells land on the interior cells they are filled
// from, so lam_in comes out folded.  The interior of lam_zero is cleared for
// the next step (a buffer neither read nor written by this one).
// gbar (internal-mass gravity, else nullptr): n0 doubles, zero on entry;
// receives dJ/dg_r of the radial table g.g_r the step read.
// exact_branches (FP64 sweep): the forward was the bit-exact FP64 step, whose
// rounding of the primitives the sweep reproduces to take its branches.
void step(const GridDev& g, const fused::StateDev& U, const fused::StateDev& lam_out, const fused::StateDev& lam_in,
          double dt, bool fp64, bool exact_branches, const fused::StateDev& lam_zero, double* gbar, cudaStream_t s);
// Internal-mass gravity: adds to the density adjoint of lam the part that
// flows through the step's gravity table (gbar from step()); shell_bar:
// nx0 + ng doubles of scratch.
void internal_mass_reverse(const GridDev& g, const double* gbar, double* shell_bar, const fused::StateDev& lam,
                           cudaStream_t s);
// Transpose of the boundary fill, in place on interior cells.
void fold(const GridDev& g, const fused::StateDev& lam, cudaStream_t s);
void zero_ghosts(const GridDev& g, const fused::StateDev& lam, cudaStream_t s);

} // namespace adjoint

} // namespace hcl
