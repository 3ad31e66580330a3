// capi.cu -- implementation of the C ABI declared in include/heracles_b200.h.
//
// Owns the per-domain handle: configuration, the grid arrays built on the
// host exactly as Grid::set_grid builds them (mesh/grid.cpp:134-155,
// mesh/geometry.cpp:32-126, mesh/grid_type.cpp:151-186), their device copies,
// the fused-path state buffers and control block, and the CUDA graphs that
// replay chunks of fused steps.  No entry point throws; failures return a
// status and set the thread's last-error message.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "heracles_b200.h"
#include "hcl_device.cuh"
#include "stages.hpp"

using hcl::GridDev;
using hcl::RunParamsDev;
using hcl::StepCtl;
using hcl::fused::StateDev;

namespace {

thread_local std::string t_last_error;

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

#define HCL_CUDA(call)                                                                                         \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) {                                                                               \
            return fail(HCL_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
        }                                                                                                      \
    } while (0)

#define HCL_LAUNCH_CHECK()                                                                                  \
    do {                                                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                                \
        if (e_ != cudaSuccess) {                                                                            \
            return fail(HCL_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                          \
        }                                                                                                   \
    } while (0)

template <class T>
int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) {
        return HCL_OK;
    }
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(HCL_ERR_CUDA, "cudaMalloc of %zu bytes failed: %s", sizeof(T) * count, cudaGetErrorString(e));
    }
    return HCL_OK;
}

struct GraphKey {
    int k;
    int precision;
    int shape;
    RunParamsDev rp;
    bool operator<(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) < 0; }
};

} // namespace

namespace hcl::host {
// Shared with the host-only entry points (host/capi_host.cpp).
int set_error(int code, std::string const& msg)
{
    t_last_error = msg;
    return code;
}
} // namespace hcl::host

struct hcl_handle {
    hcl_config cfg{};
    GridDev g{};
    // host grid arrays
    std::vector<double> hx[3], hdx[3], hxc[3], hds, hdv, hgr, hcot, hsin1, hsinxc1;
    // device grid arrays
    double *dx_nodes[3] = {}, *ddx[3] = {}, *dxc[3] = {}, *dds = nullptr, *ddv = nullptr, *dgr = nullptr;
    double *dcot = nullptr, *dsin1 = nullptr, *dsinxc1 = nullptr;
    double* grav_shell = nullptr; // InternalMassGravity: shell means of rho (nx0 + ng)
    // stage-path scratch (MUSCLHancockHydroReconstruction's P_rec/u_rec, fx_rec_old)
    double *u_rec = nullptr, *P_rec = nullptr, *fx_rec_old = nullptr;
    // reductions
    unsigned long long* red_bits = nullptr;
    int* red_flag = nullptr;
    double* red_partials = nullptr;
    double* red_out = nullptr;
    // fused state
    double* state_mem[2] = {nullptr, nullptr};
    StateDev st[2]{};
    StepCtl* ctl = nullptr;
    StepCtl* ctl_tune = nullptr;
    int64_t counter = 0;   // fused steps launched since the last prologue
    int state_valid = 0;
    int cur = 0;           // buffer holding the current state when not running
    double t_base = 0.0;
    int iter_base = 0;
    int stopped = 0;
    int mixed_shape = -1;  // autotuned tile shape of the mixed 2-D kernel
    int force_stage = 0;   // hcl_set_stage_loop
    // dt log
    double* dt_log = nullptr;
    int dt_log_cap = 0;
    double* d_dts = nullptr;
    int d_dts_cap = 0;
    // stream and graphs
    cudaStream_t stream = nullptr;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    // discrete adjoint: checkpoints, segment states, adjoint state, dts
    double* adj_ckpt = nullptr;   // nck states
    double* adj_seg = nullptr;    // k+1 states
    double* adj_lam = nullptr;    // 3 states
    double* adj_gmem = nullptr;   // internal-mass gravity: 2 (k+1) radial tables, dJ/dg_r, 2 shell scratches
    int adj_cap_gmem = 0;         // doubles
    double* adj_ddts = nullptr;   // device copy of the dts
    StepCtl* adj_ctl = nullptr;
    std::vector<double> adj_dts;
    int adj_k = 0;
    int adj_nck = 0;
    int adj_cap_ck = 0;
    int adj_cap_seg = 0;
    int adj_prec = 0;
    int adj_ready = 0;
    int adj_ddts_cap = 0;
    // reference-layout state of the stage-composed loop (passive scalars or
    // pressure fix): one allocation, carved by stage_buffers()
    double* sl_mem = nullptr;
    // output scratch of hcl_get_prim: rho, rhou, E, u, P, T in the reference layout
    double* io_mem = nullptr;
    double *sl_rho = nullptr, *sl_rhou = nullptr, *sl_E = nullptr, *sl_fx = nullptr, *sl_u = nullptr, *sl_P = nullptr;
    double *sl_rho_rec = nullptr, *sl_rhou_rec = nullptr, *sl_E_rec = nullptr, *sl_fx_rec = nullptr;
    double *sl_rho_new = nullptr, *sl_rhou_new = nullptr, *sl_E_new = nullptr, *sl_fx_new = nullptr;
    double sl_t = 0.0;
    int sl_iter = 0;
    int sl_toid = -1, sl_ioid = -1;
    int sl_status = 0;
    std::vector<double> sl_dts;
    // second stream of the reverse pass: recomputes segment s-1 while the
    // main stream sweeps segment s back; events order the two segment buffers
    cudaStream_t adj_stream = nullptr;
    cudaEvent_t adj_ev_start = nullptr;
    cudaEvent_t adj_ev_rec[2] = {nullptr, nullptr};
    cudaEvent_t adj_ev_rev[2] = {nullptr, nullptr};
};

static int adjoint_backward_impl(hcl_handle* h, const double* lam_final, double* grad, int memory);

namespace {

void free_handle(hcl_handle* h)
{
    if (!h) {
        return;
    }
    for (auto& kv : h->graphs) {
        cudaGraphExecDestroy(kv.second);
    }
    cudaFree(h->io_mem);
    for (int d = 0; d < 3; ++d) {
        cudaFree(h->dx_nodes[d]);
        cudaFree(h->ddx[d]);
        cudaFree(h->dxc[d]);
    }
    cudaFree(h->dds);
    cudaFree(h->ddv);
    cudaFree(h->dgr);
    cudaFree(h->grav_shell);
    cudaFree(h->dcot);
    cudaFree(h->dsin1);
    cudaFree(h->dsinxc1);
    cudaFree(h->u_rec);
    cudaFree(h->P_rec);
    cudaFree(h->fx_rec_old);
    cudaFree(h->red_bits);
    cudaFree(h->red_flag);
    cudaFree(h->red_partials);
    cudaFree(h->red_out);
    cudaFree(h->state_mem[0]);
    cudaFree(h->state_mem[1]);
    cudaFree(h->ctl);
    cudaFree(h->ctl_tune);
    cudaFree(h->dt_log);
    cudaFree(h->d_dts);
    cudaFree(h->adj_ckpt);
    cudaFree(h->adj_seg);
    cudaFree(h->adj_lam);
    cudaFree(h->adj_gmem);
    cudaFree(h->adj_ddts);
    cudaFree(h->adj_ctl);
    cudaFree(h->sl_mem);
    for (cudaEvent_t ev : {h->adj_ev_start, h->adj_ev_rec[0], h->adj_ev_rec[1], h->adj_ev_rev[0], h->adj_ev_rev[1]}) {
        if (ev) {
            cudaEventDestroy(ev);
        }
    }
    if (h->adj_stream) {
        cudaStreamDestroy(h->adj_stream);
    }
    if (h->stream) {
        cudaStreamDestroy(h->stream);
    }
    delete h;
}

// Regular mesh (mesh/grid_type.cpp:151-186), cell sizes and centres
// (mesh/grid.cpp:31-44), ds/dv (mesh/geometry.cpp:32-126), point-mass
// gravity (gravity/gravity.cpp:49-55), on the host with libm.
void build_grid_host(hcl_handle* h)
{
    const hcl_config& c = h->cfg;
    const int nd = c.ndim;
    int n[3], nx[3];
    for (int d = 0; d < 3; ++d) {
        nx[d] = d < nd ? c.nx[d] : 1;
        n[d] = nx[d] + (d < nd ? 2 * c.nghost : 0);
    }
    for (int d = 0; d < 3; ++d) {
        h->hx[d].assign((size_t)n[d] + 1, 0.0);
        if (c.nodes[d]) {
            std::memcpy(h->hx[d].data(), c.nodes[d], sizeof(double) * ((size_t)n[d] + 1));
        } else {
            const int ngd = d < nd ? c.nghost : 0;
            const double dxd = (c.xmax[d] - c.xmin[d]) / nx[d];
            for (int i = 0; i < n[d] + 1; ++i) {
                h->hx[d][i] = c.xmin[d] + ((i - ngd) * dxd);
            }
        }
        h->hdx[d].assign(n[d], 0.0);
        h->hxc[d].assign(n[d], 0.0);
        for (int i = 0; i < n[d]; ++i) {
            h->hdx[d][i] = h->hx[d][i + 1] - h->hx[d][i];
            h->hxc[d][i] = (h->hx[d][i] + h->hx[d][i + 1]) / 2;
        }
    }
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    h->hds.assign((size_t)N * 3, 0.0);
    h->hdv.assign((size_t)N, 0.0);
    const double pi = hcl::kPi;
    const std::vector<double>& x0 = h->hx[0];
    const std::vector<double>& x1 = h->hx[1];
    for (int k = 0; k < n[2]; ++k) {
        for (int j = 0; j < n[1]; ++j) {
            for (int i = 0; i < n[0]; ++i) {
                const int64_t id = i + (int64_t)n[0] * (j + (int64_t)n[1] * k);
                const double dx0 = h->hdx[0][i], dx1 = h->hdx[1][j], dx2 = h->hdx[2][k];
                if (c.geometry == HCL_GEOM_CARTESIAN) {
                    for (int idim = 0; idim < 3; ++idim) {
                        double a[3] = {dx0, dx1, dx2};
                        a[idim] = 1;
                        h->hds[id + N * idim] = a[0] * a[1] * a[2];
                    }
                    h->hdv[id] = dx0 * dx1 * dx2;
                } else if (nd == 1) {
                    h->hds[id] = 4 * pi * x0[i] * x0[i];
                    h->hdv[id] = (4 * pi * ((x0[i + 1] * x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i] * x0[i]))) / 3;
                } else if (nd == 2) {
                    const double dcos = std::cos(x1[j]) - std::cos(x1[j + 1]);
                    h->hds[id] = 2 * pi * x0[i] * x0[i] * dcos;
                    h->hds[id + N] = (2 * pi / 2) * ((x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i])) * std::sin(x1[j]);
                    h->hdv[id] = (2 * pi / 3) * ((x0[i + 1] * x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i] * x0[i])) * dcos;
                } else {
                    const double dcos = std::cos(x1[j]) - std::cos(x1[j + 1]);
                    h->hds[id] = x0[i] * x0[i] * dcos * dx2;
                    h->hds[id + N] = (1. / 2) * ((x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i])) * std::sin(x1[j]) * dx2;
                    h->hds[id + 2 * N] = x0[i] * dx0 * dx1;
                    h->hdv[id] = (1. / 3) * ((x0[i + 1] * x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i] * x0[i])) * dcos * dx2;
                }
            }
        }
    }
    if (c.gravity == HCL_GRAVITY_POINT_MASS) {
        h->hgr.assign(n[0], 0.0);
        for (int i = 0; i < n[0]; ++i) {
            h->hgr[i] = -hcl::kG * c.central_mass / (h->hxc[0][i] * h->hxc[0][i]);
        }
    } else if (c.gravity == HCL_GRAVITY_INTERNAL_MASS) {
        h->hgr.assign(n[0], 0.0); // filled from the density (refresh_gravity)
    }
    // spherical trig factors per index (source_terms.hpp:38, :58-59, time_step.hpp:67)
    h->hcot.assign(n[1], 0.0);
    h->hsin1.assign((size_t)n[1] + 1, 0.0);
    h->hsinxc1.assign(n[1], 0.0);
    for (int j = 0; j < n[1]; ++j) {
        h->hcot[j] = std::cos((x1[j] + x1[j + 1]) / 2) / std::sin((x1[j] + x1[j + 1]) / 2);
        h->hsinxc1[j] = std::sin(h->hxc[1][j]);
    }
    for (int j = 0; j < n[1] + 1; ++j) {
        h->hsin1[j] = std::sin(x1[j]);
    }

    GridDev& g = h->g;
    g.ndim = nd;
    g.ng = c.nghost;
    g.nfx = c.nfx;
    for (int d = 0; d < 3; ++d) {
        g.n[d] = n[d];
        g.nx[d] = nx[d];
        g.g[d] = c.g[d];
    }
    g.N = N;
    g.geom = c.geometry;
    g.limiter = c.limiter;
    g.riemann = c.riemann;
    for (int f = 0; f < 6; ++f) {
        g.bc[f] = c.bc[f];
    }
    g.gravity = c.gravity;
    g.gamma = c.gamma;
    g.gamma_m1 = c.gamma - 1;
    g.mmw = c.mmw;
    g.eos = c.eos;
    g.pressure_fix = c.pressure_fix;
    g.eps_pf = c.eps_pf;
    // uniform spacing (to 1e-12 relative): with Cartesian geometry it enables
    // the fast forms of the mixed kernel; the adjoint needs it in any geometry
    int uniform = 1;
    for (int d = 0; d < nd; ++d) {
        const double ref = h->hdx[d][c.nghost];
        for (int i = 0; i < n[d] && uniform; ++i) {
            if (std::fabs(h->hdx[d][i] - ref) > 1e-12 * std::fabs(ref)) {
                uniform = 0;
            }
        }
        g.inv_dx[d] = 1.0 / ref;
    }
    for (int d = 0; d < 3; ++d) {
        g.inv_dx_f[d] = (float)g.inv_dx[d];
    }
    g.cfl_kc2 = (float)(0.5 * g.gamma * g.gamma_m1);
    g.uniform_dx = uniform;
    g.uniform_cart = uniform && c.geometry == HCL_GEOM_CARTESIAN;
}

int validate(const hcl_config* c)
{
    if (!c) {
        return fail(HCL_ERR_ARGUMENT, "null config");
    }
    if (c->pressure_fix && !(c->eps_pf > 0)) {
        return fail(HCL_ERR_CONFIG, "eps_pf must be > 0 with the pressure fix");
    }
    if (c->ndim < 1 || c->ndim > 3) {
        return fail(HCL_ERR_CONFIG, "ndim must be 1, 2 or 3 (got %d)", c->ndim);
    }
    // thermodynamics/perfect_gas.cpp:15-21
    if (!std::isfinite(c->gamma) || c->gamma <= 1) {
        return fail(HCL_ERR_DOMAIN, "Invalid gamma");
    }
    if (!std::isfinite(c->mmw) || c->mmw <= 0) {
        return fail(HCL_ERR_DOMAIN, "Invalid mmw");
    }
    if (c->nghost < 2 || c->nghost > 4) {
        return fail(HCL_ERR_CONFIG, "Nghost must be in [2, 4] (got %d)", c->nghost);
    }
    for (int d = 0; d < c->ndim; ++d) {
        if (c->nx[d] < c->nghost) {
            return fail(HCL_ERR_CONFIG, "Nx%d_glob = %d is smaller than Nghost", d, c->nx[d]);
        }
    }
    if (c->limiter < 0 || c->limiter > 3) {
        return fail(HCL_ERR_CONFIG, "Unknown face reconstruction algorithm id %d.", c->limiter);
    }
    if (c->riemann < 0 || c->riemann > 2) {
        return fail(HCL_ERR_CONFIG, "Invalid riemann solver id %d.", c->riemann);
    }
    for (int f = 0; f < 2 * c->ndim; ++f) {
        if (c->bc[f] < 0 || c->bc[f] > 2) {
            return fail(HCL_ERR_CONFIG, "Unknown boundary condition id %d on face %d.", c->bc[f], f);
        }
        // periodicity is a property of the pair of faces (ghost_sync wraps both)
    }
    if (c->geometry != HCL_GEOM_CARTESIAN && c->geometry != HCL_GEOM_SPHERICAL) {
        return fail(HCL_ERR_CONFIG, "Unknown geometry id %d", c->geometry);
    }
    if (c->gravity != HCL_GRAVITY_UNIFORM && c->gravity != HCL_GRAVITY_POINT_MASS &&
        c->gravity != HCL_GRAVITY_INTERNAL_MASS) {
        return fail(HCL_ERR_CONFIG, "Unknown gravity id %d", c->gravity);
    }
    if (c->precision != HCL_FP64 && c->precision != HCL_FP32_MIXED && c->precision != HCL_FP64_FAST) {
        return fail(HCL_ERR_CONFIG, "Unknown precision id %d", c->precision);
    }
    if (c->eos != HCL_EOS_PERFECT_GAS && c->eos != HCL_EOS_RAD_GAS) {
        return fail(HCL_ERR_CONFIG, "Unknown eos id %d", c->eos);
    }
    if (c->eos == HCL_EOS_RAD_GAS && c->precision != HCL_FP64) {
        // the FP32-mixed kernels use the perfect-gas algebra (P = (gamma-1) e)
        return fail(HCL_ERR_CONFIG, "the RadGas EOS needs precision HCL_FP64");
    }
    if (c->nfx < 0) {
        return fail(HCL_ERR_CONFIG, "nfx must be >= 0");
    }
    return HCL_OK;
}

cudaStream_t pick(hcl_handle* h, void* s)
{
    return s ? (cudaStream_t)s : h->stream;
}

int upload(double** dst, const std::vector<double>& src)
{
    int rc = dalloc(dst, src.size());
    if (rc) {
        return rc;
    }
    if (!src.empty()) {
        HCL_CUDA(cudaMemcpy(*dst, src.data(), sizeof(double) * src.size(), cudaMemcpyHostToDevice));
    }
    return HCL_OK;
}

int ensure_dt_log(hcl_handle* h, int need)
{
    if (need <= h->dt_log_cap) {
        return HCL_OK;
    }
    int cap = std::max(need, std::max(1024, 2 * h->dt_log_cap));
    double* p = nullptr;
    int rc = dalloc(&p, (size_t)cap);
    if (rc) {
        return rc;
    }
    if (h->dt_log && h->dt_log_cap > 0) {
        HCL_CUDA(cudaMemcpyAsync(p, h->dt_log, sizeof(double) * h->dt_log_cap, cudaMemcpyDeviceToDevice, h->stream));
        HCL_CUDA(cudaStreamSynchronize(h->stream));
        cudaFree(h->dt_log);
    }
    h->dt_log = p;
    h->dt_log_cap = cap;
    return HCL_OK;
}

int read_ctl(hcl_handle* h, StepCtl* out)
{
    HCL_CUDA(cudaMemcpyAsync(out, h->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, h->stream));
    HCL_CUDA(cudaStreamSynchronize(h->stream));
    return HCL_OK;
}

void launch_step(hcl_handle* h, const RunParamsDev& rp, int64_t counter, StepCtl* ctl, int in_buf, int shape,
                 cudaStream_t s)
{
    const int slot = (int)(counter % 6);
    const int out_buf = in_buf ^ 1;
    if (h->g.gravity == HCL_GRAVITY_INTERNAL_MASS) {
        // the radial gravity of the step's input density (main.cpp:309, :528)
        hcl::stage::internal_mass_gravity(h->g, h->st[in_buf].q, h->st[in_buf].pitch, h->cfg.central_mass,
                                          h->grav_shell, h->dgr, s);
    }
    if (h->cfg.precision == HCL_FP64) {
        hcl::fused::step_exact(h->g, h->st[in_buf], h->st[out_buf], ctl, rp, slot, out_buf, s);
    } else if (h->cfg.precision == HCL_FP64_FAST) {
        hcl::fused::step_fast64(h->g, h->st[in_buf], h->st[out_buf], ctl, rp, slot, out_buf, s);
    } else {
        hcl::fused::step_mixed(h->g, h->st[in_buf], h->st[out_buf], ctl, rp, slot, out_buf, shape, s);
    }
}

// Picks the fastest tile shape of the mixed 2-D kernel by timing a few steps
// that read the current state and write the other buffer with a scratch
// control block (the current state is not modified).
int autotune_mixed(hcl_handle* h)
{
    const int nshapes = hcl::fused::mixed_shape_count(h->g.ndim);
    h->mixed_shape = 0;
    if (nshapes <= 1) {
        return HCL_OK;
    }
    const char* env = std::getenv("HCL_MIXED_SHAPE");
    if (env) {
        h->mixed_shape = std::max(0, std::min(nshapes - 1, std::atoi(env)));
        if (!hcl::fused::mixed_shape_valid(h->g, h->mixed_shape)) {
            h->mixed_shape = 0;
        }
        return HCL_OK;
    }
    if (h->g.N < 65536) {
        return HCL_OK;
    }
    RunParamsDev rp;
    std::memset(&rp, 0, sizeof(rp));
    rp.cfl = 0.4;
    rp.t_end = 1e300;
    rp.max_iter = INT_MAX;
    rp.fixed_dt = 2;
    rp.dt_value = 0.0;
    cudaEvent_t e0, e1;
    HCL_CUDA(cudaEventCreate(&e0));
    HCL_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int sh = 0; sh < nshapes; ++sh) {
        if (!hcl::fused::mixed_shape_valid(h->g, sh)) {
            continue;
        }
        hcl::fused::prologue(h->g, h->st[h->cur], h->ctl_tune, 0.0, 0, h->stream);
        // warm-up, then time 4 launches that all read the same input
        for (int r = 0; r < 2; ++r) {
            launch_step(h, rp, 0, h->ctl_tune, h->cur, sh, h->stream);
        }
        HCL_CUDA(cudaEventRecord(e0, h->stream));
        for (int r = 0; r < 4; ++r) {
            launch_step(h, rp, 0, h->ctl_tune, h->cur, sh, h->stream);
        }
        HCL_CUDA(cudaEventRecord(e1, h->stream));
        HCL_CUDA(cudaEventSynchronize(e1));
        HCL_LAUNCH_CHECK();
        float ms = 0;
        HCL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            h->mixed_shape = sh;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return HCL_OK;
}

int get_graph(hcl_handle* h, const RunParamsDev& rp, int k, cudaGraphExec_t* out)
{
    GraphKey key;
    std::memset(&key, 0, sizeof(key));
    key.k = k;
    key.precision = h->cfg.precision;
    key.shape = h->mixed_shape;
    key.rp = rp;
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) {
        *out = it->second;
        return HCL_OK;
    }
    cudaGraph_t graph;
    HCL_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t before = hcl::g_launches.load();
    for (int s = 0; s < k; ++s) {
        launch_step(h, rp, s, h->ctl, s & 1, h->mixed_shape, h->stream);
    }
    hcl::g_launches = before; // counted at replay
    HCL_CUDA(cudaStreamEndCapture(h->stream, &graph));
    cudaGraphExec_t exec;
    HCL_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    h->graphs[key] = exec;
    *out = exec;
    return HCL_OK;
}

// Handles whose time loop is composed of the FP64 stage entry points: those
// that ask for it, and passive scalars too many for the fused tile's shared
// memory (the tiles carry the pressure fix in every precision).
bool stage_mode(const hcl_handle* h)
{
    if (h->force_stage) {
        return true;
    }
    if (h->cfg.nfx == 0) {
        return false;
    }
    const size_t bytes = h->cfg.precision == HCL_FP32_MIXED ? hcl::fused::mixed_smem_bytes(h->g, 0)
                                                             : hcl::fused::exact_smem_bytes(h->g);
    return bytes + hcl::fused::kFusedStaticSmemMargin > (size_t)hcl::fused::smem_optin();
}

// The reference-layout arrays of the stage-composed loop (main.cpp:187-205).
int stage_buffers(hcl_handle* h)
{
    if (h->sl_mem) {
        return HCL_OK;
    }
    const size_t N = (size_t)h->g.N, nd = (size_t)h->g.ndim, nf = (size_t)std::max(h->g.nfx, 1);
    const size_t sizes[14] = {N, N * nd, N, N * nf, N * nd, N, N * 2 * nd, N * 2 * nd * nd, N * 2 * nd,
                              N * 2 * nd * nf, N, N * nd, N, N * nf};
    size_t total = 0;
    for (size_t v : sizes) {
        total += v;
    }
    int rc = dalloc(&h->sl_mem, total);
    if (rc) {
        return rc;
    }
    HCL_CUDA(cudaMemset(h->sl_mem, 0, sizeof(double) * total));
    double** ptrs[14] = {&h->sl_rho,     &h->sl_rhou,     &h->sl_E,       &h->sl_fx,        &h->sl_u,
                         &h->sl_P,       &h->sl_rho_rec,  &h->sl_rhou_rec, &h->sl_E_rec,   &h->sl_fx_rec,
                         &h->sl_rho_new, &h->sl_rhou_new, &h->sl_E_new,   &h->sl_fx_new};
    double* q = h->sl_mem;
    for (int i = 0; i < 14; ++i) {
        *ptrs[i] = q;
        q += sizes[i];
    }
    return HCL_OK;
}

// Normalises the fused state after a finished run so that it sits in buffer 0
// with a fresh control block (t and iteration carried over).
int restart_clock(hcl_handle* h, double t, int iter)
{
    if (h->cur != 0) {
        const size_t bytes = sizeof(double) * (size_t)h->st[0].plane * (h->g.ndim + 2 + h->g.nfx);
        HCL_CUDA(cudaMemcpyAsync(h->st[0].q, h->st[1].q, bytes, cudaMemcpyDeviceToDevice, h->stream));
        h->cur = 0;
    }
    hcl::fused::prologue(h->g, h->st[0], h->ctl, t, iter, h->stream);
    HCL_LAUNCH_CHECK();
    h->counter = 0;
    h->stopped = 0;
    h->t_base = t;
    h->iter_base = iter;
    return HCL_OK;
}

} // namespace

extern "C" {

int hcl_abi_version(void)
{
    return HCL_ABI_VERSION;
}

const char* hcl_last_error(void)
{
    return t_last_error.c_str();
}

int64_t hcl_kernel_launch_count(void)
{
    return hcl::g_launches.load();
}

int hcl_get_stream(const hcl_handle* h, void** stream)
{
    if (!h || !stream) {
        return fail(HCL_ERR_ARGUMENT, "null argument");
    }
    *stream = (void*)h->stream;
    return HCL_OK;
}

void hcl_config_default(hcl_config* c)
{
    if (!c) {
        return;
    }
    std::memset(c, 0, sizeof(*c));
    // utils/param.cpp:14-73
    c->ndim = 1;
    c->nx[0] = c->nx[1] = c->nx[2] = 1;
    c->nghost = 2;
    c->nfx = 0;
    c->geometry = HCL_GEOM_CARTESIAN;
    c->gamma = 5. / 3;
    c->mmw = 1.;
    c->limiter = HCL_LIMITER_VANLEER;
    c->riemann = HCL_RIEMANN_HLL;
    for (int f = 0; f < 6; ++f) {
        c->bc[f] = HCL_BC_PERIODIC;
    }
    c->gravity = HCL_GRAVITY_UNIFORM;
    c->central_mass = 1.0;
    for (int d = 0; d < 3; ++d) {
        c->xmin[d] = 0.0;
        c->xmax[d] = 1.0;
    }
    c->precision = HCL_FP64;
    c->device = 0;
    c->pressure_fix = 0;
    c->eps_pf = 0.000001;
    c->eos = HCL_EOS_PERFECT_GAS;
}

int hcl_create(const hcl_config* cfg, hcl_handle** out)
{
    if (!out) {
        return fail(HCL_ERR_ARGUMENT, "null output handle");
    }
    *out = nullptr;
    int rc = validate(cfg);
    if (rc) {
        return rc;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(HCL_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (cfg->device < 0 || cfg->device >= ndev) {
        return fail(HCL_ERR_CONFIG, "device %d out of range (%d devices)", cfg->device, ndev);
    }
    HCL_CUDA(cudaSetDevice(cfg->device));
    hcl::fused::configure_exact();
    hcl::fused::configure_fast64();
    hcl::fused::configure_mixed();
    hcl::adjoint::configure();
    HCL_CUDA(cudaGetLastError());
    hcl_handle* h = new hcl_handle();
    h->cfg = *cfg;
    for (int d = 0; d < 3; ++d) {
        h->cfg.nodes[d] = nullptr; // not retained
    }
    hcl_config tmp = *cfg;
    h->cfg = tmp;
    build_grid_host(h);
    for (int d = 0; d < 3; ++d) {
        h->cfg.nodes[d] = nullptr;
    }
    auto bail = [&](int code) {
        free_handle(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        return bail(fail(HCL_ERR_CUDA, "cudaStreamCreate failed"));
    }
    GridDev& g = h->g;
    for (int d = 0; d < 3; ++d) {
        if ((rc = upload(&h->dx_nodes[d], h->hx[d])) || (rc = upload(&h->ddx[d], h->hdx[d])) ||
            (rc = upload(&h->dxc[d], h->hxc[d]))) {
            return bail(rc);
        }
        g.x[d] = h->dx_nodes[d];
        g.dx[d] = h->ddx[d];
        g.xc[d] = h->dxc[d];
    }
    if ((rc = upload(&h->dds, h->hds)) || (rc = upload(&h->ddv, h->hdv)) || (rc = upload(&h->dgr, h->hgr)) ||
        (rc = upload(&h->dcot, h->hcot)) || (rc = upload(&h->dsin1, h->hsin1)) ||
        (rc = upload(&h->dsinxc1, h->hsinxc1))) {
        return bail(rc);
    }
    if (h->cfg.gravity == HCL_GRAVITY_INTERNAL_MASS &&
        (rc = dalloc(&h->grav_shell, (size_t)(g.nx[0] + g.ng)))) {
        return bail(rc);
    }
    g.ds = h->dds;
    g.dv = h->ddv;
    g.g_r = h->dgr;
    g.cot_mid1 = h->dcot;
    g.sin1 = h->dsin1;
    g.sin_xc1 = h->dsinxc1;

    const int nd = g.ndim;
    const int nv = nd + 2;
    if ((rc = dalloc(&h->red_bits, 4)) || (rc = dalloc(&h->red_flag, 4)) ||
        (rc = dalloc(&h->red_partials,
                     (size_t)std::max(2 * hcl::stage::integrate_blocks(), hcl::fused::conservation_partials_doubles(nd)))) ||
        (rc = dalloc(&h->red_out, 16))) {
        return bail(rc);
    }
    // fused state: nv + nfx planes of n2*n1*pitch doubles, pitch a multiple of 16
    const int pitch = (g.n[0] + 15) / 16 * 16;
    const int64_t plane = (int64_t)pitch * g.n[1] * g.n[2];
    const size_t nplanes = (size_t)(nv + g.nfx);
    for (int b = 0; b < 2; ++b) {
        if ((rc = dalloc(&h->state_mem[b], (size_t)plane * nplanes))) {
            return bail(rc);
        }
        HCL_CUDA(cudaMemset(h->state_mem[b], 0, sizeof(double) * (size_t)plane * nplanes));
        h->st[b].q = h->state_mem[b];
        h->st[b].plane = plane;
        h->st[b].pitch = pitch;
    }
    if ((rc = dalloc(&h->ctl, 1)) || (rc = dalloc(&h->ctl_tune, 1))) {
        return bail(rc);
    }
    HCL_CUDA(cudaMemset(h->ctl, 0, sizeof(StepCtl)));
    *out = h;
    return HCL_OK;
}

int hcl_destroy(hcl_handle* h)
{
    if (h) {
        cudaSetDevice(h->cfg.device);
        cudaStreamSynchronize(h->stream);
    }
    free_handle(h);
    return HCL_OK;
}

int hcl_get_config(const hcl_handle* h, hcl_config* out)
{
    if (!h || !out) {
        return fail(HCL_ERR_ARGUMENT, "null handle or output");
    }
    *out = h->cfg;
    for (int d = 0; d < 3; ++d) {
        out->nodes[d] = nullptr;
    }
    return HCL_OK;
}

int hcl_get_extents(const hcl_handle* h, int n_wg[3], int64_t* ncells)
{
    if (!h) {
        return fail(HCL_ERR_ARGUMENT, "null handle");
    }
    for (int d = 0; d < 3; ++d) {
        if (n_wg) {
            n_wg[d] = h->g.n[d];
        }
    }
    if (ncells) {
        *ncells = h->g.N;
    }
    return HCL_OK;
}

int hcl_get_interior(const hcl_handle* h, int nx[3], int* nghost)
{
    if (!h) {
        return fail(HCL_ERR_ARGUMENT, "null handle");
    }
    for (int d = 0; d < 3; ++d) {
        if (nx) {
            nx[d] = h->g.nx[d];
        }
    }
    if (nghost) {
        *nghost = h->g.ng;
    }
    return HCL_OK;
}

int hcl_get_grid(const hcl_handle* h, double* x[3], double* dx[3], double* xc[3], double* ds, double* dv)
{
    if (!h) {
        return fail(HCL_ERR_ARGUMENT, "null handle");
    }
    for (int d = 0; d < 3; ++d) {
        if (x && x[d]) {
            std::memcpy(x[d], h->hx[d].data(), sizeof(double) * h->hx[d].size());
        }
        if (dx && dx[d]) {
            std::memcpy(dx[d], h->hdx[d].data(), sizeof(double) * h->hdx[d].size());
        }
        if (xc && xc[d]) {
            std::memcpy(xc[d], h->hxc[d].data(), sizeof(double) * h->hxc[d].size());
        }
    }
    if (ds) {
        std::memcpy(ds, h->hds.data(), sizeof(double) * h->hds.size());
    }
    if (dv) {
        std::memcpy(dv, h->hdv.data(), sizeof(double) * h->hdv.size());
    }
    return HCL_OK;
}

int hcl_get_grid_device(const hcl_handle* h, const double* dx[3], const double** ds, const double** dv)
{
    if (!h) {
        return fail(HCL_ERR_ARGUMENT, "null handle");
    }
    for (int d = 0; d < 3; ++d) {
        if (dx) {
            dx[d] = h->ddx[d];
        }
    }
    if (ds) {
        *ds = h->dds;
    }
    if (dv) {
        *dv = h->ddv;
    }
    return HCL_OK;
}

// ---- stage entry points ----------------------------------------------------
#define HCL_CHECK_HANDLE(h)                              \
    do {                                                 \
        if (!(h)) {                                      \
            return fail(HCL_ERR_ARGUMENT, "null handle"); \
        }                                                \
        HCL_CUDA(cudaSetDevice((h)->cfg.device));        \
    } while (0)

#define HCL_CHECK_NGEFF(h, ng_eff)                                                                    \
    do {                                                                                             \
        if ((ng_eff) < 0 || (ng_eff) > (h)->g.ng) {                                                  \
            return fail(HCL_ERR_CONFIG, "NgEff > Ng"); /* range.cpp:370-372 */                        \
        }                                                                                            \
    } while (0)

int hcl_conv_prim_to_cons(hcl_handle* h, int ng_eff, const double* rho, const double* u, const double* P,
                          double* rhou, double* E, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (!rho || !u || !P || !rhou || !E) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    hcl::stage::conv_prim_to_cons(h->g, ng_eff, rho, u, P, rhou, E, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_conv_cons_to_prim(hcl_handle* h, int ng_eff, const double* rho, const double* rhou, const double* E,
                          double* u, double* P, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (!rho || !u || !P || !rhou || !E) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    hcl::stage::conv_cons_to_prim(h->g, ng_eff, rho, rhou, E, u, P, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_temperature(hcl_handle* h, int ng_eff, const double* rho, const double* P, double* T, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (!rho || !P || !T) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    hcl::stage::temperature(h->g, ng_eff, rho, P, T, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_face_reconstruction(hcl_handle* h, int ng_eff, const double* var, double* var_rec, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (ng_eff > h->g.ng - 1) {
        return fail(HCL_ERR_CONFIG, "face reconstruction needs one ghost layer beyond the range");
    }
    if (!var || !var_rec) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    hcl::stage::face_reconstruction(h->g, ng_eff, var, var_rec, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_hydro_reconstruction(hcl_handle* h, int ng_eff, double dt, const double* rho, const double* u,
                             const double* P, const double* fx, double* rho_rec, double* rhou_rec, double* E_rec,
                             double* fx_rec, double* u_rec, double* P_rec, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (ng_eff > h->g.ng - 1) {
        return fail(HCL_ERR_CONFIG, "reconstruction needs one ghost layer beyond the range");
    }
    if (!rho || !u || !P || !rho_rec || !rhou_rec || !E_rec) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    if (h->g.nfx > 0 && (!fx || !fx_rec)) {
        return fail(HCL_ERR_ARGUMENT, "nfx > 0 needs fx and fx_rec");
    }
    const int nd = h->g.ndim;
    const size_t N = (size_t)h->g.N;
    int rc;
    if (!u_rec) {
        if (!h->u_rec && (rc = dalloc(&h->u_rec, N * 2 * nd * nd))) {
            return rc;
        }
        u_rec = h->u_rec;
    }
    if (!P_rec) {
        if (!h->P_rec && (rc = dalloc(&h->P_rec, N * 2 * nd))) {
            return rc;
        }
        P_rec = h->P_rec;
    }
    if (h->g.nfx > 0 && !h->fx_rec_old && (rc = dalloc(&h->fx_rec_old, N * 2 * nd * h->g.nfx))) {
        return rc;
    }
    hcl::stage::hydro_reconstruction(h->g, ng_eff, dt, rho, u, P, fx, rho_rec, rhou_rec, E_rec, fx_rec, u_rec, P_rec,
                                     h->fx_rec_old, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_godunov_scheme(hcl_handle* h, int ng_eff, double dt, const double* rho, const double* rhou,
                       const double* E, const double* fx, const double* rho_rec, const double* rhou_rec,
                       const double* E_rec, const double* fx_rec, double* rho_new, double* rhou_new, double* E_new,
                       double* fx_new, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (ng_eff > h->g.ng - 2 + 0 && ng_eff > 0) {
        return fail(HCL_ERR_CONFIG, "the Godunov update reads face states one cell beyond the range");
    }
    if (!rho || !rhou || !E || !rho_rec || !rhou_rec || !E_rec || !rho_new || !rhou_new || !E_new) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    if (h->g.nfx > 0 && (!fx || !fx_rec || !fx_new)) {
        return fail(HCL_ERR_ARGUMENT, "nfx > 0 needs fx, fx_rec and fx_new");
    }
    hcl::stage::godunov(h->g, ng_eff, dt, rho, rhou, E, fx, rho_rec, rhou_rec, E_rec, fx_rec, rho_new, rhou_new, E_new,
                        fx_new, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_pressure_fix(hcl_handle* h, double dt, double eps, const double* rho, const double* rhou, const double* E,
                     const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* rho_new,
                     const double* rhou_new, double* E_new, void* stream)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !rhou || !E || !rho_rec || !rhou_rec || !E_rec || !rho_new || !rhou_new || !E_new) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    hcl::stage::pressure_fix(h->g, dt, eps, rho, rhou, E, rho_rec, rhou_rec, E_rec, rho_new, rhou_new, E_new,
                             pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_boundary_conditions(hcl_handle* h, double* rho, double* rhou, double* E, double* fx, void* stream)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !rhou || !E || (h->g.nfx > 0 && !fx)) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    hcl::stage::boundaries(h->g, rho, rhou, E, fx, pick(h, stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_internal_mass_gravity(hcl_handle* h, const double* rho, double* g_out, void* stream)
{
    HCL_CHECK_HANDLE(h);
    if (h->g.gravity != HCL_GRAVITY_INTERNAL_MASS) {
        return fail(HCL_ERR_CONFIG, "the handle was not created with HCL_GRAVITY_INTERNAL_MASS");
    }
    if (!rho) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    cudaStream_t s = pick(h, stream);
    hcl::stage::internal_mass_gravity(h->g, rho, h->g.n[0], h->cfg.central_mass, h->grav_shell, h->dgr, s);
    if (g_out) {
        HCL_CUDA(cudaMemcpyAsync(g_out, h->dgr, sizeof(double) * (size_t)h->g.n[0], cudaMemcpyDeviceToDevice, s));
    }
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_time_step(hcl_handle* h, int ng_eff, const double* rho, const double* u, const double* P, double* dt_out,
                  void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (!rho || !u || !P || !dt_out) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    cudaStream_t s = pick(h, stream);
    HCL_CUDA(cudaMemsetAsync(h->red_bits, 0, sizeof(unsigned long long), s));
    hcl::stage::time_step_inv(h->g, ng_eff, rho, u, P, h->red_bits, s);
    HCL_LAUNCH_CHECK();
    unsigned long long bits = 0;
    HCL_CUDA(cudaMemcpyAsync(&bits, h->red_bits, sizeof(bits), cudaMemcpyDeviceToHost, s));
    HCL_CUDA(cudaStreamSynchronize(s));
    double inv;
    std::memcpy(&inv, &bits, sizeof(inv));
    *dt_out = 1 / inv; // time_step.hpp:82
    return HCL_OK;
}

int hcl_minimum_internal_energy(hcl_handle* h, const double* rho, const double* rhou, const double* E, double* out,
                                void* stream)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !rhou || !E || !out) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    cudaStream_t s = pick(h, stream);
    HCL_CUDA(cudaMemsetAsync(h->red_bits, 0xff, sizeof(unsigned long long), s));
    HCL_CUDA(cudaMemsetAsync(h->red_flag, 0, sizeof(int), s));
    hcl::stage::min_internal_energy(h->g, rho, rhou, E, h->red_bits, h->red_flag, s);
    HCL_LAUNCH_CHECK();
    unsigned long long key = 0;
    int nanf = 0;
    HCL_CUDA(cudaMemcpyAsync(&key, h->red_bits, sizeof(key), cudaMemcpyDeviceToHost, s));
    HCL_CUDA(cudaMemcpyAsync(&nanf, h->red_flag, sizeof(nanf), cudaMemcpyDeviceToHost, s));
    HCL_CUDA(cudaStreamSynchronize(s));
    *out = nanf ? NAN : hcl::stage::decode_min_key(key);
    return HCL_OK;
}

int hcl_integrate(hcl_handle* h, const double* var, double* out, void* stream)
{
    HCL_CHECK_HANDLE(h);
    if (!var || !out) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    cudaStream_t s = pick(h, stream);
    hcl::stage::integrate(h->g, var, h->red_partials, h->red_out, s);
    HCL_LAUNCH_CHECK();
    double res[2];
    HCL_CUDA(cudaMemcpyAsync(res, h->red_out, sizeof(res), cudaMemcpyDeviceToHost, s));
    HCL_CUDA(cudaStreamSynchronize(s));
    *out = res[0];
    return HCL_OK;
}

// ---- handle-owned state ----------------------------------------------------
// InternalMassGravity handles: the radial gravity table of the current state
// (main.cpp:309 after the initial state, :528 after every step).
static int refresh_gravity(hcl_handle* h)
{
    if (h->g.gravity != HCL_GRAVITY_INTERNAL_MASS || !h->state_valid) {
        return HCL_OK;
    }
    const double* rho = stage_mode(h) ? h->sl_rho : h->st[h->cur].q;
    const int pitch = stage_mode(h) ? h->g.n[0] : h->st[h->cur].pitch;
    hcl::stage::internal_mass_gravity(h->g, rho, pitch, h->cfg.central_mass, h->grav_shell, h->dgr, h->stream);
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

int hcl_set_state(hcl_handle* h, const double* rho, const double* rhou, const double* E, const double* fx,
                  int memory)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !rhou || !E) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    const cudaMemcpyKind kind = memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (stage_mode(h)) {
        int rc = stage_buffers(h);
        if (rc) {
            return rc;
        }
        const size_t N = (size_t)h->g.N, nd = (size_t)h->g.ndim;
        cudaStream_t s = h->stream;
        HCL_CUDA(cudaMemcpyAsync(h->sl_rho, rho, sizeof(double) * N, kind, s));
        HCL_CUDA(cudaMemcpyAsync(h->sl_rhou, rhou, sizeof(double) * N * nd, kind, s));
        HCL_CUDA(cudaMemcpyAsync(h->sl_E, E, sizeof(double) * N, kind, s));
        if (h->g.nfx > 0) {
            if (fx) {
                HCL_CUDA(cudaMemcpyAsync(h->sl_fx, fx, sizeof(double) * N * h->g.nfx, kind, s));
            } else {
                HCL_CUDA(cudaMemsetAsync(h->sl_fx, 0, sizeof(double) * N * h->g.nfx, s));
            }
        }
        // main.cpp:311
        if ((rc = hcl_conv_cons_to_prim(h, h->g.ng, h->sl_rho, h->sl_rhou, h->sl_E, h->sl_u, h->sl_P, s))) {
            return rc;
        }
        HCL_CUDA(cudaStreamSynchronize(s));
        h->state_valid = 1;
        if ((rc = refresh_gravity(h))) {
            return rc;
        }
        return hcl_reset_clock(h, 0.0);
    }
    hcl::fused::pack_state(h->g, h->st[0], rho, rhou, E, kind, h->stream);
    hcl::fused::pack_fx(h->g, h->st[0], fx, kind, h->stream);
    HCL_CUDA(cudaGetLastError());
    h->cur = 0;
    h->state_valid = 1;
    int rc = refresh_gravity(h);
    return rc ? rc : restart_clock(h, 0.0, 0);
}

int hcl_get_state(hcl_handle* h, double* rho, double* rhou, double* E, double* fx, int memory)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !rhou || !E) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    const cudaMemcpyKind kind = memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (stage_mode(h)) {
        const size_t N = (size_t)h->g.N, nd = (size_t)h->g.ndim;
        cudaStream_t s = h->stream;
        HCL_CUDA(cudaMemcpyAsync(rho, h->sl_rho, sizeof(double) * N, kind, s));
        HCL_CUDA(cudaMemcpyAsync(rhou, h->sl_rhou, sizeof(double) * N * nd, kind, s));
        HCL_CUDA(cudaMemcpyAsync(E, h->sl_E, sizeof(double) * N, kind, s));
        if (fx && h->g.nfx > 0) {
            HCL_CUDA(cudaMemcpyAsync(fx, h->sl_fx, sizeof(double) * N * h->g.nfx, kind, s));
        }
        HCL_CUDA(cudaStreamSynchronize(s));
        return HCL_OK;
    }
    hcl::fused::unpack_state(h->g, h->st[h->cur], rho, rhou, E, kind, h->stream);
    if (fx) {
        hcl::fused::unpack_fx(h->g, h->st[h->cur], fx, kind, h->stream);
    }
    HCL_CUDA(cudaGetLastError());
    HCL_CUDA(cudaStreamSynchronize(h->stream));
    return HCL_OK;
}

int hcl_get_prim(hcl_handle* h, double* rho, double* u, double* P, double* T, double* fx, int memory)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !u || !P) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    const size_t N = (size_t)h->g.N, nd = (size_t)h->g.ndim;
    int rc;
    if (!h->io_mem && (rc = dalloc(&h->io_mem, N * (4 + 2 * nd)))) {
        return rc;
    }
    double* d_rho = h->io_mem;
    double* d_rhou = d_rho + N;
    double* d_E = d_rhou + N * nd;
    double* d_u = d_E + N;
    double* d_P = d_u + N * nd;
    double* d_T = d_P + N;
    if ((rc = hcl_get_state(h, d_rho, d_rhou, d_E, nullptr, HCL_DEVICE))) {
        return rc;
    }
    cudaStream_t s = h->stream;
    // main.cpp:526 and :317-318: cons -> prim and the temperature over all ghosts
    hcl::stage::conv_cons_to_prim(h->g, h->g.ng, d_rho, d_rhou, d_E, d_u, d_P, s);
    hcl::stage::temperature(h->g, h->g.ng, d_rho, d_P, d_T, s);
    HCL_LAUNCH_CHECK();
    const cudaMemcpyKind kind = memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    HCL_CUDA(cudaMemcpyAsync(rho, d_rho, sizeof(double) * N, kind, s));
    HCL_CUDA(cudaMemcpyAsync(u, d_u, sizeof(double) * N * nd, kind, s));
    HCL_CUDA(cudaMemcpyAsync(P, d_P, sizeof(double) * N, kind, s));
    if (T) {
        HCL_CUDA(cudaMemcpyAsync(T, d_T, sizeof(double) * N, kind, s));
    }
    if (fx && h->g.nfx > 0) {
        if (stage_mode(h)) {
            HCL_CUDA(cudaMemcpyAsync(fx, h->sl_fx, sizeof(double) * N * h->g.nfx, kind, s));
        } else {
            hcl::fused::unpack_fx(h->g, h->st[h->cur], fx, kind, s);
            HCL_CUDA(cudaGetLastError());
        }
    }
    HCL_CUDA(cudaStreamSynchronize(s));
    return HCL_OK;
}

int hcl_set_clock(hcl_handle* h, double t, int iter)
{
    HCL_CHECK_HANDLE(h);
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    if (iter < 0) {
        return fail(HCL_ERR_ARGUMENT, "negative iteration count");
    }
    if (stage_mode(h)) {
        h->sl_t = t;
        h->sl_iter = iter;
        h->sl_toid = h->sl_ioid = -1;
        h->sl_status = 0;
        h->sl_dts.clear();
        return HCL_OK;
    }
    return restart_clock(h, t, iter);
}

int hcl_set_state_from_prim(hcl_handle* h, const double* rho, const double* u, const double* P, const double* fx)
{
    HCL_CHECK_HANDLE(h);
    if (!rho || !u || !P) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    const int nd = h->g.ndim;
    const size_t N = (size_t)h->g.N;
    int rc;
    if (stage_mode(h)) {
        // main.cpp:305-311 on the reference-layout arrays
        if ((rc = stage_buffers(h))) {
            return rc;
        }
        cudaStream_t s = h->stream;
        HCL_CUDA(cudaMemcpyAsync(h->sl_rho, rho, sizeof(double) * N, cudaMemcpyHostToDevice, s));
        HCL_CUDA(cudaMemcpyAsync(h->sl_u, u, sizeof(double) * N * nd, cudaMemcpyHostToDevice, s));
        HCL_CUDA(cudaMemcpyAsync(h->sl_P, P, sizeof(double) * N, cudaMemcpyHostToDevice, s));
        HCL_CUDA(cudaMemsetAsync(h->sl_rhou, 0, sizeof(double) * N * nd, s));
        HCL_CUDA(cudaMemsetAsync(h->sl_E, 0, sizeof(double) * N, s));
        if (h->g.nfx > 0) {
            if (fx) {
                HCL_CUDA(cudaMemcpyAsync(h->sl_fx, fx, sizeof(double) * N * h->g.nfx, cudaMemcpyHostToDevice, s));
            } else {
                HCL_CUDA(cudaMemsetAsync(h->sl_fx, 0, sizeof(double) * N * h->g.nfx, s));
            }
        }
        if ((rc = hcl_conv_prim_to_cons(h, 0, h->sl_rho, h->sl_u, h->sl_P, h->sl_rhou, h->sl_E, s)) ||
            (rc = hcl_boundary_conditions(h, h->sl_rho, h->sl_rhou, h->sl_E, h->g.nfx > 0 ? h->sl_fx : nullptr, s)) ||
            (rc = hcl_conv_cons_to_prim(h, h->g.ng, h->sl_rho, h->sl_rhou, h->sl_E, h->sl_u, h->sl_P, s))) {
            return rc;
        }
        HCL_CUDA(cudaStreamSynchronize(s));
        h->state_valid = 1;
        if ((rc = refresh_gravity(h))) {
            return rc;
        }
        return hcl_reset_clock(h, 0.0);
    }
    const size_t nf = (size_t)h->g.nfx;
    double *d_rho = nullptr, *d_u = nullptr, *d_P = nullptr, *d_m = nullptr, *d_E = nullptr, *d_fx = nullptr;
    if ((rc = dalloc(&d_rho, N)) || (rc = dalloc(&d_u, N * nd)) || (rc = dalloc(&d_P, N)) ||
        (rc = dalloc(&d_m, N * nd)) || (rc = dalloc(&d_E, N)) || (nf > 0 && (rc = dalloc(&d_fx, N * nf)))) {
        cudaFree(d_rho);
        cudaFree(d_u);
        cudaFree(d_P);
        cudaFree(d_m);
        cudaFree(d_E);
        cudaFree(d_fx);
        return rc;
    }
    cudaStream_t s = h->stream;
    cudaMemcpyAsync(d_rho, rho, sizeof(double) * N, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_u, u, sizeof(double) * N * nd, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_P, P, sizeof(double) * N, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_m, 0, sizeof(double) * N * nd, s);
    cudaMemsetAsync(d_E, 0, sizeof(double) * N, s);
    if (nf > 0) {
        if (fx) {
            cudaMemcpyAsync(d_fx, fx, sizeof(double) * N * nf, cudaMemcpyHostToDevice, s);
        } else {
            cudaMemsetAsync(d_fx, 0, sizeof(double) * N * nf, s);
        }
    }
    // main.cpp:305-307: conv_prim_to_cons(no_ghosts) then the boundaries
    hcl::stage::conv_prim_to_cons(h->g, 0, d_rho, d_u, d_P, d_m, d_E, s);
    hcl::stage::boundaries(h->g, d_rho, d_m, d_E, d_fx, s);
    hcl::fused::pack_state(h->g, h->st[0], d_rho, d_m, d_E, cudaMemcpyDeviceToDevice, s);
    hcl::fused::pack_fx(h->g, h->st[0], d_fx, cudaMemcpyDeviceToDevice, s);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(d_rho);
    cudaFree(d_u);
    cudaFree(d_P);
    cudaFree(d_m);
    cudaFree(d_E);
    cudaFree(d_fx);
    if (e != cudaSuccess) {
        return fail(HCL_ERR_CUDA, "initial state: %s", cudaGetErrorString(e));
    }
    h->cur = 0;
    h->state_valid = 1;
    if ((rc = refresh_gravity(h))) {
        return rc;
    }
    return restart_clock(h, 0.0, 0);
}

int hcl_reset_clock(hcl_handle* h, double t_ini)
{
    HCL_CHECK_HANDLE(h);
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    if (stage_mode(h)) {
        h->sl_t = t_ini;
        h->sl_iter = 0;
        h->sl_toid = h->sl_ioid = -1;
        h->sl_status = 0;
        h->sl_dts.clear();
        return HCL_OK;
    }
    return restart_clock(h, t_ini, 0);
}

// The reference time loop (main.cpp:354-531) composed of the FP64 stage entry
// points on the reference-layout arrays: dt and the health check are read back
// each step, as the reference does.
static int run_stage_loop(hcl_handle* h, const hcl_run_params* p, hcl_run_result* r)
{
    if (h->sl_status) {
        return fail(HCL_ERR_INVALID_STATE, "the state is invalid; set a new state");
    }
    if (p->fixed_dt && (!p->dts || p->nsteps <= 0)) {
        return fail(HCL_ERR_ARGUMENT, "fixed_dt needs dts and nsteps > 0");
    }
    cudaStream_t s = h->stream;
    const int ng = h->g.ng;
    const bool pf = h->cfg.pressure_fix != 0;
    const bool has_fx = h->g.nfx > 0;
    int rc;
    int done = 0;
    int status = 0;
    bool finished = false;
    double last_dt = 0.0;
    while (p->nsteps <= 0 || done < p->nsteps) {
        double dt;
        if (p->fixed_dt) {
            dt = p->dts[done];
        } else {
            double dt_inv = 0.0;
            if ((rc = hcl_time_step(h, ng, h->sl_rho, h->sl_u, h->sl_P, &dt_inv, s))) {
                return rc;
            }
            dt = p->cfl * dt_inv; // main.cpp:355
        }
        bool should_exit = false;
        if (p->iter_frequency > 0) { // main.cpp:358-364
            const int next_output = (h->sl_ioid + 1) * p->iter_frequency;
            if ((h->sl_iter + 1) >= next_output) {
                ++h->sl_ioid;
            }
        }
        if (p->time_frequency > 0) { // main.cpp:365-375
            const double next_output = p->time_first_output + ((h->sl_toid + 1) * p->time_frequency);
            if ((h->sl_t + dt) >= next_output) {
                dt = next_output - h->sl_t;
                if (dt <= 0) {
                    status = HCL_ERR_NEGATIVE_DT;
                    break;
                }
                ++h->sl_toid;
            }
        }
        if ((h->sl_t + dt) >= p->t_end) { // main.cpp:377-381
            dt = p->t_end - h->sl_t;
            should_exit = true;
        }
        if ((h->sl_iter + 1) >= p->max_iter) { // main.cpp:382-385
            should_exit = true;
        }
        double min_evol = 0.0; // main.cpp:397-425
        if ((rc = hcl_minimum_internal_energy(h, h->sl_rho, h->sl_rhou, h->sl_E, &min_evol, s))) {
            return rc;
        }
        if (std::isnan(min_evol) || min_evol < 0) {
            status = HCL_ERR_INVALID_STATE;
            break;
        }
        h->sl_dts.push_back(dt);
        double* const fxp = has_fx ? h->sl_fx : nullptr; // the buffers swap every step
        // main.cpp:427-479
        if ((rc = hcl_hydro_reconstruction(h, 1, dt / 2, h->sl_rho, h->sl_u, h->sl_P, fxp, h->sl_rho_rec,
                                           h->sl_rhou_rec, h->sl_E_rec, fxp ? h->sl_fx_rec : nullptr, nullptr,
                                           nullptr, s)) ||
            (rc = hcl_godunov_scheme(h, 0, dt, h->sl_rho, h->sl_rhou, h->sl_E, fxp, h->sl_rho_rec, h->sl_rhou_rec,
                                     h->sl_E_rec, fxp ? h->sl_fx_rec : nullptr, h->sl_rho_new, h->sl_rhou_new,
                                     h->sl_E_new, fxp ? h->sl_fx_new : nullptr, s))) {
            return rc;
        }
        if (pf && (rc = hcl_pressure_fix(h, dt, h->cfg.eps_pf, h->sl_rho, h->sl_rhou, h->sl_E, h->sl_rho_rec,
                                         h->sl_rhou_rec, h->sl_E_rec, h->sl_rho_new, h->sl_rhou_new, h->sl_E_new,
                                         s))) {
            return rc;
        }
        if ((rc = hcl_boundary_conditions(h, h->sl_rho_new, h->sl_rhou_new, h->sl_E_new,
                                          fxp ? h->sl_fx_new : nullptr, s))) {
            return rc;
        }
        // main.cpp:481-484: the new state becomes the current one
        std::swap(h->sl_rho, h->sl_rho_new);
        std::swap(h->sl_rhou, h->sl_rhou_new);
        std::swap(h->sl_E, h->sl_E_new);
        std::swap(h->sl_fx, h->sl_fx_new);
        if ((rc = hcl_conv_cons_to_prim(h, ng, h->sl_rho, h->sl_rhou, h->sl_E, h->sl_u, h->sl_P, s))) {
            return rc;
        }
        if (h->g.gravity == HCL_GRAVITY_INTERNAL_MASS) { // main.cpp:528
            hcl::stage::internal_mass_gravity(h->g, h->sl_rho, h->g.n[0], h->cfg.central_mass, h->grav_shell,
                                              h->dgr, s);
        }
        h->sl_t += dt; // main.cpp:530-531
        ++h->sl_iter;
        ++done;
        last_dt = dt;
        if (should_exit) {
            finished = true;
            break;
        }
    }
    HCL_CUDA(cudaStreamSynchronize(s));
    HCL_LAUNCH_CHECK();
    if (r) {
        r->t = h->sl_t;
        r->iter = h->sl_iter;
        r->status = status;
        r->bad_cell = -1;
        r->finished = finished ? 1 : 0;
        r->last_dt = last_dt;
    }
    if (status == HCL_ERR_INVALID_STATE) {
        h->sl_status = status;
        return fail(HCL_ERR_INVALID_STATE, "detected invalid volumic internal energy");
    }
    if (status == HCL_ERR_NEGATIVE_DT) {
        h->sl_status = status;
        return fail(HCL_ERR_NEGATIVE_DT, "Error: the time step is negative");
    }
    return HCL_OK;
}

int hcl_run(hcl_handle* h, const hcl_run_params* p, hcl_run_result* r)
{
    HCL_CHECK_HANDLE(h);
    if (!p) {
        return fail(HCL_ERR_ARGUMENT, "null run parameters");
    }
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    if (stage_mode(h)) {
        return run_stage_loop(h, p, r);
    }
    int rc;
    StepCtl ctl;
    if (h->stopped) {
        // resume after a finished run: carry t and iteration over
        if ((rc = read_ctl(h, &ctl))) {
            return rc;
        }
        if (ctl.err) {
            return fail(HCL_ERR_INVALID_STATE, "the state is invalid; set a new state");
        }
        if ((rc = restart_clock(h, ctl.t[h->counter & 1], ctl.iter[h->counter & 1]))) {
            return rc;
        }
    }
    if (h->cfg.precision == HCL_FP32_MIXED && h->mixed_shape < 0) {
        if ((rc = autotune_mixed(h))) {
            return rc;
        }
    }
    RunParamsDev rp;
    std::memset(&rp, 0, sizeof(rp));
    rp.cfl = p->cfl;
    rp.t_end = p->t_end;
    rp.max_iter = p->max_iter;
    rp.iter_frequency = p->iter_frequency;
    rp.time_frequency = p->time_frequency;
    rp.time_first_output = p->time_first_output;
    rp.fixed_dt = p->fixed_dt ? 1 : 0;
    const int nsteps = p->nsteps;
    if ((rc = read_ctl(h, &ctl))) {
        return rc;
    }
    const int iter_now = ctl.iter[h->counter & 1];
    const int horizon = nsteps > 0 ? iter_now + nsteps : std::min(p->max_iter, iter_now + (1 << 20));
    if ((rc = ensure_dt_log(h, horizon + 8))) {
        return rc;
    }
    rp.dt_log = h->dt_log;
    rp.dt_log_cap = h->dt_log_cap;
    if (p->fixed_dt) {
        if (!p->dts || nsteps <= 0) {
            return fail(HCL_ERR_ARGUMENT, "fixed_dt needs dts and nsteps > 0");
        }
        if (h->d_dts_cap < horizon + 8) {
            cudaFree(h->d_dts);
            h->d_dts = nullptr;
            h->d_dts_cap = 0;
            if ((rc = dalloc(&h->d_dts, (size_t)horizon + 8))) {
                return rc;
            }
            h->d_dts_cap = horizon + 8;
        }
        HCL_CUDA(cudaMemsetAsync(h->d_dts, 0, sizeof(double) * h->d_dts_cap, h->stream));
        HCL_CUDA(cudaMemcpyAsync(h->d_dts + iter_now, p->dts, sizeof(double) * nsteps, cudaMemcpyHostToDevice,
                                 h->stream));
        rp.dts = h->d_dts;
    }
    const int K = p->graph_chunk > 0 ? (p->graph_chunk + 5) / 6 * 6 : 60;
    const int shape = h->mixed_shape < 0 ? 0 : h->mixed_shape;
    // A run of a fixed step count replays the largest of these graphs that
    // fits, again and again, then launches the last < 6 steps singly.  All of
    // them are built (captured once per run parameters) on the first such
    // call, so that later calls of any step count replay graphs only.
    int sizes[4] = {K, 24, 12, 6};
    int nsizes = 1;
    for (int i = 1; i < 4; ++i) {
        if (sizes[i] < K) {
            sizes[nsizes++] = sizes[i];
        }
    }
    if (nsteps > 0) {
        for (int i = 0; i < nsizes; ++i) {
            cudaGraphExec_t exec;
            if ((rc = get_graph(h, rp, sizes[i], &exec))) {
                return rc;
            }
        }
    }

    auto single = [&]() {
        launch_step(h, rp, h->counter, h->ctl, (int)(h->counter & 1), shape, h->stream);
        ++h->counter;
    };
    int done = 0;
    bool finished = false;
    while (!finished) {
        // align to the graph's slot phase with single launches
        while (h->counter % 6 != 0 && (nsteps <= 0 || done < nsteps)) {
            single();
            ++done;
        }
        const int remaining = nsteps > 0 ? nsteps - done : K;
        int chunk = 0;
        for (int i = 0; i < nsizes && chunk == 0; ++i) {
            if (remaining >= sizes[i]) {
                chunk = sizes[i];
            }
        }
        if (chunk > 0) {
            cudaGraphExec_t exec;
            if ((rc = get_graph(h, rp, chunk, &exec))) {
                return rc;
            }
            HCL_CUDA(cudaGraphLaunch(exec, h->stream));
            hcl::g_launches += chunk;
            h->counter += chunk;
            done += chunk;
        } else {
            while (done < nsteps) {
                single();
                ++done;
            }
        }
        HCL_LAUNCH_CHECK();
        if (nsteps > 0) {
            finished = done >= nsteps;
        } else {
            if ((rc = read_ctl(h, &ctl))) {
                return rc;
            }
            finished = ctl.stop[h->counter & 1] || ctl.errflag[h->counter & 1] || ctl.err;
        }
    }
    if ((rc = read_ctl(h, &ctl))) {
        return rc;
    }
    const int q = (int)(h->counter & 1);
    const bool stop = ctl.stop[q] || ctl.err;
    h->cur = stop ? ctl.final_buf : q;
    h->stopped = stop ? 1 : 0;
    if ((rc = refresh_gravity(h))) {
        return rc;
    }
    if (r) {
        r->t = ctl.t[q];
        r->iter = ctl.iter[q];
        r->status = ctl.err;
        r->bad_cell = ctl.bad_cell == ~0ull ? -1 : (int64_t)ctl.bad_cell;
        r->finished = ctl.stop[q] ? 1 : 0;
        r->last_dt = ctl.last_dt;
    }
    if (ctl.err == HCL_ERR_INVALID_STATE) {
        return fail(HCL_ERR_INVALID_STATE, "detected invalid volumic internal energy at cell %lld",
                    (long long)(ctl.bad_cell == ~0ull ? -1 : (long long)ctl.bad_cell));
    }
    if (ctl.err == HCL_ERR_NEGATIVE_DT) {
        return fail(HCL_ERR_NEGATIVE_DT, "Error: the time step is negative");
    }
    if (ctl.err == HCL_ERR_TIMEOUT) {
        return fail(HCL_ERR_TIMEOUT, "a bounded device-side wait for a staged state row gave up");
    }
    return HCL_OK;
}

int hcl_step_fixed_dt(hcl_handle* h, double dt, void* stream)
{
    HCL_CHECK_HANDLE(h);
    if (stage_mode(h)) {
        return fail(HCL_ERR_CONFIG, "hcl_step_fixed_dt runs the fused step (no passive scalars, no pressure fix)");
    }
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    if (h->stopped) {
        StepCtl ctl;
        int rc = read_ctl(h, &ctl);
        if (rc) {
            return rc;
        }
        if ((rc = restart_clock(h, ctl.t[h->counter & 1], ctl.iter[h->counter & 1]))) {
            return rc;
        }
    }
    if (h->cfg.precision == HCL_FP32_MIXED && h->mixed_shape < 0) {
        int rc = autotune_mixed(h);
        if (rc) {
            return rc;
        }
    }
    RunParamsDev rp;
    std::memset(&rp, 0, sizeof(rp));
    rp.cfl = 0.4;
    rp.t_end = 1e300;
    rp.max_iter = INT_MAX;
    rp.fixed_dt = 2;
    rp.dt_value = dt;
    cudaStream_t s = pick(h, stream);
    launch_step(h, rp, h->counter, h->ctl, (int)(h->counter & 1), h->mixed_shape < 0 ? 0 : h->mixed_shape, s);
    ++h->counter;
    h->cur = (int)(h->counter & 1);
    HCL_LAUNCH_CHECK();
    if (h->g.gravity == HCL_GRAVITY_INTERNAL_MASS) {
        hcl::stage::internal_mass_gravity(h->g, h->st[h->cur].q, h->st[h->cur].pitch, h->cfg.central_mass,
                                          h->grav_shell, h->dgr, s);
        HCL_LAUNCH_CHECK();
    }
    return HCL_OK;
}

int hcl_set_stage_loop(hcl_handle* h, int on)
{
    HCL_CHECK_HANDLE(h);
    if (h->state_valid) {
        return fail(HCL_ERR_CONFIG, "hcl_set_stage_loop: select the time loop before the state is set");
    }
    h->force_stage = on != 0;
    return HCL_OK;
}

int hcl_set_schedule(hcl_handle* h, int schedule, int* used)
{
    HCL_CHECK_HANDLE(h);
    if (schedule == -2) {
        if (used) {
            *used = h->mixed_shape;
        }
        return HCL_OK;
    }
    if (schedule < -1 || schedule >= hcl::fused::mixed_shape_count(h->g.ndim)) {
        return fail(HCL_ERR_ARGUMENT, "schedule %d out of range", schedule);
    }
    if (schedule >= 0 && !hcl::fused::mixed_shape_valid(h->g, schedule)) {
        return fail(HCL_ERR_CONFIG, "schedule %d needs a uniform Cartesian grid (and an even ghost width for 7-8)", schedule);
    }
    h->mixed_shape = schedule < 0 ? -1 : schedule;
    if (used) {
        *used = h->mixed_shape;
    }
    return HCL_OK;
}

int hcl_get_dt_log(hcl_handle* h, double* dts, int max_count, int* count)
{
    HCL_CHECK_HANDLE(h);
    if (stage_mode(h)) {
        const int n = std::min(max_count, (int)h->sl_dts.size());
        if (n > 0 && dts) {
            std::memcpy(dts, h->sl_dts.data(), sizeof(double) * n);
        }
        if (count) {
            *count = n;
        }
        return HCL_OK;
    }
    StepCtl ctl;
    int rc = read_ctl(h, &ctl);
    if (rc) {
        return rc;
    }
    const int n = std::min(max_count, std::min(ctl.iter[h->counter & 1], h->dt_log_cap));
    if (n > 0 && dts) {
        HCL_CUDA(cudaMemcpy(dts, h->dt_log, sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    if (count) {
        *count = n;
    }
    return HCL_OK;
}

int hcl_conservation_sums(hcl_handle* h, double* out)
{
    HCL_CHECK_HANDLE(h);
    if (!out) {
        return fail(HCL_ERR_ARGUMENT, "null output");
    }
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    if (stage_mode(h)) {
        const int nd = h->g.ndim;
        int rc = hcl_integrate(h, h->sl_rho, &out[0], h->stream);
        for (int d = 0; d < nd && rc == HCL_OK; ++d) {
            rc = hcl_integrate(h, h->sl_rhou + h->g.N * d, &out[1 + d], h->stream);
        }
        if (rc == HCL_OK) {
            rc = hcl_integrate(h, h->sl_E, &out[1 + nd], h->stream);
        }
        return rc;
    }
    hcl::fused::conservation_sums(h->g, h->st[h->cur], h->red_partials, h->red_out, h->stream);
    HCL_LAUNCH_CHECK();
    HCL_CUDA(cudaMemcpyAsync(out, h->red_out, sizeof(double) * (h->g.ndim + 2), cudaMemcpyDeviceToHost, h->stream));
    HCL_CUDA(cudaStreamSynchronize(h->stream));
    return HCL_OK;
}

// ---- discrete adjoint -------------------------------------------------------
int hcl_adjoint_forward(hcl_handle* h, const hcl_adjoint_params* p)
{
    HCL_CHECK_HANDLE(h);
    if (!p || p->nsteps <= 0) {
        return fail(HCL_ERR_ARGUMENT, "adjoint needs nsteps > 0");
    }
    if (!h->state_valid) {
        return fail(HCL_ERR_CONFIG, "no state set");
    }
    const GridDev& g = h->g;
    if (h->cfg.pressure_fix || g.eos != HCL_EOS_PERFECT_GAS) {
        return fail(HCL_ERR_CONFIG, "the adjoint supports Cartesian and spherical grids, uniform, point-mass or "
                                    "internal-mass gravity, every Riemann solver, passive scalars, no pressure fix, "
                                    "the perfect-gas EOS");
    }
    if (p->precision != HCL_FP64 && p->precision != HCL_FP32_MIXED) {
        return fail(HCL_ERR_CONFIG, "the reverse sweep runs in HCL_FP64 or HCL_FP32_MIXED");
    }
    if (g.nfx > 0) {
        size_t need = 0, avail = 0;
        if (!hcl::adjoint::scalar_sweep_fits(g.ndim, p->precision == HCL_FP64, g.nfx, &need, &avail)) {
            return fail(HCL_ERR_CONFIG,
                        "the reverse sweep's tile with %d passive scalars needs %zu bytes of shared memory, the device "
                        "allows %zu: use fewer scalars or the HCL_FP32_MIXED sweep",
                        g.nfx, need, avail);
        }
    }
    int rc;
    StepCtl ctl;
    if ((rc = read_ctl(h, &ctl))) {
        return rc;
    }
    if (h->stopped) {
        if ((rc = restart_clock(h, ctl.t[h->counter & 1], ctl.iter[h->counter & 1]))) {
            return rc;
        }
        if ((rc = read_ctl(h, &ctl))) {
            return rc;
        }
    }
    const int N = p->nsteps;
    const int k = p->checkpoint_every > 0 ? p->checkpoint_every : 32;
    const int nck = (N + k - 1) / k;
    const size_t sz = (size_t)h->st[0].plane * (g.ndim + 2 + g.nfx);
    if (h->adj_cap_ck < nck) {
        cudaFree(h->adj_ckpt);
        h->adj_ckpt = nullptr;
        h->adj_cap_ck = 0;
        if ((rc = dalloc(&h->adj_ckpt, sz * nck))) {
            return rc;
        }
        h->adj_cap_ck = nck;
    }
    const int iter0 = ctl.iter[h->counter & 1];
    int done = 0;
    for (int s = 0; s < nck; ++s) {
        const int cur = h->cur;
        HCL_CUDA(cudaMemcpyAsync(h->adj_ckpt + sz * s, h->st[cur].q, sizeof(double) * sz, cudaMemcpyDeviceToDevice,
                                 h->stream));
        hcl_run_params rp;
        std::memset(&rp, 0, sizeof(rp));
        rp.cfl = p->cfl > 0 ? p->cfl : 0.4;
        rp.t_end = 1e300;
        rp.max_iter = INT_MAX;
        rp.nsteps = std::min(k, N - done);
        rp.graph_chunk = 6;
        if (p->dts) {
            rp.fixed_dt = 1;
            rp.dts = p->dts + done;
        }
        hcl_run_result rr;
        if ((rc = hcl_run(h, &rp, &rr))) {
            return rc;
        }
        done += rp.nsteps;
    }
    // dts of the steps just taken
    std::vector<double> all((size_t)iter0 + N);
    int cnt = 0;
    if ((rc = hcl_get_dt_log(h, all.data(), iter0 + N, &cnt))) {
        return rc;
    }
    if (cnt < iter0 + N) {
        return fail(HCL_ERR_CONFIG, "dt log shorter than the forward run");
    }
    h->adj_dts.assign(all.begin() + iter0, all.begin() + iter0 + N);
    h->adj_k = k;
    h->adj_nck = nck;
    h->adj_prec = p->precision;
    h->adj_ready = 1;
    return HCL_OK;
}

int hcl_adjoint_dts(const hcl_handle* h, double* dts, int max_count, int* count)
{
    if (!h) {
        return fail(HCL_ERR_ARGUMENT, "null handle");
    }
    const int n = std::min(max_count, (int)h->adj_dts.size());
    if (dts && n > 0) {
        std::memcpy(dts, h->adj_dts.data(), sizeof(double) * n);
    }
    if (count) {
        *count = n;
    }
    return HCL_OK;
}

int hcl_adjoint_backward(hcl_handle* h, const double* lam_final, double* grad, int memory)
{
    int rc = adjoint_backward_impl(h, lam_final, grad, memory);
    if (rc) {
        return rc;
    }
    HCL_CUDA(cudaStreamSynchronize(h->stream));
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

} // extern "C"

// Reverse pass without the final synchronisation (the ensemble runs many concurrently).
static int adjoint_backward_impl(hcl_handle* h, const double* lam_final, double* grad, int memory)
{
    HCL_CHECK_HANDLE(h);
    if (!h->adj_ready) {
        return fail(HCL_ERR_CONFIG, "call hcl_adjoint_forward first");
    }
    if (!lam_final || !grad) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    const GridDev& g = h->g;
    const int nd = g.ndim;
    const int N = (int)h->adj_dts.size();
    const int k = h->adj_k;
    const size_t sz = (size_t)h->st[0].plane * (nd + 2 + g.nfx);
    int rc;
    // two segment buffers of k+1 states: the recompute of one overlaps the sweep of the other
    if (h->adj_cap_seg < 2 * (k + 1)) {
        cudaFree(h->adj_seg);
        h->adj_seg = nullptr;
        h->adj_cap_seg = 0;
        if ((rc = dalloc(&h->adj_seg, sz * (size_t)(2 * (k + 1))))) {
            return rc;
        }
        h->adj_cap_seg = 2 * (k + 1);
    }
    if (!h->adj_stream) {
        HCL_CUDA(cudaStreamCreateWithFlags(&h->adj_stream, cudaStreamNonBlocking));
        HCL_CUDA(cudaEventCreateWithFlags(&h->adj_ev_start, cudaEventDisableTiming));
        for (int b = 0; b < 2; ++b) {
            HCL_CUDA(cudaEventCreateWithFlags(&h->adj_ev_rec[b], cudaEventDisableTiming));
            HCL_CUDA(cudaEventCreateWithFlags(&h->adj_ev_rev[b], cudaEventDisableTiming));
        }
    }
    if (!h->adj_lam && (rc = dalloc(&h->adj_lam, sz * 3))) {
        return rc;
    }
    if (!h->adj_ctl && (rc = dalloc(&h->adj_ctl, 1))) {
        return rc;
    }
    // internal-mass gravity: the radial table of every segment state (the
    // forward rebuilds it from each step's input density), dJ/dg_r of one
    // reverse step, and shell scratch for the recompute and the reverse
    const bool imass = g.gravity == HCL_GRAVITY_INTERNAL_MASS;
    const int n0 = g.n[0];
    const int nsh = g.nx[0] + g.ng;
    const int gneed = imass ? 2 * (k + 1) * n0 + n0 + 2 * nsh : 0;
    if (h->adj_cap_gmem < gneed) {
        cudaFree(h->adj_gmem);
        h->adj_gmem = nullptr;
        h->adj_cap_gmem = 0;
        if ((rc = dalloc(&h->adj_gmem, (size_t)gneed))) {
            return rc;
        }
        h->adj_cap_gmem = gneed;
    }
    double* gtab = h->adj_gmem;
    double* gbar = imass ? gtab + 2 * (k + 1) * n0 : nullptr;
    double* shell_rev = imass ? gbar + n0 : nullptr;
    double* shell_rec = imass ? shell_rev + nsh : nullptr;
    auto grid_at = [&](int b, int j) {
        GridDev gj = g;
        if (imass) {
            gj.g_r = gtab + ((size_t)b * (k + 1) + j) * n0;
        }
        return gj;
    };
    if (h->adj_ddts_cap < N + 8) {
        cudaFree(h->adj_ddts);
        h->adj_ddts = nullptr;
        h->adj_ddts_cap = 0;
        if ((rc = dalloc(&h->adj_ddts, (size_t)N + 8))) {
            return rc;
        }
        h->adj_ddts_cap = N + 8;
    }
    cudaStream_t s = h->stream;
    HCL_CUDA(cudaMemcpyAsync(h->adj_ddts, h->adj_dts.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
    auto state_at = [&](double* base, size_t idx) {
        StateDev st = h->st[0];
        st.q = base + sz * idx;
        return st;
    };
    // three adjoint buffers in rotation: a step reads one, adds into the
    // second (zero) and clears the third for the step after it
    StateDev lam[3] = {state_at(h->adj_lam, 0), state_at(h->adj_lam, 1), state_at(h->adj_lam, 2)};
    HCL_CUDA(cudaMemsetAsync(h->adj_lam, 0, sizeof(double) * sz * 3, s));
    hcl::fused::pack_state(g, lam[0], lam_final, lam_final + g.N, lam_final + g.N * (nd + 1),
                           memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    // the passive scalars' planes follow E in the caller's buffer
    for (int f = 0; f < g.nfx; ++f) {
        const size_t w = sizeof(double) * (size_t)g.n[0];
        HCL_CUDA(cudaMemcpy2DAsync(lam[0].q + lam[0].plane * (nd + 2 + f), sizeof(double) * (size_t)lam[0].pitch,
                                   lam_final + g.N * (nd + 2 + f), w, w, (size_t)g.n[1] * g.n[2],
                                   memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    }
    // the reference layout packs rho, rhou (nd planes), E contiguously: rhou at +N, E at +N*(nd+1)
    hcl::adjoint::fold(g, lam[0], s);
    RunParamsDev rp;
    std::memset(&rp, 0, sizeof(rp));
    rp.cfl = 0.4;
    rp.t_end = 1e300;
    rp.max_iter = INT_MAX;
    rp.fixed_dt = 1;
    rp.dts = h->adj_ddts;
    const bool fp64_sweep = h->adj_prec == HCL_FP64;
    cudaStream_t a = h->adj_stream;
    // recompute U^{first} .. U^{first+len-1} of segment sg into buffer sg & 1 (stream a)
    auto recompute = [&](int sg) -> int {
        const int b = sg & 1;
        const size_t base = (size_t)b * (k + 1);
        const int first = sg * k;
        const int len = std::min(k, N - first);
        // the buffer was last read by the sweep of segment sg + 2
        HCL_CUDA(cudaStreamWaitEvent(a, h->adj_ev_rev[b], 0));
        HCL_CUDA(cudaMemcpyAsync(h->adj_seg + sz * base, h->adj_ckpt + sz * sg, sizeof(double) * sz,
                                 cudaMemcpyDeviceToDevice, a));
        hcl::fused::prologue(g, state_at(h->adj_seg, base), h->adj_ctl, 0.0, first, a);
        for (int j = 0; j < len; ++j) {
            const GridDev gj = grid_at(b, j);
            if (imass) {
                // the radial gravity of state j, which step j reads (main.cpp:309, :528)
                const StateDev sj = state_at(h->adj_seg, base + j);
                hcl::stage::internal_mass_gravity(g, sj.q, sj.pitch, h->cfg.central_mass, shell_rec,
                                                  const_cast<double*>(gj.g_r), a);
            }
            if (j + 1 == len) {
                break;
            }
            if (h->cfg.precision == HCL_FP64) {
                hcl::fused::step_exact(gj, state_at(h->adj_seg, base + j), state_at(h->adj_seg, base + j + 1),
                                       h->adj_ctl, rp, j % 6, 1, a);
            } else if (h->cfg.precision == HCL_FP64_FAST) {
                hcl::fused::step_fast64(gj, state_at(h->adj_seg, base + j), state_at(h->adj_seg, base + j + 1),
                                        h->adj_ctl, rp, j % 6, 1, a);
            } else {
                hcl::fused::step_mixed(gj, state_at(h->adj_seg, base + j), state_at(h->adj_seg, base + j + 1),
                                       h->adj_ctl, rp, j % 6, 1, h->mixed_shape < 0 ? 0 : h->mixed_shape, a);
            }
        }
        HCL_CUDA(cudaEventRecord(h->adj_ev_rec[b], a));
        return HCL_OK;
    };
    // the dts, λ^N and its fold are on stream s: stream a starts after them
    HCL_CUDA(cudaEventRecord(h->adj_ev_start, s));
    HCL_CUDA(cudaStreamWaitEvent(a, h->adj_ev_start, 0));
    // no sweep has read either buffer yet
    for (int b = 0; b < 2; ++b) {
        HCL_CUDA(cudaEventRecord(h->adj_ev_rev[b], s));
    }
    if ((rc = recompute(h->adj_nck - 1))) {
        return rc;
    }
    int ra = 0, rb = 1, rc3 = 2; // read, add into, clear
    for (int sg = h->adj_nck - 1; sg >= 0; --sg) {
        if (sg > 0 && (rc = recompute(sg - 1))) {
            return rc;
        }
        const int b = sg & 1;
        const size_t base = (size_t)b * (k + 1);
        const int first = sg * k;
        const int len = std::min(k, N - first);
        HCL_CUDA(cudaStreamWaitEvent(s, h->adj_ev_rec[b], 0));
        // backward through the segment
        for (int j = len - 1; j >= 0; --j) {
            const int n = first + j;
            // lam[rb] holds zeros here: from the initial clear, then from the
            // step before the previous one, which cleared it after the step
            // before that had read it
            if (imass) {
                HCL_CUDA(cudaMemsetAsync(gbar, 0, sizeof(double) * n0, s));
            }
            const GridDev gj = grid_at(b, j);
            hcl::adjoint::step(gj, state_at(h->adj_seg, base + j), lam[ra], lam[rb], h->adj_dts[n], fp64_sweep,
                               h->cfg.precision == HCL_FP64, lam[rc3], gbar, s);
            if (imass) {
                // the density of state j also enters through the gravity table step j read
                hcl::adjoint::internal_mass_reverse(gj, gbar, shell_rev, lam[rb], s);
            }
            const int t = ra;
            ra = rb;
            rb = rc3;
            rc3 = t;
        }
        HCL_CUDA(cudaEventRecord(h->adj_ev_rev[b], s));
    }
    HCL_LAUNCH_CHECK();
    // the gradient lives on the interior cells; ghost entries are zero
    hcl::adjoint::zero_ghosts(g, lam[ra], s);
    hcl::fused::unpack_state(g, lam[ra], grad, grad + g.N, grad + g.N * (nd + 1),
                             memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
    for (int f = 0; f < g.nfx; ++f) {
        const size_t w = sizeof(double) * (size_t)g.n[0];
        HCL_CUDA(cudaMemcpy2DAsync(grad + g.N * (nd + 2 + f), w, lam[ra].q + lam[ra].plane * (nd + 2 + f),
                                   sizeof(double) * (size_t)lam[ra].pitch, w, (size_t)g.n[1] * g.n[2],
                                   memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    }
    HCL_LAUNCH_CHECK();
    return HCL_OK;
}

// ---- batched ensemble ----------------------------------------------------------
struct hcl_ensemble {
    std::vector<hcl_handle*> h;
    std::vector<hcl::ensemble::Prob> probs;
    hcl::ensemble::Prob* d_probs = nullptr;
    hcl::ensemble::Prob* d_probs_tune = nullptr;
    int* d_items = nullptr;
    int nitems = 0;
    int items_L = 0;
    unsigned int* d_barrier = nullptr;
    int* d_status = nullptr;
    cudaStream_t stream = nullptr;
    int lim = 0, rs = 0;
    int L = 0, bps = 0, nw = 4; // tuned schedule: strip rows, CTAs per SM, warps per CTA
    int64_t cells = 0;
    // (nsteps, step0, L, bps, nw, barrier spin limit, extra barrier arrivals)
    std::map<std::tuple<int, int, int, int, int, long long, unsigned int>, cudaGraphExec_t> graphs;
    // batched reverse pass: problem tables, tile work list, dts of all problems
    hcl::ensemble::AdjProb* d_adjprobs = nullptr;
    hcl::ensemble::Prob* d_rec_probs = nullptr;
    int* d_tiles = nullptr;
    double* d_adj_dts = nullptr;
};

namespace {

void free_ensemble(hcl_ensemble* e)
{
    if (!e) {
        return;
    }
    for (auto& kv : e->graphs) {
        cudaGraphExecDestroy(kv.second);
    }
    cudaFree(e->d_probs);
    cudaFree(e->d_probs_tune);
    cudaFree(e->d_adjprobs);
    cudaFree(e->d_rec_probs);
    cudaFree(e->d_tiles);
    cudaFree(e->d_adj_dts);
    cudaFree(e->d_items);
    cudaFree(e->d_barrier);
    cudaFree(e->d_status);
    if (e->stream) {
        cudaStreamDestroy(e->stream);
    }
    for (hcl_handle* h : e->h) {
        free_handle(h);
    }
    delete e;
}

// Work list of warp strips of L rows over every problem.
int ensemble_build_items(hcl_ensemble* e, int L)
{
    if (e->items_L == L) {
        return HCL_OK;
    }
    std::vector<int> items;
    for (size_t p = 0; p < e->h.size(); ++p) {
        hcl::ensemble::Prob& P = e->probs[p];
        P.ncolw = (P.g.nx[0] + hcl::fused::kStripLanesOut - 1) / hcl::fused::kStripLanesOut;
        P.nstrip = (P.g.nx[1] + L - 1) / L;
        P.item0 = (int)items.size();
        items.insert(items.end(), (size_t)P.ncolw * P.nstrip, (int)p);
    }
    cudaFree(e->d_items);
    e->d_items = nullptr;
    int rc = dalloc(&e->d_items, items.size());
    if (rc) {
        return rc;
    }
    HCL_CUDA(cudaMemcpy(e->d_items, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice));
    e->nitems = (int)items.size();
    e->items_L = L;
    // device copies of the problem table (live control blocks and tuning copies)
    std::vector<hcl::ensemble::Prob> tune = e->probs;
    for (size_t p = 0; p < e->h.size(); ++p) {
        tune[p].ctl = e->h[p]->ctl_tune;
        tune[p].dt_log = nullptr;
    }
    HCL_CUDA(cudaMemcpy(e->d_probs, e->probs.data(), sizeof(hcl::ensemble::Prob) * e->probs.size(),
                        cudaMemcpyHostToDevice));
    HCL_CUDA(cudaMemcpy(e->d_probs_tune, tune.data(), sizeof(hcl::ensemble::Prob) * tune.size(), cudaMemcpyHostToDevice));
    return HCL_OK;
}

int ensemble_launch(hcl_ensemble* e, const hcl::ensemble::Prob* probs, int nsteps, int step0, int L, int bps, int nw,
                    int use_graph, double cfl, int* graphed, long long spin_limit = 0, int extra_arrivals = 0)
{
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->h[0]->cfg.device);
    const int grid = bps * nsm;
    hcl::ensemble::Params ep;
    std::memset(&ep, 0, sizeof(ep));
    ep.cfl = cfl;
    ep.nsteps = nsteps;
    ep.step0 = step0;
    ep.L = L;
    ep.nitems = e->nitems;
    ep.nprob = (int)e->h.size();
    ep.spin_limit = spin_limit > 0 ? spin_limit : hcl::ensemble::kSpinLimit;
    ep.extra_arrivals = (unsigned int)(extra_arrivals > 0 ? extra_arrivals : 0);
    auto issue = [&]() -> cudaError_t {
        cudaError_t err = cudaMemsetAsync(e->d_barrier, 0, sizeof(unsigned int), e->stream);
        if (err == cudaSuccess) {
            err = cudaMemsetAsync(e->d_status, 0, sizeof(int), e->stream);
        }
        if (err == cudaSuccess) {
            err = hcl::ensemble::launch(e->lim, e->rs, nw, grid, probs, e->d_items, ep, e->d_barrier, e->d_status,
                                        e->stream);
        }
        return err;
    };
    *graphed = 0;
    if (use_graph && probs == e->d_probs) {
        const auto key = std::make_tuple(nsteps, step0, L, bps, nw, ep.spin_limit, ep.extra_arrivals);
        auto it = e->graphs.find(key);
        if (it == e->graphs.end()) {
            cudaGraph_t graph;
            HCL_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            const cudaError_t err = issue();
            cudaError_t err2 = cudaStreamEndCapture(e->stream, &graph);
            if (err == cudaSuccess && err2 == cudaSuccess) {
                cudaGraphExec_t exec;
                if (cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                    it = e->graphs.emplace(key, exec).first;
                }
                cudaGraphDestroy(graph);
            }
            cudaGetLastError(); // a failed capture falls back to a direct launch
        }
        if (it != e->graphs.end()) {
            HCL_CUDA(cudaGraphLaunch(it->second, e->stream));
            *graphed = 1;
            return HCL_OK;
        }
    }
    HCL_CUDA(issue());
    return HCL_OK;
}

// Picks (strip rows, CTAs per SM, warps per CTA) by timing one step of every
// candidate on the tuning control blocks (reads buffer 0, writes buffer 1;
// the state is kept).  Candidates: CTAs of 4 warps at the resident maximum
// per SM and the two counts below it; one CTA of 16 warps per SM.
int ensemble_autotune(hcl_ensemble* e, double cfl)
{
    const int maxb4 = hcl::ensemble::max_blocks_per_sm(e->lim, e->rs, 4);
    const int maxb16 = hcl::ensemble::max_blocks_per_sm(e->lim, e->rs, 16);
    if (maxb4 <= 0) {
        return fail(HCL_ERR_CUDA, "ensemble kernel cannot be resident");
    }
    cudaEvent_t e0, e1;
    HCL_CUDA(cudaEventCreate(&e0));
    HCL_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    const int Ls[3] = {32, 64, 128};
    for (int L : Ls) {
        int rc = ensemble_build_items(e, L);
        if (rc) {
            return rc;
        }
        std::vector<std::pair<int, int>> cands; // (bps, nw)
        for (int bps = maxb4; bps >= 1 && bps >= maxb4 - 2; --bps) {
            cands.emplace_back(bps, 4);
        }
        if (maxb16 >= 1) {
            cands.emplace_back(1, 16);
        }
        for (const auto& cand : cands) {
            const int bps = cand.first, nw = cand.second;
            float tot = 0;
            for (int r = 0; r < 3; ++r) {
                for (hcl_handle* h : e->h) {
                    hcl::fused::prologue(h->g, h->st[0], h->ctl_tune, 0.0, 0, e->stream);
                }
                int graphed = 0;
                HCL_CUDA(cudaEventRecord(e0, e->stream));
                if ((rc = ensemble_launch(e, e->d_probs_tune, 1, 0, L, bps, nw, 0, cfl, &graphed))) {
                    return rc;
                }
                HCL_CUDA(cudaEventRecord(e1, e->stream));
                HCL_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                HCL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (r > 0) {
                    tot += ms;
                }
            }
            if (tot < best) {
                best = tot;
                e->L = L;
                e->bps = bps;
                e->nw = nw;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ensemble_build_items(e, e->L);
}

} // namespace

extern "C" {

int hcl_ensemble_create(const hcl_config* cfgs, int nprob, hcl_ensemble** out)
{
    if (!cfgs || nprob <= 0 || !out) {
        return fail(HCL_ERR_ARGUMENT, "ensemble needs configurations");
    }
    *out = nullptr;
    hcl_ensemble* e = new hcl_ensemble();
    auto bail = [&](int rc) {
        free_ensemble(e);
        return rc;
    };
    for (int p = 0; p < nprob; ++p) {
        const hcl_config& c = cfgs[p];
        if (c.ndim != 2 || c.precision != HCL_FP32_MIXED || c.geometry != HCL_GEOM_CARTESIAN ||
            c.gravity != HCL_GRAVITY_UNIFORM || c.nfx != 0 || c.pressure_fix != 0 || c.limiter != cfgs[0].limiter ||
            c.riemann != cfgs[0].riemann) {
            return bail(fail(HCL_ERR_CONFIG, "ensemble problem %d: needs 2-D Cartesian FP32-mixed, uniform gravity, "
                                             "and the limiter and Riemann solver of problem 0", p));
        }
        hcl_handle* h = nullptr;
        int rc = hcl_create(&c, &h);
        if (rc) {
            return bail(rc);
        }
        e->h.push_back(h);
        if (!h->g.uniform_cart) {
            return bail(fail(HCL_ERR_CONFIG, "ensemble problem %d: the grid must be uniform", p));
        }
        hcl::ensemble::Prob P;
        std::memset(&P, 0, sizeof(P));
        P.g = h->g;
        P.q[0] = h->st[0].q;
        P.q[1] = h->st[1].q;
        P.plane = h->st[0].plane;
        P.pitch = h->st[0].pitch;
        P.ctl = h->ctl;
        e->probs.push_back(P);
        e->cells += (int64_t)h->g.nx[0] * h->g.nx[1];
    }
    e->lim = cfgs[0].limiter;
    e->rs = cfgs[0].riemann;
    HCL_CUDA(cudaSetDevice(cfgs[0].device));
    int rc;
    if ((rc = dalloc(&e->d_probs, (size_t)nprob)) || (rc = dalloc(&e->d_probs_tune, (size_t)nprob)) ||
        (rc = dalloc(&e->d_barrier, 1)) || (rc = dalloc(&e->d_status, 1))) {
        return bail(rc);
    }
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        return bail(fail(HCL_ERR_CUDA, "cudaStreamCreate failed"));
    }
    *out = e;
    return HCL_OK;
}

int hcl_ensemble_destroy(hcl_ensemble* e)
{
    if (e) {
        cudaStreamSynchronize(e->stream);
    }
    free_ensemble(e);
    return HCL_OK;
}

int hcl_ensemble_handle(hcl_ensemble* e, int p, hcl_handle** h)
{
    if (!e || !h || p < 0 || p >= (int)e->h.size()) {
        return fail(HCL_ERR_ARGUMENT, "bad ensemble index");
    }
    *h = e->h[p];
    return HCL_OK;
}

int hcl_ensemble_stream(const hcl_ensemble* e, void** stream)
{
    if (!e || !stream) {
        return fail(HCL_ERR_ARGUMENT, "null argument");
    }
    *stream = (void*)e->stream;
    return HCL_OK;
}

int hcl_ensemble_run(hcl_ensemble* e, const hcl_ensemble_params* p, hcl_ensemble_result* r)
{
    if (!e || !p || p->nsteps <= 0) {
        return fail(HCL_ERR_ARGUMENT, "ensemble run needs nsteps > 0");
    }
    HCL_CUDA(cudaSetDevice(e->h[0]->cfg.device));
    const int N = p->nsteps;
    int rc;
    // every problem: state in buffer 0, fresh control block at its current t and iteration
    std::vector<int> iter0(e->h.size());
    for (size_t q = 0; q < e->h.size(); ++q) {
        hcl_handle* h = e->h[q];
        if (!h->state_valid) {
            return fail(HCL_ERR_CONFIG, "ensemble problem %zu has no state", q);
        }
        StepCtl ctl;
        if ((rc = read_ctl(h, &ctl))) {
            return rc;
        }
        if (ctl.err) {
            return fail(HCL_ERR_INVALID_STATE, "ensemble problem %zu holds an invalid state", q);
        }
        const int qq = (int)(h->counter & 1);
        if ((rc = restart_clock(h, ctl.t[qq], ctl.iter[qq]))) {
            return rc;
        }
        iter0[q] = ctl.iter[qq];
        if ((rc = ensure_dt_log(h, iter0[q] + N + 8))) {
            return rc;
        }
        e->probs[q].dt_log = h->dt_log;
        e->probs[q].dt_cap = h->dt_log_cap;
        HCL_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (p->strip_rows != 0 && p->strip_rows != 32 && p->strip_rows != 64 && p->strip_rows != 128) {
        return fail(HCL_ERR_ARGUMENT, "strip_rows must be 0 (autotune), 32, 64 or 128");
    }
    if (p->warps_per_cta != 0 && p->warps_per_cta != 4 && p->warps_per_cta != 16) {
        return fail(HCL_ERR_ARGUMENT, "warps_per_cta must be 0 (autotune), 4 or 16");
    }
    const int nw_req = p->warps_per_cta > 0 ? p->warps_per_cta : 4;
    const int maxb = hcl::ensemble::max_blocks_per_sm(e->lim, e->rs, nw_req);
    if (p->blocks_per_sm < 0 || p->blocks_per_sm > maxb) {
        return fail(HCL_ERR_ARGUMENT, "blocks_per_sm must be in [0, %d] for a co-resident launch", maxb);
    }
    e->items_L = 0; // the table carries the dt logs: rebuild it
    if (p->strip_rows > 0 || p->blocks_per_sm > 0 || p->warps_per_cta > 0) {
        e->L = p->strip_rows > 0 ? p->strip_rows : 64;
        e->nw = nw_req;
        e->bps = p->blocks_per_sm > 0 ? p->blocks_per_sm : maxb;
    } else if (e->L == 0) {
        if ((rc = ensemble_autotune(e, p->cfl))) {
            return rc;
        }
    }
    if ((rc = ensemble_build_items(e, e->L))) {
        return rc;
    }
    const int k = p->checkpoint_every > 0 ? p->checkpoint_every : N;
    const int nseg = (N + k - 1) / k;
    if (p->checkpoint_every > 0) {
        for (hcl_handle* h : e->h) {
            const size_t sz = (size_t)h->st[0].plane * (h->g.ndim + 2);
            if (h->adj_cap_ck < nseg) {
                cudaFree(h->adj_ckpt);
                h->adj_ckpt = nullptr;
                h->adj_cap_ck = 0;
                if ((rc = dalloc(&h->adj_ckpt, sz * nseg))) {
                    return rc;
                }
                h->adj_cap_ck = nseg;
            }
        }
    }
    int graphed_all = 1;
    int done = 0;
    for (int sgm = 0; sgm < nseg; ++sgm) {
        const int len = std::min(k, N - done);
        if (p->checkpoint_every > 0) {
            for (hcl_handle* h : e->h) {
                const size_t sz = (size_t)h->st[0].plane * (h->g.ndim + 2);
                HCL_CUDA(cudaMemcpyAsync(h->adj_ckpt + sz * sgm, h->st[done & 1].q, sizeof(double) * sz,
                                         cudaMemcpyDeviceToDevice, e->stream));
            }
        }
        int graphed = 0;
        if ((rc = ensemble_launch(e, e->d_probs, len, done, e->L, e->bps, e->nw, p->use_graph, p->cfl, &graphed,
                                  p->barrier_spin_limit, p->barrier_extra_arrivals))) {
            return rc;
        }
        graphed_all &= graphed;
        done += len;
    }
    int status = 0;
    HCL_CUDA(cudaMemcpyAsync(&status, e->d_status, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    HCL_CUDA(cudaStreamSynchronize(e->stream));
    HCL_LAUNCH_CHECK();
    for (size_t q = 0; q < e->h.size(); ++q) {
        hcl_handle* h = e->h[q];
        h->counter = N;
        h->cur = N & 1;
        h->stopped = 0;
        // later single-problem steps (and the adjoint's recomputation) use the
        // same warp-strip code as the ensemble
        h->mixed_shape = e->L == 32 ? 3 : (e->L == 64 ? 4 : 5);
        if (p->checkpoint_every > 0) {
            std::vector<double> all((size_t)iter0[q] + N);
            HCL_CUDA(cudaMemcpy(all.data(), h->dt_log, sizeof(double) * all.size(), cudaMemcpyDeviceToHost));
            h->adj_dts.assign(all.begin() + iter0[q], all.end());
            h->adj_k = k;
            h->adj_nck = nseg;
            h->adj_prec = p->adjoint_precision;
            h->adj_ready = 1;
        }
    }
    if (r) {
        r->status = status;
        r->strip_rows = e->L;
        r->blocks_per_sm = e->bps;
        r->warps_per_cta = e->nw;
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->h[0]->cfg.device);
        r->grid = e->bps * nsm;
        r->launches = nseg;
        r->graph = graphed_all;
        r->cells = e->cells;
    }
    if (status == HCL_ERR_TIMEOUT) {
        return fail(HCL_ERR_TIMEOUT, "ensemble grid barrier timed out");
    }
    if (status == HCL_ERR_INVALID_STATE) {
        return fail(HCL_ERR_INVALID_STATE, "detected invalid volumic internal energy in the ensemble");
    }
    return HCL_OK;
}

int hcl_ensemble_adjoint(hcl_ensemble* e, const double* const* lam_final, double* const* grads, int memory)
{
    using hcl::ensemble::AdjProb;
    using hcl::ensemble::Prob;
    if (!e || !lam_final || !grads) {
        return fail(HCL_ERR_ARGUMENT, "null argument");
    }
    const size_t np = e->h.size();
    hcl_handle* h0 = e->h[0];
    const int N = (int)h0->adj_dts.size();
    const int k = h0->adj_k;
    const int nck = h0->adj_nck;
    for (hcl_handle* h : e->h) {
        if (!h->adj_ready || (int)h->adj_dts.size() != N || h->adj_k != k || N <= 0) {
            return fail(HCL_ERR_CONFIG, "run the ensemble with checkpoint_every > 0 before its adjoint");
        }
    }
    const bool fp64 = h0->adj_prec == HCL_FP64;
    HCL_CUDA(cudaSetDevice(h0->cfg.device));
    cudaStream_t s = e->stream;
    int rc;
    // per-problem buffers and tables
    std::vector<AdjProb> ap(np);
    std::vector<Prob> rec = e->probs;
    std::vector<int> tiles;
    std::vector<double> dts_all(np * (size_t)N);
    for (size_t q = 0; q < np; ++q) {
        hcl_handle* h = e->h[q];
        const GridDev& g = h->g;
        const size_t sz = (size_t)h->st[0].plane * (g.ndim + 2);
        if (h->adj_cap_seg < k + 1) {
            cudaFree(h->adj_seg);
            h->adj_seg = nullptr;
            h->adj_cap_seg = 0;
            if ((rc = dalloc(&h->adj_seg, sz * (size_t)(2 * (k + 1))))) {
                return rc;
            }
            h->adj_cap_seg = 2 * (k + 1);
        }
        if (!h->adj_lam && (rc = dalloc(&h->adj_lam, sz * 3))) {
            return rc;
        }
        if (!h->adj_ctl && (rc = dalloc(&h->adj_ctl, 1))) {
            return rc;
        }
        AdjProb& A = ap[q];
        std::memset(&A, 0, sizeof(A));
        A.g = g;
        A.seg0 = h->st[0];
        A.seg0.q = h->adj_seg;
        A.sz = (int64_t)sz;
        A.lam[0] = h->st[0];
        A.lam[0].q = h->adj_lam;
        A.lam[1] = h->st[0];
        A.lam[1].q = h->adj_lam + sz;
        A.lam[2] = h->st[0];
        A.lam[2].q = h->adj_lam + 2 * sz;
        A.ckpt = h->adj_ckpt;
        A.ctl = h->adj_ctl;
        A.tile0 = (int)tiles.size();
        const int nt = ((g.nx[0] + hcl::ensemble::kRevTile - 1) / hcl::ensemble::kRevTile) *
                       ((g.nx[1] + hcl::ensemble::kRevTile - 1) / hcl::ensemble::kRevTile);
        tiles.insert(tiles.end(), (size_t)nt, (int)q);
        rec[q].q[0] = h->adj_seg;
        rec[q].q[1] = nullptr;
        rec[q].seg_stride = (int64_t)sz;
        rec[q].ctl = h->adj_ctl;
        rec[q].dt_log = nullptr;
        rec[q].dt_cap = 0;
        std::copy(h->adj_dts.begin(), h->adj_dts.end(), dts_all.begin() + q * (size_t)N);
    }
    cudaFree(e->d_adjprobs);
    cudaFree(e->d_rec_probs);
    cudaFree(e->d_tiles);
    cudaFree(e->d_adj_dts);
    e->d_adjprobs = nullptr;
    e->d_rec_probs = nullptr;
    e->d_tiles = nullptr;
    e->d_adj_dts = nullptr;
    if ((rc = dalloc(&e->d_adjprobs, np)) || (rc = dalloc(&e->d_rec_probs, np)) ||
        (rc = dalloc(&e->d_tiles, tiles.size())) || (rc = dalloc(&e->d_adj_dts, dts_all.size()))) {
        return rc;
    }
    for (size_t q = 0; q < np; ++q) {
        ap[q].dts = e->d_adj_dts + q * (size_t)N;
    }
    HCL_CUDA(cudaMemcpyAsync(e->d_adj_dts, dts_all.data(), sizeof(double) * dts_all.size(), cudaMemcpyHostToDevice, s));
    HCL_CUDA(cudaMemcpyAsync(e->d_adjprobs, ap.data(), sizeof(AdjProb) * np, cudaMemcpyHostToDevice, s));
    HCL_CUDA(cudaMemcpyAsync(e->d_rec_probs, rec.data(), sizeof(Prob) * np, cudaMemcpyHostToDevice, s));
    HCL_CUDA(cudaMemcpyAsync(e->d_tiles, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, s));
    // lambda^N, folded onto the interior
    const cudaMemcpyKind kin = memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (size_t q = 0; q < np; ++q) {
        const GridDev& g = e->h[q]->g;
        const int nd = g.ndim;
        HCL_CUDA(cudaMemsetAsync(ap[q].lam[0].q, 0, sizeof(double) * ap[q].sz * 3, s));
        hcl::fused::pack_state(g, ap[q].lam[0], lam_final[q], lam_final[q] + g.N, lam_final[q] + g.N * (nd + 1), kin,
                               s);
        hcl::adjoint::fold(g, ap[q].lam[0], s);
    }
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h0->cfg.device);
    const int rev_bps = hcl::ensemble::reverse_blocks_per_sm(fp64);
    if (rev_bps <= 0) {
        return fail(HCL_ERR_CUDA, "the batched reverse kernel cannot be resident");
    }
    if (e->L == 0 || e->items_L != e->L) {
        return fail(HCL_ERR_CONFIG, "run the ensemble before its adjoint");
    }
    hcl::ensemble::Params ep;
    std::memset(&ep, 0, sizeof(ep));
    ep.cfl = 0.4;
    ep.step0 = 0;
    ep.L = e->L;
    ep.nitems = e->nitems;
    ep.nprob = (int)np;
    ep.fixed_dt = 1;
    ep.dts = e->d_adj_dts;
    ep.dts_stride = N;
    ep.seg_mode = 1;
    ep.spin_limit = hcl::ensemble::kSpinLimit;
    HCL_CUDA(cudaMemsetAsync(e->d_status, 0, sizeof(int), s));
    // the segment loop (2 persistent launches per checkpoint segment) is
    // captured in a CUDA graph and replayed; it is rebuilt for every call
    // because the tables it reads are reallocated above
    int cur = 0;
    auto issue = [&]() -> cudaError_t {
        cudaError_t err = cudaSuccess;
        for (int sg = nck - 1; sg >= 0 && err == cudaSuccess; --sg) {
            const int first = sg * k;
            const int len = std::min(k, N - first);
            hcl::ensemble::seg_init(e->d_adjprobs, (int)np, sg, first, s);
            if (len > 1) {
                ep.nsteps = len - 1;
                err = cudaMemsetAsync(e->d_barrier, 0, sizeof(unsigned int), s);
                if (err == cudaSuccess) {
                    err = hcl::ensemble::launch(e->lim, e->rs, e->nw, e->bps * nsm, e->d_rec_probs, e->d_items, ep,
                                                e->d_barrier, e->d_status, s);
                }
            }
            hcl::ensemble::AdjParams prm;
            prm.nprob = (int)np;
            prm.ntiles = (int)tiles.size();
            prm.first = first;
            prm.len = len;
            prm.cur = cur;
            if (err == cudaSuccess) {
                err = cudaMemsetAsync(e->d_barrier, 0, sizeof(unsigned int), s);
            }
            if (err == cudaSuccess) {
                err = hcl::ensemble::reverse(fp64, rev_bps * nsm, e->d_adjprobs, e->d_tiles, prm, e->d_barrier,
                                             e->d_status, s);
            }
            cur = (cur + len) % 3;
        }
        return err;
    };
    {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        HCL_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const cudaError_t err = issue();
        const cudaError_t err2 = cudaStreamEndCapture(s, &graph);
        bool replayed = false;
        if (err == cudaSuccess && err2 == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
            replayed = cudaGraphLaunch(exec, s) == cudaSuccess;
        }
        if (graph) {
            cudaGraphDestroy(graph);
        }
        if (exec) {
            cudaGraphExecDestroy(exec); // a launched graph may be destroyed; its work completes
        }
        cudaGetLastError();
        if (!replayed) {
            cur = 0;
            HCL_CUDA(issue());
        }
    }
    const cudaMemcpyKind kout = memory == HCL_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (size_t q = 0; q < np; ++q) {
        const GridDev& g = e->h[q]->g;
        const int nd = g.ndim;
        hcl::adjoint::zero_ghosts(g, ap[q].lam[cur], s);
        hcl::fused::unpack_state(g, ap[q].lam[cur], grads[q], grads[q] + g.N, grads[q] + g.N * (nd + 1), kout, s);
    }
    int status = 0;
    HCL_CUDA(cudaMemcpyAsync(&status, e->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    HCL_CUDA(cudaStreamSynchronize(s));
    HCL_LAUNCH_CHECK();
    if (status == HCL_ERR_TIMEOUT) {
        return fail(HCL_ERR_TIMEOUT, "ensemble adjoint grid barrier timed out");
    }
    if (status != 0) {
        return fail(HCL_ERR_INVALID_STATE, "invalid state in the ensemble adjoint's recomputation");
    }
    return HCL_OK;
}

} // extern "C"

// ---- hydro reconstruction with fixed scratch (no allocation) ------------------------
// hcl_hydro_reconstruction_noalloc keeps the scratch of one call (u_rec, P_rec and
// fx_rec_old of MUSCLHancockHydroReconstruction) in one fixed device array per
// device instead of the handle's lazily allocated buffers.
namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(1) << 22; // 32 MiB
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_base[kNoAllocMaxDevices] = {};

// Device address of this device's copy of the array, looked up on the first
// call on each device (the caller has made that device current) and kept for
// the process: a cudaDeviceReset of that device after the first call leaves
// the kept address stale, which the header states.
int noalloc_scratch(int dev, double** out)
{
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        return fail(HCL_ERR_ARGUMENT, "device %d out of range for the fixed scratch", dev);
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_base[dev]) {
        void* p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || !p) {
            return fail(HCL_ERR_CUDA, "cudaGetSymbolAddress of the fixed scratch failed: %s", cudaGetErrorString(err));
        }
        g_noalloc_base[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_base[dev];
    return HCL_OK;
}

} // namespace

extern "C" {

int hcl_hydro_reconstruction_noalloc(hcl_handle* h, int ng_eff, double dt, const double* rho, const double* u,
                                     const double* P, const double* fx, double* rho_rec, double* rhou_rec,
                                     double* E_rec, double* fx_rec, void* stream)
{
    HCL_CHECK_HANDLE(h);
    HCL_CHECK_NGEFF(h, ng_eff);
    if (ng_eff > h->g.ng - 1) {
        return fail(HCL_ERR_CONFIG, "reconstruction needs one ghost layer beyond the range");
    }
    if (!rho || !u || !P || !rho_rec || !rhou_rec || !E_rec) {
        return fail(HCL_ERR_ARGUMENT, "null array");
    }
    if (h->g.nfx > 0 && (!fx || !fx_rec)) {
        return fail(HCL_ERR_ARGUMENT, "nfx > 0 needs fx and fx_rec");
    }
    const size_t nd = (size_t)h->g.ndim;
    const size_t N = (size_t)h->g.N;
    const size_t n_u = N * 2 * nd * nd, n_p = N * 2 * nd, n_fx = N * 2 * nd * (size_t)h->g.nfx;
    if (n_u + n_p + n_fx > kNoAllocScratchDoubles) {
        return fail(HCL_ERR_CONFIG,
                    "hcl_hydro_reconstruction_noalloc: this grid needs %zu scratch doubles (%zu cells x 2*ndim*(ndim+1+nfx)), "
                    "the fixed buffer holds %zu; use hcl_hydro_reconstruction",
                    n_u + n_p + n_fx, N, kNoAllocScratchDoubles);
    }
    int prev = -1;
    HCL_CUDA(cudaGetDevice(&prev));
    if (prev != h->cfg.device) {
        HCL_CUDA(cudaSetDevice(h->cfg.device));
    }
    double* base = nullptr;
    int rc = noalloc_scratch(h->cfg.device, &base);
    if (rc == HCL_OK) {
        hcl::stage::hydro_reconstruction(h->g, ng_eff, dt, rho, u, P, fx, rho_rec, rhou_rec, E_rec, fx_rec, base,
                                         base + n_u, h->g.nfx > 0 ? base + n_u + n_p : nullptr, pick(h, stream));
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            rc = fail(HCL_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        }
    }
    if (prev != h->cfg.device) {
        cudaSetDevice(prev);
    }
    return rc;
}

} // extern "C"
