/*
 * heracles_b200.h -- C ABI of the B200-native MUSCL-Hancock step.
 *
 * One shared library (libheracles_b200.so) exports these entry points.  They
 * take plain pointers, sizes and enums; no C++ or torch types cross the ABI.
 * Every call returns an int status (HCL_OK = 0) and never throws; the message
 * of the last failure on the calling thread is hcl_last_error().
 *
 * Arrays follow the reference's Kokkos::LayoutLeft Views exactly
 * (src/utils/kokkos_shortcut.hpp:22-41): x0 index fastest, trailing component
 * indices slowest, extents including Nghost ghost cells on active dimensions
 * (src/mesh/grid.cpp:56-58,119).  With N = n0*n1*n2:
 *   rho(i,j,k)             rho[c],   c = i + n0*(j + n1*k)
 *   rhou(i,j,k,d)          rhou[c + N*d]
 *   var_rec(i,j,k,s,d)     rec[c + N*(s + 2*d)]
 *   rhou_rec(i,j,k,s,d,r)  rec[c + N*(s + 2*(d + ndim*r))]
 *
 * The stage entry points (hcl_conv_*, hcl_face_reconstruction,
 * hcl_hydro_reconstruction, hcl_godunov_scheme, hcl_boundary_conditions,
 * hcl_time_step, ...) operate on caller-owned DEVICE arrays in that layout, so
 * each one can replace one plugin of the reference's time loop
 * (src/main.cpp:354-531).  The fused entry points (hcl_run, hcl_step, ...)
 * operate on a state owned by the handle and are the fast path.
 *
 * Reference citations are path:line inside the HERACLES++ project.
 */
#ifndef HERACLES_B200_H
#define HERACLES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HCL_ABI_VERSION 4

/* ---- status codes ------------------------------------------------------ */
enum hcl_status {
    HCL_OK = 0,
    HCL_ERR_CONFIG = 1,        /* invalid configuration (maps to std::runtime_error) */
    HCL_ERR_DOMAIN = 2,        /* invalid EOS parameter (maps to std::domain_error, perfect_gas.cpp:15-21) */
    HCL_ERR_CUDA = 3,          /* CUDA runtime error */
    HCL_ERR_INVALID_STATE = 4, /* NaN or negative internal energy (main.cpp:397-425) */
    HCL_ERR_NEGATIVE_DT = 5,   /* main.cpp:368-371 */
    HCL_ERR_TIMEOUT = 6,       /* a device-side wait gave up (bounded spin) */
    HCL_ERR_NO_DEVICE = 7,     /* no CUDA device / library built without the device code */
    HCL_ERR_ARGUMENT = 8       /* null pointer, wrong size, unknown name */
};

/* ---- enumerations (factory keys of the reference) ----------------------- */
enum hcl_limiter {             /* hydro/face_reconstruction.cpp:31-50 */
    HCL_LIMITER_CONSTANT = 0,
    HCL_LIMITER_VANLEER = 1,
    HCL_LIMITER_MINMOD = 2,
    HCL_LIMITER_VANALBADA = 3
};
enum hcl_riemann {             /* hydro/godunov_scheme.hpp:305-321 */
    HCL_RIEMANN_HLL = 0,
    HCL_RIEMANN_HLLC = 1,
    HCL_RIEMANN_LOW_MACH = 2   /* "Low Mach" = Splitting */
};
enum hcl_bc {                  /* boundary_factory.hpp:31-47 */
    HCL_BC_NULLGRADIENT = 0,
    HCL_BC_PERIODIC = 1,
    HCL_BC_REFLEXIVE = 2
};
enum hcl_geometry { HCL_GEOM_CARTESIAN = 0, HCL_GEOM_SPHERICAL = 1 };   /* utils/geom.hpp.in:17-25 */
enum hcl_gravity { /* main.cpp:73-96 */
    HCL_GRAVITY_UNIFORM = 0,
    HCL_GRAVITY_POINT_MASS = 1,
    HCL_GRAVITY_INTERNAL_MASS = 2 /* g(r) = -G M(r) / r^2 with M(r) from the density, gravity.cpp:59-128 */
};
enum hcl_precision {
    HCL_FP64 = 0,              /* reference arithmetic, bitwise-comparable to the FP64 CPU build */
    HCL_FP32_MIXED = 1,        /* FP32 prim/slopes/faces/fluxes, FP64 state, energy recovery, dt, sums */
    HCL_FP64_FAST = 2          /* all FP64, FMA contraction and the perfect gas without the temperature
                                * round trip (fewer divisions): within 1e-12 relative L1 of HCL_FP64 */
};
enum hcl_memory { HCL_HOST = 0, HCL_DEVICE = 1 };
enum hcl_eos { /* eos.hpp.in, selected at CMake time in the reference */
    HCL_EOS_PERFECT_GAS = 0, /* thermodynamics/perfect_gas.hpp */
    HCL_EOS_RAD_GAS = 1      /* thermodynamics/rad_gas.hpp: gas plus radiation (FP64 precision only) */
};

/* ---- configuration ------------------------------------------------------ */
/* Everything Param (utils/param.cpp:14-73), Grid (mesh/grid.cpp:48-76), the
 * EOS (thermodynamics/perfect_gas.cpp:13-22), the gravity plugin
 * (gravity/gravity.cpp:29-55) and the factories decide for the hot path. */
typedef struct hcl_config {
    int ndim;                 /* 1, 2 or 3 (utils/ndim.hpp.in) */
    int nx[3];                /* [Grid] Nx{0,1,2}_glob; set inactive dims to 1 */
    int nghost;               /* [Grid] Nghost (2; the MUSCL stencil needs >= 2) */
    int nfx;                  /* [Passive Scalar] nfx */
    int geometry;             /* enum hcl_geometry */
    double gamma;             /* [Perfect Gas] gamma */
    double mmw;               /* [Perfect Gas] mu */
    int limiter;              /* enum hcl_limiter   ([Hydro] reconstruction) */
    int riemann;              /* enum hcl_riemann   ([Hydro] riemann_solver) */
    int bc[6];                /* enum hcl_bc, index 2*idim + iface (main.cpp:174-185) */
    int gravity;              /* enum hcl_gravity */
    double g[3];              /* [Gravity] gx0..gx2 (uniform) */
    double central_mass;      /* [Gravity] M (point mass; central mass of the internal mass) */
    double xmin[3], xmax[3];  /* [Grid] x{0,1,2}{min,max} for the Regular grid */
    const double* nodes[3];   /* optional host node coordinates (length n_d + 1) for a
                                 UserDefined grid; NULL selects Regular (grid_type.cpp:151-186) */
    int precision;            /* enum hcl_precision, fused path */
    int device;               /* CUDA device ordinal */
    int pressure_fix;         /* [Pressure fix] pressure_fix == "On" (main.cpp:459-474) */
    double eps_pf;            /* [Pressure fix] eps_pf */
    int eos;                  /* enum hcl_eos ([Perfect Gas] gamma and mu serve both) */
} hcl_config;

typedef struct hcl_handle hcl_handle;

/* Fills *cfg with the reference's defaults (utils/param.cpp:14-73). */
void hcl_config_default(hcl_config* cfg);

/* Creates a solver for one domain on one GPU.  Builds the grid arrays
 * (x, dx, centres, ds, dv, point-mass g) on the host exactly as Grid::set_grid
 * does (mesh/grid.cpp:134-155, mesh/geometry.cpp:32-126) and uploads them.
 * Replaces the construction block of main.cpp:138-289. */
int hcl_create(const hcl_config* cfg, hcl_handle** out);
int hcl_destroy(hcl_handle* h);
const char* hcl_last_error(void);
int hcl_abi_version(void);

/* The configuration the handle was created with (node pointers not kept). */
int hcl_get_config(const hcl_handle* h, hcl_config* out);
/* Extents with ghosts (Nx_local_wg, grid.cpp:119) and cell count. */
int hcl_get_extents(const hcl_handle* h, int n_wg[3], int64_t* ncells);
/* Interior extents (Nx_glob_ng; 1 on inactive dims) and ghost width. */
int hcl_get_interior(const hcl_handle* h, int nx[3], int* nghost);
/* Host copies of the grid arrays: x_d (n_d+1), dx_d (n_d), xc_d (n_d) for d<3,
 * ds (N*3) and dv (N); any pointer may be NULL. */
int hcl_get_grid(const hcl_handle* h, double* x[3], double* dx[3], double* xc[3], double* ds, double* dv);
/* Device pointers of the handle's grid arrays (Grid::dx0.., ds, dv). */
int hcl_get_grid_device(const hcl_handle* h, const double* dx[3], const double** ds, const double** dv);

/* ---- stage entry points: one per reference plugin ----------------------- */
/* All arrays are DEVICE pointers in the layout above; ng_eff selects
 * Range::with_ghosts(ng_eff) (mesh/range.cpp:367-403).  stream may be NULL
 * (the handle's stream).  None of these synchronise. */

/* conv_prim_to_cons (hydro/array_conversion.hpp:32-104) */
int hcl_conv_prim_to_cons(hcl_handle* h, int ng_eff, const double* rho, const double* u, const double* P,
                          double* rhou, double* E, void* stream);
/* conv_cons_to_prim (hydro/array_conversion.hpp:106-172) */
int hcl_conv_cons_to_prim(hcl_handle* h, int ng_eff, const double* rho, const double* rhou, const double* E,
                          double* u, double* P, void* stream);
/* temperature (analysis/temperature.hpp:18-25): T = compute_temp_from_pres(rho,
 * P) of the configured EOS over the range with ng_eff ghost layers. */
int hcl_temperature(hcl_handle* h, int ng_eff, const double* rho, const double* P, double* T, void* stream);
/* IFaceReconstruction::execute (hydro/face_reconstruction.hpp:40-43,
 * limited_linear_reconstruction.hpp:46-64): var -> var_rec(.., 2, ndim) */
int hcl_face_reconstruction(hcl_handle* h, int ng_eff, const double* var, double* var_rec, void* stream);
/* IHydroReconstruction::execute (hydro/hydro_reconstruction.hpp:46-58,85-129)
 * including HancockExtrapolationReconstruction (extrapolation_reconstruction.hpp:65-338).
 * dt is the reconstruction time step (the reference passes dt/2, main.cpp:427-439).
 * u_rec/P_rec are the scratch views MUSCLHancockHydroReconstruction owns
 * (hydro_reconstruction.hpp:67-68); pass NULL to use the handle's own.
 * fx/fx_rec may be NULL when nfx == 0. */
int hcl_hydro_reconstruction(hcl_handle* h, int ng_eff, double dt, const double* rho, const double* u,
                             const double* P, const double* fx, double* rho_rec, double* rhou_rec, double* E_rec,
                             double* fx_rec, double* u_rec, double* P_rec, void* stream);
/* hcl_hydro_reconstruction with its scratch (u_rec, P_rec, fx_rec_old) in one
 * fixed 32 MiB device array per device (2^22 doubles) instead of buffers the
 * handle allocates on first use: the call itself allocates and frees no
 * device memory.  No counterpart in the reference (its
 * MUSCLHancockHydroReconstruction owns Kokkos views allocated at
 * construction).  For host code whose time loop must not allocate after
 * set-up: an allocation there can synchronise the whole device, and a caller
 * that hands all free device memory to its own pool has none to give.
 * Limit: N * 2*ndim*(ndim + 1 + nfx) <= 2^22 doubles, N the cell count with
 * ghosts (2-D, nfx = 0: N <= 349525; 3-D: N <= 174762); larger grids get
 * HCL_ERR_CONFIG.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and switches to the handle's device for it; make
 * that first call before any stream capture.  The looked-up address is kept
 * for the life of the process: after a cudaDeviceReset of that device (or an
 * unload and reload of this library's module) it no longer names the array,
 * so do not call this entry point on a device that was reset after its first
 * call.  Nothing in the scratch needs to
 * start at zero (each call writes every entry it reads).  The array is shared
 * by all handles on a device: calls whose work overlaps in time on one device
 * (different streams, threads or handles) race on it; order them. */
int hcl_hydro_reconstruction_noalloc(hcl_handle* h, int ng_eff, double dt, const double* rho, const double* u,
                                     const double* P, const double* fx, double* rho_rec, double* rhou_rec,
                                     double* E_rec, double* fx_rec, void* stream);
/* pressure_fix (hydro/pressure_fix.hpp:19-172, called at main.cpp:459-474) on
 * no_ghosts: where the old internal energy is below eps times the kinetic
 * energy, E_new is rebuilt from a blend of the Godunov increment and a
 * pressure-work estimate.  Updates E_new in place; FP64, reference order. */
int hcl_pressure_fix(hcl_handle* h, double dt, double eps, const double* rho, const double* rhou, const double* E,
                     const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* rho_new,
                     const double* rhou_new, double* E_new, void* stream);
/* IGodunovScheme::execute (hydro/godunov_scheme.hpp:47-63,77-302) with the
 * Riemann solver chosen at hcl_create (factory_godunov_scheme, :305-321). */
int hcl_godunov_scheme(hcl_handle* h, int ng_eff, double dt, const double* rho, const double* rhou,
                       const double* E, const double* fx, const double* rho_rec, const double* rhou_rec,
                       const double* E_rec, const double* fx_rec, double* rho_new, double* rhou_new,
                       double* E_new, double* fx_new, void* stream);
/* DistributedBoundaryCondition::operator() on one rank
 * (boundary_distribute.hpp:42-76) + every IBoundaryCondition::execute
 * (boundary.hpp:81-87, boundary.cpp:221-296): fills all ghost cells in place. */
int hcl_boundary_conditions(hcl_handle* h, double* rho, double* rhou, double* E, double* fx, void* stream);
/* make_internal_mass_gravity (gravity/gravity.cpp:59-128) for handles created
 * with HCL_GRAVITY_INTERNAL_MASS: recomputes the handle's radial gravity table
 * from the density rho (device, with the ghost layers of dimension 0 filled):
 * shell means of rho over the interior (j, k), the enclosed mass at the cell
 * centres from the central mass outwards, g(i) = -G M(i) / xc(i)^2.  The
 * stage entry points that take gravity use the table from then on (the
 * reference rebuilds its Gravity object the same way, main.cpp:309 and :528).
 * g_out (device, n0 doubles, may be NULL) receives a copy of the table.
 * hcl_run and hcl_set_state* keep the table current by themselves. */
int hcl_internal_mass_gravity(hcl_handle* h, const double* rho, double* g_out, void* stream);
/* time_step (hydro/time_step.hpp:35-82): writes 1/max_cells(sum_d (|u_d|+c)/dx_d)
 * to *dt_out (host), i.e. the value the reference returns before main
 * multiplies by cfl.  Synchronises the stream. */
int hcl_time_step(hcl_handle* h, int ng_eff, const double* rho, const double* u, const double* P, double* dt_out,
                  void* stream);
/* minimum_internal_energy (analysis/internal_energy.cpp:20-45), no_ghosts. Synchronises. */
int hcl_minimum_internal_energy(hcl_handle* h, const double* rho, const double* rhou, const double* E,
                                double* out, void* stream);
/* integrate (analysis/integration.cpp:22-37): sum var*dv over no_ghosts,
 * compensated and deterministic.  Synchronises. */
int hcl_integrate(hcl_handle* h, const double* var, double* out, void* stream);

/* ---- handle-owned state and the fused step ------------------------------ */
/* Copies the conserved state in (rho, rhou, E, fx: full arrays with ghosts,
 * layout above) from host or device memory. fx may be NULL when nfx == 0. */
int hcl_set_state(hcl_handle* h, const double* rho, const double* rhou, const double* E, const double* fx,
                  int memory);
int hcl_get_state(hcl_handle* h, double* rho, double* rhou, double* E, double* fx, int memory);
/* Initial state from primitives on the interior (what a setup plugin's
 * InitializationSetup::execute writes, initialization_interface.hpp:33-39),
 * then conv_prim_to_cons + boundaries (main.cpp:305-307).  Host arrays of
 * full extent; ghost entries are ignored. */
int hcl_set_state_from_prim(hcl_handle* h, const double* rho, const double* u, const double* P,
                            const double* fx);

/* The primitive arrays main() holds when it writes an output (main.cpp:526 and
 * :317-318): rho, u (ndim components), P and, when T is not NULL, the
 * temperature, over all cells including ghosts (reference layout), plus the
 * passive scalars when fx is not NULL.  Host or device destination. */
int hcl_get_prim(hcl_handle* h, double* rho, double* u, double* P, double* T, double* fx, int memory);
/* Sets the time and the iteration count of the loop without touching the state
 * (a restart from an output: main.cpp:234-248 reads iter and current_time). */
int hcl_set_clock(hcl_handle* h, double t, int iter);

/* Parameters of the time loop (utils/param.cpp:40-50, main.cpp:354-385). */
typedef struct hcl_run_params {
    double cfl;               /* [Run] cfl */
    double t_end;             /* [Run] t_end */
    int max_iter;             /* [Output] max_iter (absolute iteration bound) */
    int iter_frequency;       /* [Output] iter_frequency (0 = off) */
    double time_frequency;    /* [Output] time_frequency (0 = off): dt is clamped to output times */
    double time_first_output; /* [Output] time_first_output */
    int nsteps;               /* steps to take in this call (<= 0: until t_end / max_iter) */
    int graph_chunk;          /* steps per CUDA-graph replay (0 = 60; rounded up to a multiple
                                 of 6).  A run of a fixed step count replays that graph and,
                                 for its remainder, graphs of 24, 12 and 6 steps (all captured
                                 on the handle's first fixed-count run), then launches the last
                                 < 6 steps singly */
    int fixed_dt;             /* 1: use dts[] (host, one per step) instead of the CFL dt */
    const double* dts;
} hcl_run_params;

typedef struct hcl_run_result {
    double t;                 /* time after the last step */
    int iter;                 /* iterations done since the state was set */
    int status;               /* HCL_OK, HCL_ERR_INVALID_STATE, HCL_ERR_NEGATIVE_DT, HCL_ERR_TIMEOUT */
    int64_t bad_cell;         /* first cell with NaN / negative internal energy, or -1 */
    int finished;             /* 1 when t_end or max_iter was reached */
    double last_dt;
} hcl_run_result;

/* Runs the reference time loop (main.cpp:354-531) with the fused step kernel,
 * everything on the device: CFL dt reduced inside the step kernel, dt clamps,
 * health check and ghost filling in place; steps are replayed from CUDA graphs.
 * Synchronises at the end (and between graph chunks when nsteps <= 0).
 * Passive scalars (nfx > 0) and the pressure fix ride in the fused
 * shared-memory tile kernels (FP64, fast FP64 and FP32-mixed, which applies
 * the fix in FP64 to its FP32 face states); the state then includes fx.
 * Handles with more passive scalars than the tile's shared memory holds, and
 * handles set to it by hcl_set_stage_loop, run the same loop composed of the
 * FP64 stage entry points (reconstruction, Godunov, pressure fix, boundaries,
 * cons->prim) in the reference's order, with dt and the health check read
 * back each step. */
int hcl_run(hcl_handle* h, const hcl_run_params* p, hcl_run_result* r);
/* One step of the fused kernel with the given dt (no CFL clamp logic, no
 * synchronisation): the building block the adapters use. */
int hcl_step_fixed_dt(hcl_handle* h, double dt, void* stream);
/* Resets time/iteration counters (t = t_ini) without touching the state. */
int hcl_reset_clock(hcl_handle* h, double t_ini);
/* Records the dt of each step taken by hcl_run into a device log that
 * hcl_get_dt_log copies out (adjoint and parity tools). */
int hcl_get_dt_log(hcl_handle* h, double* dts, int max_count, int* count);

/* Schedule of the FP32-mixed fused kernel.  -1 (default): autotuned on the
 * first run; -2: leaves the schedule unchanged (query).  2-D: 0-2
 * shared-memory tiles (16x16, 32x8, 32x16); on uniform Cartesian grids 3-5
 * warp strips of 32/64/128 rows, 6 warp strips fitted to one wave of
 * resident warps (7-8 unused), 9 fitted warp strips in 16-warp CTAs that march in step with their
 * rows staged by the Tensor Memory Accelerator (even ghost width), 10 the same
 * with per-lane cp.async staging.  3-D: 0
 * shared-memory tiles, 1 column march (uniform Cartesian grids).  With
 * passive scalars only the tiles qualify, and for one or two scalars also
 * 3-6 in 2-D, for one scalar 1 in 3-D.  Returns the schedule in use through *used (may be NULL; -1 before
 * the autotuner ran). */
int hcl_set_schedule(hcl_handle* h, int schedule, int* used);

/* Selects the time loop of hcl_run: 0 (default) the fused loop wherever the
 * fused kernels carry the handle's features, 1 the loop composed of the FP64
 * stage entry points in the reference's order (main.cpp:354-531, one kernel
 * per Kokkos kernel, dt and the health check read back each step).  Both
 * give the same FP64 results; the staged loop is the reference's own
 * structure, for stage-wise comparisons.  Call before the first state is
 * set (HCL_ERR_CONFIG afterwards). */
int hcl_set_stage_loop(hcl_handle* h, int on);

/* Compensated FP64 sums over no_ghosts: out[0] = sum rho dv, out[1..ndim] =
 * sum rhou_d dv, out[ndim+1] = sum E dv.  Deterministic. */
int hcl_conservation_sums(hcl_handle* h, double* out);

/* Number of kernels of this library launched by the calling process so far
 * (host-side counter of launches issued). */
int64_t hcl_kernel_launch_count(void);

/* The CUDA stream (cudaStream_t) the handle launches on, so callers can order
 * their own work or record timing events on it. */
int hcl_get_stream(const hcl_handle* h, void** stream);

/* ---- discrete adjoint of the fused step ------------------------------------ */
/* Reverse-mode derivative of nsteps fused steps with dt held fixed per step
 * (recorded by the forward pass or given).  Supported: Cartesian and
 * spherical grids, regular or of user-defined nodes (the spherical face areas,
 * volumes and geometric source terms included), uniform, point-mass and
 * internal-mass gravity, HLL/HLLC/Low Mach, every limiter, ndim 1-3, passive
 * scalars (as many as the reverse tile's shared memory holds: 3-D FP64 sweeps
 * take one), no pressure fix, the perfect-gas EOS; anything else returns
 * HCL_ERR_CONFIG.  Branches (limiter sign tests, wave-speed min/max, HLLC
 * switches) are differentiated along the branch the forward evaluation took;
 * for the passive scalars (their limiters, the upwind choice of each face and
 * the clamp of x' to [0, 1]) along the branch of the sweep's own
 * recomputation.  No reference counterpart: the reference has no adjoint. */
typedef struct hcl_adjoint_params {
    int nsteps;
    const double* dts;        /* host, nsteps values; NULL: CFL dt of this forward run (recorded) */
    double cfl;               /* CFL number when dts == NULL */
    int checkpoint_every;     /* store the state every k steps (0: 32) */
    int precision;            /* reverse sweep: HCL_FP64 or HCL_FP32_MIXED (state and adjoint stay FP64) */
} hcl_adjoint_params;

/* Forward pass: runs nsteps fused steps from the current state U^0 (in the
 * handle's precision), checkpointing the state every k steps.  The handle's
 * state becomes U^N; dts used are available through hcl_adjoint_dts. */
int hcl_adjoint_forward(hcl_handle* h, const hcl_adjoint_params* p);
/* Reverse pass: given lam_final = dJ/dU^N, writes grad = dJ/dU^0 for the
 * interior cells (ghost entries are zero: ghosts are functions of the
 * interior).  Both are one contiguous buffer of (ndim+2+nfx)*N doubles holding
 * the full arrays rho, rhou (ndim planes), E and the nfx passive scalars (the
 * mass fractions fx, not rho*fx) in the layout above.  Each
 * checkpoint segment is recomputed forward on the device, then swept
 * backward step by step. */
int hcl_adjoint_backward(hcl_handle* h, const double* lam_final, double* grad, int memory);
/* The dt of each step of the last hcl_adjoint_forward (host array of nsteps). */
int hcl_adjoint_dts(const hcl_handle* h, double* dts, int max_count, int* count);

/* ---- batched ensemble of independent 2-D problems --------------------------- */
/* Many independent domains (uneven grids) stepped together by one persistent
 * cooperative kernel: warp strips of every problem are the work items, each
 * problem keeps its own CFL dt, and a bounded grid barrier (HCL_ERR_TIMEOUT
 * instead of a hang) separates steps.  Every problem must be 2-D, uniform
 * Cartesian, uniform gravity, FP32-mixed, and share one limiter and Riemann
 * solver.  No reference counterpart: the reference runs one domain per
 * executable. */
typedef struct hcl_ensemble hcl_ensemble;

typedef struct hcl_ensemble_params {
    int nsteps;               /* steps every problem takes */
    double cfl;
    int checkpoint_every;     /* > 0: store checkpoints for hcl_ensemble_adjoint */
    int strip_rows;           /* 0: autotune among 32/64/128 */
    int blocks_per_sm;        /* 0: autotune */
    int use_graph;            /* 1: capture the persistent launch in a CUDA graph and replay it */
    int adjoint_precision;    /* HCL_FP64 or HCL_FP32_MIXED reverse sweep for hcl_ensemble_adjoint */
    int warps_per_cta;        /* 0: autotune; 4 or 16 warps per CTA of the persistent launch */
    long long barrier_spin_limit; /* polls of the step barrier before it gives up with HCL_ERR_TIMEOUT
                                   * (every CTA then returns); 0: 2^26 polls, a few seconds */
    int barrier_extra_arrivals;   /* failure-path tests only: the step barrier waits for this many
                                   * arrivals beyond the CTA count, which never come, so it runs out
                                   * its limit; 0 in normal use */
} hcl_ensemble_params;

typedef struct hcl_ensemble_result {
    int status;               /* HCL_OK, HCL_ERR_INVALID_STATE, HCL_ERR_TIMEOUT */
    int strip_rows;           /* schedule used */
    int blocks_per_sm;
    int grid;                 /* CTAs of the persistent launch */
    int launches;             /* persistent launches issued (1 per checkpoint segment) */
    int graph;                /* 1 when replayed from a CUDA graph */
    int64_t cells;            /* interior cells over all problems */
    int warps_per_cta;
} hcl_ensemble_result;

/* Creates one handle per configuration (hcl_create) plus the batch. */
int hcl_ensemble_create(const hcl_config* cfgs, int nprob, hcl_ensemble** out);
int hcl_ensemble_destroy(hcl_ensemble* e);
/* Handle of problem p (set its state, read results, per-problem queries). */
int hcl_ensemble_handle(hcl_ensemble* e, int p, hcl_handle** h);
int hcl_ensemble_stream(const hcl_ensemble* e, void** stream);
/* Advances every problem by nsteps (synchronises at the end). */
int hcl_ensemble_run(hcl_ensemble* e, const hcl_ensemble_params* p, hcl_ensemble_result* r);
/* Reverse pass of the last run (which needs checkpoint_every > 0): for every
 * problem p, lam_final[p] = dJ/dU_p^N and grads[p] receives dJ/dU_p^0 (same
 * buffer layout as hcl_adjoint_backward).  The problems' sweeps run
 * concurrently on their own streams. */
int hcl_ensemble_adjoint(hcl_ensemble* e, const double* const* lam_final, double* const* grads, int memory);

/* ---- outputs and restarts (host only) --------------------------------------- */
/* The reference writes one HDF5 file per output through PDI
 * (io/io.cpp:185-318 write_pdi, dataset set io/config.yaml.cpp:7-265) and
 * restarts from one (read_pdi, io/io.hpp:40-53).  No HDF5 library is used
 * here: the same datasets -- output_id, iter_output_id, time_output_id, iter,
 * current_time, gamma, x0..x2 (nodes with ghosts), x0_ng..x2_ng (interior
 * nodes), rho, ux0..ux{ndim-1}, P, E, T, fx0..fx{nfx-1} (interior cells,
 * C order [nx2][nx1][nx0]) -- go into one raw file "<prefix>_<output_id,
 * 8 digits>.hclraw": the magic "HCLRAW01", the byte length of a text index,
 * the index (one line per dataset: name, type f64|i32, byte offset, extents),
 * then little-endian data at 64-byte aligned offsets.  An XDMF file
 * "<prefix>.xmf" lists every output written so far as a time series whose
 * attributes point into the raw files (Format="Binary", Seek = offset), like
 * the reference's XmlWriter (io/io.hpp:56-81) does into its HDF5 files. */
int hcl_write_output(hcl_handle* h, const char* directory, const char* prefix, int output_id, int iter_output_id,
                     int time_output_id, int iter, double t);
/* Restart (main.cpp:225-246): reads rho, u, P, fx and the clock from an output
 * file into a handle of the same grid (the file's nodes must equal the
 * handle's, else HCL_ERR_CONFIG), sets the state from the primitives
 * (conv_prim_to_cons + boundaries, as hcl_set_state_from_prim) and the clock
 * (hcl_set_clock); returns the output counters through the pointers (each may
 * be NULL). */
int hcl_read_restart(hcl_handle* h, const char* path, int* output_id, int* iter_output_id, int* time_output_id,
                     int* iter, double* t);

/* ---- .ini front end (host only) ------------------------------------------ */
/* Compile-time choices of the reference (CMake Heraclespp_NDIM, _GEOM,
 * _GRAVITY, _SETUP; CMakeLists.txt:11-79) given at run time. */
typedef struct hcl_build_options {
    int ndim;                 /* 0: infer from Nx1_glob/Nx2_glob > 1 */
    int geometry;             /* enum hcl_geometry */
    int gravity;              /* enum hcl_gravity */
    int precision;            /* enum hcl_precision */
    int device;
    const char* setup;        /* setup plugin name, e.g. "shock_tube" */
    int eos;                  /* enum hcl_eos */
} hcl_build_options;

/* Initial primitives of a setup plugin (InitializationSetup::execute,
 * initialization_interface.hpp:33-39) on the interior cells, parameterised by
 * the [Initialisation] keys of ini_path (NULL: the setup's defaults).  Host
 * arrays of full extent n_wg; xc_d are the cell centres (Grid::x{d}_center). */
int hcl_setup_initial_prim(const char* setup, const char* ini_path, int ndim, const int n_wg[3], int nghost,
                           const double* xc0, const double* xc1, const double* xc2, double* rho, double* u,
                           double* P);

/* Everything main.cpp:138-311 does before the time loop, from an .ini file:
 * Param, BC resolution and factories, grid, setup plugin, prim->cons and
 * boundaries; fills *run from [Run]/[Output] (nsteps = 0: run to t_end). */
int hcl_create_from_ini(const char* ini_path, const hcl_build_options* opt, hcl_handle** out, hcl_run_params* run);

#ifdef __cplusplus
}
#endif
#endif /* HERACLES_B200_H */
