/*
 * hcl_oracle.h -- CPU restatement of HERACLES++'s MUSCL-Hancock step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA product is
 * checked against: it is never linked into, loaded by, or called from the
 * product library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may use it.
 *
 * Every function restates one reference function or Kokkos kernel, in the
 * same operation order, so that an FP64 build without FMA contraction gives
 * the same bits as the reference's own FP64 CPU build.  Citations are
 * path:line inside the reference project.
 *
 * Array layout follows Kokkos::LayoutLeft (src/utils/kokkos_shortcut.hpp:22-41):
 * the first index (i, along x0) is fastest, trailing component indices are
 * slowest.  With N = n0*n1*n2 cells (ghosts included):
 *   rho(i,j,k)            -> rho[c]                    c = i + n0*(j + n1*k)
 *   rhou(i,j,k,d)         -> rhou[c + N*d]
 *   rho_rec(i,j,k,s,d)    -> rho_rec[c + N*(s + 2*d)]
 *   rhou_rec(i,j,k,s,d,r) -> rhou_rec[c + N*(s + 2*(d + ndim*r))]
 *   ds(i,j,k,d)           -> ds[c + N*d]   (d < 3)
 */
#ifndef HCL_ORACLE_H
#define HCL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_LIM_CONSTANT = 0, OR_LIM_VANLEER = 1, OR_LIM_MINMOD = 2, OR_LIM_VANALBADA = 3 };
enum { OR_RS_HLL = 0, OR_RS_HLLC = 1, OR_RS_SPLITTING = 2 };
enum { OR_BC_NULLGRADIENT = 0, OR_BC_PERIODIC = 1, OR_BC_REFLEXIVE = 2 };
enum { OR_GEOM_CARTESIAN = 0, OR_GEOM_SPHERICAL = 1 };
enum { OR_GRAV_UNIFORM = 0, OR_GRAV_POINT_MASS = 1, OR_GRAV_INTERNAL_MASS = 2 };
enum { OR_EOS_PERFECT_GAS = 0, OR_EOS_RAD_GAS = 1 };

/* Everything the reference keeps in Grid, EOS, Gravity and the factories. */
typedef struct or_ctx {
    int ndim;          /* ndim.hpp.in:6 */
    int ng;            /* [Grid] Nghost, param.cpp:26 */
    int nfx;           /* [Passive Scalar] nfx, param.cpp:66 */
    int nx[3];         /* Nx_glob_ng (interior cells; 1 on inactive dims) */
    int n[3];          /* Nx_local_wg (cells incl. ghosts) */
    int geom;
    double gamma, gamma_m1, mmw; /* perfect_gas.cpp:13 */
    int limiter, riemann;
    int bc[6];         /* index 2*idim + iface */
    int bc_order[6];   /* boundary_distribute.cpp:33-71 */
    int gravity;
    double g[3];       /* UniformGravity values */
    double central_mass;
    /* grid arrays, owned by the context (grid.cpp:48-76) */
    double *x[3];      /* nodes, n[d]+1 */
    double *dx[3];     /* n[d] */
    double *xc[3];     /* n[d] */
    double *ds;        /* N*3 */
    double *dv;        /* N */
    double *g_r;       /* PointMassGravity / InternalMassGravity g(i), n[0] (NULL for uniform) */
    int eos;           /* OR_EOS_PERFECT_GAS or OR_EOS_RAD_GAS (eos.hpp.in) */
} or_ctx;

/* ---- grid / context -------------------------------------------------- */
/* Regular grid (grid_type.cpp:151-186), cell sizes/centres (grid.cpp:31-44),
 * ds/dv (geometry.cpp:32-126), point-mass g (gravity.cpp:49-55).
 * Returns 0 or a negative code for invalid EOS parameters (perfect_gas.cpp:13-22). */
int or_ctx_init(or_ctx* c, int ndim, const int nx[3], int ng, int nfx, int geom,
                double gamma, double mmw, int limiter, int riemann, const int bc[6],
                int gravity, const double g[3], double central_mass,
                const double xmin[3], const double xmax[3]);
/* Same but with caller-given node coordinates (UserDefined grid). */
int or_ctx_init_nodes(or_ctx* c, int ndim, const int nx[3], int ng, int nfx, int geom,
                      double gamma, double mmw, int limiter, int riemann, const int bc[6],
                      int gravity, const double g[3], double central_mass,
                      const double* x0, const double* x1, const double* x2);
void or_ctx_free(or_ctx* c);
long or_ncells(const or_ctx* c);
/* Sets OpenMP threads used by the array kernels (0 = leave default). */
void or_set_threads(int nthreads);
int or_get_threads(void);

/* ---- per-cell physics (for known-answer tests) ------------------------ */
/* prim/cons/flux are arrays [rho, v_0..v_{ndim-1}, last] */
void or_to_prim(const or_ctx* c, const double* cons, double* prim);          /* euler_equations.hpp:111-122 */
void or_to_cons(const or_ctx* c, const double* prim, double* cons);          /* euler_equations.hpp:124-134 */
void or_flux_from_prim(const or_ctx* c, const double* prim, int locdim, double* flux); /* :72-86 */
void or_flux_from_cons(const or_ctx* c, const double* cons, int locdim, double* flux); /* :93-109 */
double or_ek_prim(const or_ctx* c, const double* prim);                      /* :51-59 */
double or_ek_cons(const or_ctx* c, const double* cons);                      /* :41-49 */
double or_slope(int limiter, double diffR, double diffL);                    /* slope_limiters.hpp */
void or_riemann(const or_ctx* c, int solver, const double* consL, const double* consR, int locdim, double* flux);
double or_speed_of_sound(const or_ctx* c, double rho, double P);             /* perfect_gas.hpp:80-83 */
double or_evol_from_pres(const or_ctx* c, double rho, double P);             /* perfect_gas.hpp:46-50 */
double or_pres_from_evol(const or_ctx* c, double rho, double evol);          /* perfect_gas.hpp:58-62 */
int or_eos_valid(double rho, double P);                                      /* perfect_gas.hpp:85-89 */
/* selects the EOS of a context (PerfectGas after or_create); RadGas:
 * thermodynamics/rad_gas.hpp:47-141 with the constructor checks of
 * rad_gas.cpp:13-22, which are the PerfectGas ones */
void or_set_eos(or_ctx* c, int eos);
double or_temperature(const or_ctx* c, double rho, double P);                /* compute_temp_from_pres */

/* ---- array kernels ---------------------------------------------------- */
/* ng_eff selects Range::with_ghosts(ng_eff) (range.cpp:367-403). */
void or_conv_prim_to_cons(const or_ctx* c, int ng_eff, const double* rho, const double* u, const double* P,
                          double* rhou, double* E);                                   /* array_conversion.hpp:32-104 */
void or_conv_cons_to_prim(const or_ctx* c, int ng_eff, const double* rho, const double* rhou, const double* E,
                          double* u, double* P);                                      /* array_conversion.hpp:106-172 */
void or_face_reconstruction(const or_ctx* c, int ng_eff, const double* var, double* var_rec, long rec_stride_d);
                                                                                      /* limited_linear_reconstruction.hpp:46-64 */
void or_hydro_reconstruction(const or_ctx* c, int ng_eff, double dt, const double* rho, const double* u,
                             const double* P, const double* fx, double* rho_rec, double* rhou_rec,
                             double* E_rec, double* fx_rec, double* u_rec, double* P_rec);
                                                                                      /* hydro_reconstruction.hpp:85-129 + extrapolation_reconstruction.hpp:65-338 */
void or_godunov(const or_ctx* c, int ng_eff, double dt, const double* rho, const double* rhou, const double* E,
                const double* fx, const double* rho_rec, const double* rhou_rec, const double* E_rec,
                const double* fx_rec, double* rho_new, double* rhou_new, double* E_new, double* fx_new);
                                                                                      /* godunov_scheme.hpp:77-302 */
void or_boundaries(const or_ctx* c, double* rho, double* rhou, double* E, double* fx); /* boundary_distribute.hpp:42-76 */
double or_time_step(const or_ctx* c, int ng_eff, const double* rho, const double* u, const double* P);
                                                                                      /* time_step.hpp:35-82 (returns 1/max) */
double or_min_internal_energy(const or_ctx* c, const double* rho, const double* rhou, const double* E);
                                                                                      /* internal_energy.cpp:20-45 */
double or_integrate(const or_ctx* c, const double* var);                              /* integration.cpp:22-37 */

/* ---- time loop ---------------------------------------------------------- */
typedef struct or_run_params {
    double cfl, t_ini, t_end;
    int max_iter;              /* [Output] max_iter, main.cpp:382 */
    int iter_frequency;        /* [Output] iter_frequency */
    double time_frequency;     /* [Output] time_frequency */
    double time_first_output;  /* [Output] time_first_output */
    int fixed_dt;              /* 1: use dts[] instead of the CFL dt (adjoint checks) */
    const double* dts;
    int pressure_fix;          /* [Pressure fix] pressure_fix == "On" (main.cpp:459) */
    double eps_pf;             /* [Pressure fix] eps_pf */
} or_run_params;

typedef struct or_run_result {
    double t;
    int iter;
    int status;                /* 0 ok, 1 invalid internal energy (main.cpp:397-425), 2 negative dt */
    double initial_mass, final_mass;
} or_run_result;

/* Runs the main loop of main.cpp:354-531 in place on the conserved state
 * (ghost cells included).  If dts_out is non-NULL, the dt of each step is stored. */
int or_run(const or_ctx* c, double* rho, double* rhou, double* E, double* fx, const or_run_params* p,
           or_run_result* r, double* dts_out);

/* pressure_fix.hpp:19-172 on no_ghosts; updates E_new in place. */
/* InternalMassGravity (gravity.cpp:59-128) on one rank: recomputes c->g_r
 * from the density rho (shell means over the interior (j, k), enclosed mass at
 * the cell centres by a running sum from the central mass). */
void or_internal_mass_gravity(const or_ctx* c, const double* rho);
void or_pressure_fix(const or_ctx* c, double dt, double eps, const double* rho, const double* rhou, const double* E,
                     const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* rho_new,
                     const double* rhou_new, double* E_new);

/* Initial state helper: given primitives on the interior, computes the
 * conserved state and fills the ghosts (main.cpp:305-307). */
void or_init_from_prim(const or_ctx* c, const double* rho_prim, const double* u, const double* P,
                       double* rho, double* rhou, double* E, double* fx);

#ifdef __cplusplus
}
#endif
#endif
