/*
 * gfsph.h — C ABI of the B200 (sm_100a) implementation of Geoflow-SPH's
 * per-time-step depth-integrated SPH hot path.
 *
 * Reference program: EL-BID/Deslizamientos-y-flujos, the Fortran sources in "Codes Geoflow_SPH"
 * (files are cited by base name without their numeric prefix).
 *
 * In the reference the step is a set of argument-less Fortran module procedures
 * working on module globals:
 *   - adaptive_dt_sph        SPH_MAIN_2019.f90:289 -> Adaptive_dt_sph_SW SPH_SW_2019.f90:6521-6664
 *   - time_integration_sph   SPH_MAIN_2019.f90:220-283 -> RK45 SPH_MAIN_2019.f90:746-1005
 *   - called from Driver_Flow's DTGT loop SPH_FEM_Driver_2019.f90:1580-1697
 *     (adaptive_dt_sph at :1590, time_integration_sph at :1617)
 * The globals it reads and writes are x, vx, rho (= flow depth h), mass
 * (= volume), hsml, itype, If_Out_Domain (SPH_Main_Vars_2019.f90), dt_sph and
 * time_sph (SPH_FEM_Driver_time_vars_2019.f90), const(1..110)
 * (SPH_SW_Vars_2019.f90:27) and topol/coorg/xming/deltxg/npoigx
 * (SPH_FEM_topo_2019.f90:94-110).
 *
 * This ABI replaces those procedures with explicit calls on an opaque handle
 * that owns all device memory.  Host arrays are caller-owned and only copied.
 * Particle arrays use the reference's Fortran layout: vectors are (2,n)
 * column-major FP32, i.e. x[2*i+0] = x(1,i+1), x[2*i+1] = x(2,i+1).
 * Every call returns an int status: 0 ok, > 0 warning, < 0 error.
 * Calls on one handle must not run concurrently.  Nothing here falls back to
 * the CPU: without a usable CUDA device every compute call fails with
 * GFSPH_ERR_NO_DEVICE.
 */
#ifndef GFSPH_H
#define GFSPH_H

#ifdef __cplusplus
extern "C" {
#endif

#define GFSPH_NCONST 110
#define GFSPH_NTOPO 16

/* status codes */
#define GFSPH_OK 0
#define GFSPH_T_END_REACHED 1        /* warning: stopped early because time >= t_end */
#define GFSPH_ERR_ARG (-1)           /* bad argument (null pointer, bad size) */
#define GFSPH_ERR_CUDA (-2)          /* CUDA runtime error; when a device allocation failed
                                        (in gfsph_upload or while growing the grid or the
                                        neighbour table during a step) the handle holds no
                                        state until the next gfsph_upload */
#define GFSPH_ERR_CAPACITY (-3)      /* cell grid / neighbour table could not be grown */
#define GFSPH_ERR_UNSUPPORTED (-4)   /* option outside the implemented path */
#define GFSPH_ERR_STATE (-5)         /* call out of order (e.g. step before upload) */
#define GFSPH_ERR_NO_DEVICE (-6)     /* no usable CUDA device */
#define GFSPH_ERR_NONFINITE (-7)     /* a non-finite value appeared in the state */
#define GFSPH_ERR_DOMAIN (-8)        /* all particles left the DEM box */
#define GFSPH_ERR_HOST (-9)          /* host memory could not be allocated */

/*
 * Control parameters.  cst[k-1] holds the reference's const(k)
 * (read in blocks of 15 by Input_SW, SPH_SW_2019.f90:1151-1204).  The ones the
 * step uses: const(1) g, const(2) density, const(3) Voellmy xi (or Manning n,
 * or Bagnold K), const(5) nfric, const(6) yield stress, const(7) viscosity K,
 * const(8) Herschel-Bulkley exponent m,
 * const(9) tan(phi), const(10) hfrict0, const(15) comp, const(16) ic_cosTheta
 * (0 g, 1 g/sqrt(1+|grad Z|^2) in the pressure and the friction, IntForces_SW
 * SPH_SW_2019.f90:6775-6783, Get_Grav_Ext_SW :9264-9270), const(20)
 * density-factor switch (0 or 1), const(21)
 * erosion law (1 = Hungr, 2 = bed angle above the equilibrium angle, with a
 * frictional law, 3 = basal shear above the bed strength; 2 and 3 with
 * const(17)/(18) solid and fluid densities), const(22) erosion constant,
 * const(23) law 2's C* or law 3's bed cohesion, const(24)/(25) law 3's
 * tan(phi) and pore-pressure factor, const(47) slip factor alpha, const(48)
 * maximum erodible depth.
 */
typedef struct gfsph_params {
    float cst[GFSPH_NCONST];
    int pa_sph;            /* 1 or 2, SPH_SW_2019.f90:6905-6920 */
    int nnps;              /* 2 or 4 (grid_find_NEW_tools / _tools3); the same sets for skf 1 and 4 */
    int sle;               /* 0 keep hsml, 1 hsml = 2 sqrt(m/h) (h_upgrade SPH_MAIN_2019.f90:2925-2931) */
    int skf;               /* 1 cubic spline, 2 Gaussian, 3 quintic, 4 Wendland C2 (kernel_TOOLS
                              My_SPH_Tools_2019.f90:2062); 2 and 3 (support 3h) need nnps 2 */
    int summation_density; /* must be 1 (sum_density_Tools) */
    int average_velocity;  /* 1 applies av_vel (XSPH, SPH_MAIN_2019.f90:3042-3099) */
    int nor_density;       /* 1 divides each density sum by sum_j (m_j/h_j) W_ij
                              (sum_density_Tools My_SPH_Tools_2019.f90:1841-1846) */
    int ic_adapt;          /* ic_adapt_dt_sph: 0 fixed, 1 hsml/(3c), 2 hsml/(3(c+|v|)),
                              4 |DEM cell diagonal|/|v|, 10 min of modes 1 and 4 */
    float h_inf;           /* h_inf_SW */
    float dt;              /* initial dt_sph */
    int dem_deriv;         /* slopes when not supplied: 0 FEM projection (Get_Topol), 1 finite differences */
    int max_neighbours;    /* initial neighbour-table capacity per particle, 0..65536;
                              0 = 96 (grows on demand) */
    int icpwp;             /* 0 none; 1 basal pore-water pressure u integrated by the RK45 with the
                              dissipation of ExtForces_SW (SPH_SW_2019.f90:8648-8652); 3 with one point
                              (Get_Pwp_SW, nUaux = 1) */
    float pwp0rel;         /* icpwp = 1, 3: initial u, Uaux = pwp0rel * rho * const(14)
                              (Input_SW SPH_SW_2019.f90:1724-1737, 1829-1852) */
    int ws_interact;       /* ic_ws_Interact: 0 one material; 1 soil and water particles (ic_soil = ic_water = 1,
                              Input_SW SPH_SW_2019.f90:947-951): species from gfsph_set_species */
    int sw_alg;            /* ic_SWalg with ws_interact 1: 0 both as landslides; 1 water over the soil surface
                              (pressure g/2 (h^2 - Zp^2), Zp = Z + hs, SPH_SW_2019.f90:6809-6828) */
    int reserved[4];
} gfsph_params;

/*
 * The DEM ("topo grid"): npoigx x npoigy nodes, x fastest, node (ix,iy) at
 * (xmin + ix*dx, ymin + iy*dy).  Either pass the reference's topol(ntopo,npoig)
 * array as-is (topol != NULL, column-major, ntopo >= 15: Z, Zx, Zy, the six
 * curvature terms, ..., eroded depth (14), erodible depth (15)), or pass only
 * z (topol == NULL) and the slopes are derived with params->dem_deriv and the
 * erodible depth is initialised as Input_SW does (SPH_SW_2019.f90:1290-1310).
 */
typedef struct gfsph_dem {
    int nx, ny;            /* npoigx, npoigy */
    float xmin, ymin;      /* xming, yming */
    float dx, dy;          /* deltxg, deltyg */
    const float* topol;    /* optional, topol(ntopo, nx*ny) */
    int ntopo;
    const float* z;        /* used when topol == NULL: Z(nx*ny) */
} gfsph_dem;

typedef struct gfsph_handle gfsph_handle;

/* raster kinds for gfsph_raster (one value per DEM node, nx*ny) */
#define GFSPH_RASTER_DEPTH_IDW 0  /* IDW of h over the 4x4 node stencil, SPH_SW_2019.f90:14310-14400 */
#define GFSPH_RASTER_MAX_DEPTH 1  /* per-node max h over hazard samples, Get_MC_pixel_Vars_SW :20800-20812 */
#define GFSPH_RASTER_MAX_VEL 2    /* per-node max |v| over hazard samples */
#define GFSPH_RASTER_SUM_DEPTH 3  /* per-node sum of h over hazard samples */
#define GFSPH_RASTER_SUM_VEL 4    /* per-node sum of |v| over hazard samples */
#define GFSPH_RASTER_COUNT 5      /* per-node count of particle visits over hazard samples */
#define GFSPH_RASTER_Z 6          /* current terrain elevation topol(1,:) (lowered by erosion) */
#define GFSPH_RASTER_ERODED 7     /* accumulated eroded depth topol(14,:) */
#define GFSPH_RASTER_AVAILABLE 8  /* remaining erodible depth topol(15,:) */

/* Replaces Init_sph's SPH setup (SPH_MAIN_2019.f90:74) for the step: validates
 * the options, copies the DEM to the device, derives slopes if needed.
 * Basal laws (basal_friction_Ext_SW, SPH_SW_2019.f90:9355-9828): nfric 1
 * Manning, 2 laminar, 3 Bingham scaled by the eroded soil fraction (m - m0)/m
 * with m0 the mass at gfsph_upload (masses <= 1e-6 refused there with
 * GFSPH_ERR_ARG), 4 Bingham, 5/6 frictional with Voellmy (xi > 0) or
 * Coulomb-viscous (xi < 0), 7 with v^2/R, 8/26/27 mu(I), 11 Bagnold, 23
 * Herschel-Bulkley (m = 1, 2, 1/3 or 1/2) and 24/25 its approximations
 * (m > 0); yield stress const(6) >= 1e-32 for 4 and 23-25 (else
 * GFSPH_ERR_ARG); other laws GFSPH_ERR_UNSUPPORTED. */
int gfsph_create(const gfsph_params* params, const gfsph_dem* dem, gfsph_handle** out);

/* Frees all device memory of the handle. */
int gfsph_destroy(gfsph_handle* h);

/* Replaces the particle arrays filled by Setup_Global_Arrays_SW
 * (SPH_SW_2019.f90:6223-6246).  x, v: (2,n); rho, mass, hsml: (n); itype (n)
 * is 1 (soil) for every particle, or 1 or 2 (water) with ws_interact = 1
 * (NULL = all soil); out_flag (n) is If_Out_Domain (may be NULL = all
 * inside).  With soil and water (ic_ws_Interact = 1, SPH_SW_2019.f90:947-951)
 * the density, internal force and av_vel take pairs of one material only
 * (Pint_Update_SW_tools My_SPH_Tools_2019.f90:1652-1710); the soil-water pairs
 * push the soil (ExtForces_SW :8502-8521); the water is a Manning fluid whose
 * bed, with sw_alg 1, is the soil surface Z + hs (Get_hs_at_w_SW
 * :17789-17938, IntForces_SW :6809-6828, Get_Grav_Ext_SW :9322-9331).  That
 * option runs the staged RK45 (the soil surface of every stage); it excludes
 * erosion, pore pressure, nor_density and ic_cosTheta = 1, and the adjoint. */
int gfsph_upload(gfsph_handle* h, int n, const float* x, const float* v, const float* rho,
                 const float* mass, const float* hsml, const int* itype, const int* out_flag);

/* Copies the particle state back in the original particle order.  Any
 * pointer may be NULL to skip that array. */
int gfsph_download(gfsph_handle* h, float* x, float* v, float* rho, float* mass, float* hsml,
                   int* out_flag);

/* Basal pore-water pressure, u(:) (icpwp = 1) or Uaux(1,:) (icpwp = 3), n
 * values in the original particle order: gfsph_upload starts it as Input_SW
 * does (pwp0rel * rho * const(14), SPH_SW_2019.f90:1724-1737, 1829-1852);
 * these replace or read it (the reference's u or Uaux global, integrated by
 * the RK45 with ExtForces_SW's du, or updated by Get_Pwp_SW
 * SPH_SW_2019.f90:11176-11371 at the end of every step). */
int gfsph_set_pwp(gfsph_handle* h, const float* pwp);
int gfsph_get_pwp(gfsph_handle* h, float* pwp);

/* Replaces up to nsteps iterations of the DTGT loop body
 * (SPH_FEM_Driver_2019.f90:1580-1617): adaptive_dt_sph, time_integration_sph
 * (RK45 with summation density, internal and external forces, erosion,
 * h_upgrade, av_vel) and time += dt.  Stops early, returning
 * GFSPH_T_END_REACHED, once time >= t_end.  All steps run on the device
 * without host synchronisation.  t_out / steps_done may be NULL. */
int gfsph_step(gfsph_handle* h, int nsteps, double t_end, double* t_out, int* steps_done);

/* time_sph and dt_sph of the handle. */
int gfsph_get_time(gfsph_handle* h, double* t, float* dt);
int gfsph_set_time(gfsph_handle* h, double t, float dt);

/* Summation density on the current state without advancing it: the
 * neighbour search of grid_find_NEW_tools (My_SPH_Tools_2019.f90:1109-1370)
 * followed by sum_density_Tools (My_SPH_Tools_2019.f90:1763-1859); with
 * nor_density normalised with the depths held (after the h_inf clamp of
 * adaptive dt modes 1, 2 and 10).  Writes h per particle (original order) and
 * keeps the neighbour table for gfsph_neighbours. */
int gfsph_density(gfsph_handle* h, float* rho_out);

/* Neighbour sets of the last search (start of the last step, or
 * gfsph_density), original particle indices, CSR: offsets[n+1], idx[cap].
 * Each list is sorted ascending.  Returns GFSPH_ERR_CAPACITY when cap is too
 * small (offsets[n] then holds the needed size). */
int gfsph_neighbours(gfsph_handle* h, int cap, int* offsets, int* idx);

/* Per-particle internal (pressure) acceleration of IntForces_SW
 * (SPH_SW_2019.f90:6669-6941) on the current state, (2,n), original order.
 * Runs the search and density first (the first RK45 stage's pressure: with
 * nor_density the normalised depth, with ic_cosTheta = 1 g/deng at the
 * particles' positions). */
int gfsph_internal_forces(gfsph_handle* h, float* indvxdt);

/* One raster per DEM node, nx*ny values, x fastest. */
int gfsph_raster(gfsph_handle* h, int kind, float* out);

/* Misfit of the depth raster (GFSPH_RASTER_DEPTH_IDW) of the current state
 * against a target raster T (nx*ny): L = sum over DEM nodes of (R - T)^2, and,
 * when gx / gh are not NULL, its gradient with respect to the current
 * positions dL/dx (2,n) and depths dL/dh (n), caller order, zero for
 * particles outside the DEM.  After gfsph_adjoint_forward these are the
 * final-state gradients gfsph_adjoint_backward takes (with dL/dv = 0), which
 * gives dL/d(rheology) and dL/d(volumes) of a deposit-raster calibration.
 * No counterpart in the reference (it has no back-analysis). */
int gfsph_raster_misfit(gfsph_handle* h, const float* target, double* loss, float* gx, float* gh);

/* Adds the current particles to the per-node hazard statistics
 * (Get_MC_pixel_Vars_SW, SPH_SW_2019.f90:20717-20833: sum/max of h and |v|
 * over the particles in each node's cell).  Called at plot times. */
int gfsph_hazard_sample(gfsph_handle* h);
int gfsph_hazard_reset(gfsph_handle* h);

/* Runs the handle's kernels on this cudaStream_t (NULL = the handle's own). */
int gfsph_set_stream(gfsph_handle* h, void* cuda_stream);

/* Device timing with CUDA events on the handle's stream.  enable = 1: one
 * event pair around every kernel launch (graph replay off while on);
 * enable = 2: one event pair around the device work of each gfsph_step
 * call (graphs kept), read back as the last "kernel" slot ("step_batches",
 * launches = steps).  enable = 0: off.  Enabling resets the counters. */
int gfsph_profile(gfsph_handle* h, int enable);
int gfsph_profile_read(gfsph_handle* h, int kernel, double* total_ms, long long* launches);
int gfsph_num_kernels(void);
const char* gfsph_kernel_name(int kernel);

/* Number of kernels this handle has launched so far (graph replays count
 * each kernel node). */
long long gfsph_launch_count(gfsph_handle* h);

/* Search statistics of the last step: out[0] active particles, [1] regular
 * particles (a thread each and the neighbour table), [2] particles on the
 * coarse levels (a warp each), [3] levels, [4] cells,
 * [5] neighbour-table capacity per particle, [6] cell capacity, [7] particles
 * outside the DEM box.  Up to nout values are written. */
int gfsph_stats(gfsph_handle* h, int* out, int nout);

/* Derives the DEM slope/curvature rows topol(2..13,:) from topol(1,:) on the
 * host, once, as Topo_main does before the time loop: mode 0 = lumped-mass
 * FEM projection with 5 Jacobi sweeps (Get_Topol, SPH_FEM_topo_2019.f90:1723-1939),
 * mode 1 = central differences (Fdiff_derivs, :2812-2877).  topol is
 * (GFSPH_NTOPO, nx*ny) column-major; row 1 is read, rows 2..13 written. */
int gfsph_dem_topol(int mode, int nx, int ny, float dx, float dy, float* topol);

/*
 * The SPH -> FEM coupling pass get_gradhs_w (SPH_GFL_SW_Interactions_2019.f90:368-564)
 * on the node window [ix0, ix0+nwx) x [iy0, iy0+nwy) of the DEM background
 * triangulation (SPH_FEM_topo_2019.f90:583-604: two triangles per DEM cell,
 * (n, n+1, n+1+nx) and (n, n+1+nx, n+nx)), from the current particles:
 *   hs_w[nwx*nwy]        node depths, inverse-distance averages of the depth
 *                        of the particles in each node's triangles;
 *   gradhs_w[2*nwx*nwy]  (x, y) per node: the P1 projection g of the element
 *                        gradients, M g = sum_e (A_e/3) grad_e.
 * niter >= 1 solves as the reference does: niter sweeps
 * g += (rhs - M g)/mmatl from g = 0, the first of which leaves g = 0
 * (:497-501; the reference uses 5).  niter = 0 solves M g = rhs with the
 * device CG (solvegc2 semantics) to the squared-norm tolerance tol.
 * Either output may be NULL.
 */
int gfsph_gradhs(gfsph_handle* h, int ix0, int iy0, int nwx, int nwy, int niter, float tol, float* hs_w,
                 float* gradhs_w);

/*
 * Neighbour-search tunables, which change the speed of the search and never
 * its neighbour sets: level 0 holds the particles with hsml <= Hc =
 * min(max hsml, level_factor * mean hsml) (default 1.5, range [1, 16]), level
 * k >= 1 those with hsml in (Hc 2^(k-1), Hc 2^k]; level k's cells are
 * Hc * 2^k / cell_div wide (default 3, range [1, 8]).  Levels 0 and 1 are
 * searched by a thread per particle, coarser ones by a warp per particle.
 * gfsph_autotune times `steps` steps for each of 12 candidate pairs from
 * the current state (restored after every trial), keeps the fastest and
 * returns it with its time per step; the handle's state is unchanged.  The
 * per-particle sums then run in another neighbour order, so results may
 * differ from the defaults' in the last FP32 bit.
 */
int gfsph_set_search(gfsph_handle* h, float level_factor, float cell_div);
int gfsph_get_search(gfsph_handle* h, float* level_factor, float* cell_div);
int gfsph_autotune(gfsph_handle* h, int steps, float* level_factor, float* cell_div, float* best_ms_per_step);

/*
 * Adjoint of the step: gradients of a loss on the final state of nsteps steps
 * with respect to the initial positions and velocities, the particle volumes
 * and the basal rheology (tanfi = const(9), xi = const(3)), for
 * back-analysis.  This is a new capability; the reference has none.
 *
 * gfsph_adjoint_forward runs nsteps steps from the handle's state (the
 * handle ends at the final state) and keeps the state every `every` steps in
 * device memory (16 bytes per particle per kept state).
 * gfsph_adjoint_backward takes dL/dx, dL/dv (2n each, caller order) and
 * optionally dL/dh (n, the final depth) of the final state and returns
 * dL/dx0, dL/dv0 (2n), dL/dvolume (n), dL/dtanfi and dL/dxi.  It recomputes
 * every step from the kept states (each step's neighbour list is held fixed,
 * as the forward step freezes it) and leaves the handle at the final state.
 *
 * Supported: nfric 5/6 with xi >= 0 and the Bingham law nfric 4, no erosion
 * or pore pressure, pa_sph 2, sle 0 or 1 (with sle 1 the smoothing lengths of
 * every step are differentiated through h_upgrade and every pair's kernel),
 * ic_adapt 0, one grid level and no particle leaving the DEM
 * (GFSPH_ERR_UNSUPPORTED otherwise), one material (ws_interact 0).
 *
 * The record refers to its handle: call gfsph_adjoint_backward only while
 * that handle exists (gfsph_adjoint_destroy does not touch it, so the record
 * may be destroyed before or after the handle).
 */
typedef struct gfsph_adjoint gfsph_adjoint;
int gfsph_adjoint_forward(gfsph_handle* h, int nsteps, int every, gfsph_adjoint** out);
int gfsph_adjoint_backward(gfsph_adjoint* a, const float* gx, const float* gv, const float* gh, float* gx0,
                           float* gv0, float* gm, double* gmu, double* gxi);
/* One rheology gradient of the last gfsph_adjoint_backward on a: which = 0
 * dL/dtanfi (const(9)), 1 dL/dxi (const(3)), 2 dL/d(Bingham yield stress,
 * const(6); nfric 4).  GFSPH_ERR_STATE before the first backward pass. */
#define GFSPH_ADJ_TANFI 0
#define GFSPH_ADJ_XI 1
#define GFSPH_ADJ_TAUY 2
int gfsph_adjoint_param(gfsph_adjoint* a, int which, double* value);
int gfsph_adjoint_destroy(gfsph_adjoint* a);

/*
 * Monte-Carlo ensembles (the realization loop of SPH_FEM_Driver_2019.f90:88-139
 * with Get_MC_pixel_Vars_SW at plot times): nreal independent runs on one
 * DEM, each with its own parameters (params[r], e.g. sampled mu = const(9)
 * and xi = const(3)) and particles, advanced together: every member's graph
 * launches go out on its own stream before any wait, so small realizations
 * share the GPU.  Each member is an ordinary handle (gfsph_ensemble_member)
 * for upload, download and rasters.  The DEM slope and curvature rows (which
 * erosion does not change) are one device copy for all members; each member
 * keeps its own Z, eroded and erodible depth, which erode independently.  The
 * ensemble owns its members: gfsph_ensemble_destroy frees them, and a
 * member must not be passed to gfsph_destroy.
 */
typedef struct gfsph_ensemble gfsph_ensemble;
int gfsph_ensemble_create(const gfsph_params* params /* nreal entries */, const gfsph_dem* dem, int nreal,
                          gfsph_ensemble** out);
int gfsph_ensemble_destroy(gfsph_ensemble* e);
int gfsph_ensemble_member(gfsph_ensemble* e, int r, gfsph_handle** member);
/* Up to nsteps steps of every member (each stops at t_end); min_steps_done
 * receives the fewest steps any member completed. */
int gfsph_ensemble_step(gfsph_ensemble* e, int nsteps, double t_end, int* min_steps_done);
/* Hazard sample of every member (call at plot times). */
int gfsph_ensemble_sample(gfsph_ensemble* e);
/* Per DEM node, the fraction of members whose sampled maximum depth
 * exceeds `threshold` (nx*ny values). */
int gfsph_ensemble_exceedance(gfsph_ensemble* e, float threshold, float* prob);

/*
 * Conjugate gradients of solvegc2 (SPH_GCsolver_2019.f90:16-316) on the device:
 * Jacobi-preconditioned CG on the element-by-element system sum_e gstif_e
 * (every iteration of a solve runs in one persistent cooperative kernel),
 * prescribed dofs (iffix != 0) held at their `fixed` values and masked out
 * of the products (kbyp, :273-313), stop when r.r / r0.r0 <= tol (squared
 * norms, :112), at most 10*ntotv iterations.  Vectors and dot products are
 * FP64 on the device.  Layouts are the reference's: intmat(nnode, nelem)
 * with 1-based node numbers, gstif(nevab, nevab, nelem) with
 * nevab = nnode*ndofn, dof index (node-1)*ndofn + idofn; iffix, fixed, rcg,
 * ficg have ntotv = npoin*ndofn entries.  As in the reference, rcg returns
 * the last residual and free dofs with a zero diagonal are held (marked -999
 * during the solve).
 */
typedef struct gfsph_cg gfsph_cg;

/* Assembles the element matrices once (CSR on the device). */
int gfsph_cg_create(int npoin, int nelem, int nnode, int ndofn, const int* intmat, const float* gstif,
                    gfsph_cg** out);
/* One solve; replaces a call of solvegc2 on the system made by gfsph_cg_create. */
int gfsph_cg_solve(gfsph_cg* cg, int* iffix, const float* fixed, float* rcg, float* ficg, float tol,
                   int* iterations);
int gfsph_cg_destroy(gfsph_cg* cg);
long long gfsph_cg_launch_count(gfsph_cg* cg);
/* Device time of the last gfsph_cg_solve on cg (CUDA events around its
 * kernels: set-up, every iteration, results), without the host copies.  No
 * counterpart in the reference. */
int gfsph_cg_device_ms(gfsph_cg* cg, double* ms);
/* solvegc2 with the reference's argument list (create + solve + destroy). */
int gfsph_solvegc2(int npoin, int nelem, int nnode, int ndofn, const int* intmat, int* iffix, const float* fixed,
                   const float* gstif, float* rcg, float* ficg, float tol, int* iterations);

/* Allocation-free variant of the depth raster (GFSPH_RASTER_DEPTH_IDW), for
 * callers that cannot allocate device memory once their run has started (a
 * host that reserves all device memory up front, or one embedded in a
 * framework that owns the allocator).  It has no counterpart in the
 * reference.  Inputs and output are device pointers owned by the caller:
 * d_x (2,n), d_rho (n), d_flag (n, may be NULL = all inside), d_out (nx*ny).
 * d_x is read as interleaved (x, y) pairs and must be 8-byte aligned, the
 * other arrays 4-byte aligned (GFSPH_ERR_ARG otherwise).
 * The per-node accumulators live in a fixed device array of
 * GFSPH_NOALLOC_MAX_NODES nodes (16 MiB, held by every GPU that loads the
 * library until exit); larger grids are rejected with GFSPH_ERR_CAPACITY.
 * The first call on a device looks up that array's device address (make it
 * before any stream capture); the address is kept for the life of the
 * process, so after a cudaDeviceReset this entry point must not be used.  Every call shares the array: calls that
 * overlap on the GPU race.  The work is enqueued on `stream`
 * (cudaStream_t, NULL = default stream) and nothing is allocated or freed. */
#define GFSPH_NOALLOC_MAX_NODES (1 << 20)
int gfsph_raster_idw_noalloc(int n, const float* d_x, const float* d_rho, const int* d_flag, int nx, int ny,
                             float xmin, float ymin, float dx, float dy, float* d_out, void* stream);

/*
 * The Taylor-Galerkin shallow-water step of the GFL module
 * (Time_Integration_GFL, GFL_MAIN_2019.f90:216-284) on the device: the mesh
 * side of the SPH <-> FEM coupling (SPH_FEM_Driver_2019.f90:1630-1650).
 * gfsph_gfl_create does the set-up of Init_GFL (:65-214: element geometry,
 * lumped mass, Get_Topol's nodal slopes and curvatures, the boundary nodes
 * and their tangents, the boundary sides) on the host in single precision;
 * gfsph_gfl_step runs nsteps steps of first_step, second_step, solve
 * (niter sweeps of the consistent-mass system), addthem and check, with the
 * reference's summation orders (results equal an FP32 restatement bit for
 * bit).  Scope: nsour 1, itens 0 (const(11)), no pore pressure, every
 * boundary node a wall (no prescribed, absorbing or loaded nodes), no
 * atmospheric pressure or wind, a fixed dt per call, nfric 0-8 with Manning
 * added when const(3) != 0; GFSPH_ERR_UNSUPPORTED outside it.
 */
typedef struct gfsph_gfl gfsph_gfl;
typedef struct gfsph_gfl_params {
    float constF[15]; /* constF[k-1] = constF(k) of the .dat as Input_GFL keeps them (absolute values; hfrict0
                         above 1e-32, dens above 0.001 for nfric 2, else GFSPH_ERR_ARG): cgra, dens, Manning,
                         Coriolis, nfric, tauy, K, -, tanfi8, hfrict0, itens, tanfi0, Bfact, hrelpw, - */
    int ntype;        /* 2: flow under a still-water level swl (pressure of h - HH); 3: flow over a dry bed */
    int ngaus;        /* Gauss points per triangle: 1 or 3 */
    int niter;        /* sweeps of the consistent-mass iteration in solve (>= 1) */
    float swl;        /* still-water level (ntype 2) */
    float comp;       /* depth below which a node is dry (check) */
} gfsph_gfl_params;

/* coord (npoin, 2), intmat (nelem, 3) 1-based and counter-clockwise, z the
 * nodal bed elevation (npoin).  The state h, hu, hv starts at zero. */
int gfsph_gfl_create(const gfsph_gfl_params* p, int npoin, int nelem, const float* coord, const int* intmat,
                     const float* z, gfsph_gfl** out);
int gfsph_gfl_destroy(gfsph_gfl* g);
/* unkno (npoin, 3): h, hu, hv per node; time is the GFL clock (the tanfi decay) */
int gfsph_gfl_set_state(gfsph_gfl* g, const float* unkno, double time);
int gfsph_gfl_get_state(gfsph_gfl* g, float* unkno, double* time);
/* The soil of the SPH flow under the water (WIR interaction, ntype 2):
 * hs_w (npoin) raises the bed and gradhs_w (npoin, 2), as gfsph_gradhs
 * returns it, adds to the nodal slopes; the element slopes take the element
 * gradient of hs_w (get_gradhs_w, SPH_GFL_SW_Interactions_2019.f90:469-481).
 * NULL, NULL switches it off. */
int gfsph_gfl_set_wir(gfsph_gfl* g, const float* hs_w, const float* gradhs_w);
int gfsph_gfl_step(gfsph_gfl* g, int nsteps, float dt);
/* The set-up's nodal (npoin, 9) and element (nelem, 9) topography rows
 * (Topol and Topel: Z, Zx, Zy, 1+Zx^2, ZxZy, 1+Zy^2, curvatures); either may be NULL. */
int gfsph_gfl_topol(gfsph_gfl* g, float* topol, float* topel);
long long gfsph_gfl_launch_count(gfsph_gfl* g);
/* Device time of the last gfsph_gfl_step (CUDA events around its kernels).
 * No counterpart in the reference. */
int gfsph_gfl_device_ms(gfsph_gfl* g, double* ms);

const char* gfsph_strerror(int status);
int gfsph_version(void);

/* The architecture the library's kernels were built for, as the CUDA runtime
 * reports it for a loaded kernel (cudaFuncGetAttributes binaryVersion,
 * major * 10 + minor: 100 for sm_100a).  Needs a device.  No counterpart in
 * the reference. */
int gfsph_binary_version(int* version);

#ifdef __cplusplus
}
#endif
#endif /* GFSPH_H */
