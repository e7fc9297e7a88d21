/*
 * fall3d_ads.h -- C ABI of libfall3d_ads.so, the B200 implementation of the
 * FALL3D advection-diffusion-sedimentation (ADS) time step.
 *
 * The Fortran host (task_Fall3d / mod_F3D) reaches the GPU through these
 * entry points with ISO_C_BINDING; every array argument is a plain pointer
 * to the first element of the reference's own array, in the reference's own
 * column-major layout and bounds (serial build: my_ips = 1 .. my_ipe = nx).
 * The library copies what it needs and never keeps a host pointer.
 *
 * Every function returns 0 on success, 1 on error (message available from
 * f3d_last_error) or 2 when a settling-velocity solve did not converge
 * (the reference's MY_ERR%flag = 2, mod_Phys.F90:947-948).  Nothing aborts.
 *
 * One context = one model domain on one GPU with its own CUDA stream.
 * Calls on one context must come from one host thread at a time.
 */
#ifndef FALL3D_ADS_H
#define FALL3D_ADS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct f3d_ctx f3d_ctx;
typedef struct f3d_mlp f3d_mlp;

/* Interior mass points of the domain (my_ipe-my_ips+1, ...) and bins. */
typedef struct {
  int nx, ny, nz, nbins;
} f3d_dims;

/* Arithmetic forms. */
#define F3D_PREC_FP64 0 /* FP64 state and stencil, reference operation order  */
#define F3D_PREC_FP32 1 /* FP32 state and stencil; FP64 deposit, budget, CFL */
#define F3D_PREC_FP32C 2 /* FP32 stencil on a compensated state: FP32 pair hi + lo
                            (~48 bits), conservative FP64 final update per cell */
/* The two precision forms address a bin's cells with 32-bit offsets: their
 * grids need (nx+1)(ny+1)(nz+1) < 2^31 (creation fails otherwise). */

/* Limiters (mod_Phys.F90:58-61) and time marching (mod_Phys.F90:64-65). */
#define F3D_LIMITER_MINMOD 1
#define F3D_LIMITER_SUPERBEE 2
#define F3D_LIMITER_OSPRE 3
#define F3D_TIME_MARCHING_EULER 1
#define F3D_TIME_MARCHING_RK 2

/* ---- lifetime --------------------------------------------------------- */

/* ADS_initialize(limitertype, time_marching)  mod_ADS.F90:98.
 * Allocates every device buffer of the domain (state, meteo, scratch). */
int f3d_ads_create(const f3d_dims *dims, int limiter, int time_marching,
                   int precision, int device, f3d_ctx **out);

/* ADS_release()  mod_ADS.F90:208. */
int f3d_ads_destroy(f3d_ctx *ctx);

/* Copies the message of the last failed call on this host thread. */
int f3d_last_error(char *buf, int len);

/* ---- inputs ------------------------------------------------------------ */

/* ARAKAWA_C_GRID metric arrays (mod_KindType.F90:465-502), built by
 * grid_build_arakawa_c (mod_Grid.F90:286-676):
 *   dX1_p(ips-2:ipe+2) dX1_b(ibs-1:ibe+1) dX2_p(jps-2:jpe+2)
 *   dX2_b(jbs-1:jbe+1) dX3_p(kps-2:kpe+2) dX3_b(kbs-1:kbe+1)
 *   Hm1_p(jps:jpe) Hm2_p(jps-2:jpe+2) Hm3_p(ips:ipe,jps:jpe) */
int f3d_ads_set_grid(f3d_ctx *ctx, const double *dX1_p, const double *dX1_b,
                     const double *dX2_p, const double *dX2_b,
                     const double *dX3_p, const double *dX3_b,
                     const double *Hm1_p, const double *Hm2_p,
                     const double *Hm3_p);

/* Meteo term produced by F3D_update_meteo_term (mod_F3D.F90:564-969):
 *   u  MY_MET%my_u (ibs-1:ibe+1, jps:jpe, kps:kpe, 2)   scaled, staggered
 *   v  MY_MET%my_v (jbs-1:jbe+1, ips:ipe, kps:kpe, 2)
 *   w  MY_MET%my_w (kbs-1:kbe+1, ips:ipe, jps:jpe, 2)
 *   k1 MY_MET%my_k1(ips-2:ipe+2, jps:jpe, kps:kpe)
 *   k2 MY_MET%my_k2(jps-2:jpe+2, ips:ipe, kps:kpe)
 *   k3 MY_MET%my_k3(kps-2:kpe+2, ips:ipe, jps:jpe)
 *   vs MY_TRA%my_vs(ips:ipe, jps:jpe, kbs-1:kbe+1, nbins)  (scaled by 1/Hm3)
 *   t_its, t_ite = MY_MET%timesec(its), timesec(ite)
 * vs may be NULL to keep the field from f3d_ads_compute_vset. */
int f3d_ads_set_meteo(f3d_ctx *ctx, const double *u, const double *v,
                      const double *w, const double *k1, const double *k2,
                      const double *k3, const double *vs, double t_its,
                      double t_ite);

/* Vertical mapping of the terrain-following grid for f3d_ads_set_meteo_corners
 * (MY_GRID%map_v, mod_Grid.F90:761-870, 879-1017): 0 Cartesian (default),
 * 1 sigma without decay, 2 sigma with linear decay of the terrain slopes.
 * X3_c(kbs:kbe) heights of the w levels, X3_p(kps:kpe) of the mass levels,
 * dhdx_p, dhdy_p(ips:ipe,jps:jpe) terrain slopes; ignored for map_v = 0. */
int f3d_ads_set_terrain(f3d_ctx *ctx, int map_v, double X3max,
                        const double *X3_c, const double *X3_p,
                        const double *dhdx_p, const double *dhdy_p);

/* The compute part of F3D_update_meteo_term (mod_F3D.F90:673-944) on the
 * device, in place of f3d_ads_set_meteo: from the corner winds of the two
 * time levels of the interval, MY_MET%my_uc/my_vc/my_wc(ibs:ibe,jbs:jbe,
 * kbs:kbe) at its and ite (two consecutive blocks each), and the unscaled
 * diffusion at mass points k1(ips-2:ipe+2,jps:jpe,kps:kpe),
 * k2(ips:ipe,jps-2:jpe+2,kps:kpe), k3(ips:ipe,jps:jpe,kps-2:kpe+2) -- or, with
 * all three NULL, constants kh, kv (phys_get_kdiffu CONSTANT,
 * mod_Phys.F90:477-480) -- builds the ground-zeroed, staggered
 * (mod_Grid.F90:685-752), scaled (mod_Grid.F90:761-870, 879-1017) fields of
 * the step directly in device memory.  The settling velocity stays with
 * f3d_ads_compute_vset(_mlp). */
int f3d_ads_set_meteo_corners(f3d_ctx *ctx, const double *uc, const double *vc,
                              const double *wc, const double *k1,
                              const double *k2, const double *k3, double kh,
                              double kv, double t_its, double t_ite);

/* Wet deposition, phys_wet_deposition (mod_Phys.F90:1358-1427), applied in
 * every step after the sweeps (mod_F3D.F90:1497-1513) to the bins of
 * category 1 (particle) or 3 (radionuclide) with diameter <= 1e-4 m:
 * scavenging lambda = min(1, dt a P^b) (MY_MOD%wet_deposition_a/_b),
 * below the boundary-layer top only.  pre, pblh(ips:ipe,jps:jpe) precipitation
 * rate and boundary-layer height of the meteo interval; h_c(ibs:ibe,jbs:jbe)
 * topography and z_c(ibs:ibe,jbs:jbe,kbs:kbe) heights of the cell corners.
 * Call again at each meteo update; bin_cat = NULL switches it off.  The wet
 * deposit starts at zero and is read with f3d_ads_get_awet. */
int f3d_ads_set_wet_deposition(f3d_ctx *ctx, double a, double b,
                               const double *pre, const double *pblh,
                               const double *h_c, const double *z_c,
                               const int *bin_cat, const double *bin_diam);
/* Radioactive decay, phys_radionuclides (mod_Phys.F90:1216-1342), applied in
 * every step after wet deposition to the bins of category 3 in the air and in
 * the dry and wet deposits.  bin_spe: species 5 Cs134, 6 Cs137, 7 I131,
 * 8 Sr90, 9 Y90 (mod_KindType.F90:62-66); NULL switches it off. */
int f3d_ads_set_radionuclides(f3d_ctx *ctx, const int *bin_cat,
                              const int *bin_spe);
/* MY_TRA%my_awet(ips-2:ipe+2, jps-2:jpe+2, nbins), halos zero. */
int f3d_ads_get_awet(f3d_ctx *ctx, double *my_awet);

/* Diffusion model of phys_get_kdiffu (mod_Phys.F90:406-664). */
typedef struct {
  int modkh;       /* MY_MOD%modkh: 1 CONSTANT, 2 CMAQ, 4 RAMS */
  int modkv;       /* MY_MOD%modkv: 1 CONSTANT, 3 SIMILARITY */
  int map_h;       /* MY_GRID%map_h: 0 Cartesian, 1 spherical */
  double kh0, kv0; /* MY_MOD%kh0, kv0 (CONSTANT) */
  double rams_cs;  /* MY_MOD%RAMS_CS */
  double dlon, dlat; /* MY_GRID%dlon, dlat */
  double s_time;   /* interpolation factor of the corner fields at the update
                      time (mod_F3D.F90:760-767) */
} f3d_kdiffu;

/* f3d_ads_set_meteo_corners with the diffusion computed on the device by
 * phys_get_kdiffu from the corner winds and virtual temperature interpolated
 * at kd->s_time (CMAQ/RAMS horizontal, similarity vertical, or constants),
 * then scaled like the given K's.  tvc: MY_MET%my_tvc(ibs:ibe, jbs:jbe,
 * kbs:kbe, its:ite) (2 snapshots); pblh, mon, ust: MY_MET%my_pblh, my_mon
 * (already limited to |L| >= 10, mod_F3D.F90:740), my_ust at mass points;
 * h_c: MY_GRID%h_c.  These five may be NULL unless modkv is SIMILARITY, which
 * also needs the corner heights (f3d_ads_set_corner_heights).  Errors as
 * phys_get_kdiffu's. */
int f3d_ads_set_meteo_corners_kdiffu(f3d_ctx *ctx, const double *uc,
                                     const double *vc, const double *wc,
                                     const double *tvc, const double *pblh,
                                     const double *mon, const double *ust,
                                     const double *h_c, const f3d_kdiffu *kd,
                                     double t_its, double t_ite);

/* Gravity current, F3D_add_radial_wind (mod_F3D.F90:978-1226).  params =
 * MY_MOD%MY_GC {lon, lat, start_time, end_time, c_flow_rate, k_entrain,
 * brunt_vaisala, lambda, mass_flow_rate, h_tot, input_min_radius}; the
 * coordinates MY_GRID%lon_c(ibs:ibe), lat_c(jbs:jbe), lon_p(ips:ipe),
 * lat_p(jps:jpe), Hm1_c(jbs:jbe) (all five, or all NULL to keep the ones
 * given before, e.g. when only mass_flow_rate changes).  Needs the corner
 * heights (f3d_ads_set_corner_heights).  From then on every f3d_ads_step at a
 * time inside [start_time, end_time] with mass_flow_rate > 0 adds the radial
 * wind to the interpolated u and v before its sweeps (:1443-1445). */
int f3d_ads_set_gravity_current(f3d_ctx *ctx, const double params[11],
                                const double *lon_c, const double *lat_c,
                                const double *lon_p, const double *lat_p,
                                const double *Hm1_c);
/* The update_step time step of a gravity-current step (mod_F3D.F90:1449-1452):
 * *active = 1 when the current acts at `time`, and then my_dt, gl_dt are
 * grid_get_time_step on the winds that step uses (interpolated at stime, with
 * the radial wind).  *active = 0 leaves them untouched.  state (may be NULL)
 * gets {vol_flow_rate, min_radius, radius_grav, c_grav_factor, th_grav, hmin,
 * hmax}, the values the reference stores in MY_MOD%MY_GC. */
int f3d_ads_gravity_current_time_step(f3d_ctx *ctx, double time, double stime,
                                      int criterion, double cfl,
                                      double run_end, int *active,
                                      double *my_dt, double *gl_dt,
                                      double state[7]);

/* Keep (on != 0) the state's boundary halo layers on the device: the
 * free-flow ghost value each sweep writes into the first halo cell at both
 * ends of its pencils (freeflow, mod_ADS.F90:1227-1326, applied to MY_TRA%my_c
 * at :270, :460, :676), decayed with the state by phys_radionuclides.  The
 * output reductions read them at the domain edges, f3d_ads_upload_state takes
 * them from the halo of my_c and f3d_ads_download_state returns them there.
 * Off (the default), the halo reads as zero in the output reductions. */
int f3d_ads_keep_boundary_halo(f3d_ctx *ctx, int on);
/* Heights of the cell corners MY_GRID%z_c(ibs:ibe,jbs:jbe,kbs:kbe), for the
 * output reductions. */
int f3d_ads_set_corner_heights(f3d_ctx *ctx, const double *z_c);
/* The per-species reductions of nc_IO_out_res (mod_nc_IO.F90:3206-4335) on
 * the device, at the cell corners (ibs:ibe, jbs:jbe), Fortran order:
 *   CON_SUR   surface concentration, g/m3 (:3624-3633)
 *   COL_MASS  column load, g/m2, or DU when col_du != 0 (SO2, :3682-3703)
 *   CLOUD_TOP z_c of the highest corner above 50 ug/m3, else 0 (:3828-3858)
 *   GRN_LOAD  dry + wet deposit, kg/m2 (:3428-3446, :3909-3920)
 * from 1e3 c/(Hm1 Hm2 Hm3) clipped at 0 and averaged to corners as grid_p2c
 * and grid_p2c_2D do (mod_Grid.F90:1150-1220).  bin_in[nbins] selects the
 * bins summed: those of the species, or of the species with diameter <= PM
 * for the PMxx column loads (:3753-3777).  Any output may be NULL.  Mass
 * points outside the domain are the state's halo: the kept boundary halo
 * layers (f3d_ads_keep_boundary_halo), else zero. */
int f3d_ads_output_species(f3d_ctx *ctx, const int *bin_in, int col_du,
                           double *con_sur, double *col_mass,
                           double *cloud_top, double *grn_load);

/* Source term MY_TRA%my_s(ips:ipe,jps:jpe,kps:kpe,nbins) after
 * F3D_set_source_term (mod_F3D.F90:349-555), given sparsely: n cells with
 * 1-based Fortran indices ijk[3*q+0..2] and values s[nbins*q + bin] (the
 * already Hm1*Hm2*Hm3-scaled my_s).  n = 0 clears the source. */
int f3d_ads_set_source(f3d_ctx *ctx, int n, const int *ijk, const double *s);

/* Same, from the dense my_s array; zero cells are skipped. */
int f3d_ads_set_source_dense(f3d_ctx *ctx, const double *my_s);

/* Initial condition / restart (task_Fall3d.F90:233-249):
 *   my_c   (ips-2:ipe+2, jps-2:jpe+2, kps-2:kpe+2, nbins)
 *   my_acum(ips-2:ipe+2, jps-2:jpe+2, nbins)            (either may be NULL) */
int f3d_ads_upload_state(f3d_ctx *ctx, const double *my_c,
                         const double *my_acum);

/* Copies the device state back into the reference arrays (interior cells;
 * ghost cells receive the free-flow values of the final state). */
int f3d_ads_download_state(f3d_ctx *ctx, double *my_c, double *my_acum);

/* ---- the time step ----------------------------------------------------- */

/* Body of F3D_time_step (mod_F3D.F90:1397-1491): u/v time interpolation,
 * source injection, x/y sweeps (order alternating with iiter parity), z sweep
 * with settling, ground deposit and boundary fluxes.  fluxes[6] =
 * {W,E,S,N,U,D} (MY_TRA%my_W_flux ...) are INOUT accumulators, as in
 * ADS_solve_along_x/y/z.  Blocks until the step completed. */
int f3d_ads_step(f3d_ctx *ctx, double dt, double time, int iiter,
                 double fluxes[6]);

/* Same step, enqueued without waiting; flux increments accumulate on the
 * device and are read with f3d_ads_get_fluxes. */
int f3d_ads_step_async(f3d_ctx *ctx, double dt, double time, int iiter);

/* Adds the device-accumulated flux increments to fluxes[6] and zeroes them. */
int f3d_ads_get_fluxes(f3d_ctx *ctx, double fluxes[6]);

/* Waits for every call enqueued on the context. */
int f3d_ads_synchronize(f3d_ctx *ctx);

/* The CUDA stream (cudaStream_t) the context enqueues on, for event timing
 * and for ordering the caller's own work after a step. */
int f3d_ads_get_stream(f3d_ctx *ctx, void **stream);

/* Per-phase device timing with CUDA events on the context stream.  When on,
 * every step records events around its phases and waits for them; the
 * accumulated milliseconds are ms[0] prep+source, ms[1] x sweep, ms[2] y
 * sweep, ms[3] z sweep, ms[4] flux reduction, ms[5] whole step. */
int f3d_ads_set_profiling(f3d_ctx *ctx, int on);
int f3d_ads_get_profile(f3d_ctx *ctx, double ms[6], int *nsteps);

/* Number of CUDA kernels this context has launched since creation. */
int f3d_ads_launch_count(f3d_ctx *ctx, long long *count);

/* The pieces of the step, for unit parity with the ADS_* routines. */
/* ADS_update_horizontal_vcomps(u1,u2,v1,v2,stime)  mod_ADS.F90:187 */
int f3d_ads_update_vcomps(f3d_ctx *ctx, double stime);
/* ADS_solve_along_x(W_flux,E_flux,dt,...)  mod_ADS.F90:233 */
int f3d_ads_solve_along_x(f3d_ctx *ctx, double dt, double *W_flux,
                          double *E_flux);
/* ADS_solve_along_y(S_flux,N_flux,dt,...)  mod_ADS.F90:422 */
int f3d_ads_solve_along_y(f3d_ctx *ctx, double dt, double *S_flux,
                          double *N_flux);
/* ADS_solve_along_z(D_flux,U_flux,dt,...,stime,my_vs,...)  mod_ADS.F90:612 */
int f3d_ads_solve_along_z(f3d_ctx *ctx, double dt, double stime,
                          double *D_flux, double *U_flux);
/* Source injection loop of F3D_time_step, mod_F3D.F90:1456-1473 */
int f3d_ads_add_source(f3d_ctx *ctx, double dt);

/* ---- diagnostics ------------------------------------------------------- */

/* grid_get_time_step (mod_Grid.F90:1026-1141) with winds interpolated at
 * stime (mod_F3D.F90:957-961).  criterion 1 (ONE_DIMENSIONAL) or
 * 2 (ALL_DIMENSIONS).  FP64 max-reduction on the device. */
int f3d_ads_get_time_step(f3d_ctx *ctx, double stime, int criterion,
                          double cfl, double run_end, double *my_dt,
                          double *gl_dt);

/* grid_get_mass_volume (mod_Grid.F90:1340-1389): sum c dX dY dZ over the
 * interior.  per_bin (nbins, may be NULL) receives the per-bin masses. */
int f3d_ads_mass_volume(f3d_ctx *ctx, double *mass, double *per_bin);

/* ADS_solve_1D (mod_ADS.F90:820-1053): RK4 on one pencil of n >= 2 cells
 * with boundary codes bcode[2] (-1 periodic when the face velocity enters,
 * 0 ghosts as given, 1 Dirichlet bvalue, 2 free flow: Dirichlet bvalue on
 * inflow, zero gradient on outflow).  Host arrays, reference layouts:
 * c(ips-2:ipe+2) INOUT (n+4), dxp and k (n+4), dxb and u (ibs-1:ibe+1,
 * n+3); flux[2] receives the 4th-stage boundary fluxes (F + P).  Off the
 * reference's time loop; it is the 1-D entry of the known-answer tests. */
int f3d_ads_solve_1d(int n, int limiter, double *c, const double *dxp,
                     const double *dxb, const double *u, const double *k,
                     double dt, const double bvalue[2], double flux[2],
                     const int bcode[2], int device);

/* Failure detection (mod_KindType.F90:85-95, MY_ERR; the reference checks
 * no values, so these have no direct counterpart).
 * f3d_ads_check_finite: an on-device scan of the resident inputs and state
 * for NaN or infinite values; *mask (0 = all finite) has bit 1 state,
 * 2 ground deposit, 4 u, 8 v, 16 w (both meteo snapshots), 32 k1, 64 k2,
 * 128 k3, 256 settling velocity. */
int f3d_ads_check_finite(f3d_ctx *ctx, int *mask);
/* Process-wide poll limit of every bounded device wait in the kernels
 * launched from now on (the persistent step kernel's grid barriers and the
 * surrogate's tensor-core completion waits), for tests of the failure path:
 * a wait that runs out records an error status (f3d_ens_status, or an
 * error return) instead of waiting on.  polls < 0 restores the default
 * (2^25 polls, about a second).  A kernel whose first wait gave up still
 * waits, with the default limit, for its own tensor-core work in flight
 * before it frees its tensor memory.  CUDA graphs keep the limit of the
 * launches they captured. */
int f3d_set_wait_limit(long long polls);
/* Process-wide iteration limit of the settling-velocity fixed point
 * (phys_get_vset_point's maxit = 1000, mod_Phys.F90:794) for the next
 * f3d_vset_points / f3d_ads_compute_vset / f3d_ens_compute_class_vset
 * calls; a point that has not converged within it returns flag 2
 * (mod_Phys.F90:944-948).  maxit = -1 restores 1000. */
int f3d_set_vset_maxit(int maxit);
/* Process-wide choice of how the steps run wet deposition and radioactive
 * decay (phys_wet_deposition and phys_radionuclides after the sweeps,
 * mod_F3D.F90:1493-1520).  on = 0 (the default): as separate passes over the
 * state after the z sweep.  on = 1: as the z sweep's epilogue, each cell
 * scavenged and decayed as it leaves the sweep and the column's deposits
 * updated by the thread that owns them, with a separate pass left only for
 * Y90 bins (set from their Sr90 parent) and the kept boundary halo layers.
 * The exact and plain FP32 forms give the same bits either way; the
 * compensated form rounds its pair once instead of after each process.  The
 * epilogue saves the passes' memory traffic but adds FP64 arithmetic to the
 * issue-bound sweep, and measured slower on a B200.  Takes effect at the
 * next step (an ensemble re-captures its step graphs). */
int f3d_set_zsweep_epilogue(int on);

/* Mass in the volume for callers that cannot allocate device memory.  No
 * counterpart in the reference: a variant of f3d_ads_mass_volume for code
 * whose device memory is owned by its own runtime (an OpenACC or CUDA
 * Fortran port holding my_c on the device, a pool reserved at start-up, a
 * framework that forbids allocation in its time loop).  It calls no
 * allocating routine: the per-block partial sums use a fixed device array
 * of 64 bins x 296 blocks (148 KiB).  The CUDA runtime commits that array
 * when it loads this library's device code on a device, which under the
 * default lazy module loading is the FIRST call on that device; the device
 * then keeps it until its context ends.  So make the first call on each
 * device before any region where allocation is forbidden and before any
 * stream capture.  All pointers are DEVICE pointers:
 *   c      my_c (ips-2:ipe+2, jps-2:jpe+2, kps-2:kpe+2, nbins), FP64
 *   dX1_p, dX2_p, dX3_p   the grid arrays with their halos (as in set_grid)
 *   per_bin (nbins) and/or total (1): outputs, either may be NULL
 * nbins above 64 is rejected.  Work is enqueued on `stream` (a
 * cudaStream_t, NULL = default stream) and not waited for.  The array's
 * device address is looked up on every call, for the current device.
 * Calls share the array, so calls that overlap on the GPU race; order them
 * on one stream. */
int f3d_mass_volume_noalloc(int nx, int ny, int nz, int nbins, const double *c,
                            const double *dX1_p, const double *dX2_p,
                            const double *dX3_p, double *per_bin,
                            double *total, void *stream);

/* grid_get_mass_sink (mod_Grid.F90:1400-1450): the mass removed by wet
 * deposition, sum over columns of (sum over bins of awet) dX dY, added in the
 * reference's serial order (the column terms are formed on the device). 0
 * without wet deposition. */
int f3d_ads_mass_sink(f3d_ctx *ctx, double *mass);
/* grid_get_mass_boundaries (mod_Grid.F90:1461-1511) from fluxes {W,E,S,N,U,D}. */
int f3d_ads_mass_boundaries(const double fluxes[6], double *ground,
                            double *lateral);

/* ---- settling velocity ---------------------------------------------------- */

/* phys_get_vset_point (mod_Phys.F90:757-954) for n independent points on the
 * GPU (host arrays).  model 1..7 (mod_Phys.F90:44-50).  flags[q] receives
 * 0 / 2 (no convergence); iters (may be NULL) the iteration counts.
 * Returns 2 when any point failed to converge. */
int f3d_vset_points(int model, int n, const double *diam, const double *rhop,
                    const double *psi, const double *rhoa, const double *visc,
                    double *vset, int *flags, int *iters);

/* phys_get_vset (mod_Phys.F90:673-740) + the vs/Hm3 scaling of
 * grid_get_scaled_variables (mod_Grid.F90:996-1005) on the device, writing
 * the context's settling-velocity field.  rhoc, tc: corner air density and
 * temperature (ibs:ibe, jbs:jbe, kbs:kbe).  bin_cat: 1 particle,
 * 2 aerosol, 3 radionuclide; is_aggregate (may be NULL) with vset_fac.
 * vs_out (may be NULL) receives my_vs in the reference layout. */
int f3d_ads_compute_vset(f3d_ctx *ctx, int model, const double *rhoc,
                         const double *tc, const double *diam,
                         const double *rhop, const double *psi,
                         const int *bin_cat, const int *is_aggregate,
                         double vset_fac, double *vs_out);

/* Same as f3d_ads_compute_vset, with the learned surrogate (see f3d_mlp_*)
 * in place of the drag-law iteration; w-faces outside the surrogate's
 * envelope (and every face of a bin outside it) take the iteration.
 * refine = 1 adds one Steffensen correction (two drag-law evaluations) to the
 * surrogate value.  nfallback (may be NULL) = faces that took the iteration.
 * No reference counterpart: replaces the phys_get_vset_point call inside
 * phys_get_vset (mod_Phys.F90:717-718). */
int f3d_ads_compute_vset_mlp(f3d_ctx *ctx, f3d_mlp *mlp, const double *rhoc,
                             const double *tc, const double *diam,
                             const double *rhop, const double *psi,
                             const int *bin_cat, const int *is_aggregate,
                             double vset_fac, int refine, long long *nfallback,
                             double *vs_out);

/* ---- batched ensemble -------------------------------------------------------
 * Ensemble members of FALL3D run as independent jobs in separate MPI
 * communicators (mod_Parallel.F90:188-217, task_SetEns.F90).  Here every
 * member of an ensemble lives on one GPU and all members advance together,
 * one batched step per call.  Members are grouped into grid classes: the
 * members of a class share the grid, the meteo term and the settling
 * velocity (the ensemble perturbs the winds by one factor per member,
 * task_Fall3d.F90:194-198, applied on the device), and own their
 * concentration, deposit, source, time step and clock. */
typedef struct f3d_ens f3d_ens;

typedef struct {
  int grid_class;     /* 0 .. nclasses-1 */
  double wind_factor; /* multiplier of u and v: 1 + r range/100 (RELATIVE perturbation) */
} f3d_ens_member;

#define F3D_ENS_MODE_KERNELS 0    /* one kernel per phase, replayed from CUDA graphs */
#define F3D_ENS_MODE_PERSISTENT 1 /* one persistent cooperative kernel per step */

int f3d_ens_create(int nclasses, const f3d_dims *class_dims, int nmembers,
                   const f3d_ens_member *members, int limiter, int time_marching,
                   int precision, int device, f3d_ens **out);
int f3d_ens_destroy(f3d_ens *ens);
/* Same arrays and layouts as f3d_ads_set_grid / f3d_ads_set_meteo, per class. */
int f3d_ens_set_class_grid(f3d_ens *ens, int cls, const double *dX1_p,
                           const double *dX1_b, const double *dX2_p,
                           const double *dX2_b, const double *dX3_p,
                           const double *dX3_b, const double *Hm1_p,
                           const double *Hm2_p, const double *Hm3_p);
int f3d_ens_set_class_meteo(f3d_ens *ens, int cls, const double *u,
                            const double *v, const double *w, const double *k1,
                            const double *k2, const double *k3, const double *vs,
                            double t_its, double t_ite);
/* f3d_ads_set_terrain and f3d_ads_set_meteo_corners for a grid class. */
int f3d_ens_set_class_terrain(f3d_ens *ens, int cls, int map_v, double X3max,
                              const double *X3_c, const double *X3_p,
                              const double *dhdx_p, const double *dhdy_p);
int f3d_ens_set_class_meteo_corners(f3d_ens *ens, int cls, const double *uc,
                                    const double *vc, const double *wc,
                                    const double *k1, const double *k2,
                                    const double *k3, double kh, double kv,
                                    double t_its, double t_ite);
/* phys_get_vset + vs/Hm3 of a class on the device (see f3d_ads_compute_vset). */
int f3d_ens_compute_class_vset(f3d_ens *ens, int cls, int model,
                               const double *rhoc, const double *tc,
                               const double *diam, const double *rhop,
                               const double *psi, const int *bin_cat,
                               const int *is_aggregate, double vset_fac);
/* The same with the learned surrogate (see f3d_ads_compute_vset_mlp). */
int f3d_ens_compute_class_vset_mlp(f3d_ens *ens, int cls, f3d_mlp *mlp,
                                   const double *rhoc, const double *tc,
                                   const double *diam, const double *rhop,
                                   const double *psi, const int *bin_cat,
                                   const int *is_aggregate, double vset_fac,
                                   int refine, long long *nfallback);
/* Device time (ms) of the last class settling-velocity kernel. */
int f3d_ens_vset_ms(f3d_ens *ens, float *ms);
int f3d_ens_set_member_source(f3d_ens *ens, int member, int n, const int *ijk,
                              const double *s);
int f3d_ens_upload_member_state(f3d_ens *ens, int member, const double *my_c,
                                const double *my_acum);
int f3d_ens_download_member_state(f3d_ens *ens, int member, double *my_c,
                                  double *my_acum);
/* grid_get_time_step for every member at stime (each with its own winds);
 * the members' dt are set on the device and copied to dt[nmembers] if given. */
int f3d_ens_compute_time_steps(f3d_ens *ens, double stime, int criterion,
                               double cfl, double run_end, double *dt);
/* Model clock of every member (time[nmembers]) and the common iteration. */
int f3d_ens_set_clock(f3d_ens *ens, const double *time, int iiter);
int f3d_ens_get_clock(f3d_ens *ens, double *time, int *iiter);
/* Execution shape: mode, bins per sweep block (1, 2, 4) and, for the
 * persistent mode, resident blocks per SM (0 = as many as fit). */
int f3d_ens_set_tuning(f3d_ens *ens, int mode, int bins_per_block,
                       int ctas_per_sm);
/* Advance every member nsteps times with its own dt on the device clock
 * (time += dt, iiter += 1 after each step); enqueued, not waited for. */
int f3d_ens_run(f3d_ens *ens, int nsteps);
/* One step with host-given dt[m], time[m]; fluxes[6*m..] INOUT {W,E,S,N,U,D}
 * (may be NULL: increments stay on the device).  Blocks when fluxes given. */
int f3d_ens_step(f3d_ens *ens, const double *dt, const double *time, int iiter,
                 double *fluxes);
/* Adds the device-accumulated flux totals to fluxes[6*nmembers], zeroes them. */
int f3d_ens_get_fluxes(f3d_ens *ens, double *fluxes);
int f3d_ens_mass_volume(f3d_ens *ens, int member, double *mass);
/* Zero every member's concentration, deposit and flux totals on the device
 * (a fresh start without host transfers; the clocks are left to
 * f3d_ens_set_clock). */
int f3d_ens_reset_state(f3d_ens *ens);
/* grid_get_mass_sink (mod_Grid.F90:1400-1450) of one member. */
int f3d_ens_mass_sink(f3d_ens *ens, int member, double *mass);
/* Wet deposition and radioactive decay for every member after its sweeps,
 * as f3d_ads_set_wet_deposition / f3d_ads_set_radionuclides do for one
 * domain (mod_F3D.F90:1493-1520).  The precipitation, boundary layer,
 * terrain and heights are per grid class; a, bin_cat and bin_diam are the
 * ensemble's (bin_cat NULL switches wet deposition off).  Each member's
 * lambda uses its own dt on the device; the decay factors exp(-kn dt) are
 * evaluated on the host for each member's dt whenever the time steps change
 * (f3d_ens_compute_time_steps, f3d_ens_step). */
int f3d_ens_set_class_wet_deposition(f3d_ens *ens, int grid_class, double a,
                                     double b, const double *pre,
                                     const double *pblh, const double *h_c,
                                     const double *z_c, const int *bin_cat,
                                     const double *bin_diam);
int f3d_ens_set_radionuclides(f3d_ens *ens, const int *bin_cat,
                              const int *bin_spe);
/* A member's wet deposit MY_TRA%my_awet(ips-2:ipe+2, jps-2:jpe+2, nbins). */
int f3d_ens_get_member_awet(f3d_ens *ens, int member, double *my_awet);
/* Corner heights of a grid class, and the per-species output reductions of
 * nc_IO_out_res for one member (f3d_ads_output_species; the halo reads as
 * zero). */
int f3d_ens_set_class_corner_heights(f3d_ens *ens, int grid_class,
                                     const double *z_c);
int f3d_ens_output_member_species(f3d_ens *ens, int member, const int *bin_in,
                                  int col_du, double *con_sur,
                                  double *col_mass, double *cloud_top,
                                  double *grn_load);
/* Per-phase device timing: while on, f3d_ens_run enqueues steps without the
 * graph and records events between phases; ms[5] accumulates
 * {prep+source, x sweep, y sweep, z sweep, flux+clock} (persistent mode: the
 * fused step kernel in ms[1]) over nsteps steps.  Turning it on resets. */
int f3d_ens_set_profiling(f3d_ens *ens, int on);
int f3d_ens_get_profile(f3d_ens *ens, double *ms, int *nsteps);
int f3d_ens_synchronize(f3d_ens *ens);
int f3d_ens_get_stream(f3d_ens *ens, void **stream);
int f3d_ens_launch_count(f3d_ens *ens, long long *count);
/* Device error status: 1 after a bounded grid-barrier wait gave up (the
 * persistent step kernel then winds down instead of waiting; the state of
 * that step is not valid).  Waits for the ensemble's stream first.  No
 * counterpart in the reference, which has no device waits; it stands for
 * MY_ERR%flag = 1 (mod_KindType.F90:85-95). */
int f3d_ens_status(f3d_ens *ens, int *device_error);
/* Boundary halo layers of every member, as f3d_ads_keep_boundary_halo: the
 * free-flow ghost values of the sweeps are kept (and decayed), the output
 * reductions read them at the edge corners, and member up/downloads carry
 * them in the halo cells of my_c.  on = 0 stops keeping them. */
int f3d_ens_keep_boundary_halo(f3d_ens *ens, int on);
/* Gravity current of member mi (F3D_add_radial_wind, mod_F3D.F90:978-1226),
 * as f3d_ads_set_gravity_current for a single domain: params[11] = {lon,
 * lat, start_time, end_time, c_flow_rate, k_entrain, brunt_vaisala,
 * lambda_grav, mass_flow_rate, h_tot, input_min_radius}; the five
 * coordinate arrays of the member's class grid are needed on the first call
 * of a class (may be NULL afterwards); the class's corner heights must be set
 * (f3d_ens_set_class_corner_heights).  params NULL switches the member's
 * current off.  While any member has a current the ensemble advances with
 * host-driven steps only (f3d_ens_step; f3d_ens_run refuses): every step
 * inside the member's window adds the radial wind to its interpolated winds
 * (mod_F3D.F90:1443-1445). */
int f3d_ens_set_member_gravity_current(f3d_ens *ens, int mi, const double params[11],
                                       const double *lon_c, const double *lat_c,
                                       const double *lon_p, const double *lat_p,
                                       const double *Hm1_c);
/* The update_step time step of every member whose current acts at times[m]
 * (mod_F3D.F90:1446-1452): grid_get_time_step on its winds with the radial
 * wind at interpolation factor stimes[m]; active[m] = 1 and dts[m] set for
 * those members, active[m] = 0 and dts[m] untouched for the others. */
int f3d_ens_gravity_current_time_steps(f3d_ens *ens, const double *times, const double *stimes,
                                       int criterion, double cfl, double run_end, int *active,
                                       double *dts);
/* Autotuner of the batched step (no counterpart in the reference, whose
 * members run as separate jobs).  Times each candidate execution shape on
 * the device -- per-phase kernels replayed from CUDA graphs with 4, 2 or 1
 * bins per block, the persistent step kernel with 4 or 2 -- for one warm-up
 * and `steps` timed steps (CUDA events on the ensemble's stream), keeps the
 * fastest and sets it.  Member state and clocks advance while tuning: reset
 * them afterwards if needed.  With cache_file and key (a single token, e.g.
 * class shapes, bins, precision and GPU name) the result is read from and
 * written to that text file, so a later run with the same key sets the
 * cached shape without timing.  tuning[3] = {mode, bins per block, blocks
 * per SM (0 = as many as fit)}; cand_ms (may be NULL) receives the
 * F3D_ENS_TUNE_CANDIDATES candidates' ms per step (-1 where one failed). */
#define F3D_ENS_TUNE_CANDIDATES 5
int f3d_ens_autotune(f3d_ens *ens, int steps, const char *cache_file, const char *key,
                     int tuning[3], double *ms_per_step, double *cand_ms);
/* Clears the device error status, so that the host may continue after it
 * has handled the failure (for example, restored the state). */
int f3d_ens_clear_status(f3d_ens *ens);
/* Finite scan of member mi's state and its class's device inputs; bits of
 * *mask as in f3d_ads_check_finite. */
int f3d_ens_check_finite(f3d_ens *ens, int mi, int *mask);

/* ---- learned settling velocity ----------------------------------------------
 * A 5 -> 64 -> 64 -> 1 tanh network standing in for the fixed-point drag-law
 * solve of phys_get_vset_point (mod_Phys.F90:757-954); no reference
 * counterpart.  Inputs (diameter, particle density, sphericity, air density,
 * air viscosity) enter as normalised log features; the output is the log
 * ratio of the particle Reynolds number to its Stokes value.  Training data
 * are generated and labelled on the device by the model's own iteration;
 * training (forward, backward, Adam) runs in the library's own kernels;
 * inference runs layer 2 on the tensor cores (tcgen05, split BF16 operands,
 * FP32 accumulate).  Parameter vector (F3D_MLP_NPARAMS floats): W1[64][5],
 * b1[64], W2[64][64], b2[64], W3[64], b3 (row-major, out x in). */
#define F3D_MLP_NPARAMS 4609

/* envelope[10] = {d_lo, d_hi, rhop_lo, rhop_hi, psi_lo, psi_hi, rhoa_lo,
 * rhoa_hi, visc_lo, visc_hi} (SI units).  Training samples are drawn from the
 * envelope widened by margin (diameter by exp(+-3 margin), the others by
 * (1 -+ margin), sphericity capped at 1).  model: 1,2,3,5,6,7 (the iterative
 * models of phys_get_vset_point).  seed: parameter initialisation. */
int f3d_mlp_create(int model, const double *envelope, double margin,
                   unsigned long long seed, int device, f3d_mlp **out);
int f3d_mlp_destroy(f3d_mlp *mlp);
/* nsamples uniform draws over the training box, labelled by the iteration;
 * nfail (may be NULL) = draws whose iteration did not converge (unused). */
int f3d_mlp_generate(f3d_mlp *mlp, long long nsamples, unsigned long long seed,
                     long long *nfail);
/* raw[5 n] = (d, rhop, psi, rhoa, visc) per sample; rec[8 n] = (5 features,
 * target, 0, 0) per sample.  Either may be NULL. */
int f3d_mlp_get_samples(f3d_mlp *mlp, long long first, long long n,
                        double *raw, float *rec);
/* Adam over steps minibatches of batch samples (a multiple of 128), cosine
 * learning rate lr_max -> lr_min.  loss_hist[steps] and train_ms may be NULL. */
int f3d_mlp_train(f3d_mlp *mlp, int steps, int batch, double lr_max,
                  double lr_min, unsigned long long seed, float *loss_hist,
                  float *train_ms);
/* Gradient (F3D_MLP_NPARAMS) and value of the mean squared error over n
 * given samples (features[5 n], targets[n]) at the current parameters. */
int f3d_mlp_gradient(f3d_mlp *mlp, long long n, const float *features,
                     const float *targets, float *grad, float *loss);
int f3d_mlp_get_params(f3d_mlp *mlp, float *params);
int f3d_mlp_set_params(f3d_mlp *mlp, const float *params);
/* out[19]: lar_c, lar_sinv, sg_scale, psi_lo, psi_sinv, lnd_lo, lnd_sinv,
 * lnmu_lo, lnmu_sinv, then the training box (lo, hi) per coordinate. */
int f3d_mlp_get_norm(f3d_mlp *mlp, double *out);
/* Settling velocity of n points; used[n] (may be NULL) = 1 where the
 * surrogate answered, 0 where the point was outside the envelope. */
int f3d_mlp_predict(f3d_mlp *mlp, long long n, const double *diam,
                    const double *rhop, const double *psi, const double *rhoa,
                    const double *visc, int refine, double *vset, int *used);
/* Device time (ms) of the last inference kernel. */
int f3d_mlp_last_ms(f3d_mlp *mlp, float *ms);

/* ---- pinned host memory for fast transfers --------------------------------- */
int f3d_host_alloc(size_t bytes, void **ptr);
int f3d_host_free(void *ptr);

#ifdef __cplusplus
}
#endif
#endif /* FALL3D_ADS_H */
