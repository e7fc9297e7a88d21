/*
 * f3d_oracle.h -- CPU FP64 oracle for the FALL3D ADS time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Fortran routines on the advection-diffusion-sedimentation path, used as the
 * checker for the CUDA library and as the timed CPU baseline.  The product
 * library (libfall3d_ads.so) never links or calls it.
 *
 * Parity status: the reference (Fortran 90, autotools, netCDF) cannot be
 * compiled in this environment and ships no golden outputs, so this oracle is
 * "parity unpinned" against the reference binary.  It is pinned instead by
 * analytic known-answer tests (pure advection, pure diffusion, Stokes-limit
 * settling, exact mass conservation) in tests/test_oracle_kat.py.
 *
 * Array layouts follow the reference exactly (column-major, first index
 * fastest, serial build so my_ips = 1 ... my_ipe = nx):
 *   c     my_c   (ips-2:ipe+2, jps-2:jpe+2, kps-2:kpe+2, nbins)   mod_KindType.F90:388
 *   acum  my_acum(ips-2:ipe+2, jps-2:jpe+2, nbins)                mod_KindType.F90:391
 *   s     my_s   (ips:ipe, jps:jpe, kps:kpe, nbins)               mod_KindType.F90:389
 *   vs    my_vs  (ips:ipe, jps:jpe, kbs-1:kbe+1, nbins)           mod_KindType.F90:390
 *   u     my_u   (ibs-1:ibe+1, jps:jpe, kps:kpe[,2])              mod_KindType.F90:547
 *   v     my_v   (jbs-1:jbe+1, ips:ipe, kps:kpe[,2])              mod_KindType.F90:548
 *   w     my_w   (kbs-1:kbe+1, ips:ipe, jps:jpe[,2])              mod_KindType.F90:549
 *   k1    my_k1  (ips-2:ipe+2, jps:jpe, kps:kpe)                  mod_KindType.F90:559
 *   k2    my_k2  (jps-2:jpe+2, ips:ipe, kps:kpe)                  mod_KindType.F90:560
 *   k3    my_k3  (kps-2:kpe+2, ips:ipe, jps:jpe)                  mod_F3D.F90:605
 *   dX1_p (ips-2:ipe+2)  dX1_b (ibs-1:ibe+1)   and likewise for 2, 3
 *   Hm1_p (jps:jpe)  Hm2_p (jps-2:jpe+2)  Hm3_p (ips:ipe, jps:jpe)
 */
#ifndef F3D_ORACLE_H
#define F3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz, nbins;
  int limiter;       /* 1 minmod, 2 superbee, 3 ospre      (mod_ADS.F90:121-131) */
  int time_marching; /* 1 Euler, 2 RK4                     (mod_ADS.F90:43-44)   */
} or_dims;

typedef struct {
  const double *dX1_p, *dX1_b, *dX2_p, *dX2_b, *dX3_p, *dX3_b;
  const double *Hm1_p, *Hm2_p, *Hm3_p;
} or_grid;

/* One 1-D pencil KT right-hand side (mod_ADS.F90:1057-1120).  Arrays are
 * passed with the reference offsets: c,dxp,k start at index ips-2, u,dxb at
 * ibs-1.  rhs has n entries. */
void or_kt_rhs(int n, int limiter, const double *c, const double *dxp,
               const double *dxb, const double *u, const double *k,
               double flux[2], double *rhs);

/* ADS_solve_1D (mod_ADS.F90:820-1053) with bcode (0,-1,1,2) per side. */
void or_ads_solve_1d(int n, int limiter, double *c, const double *dxp,
                     const double *dxb, const double *u, const double *k,
                     double dt, const double bvalue[2], double flux[2],
                     const int bcode[2]);

/* ADS_solve_along_x/y/z (mod_ADS.F90:233, 422, 612).  u/v/w are the current
 * velocity (CB%u, CB%v and w1/w2 for z).  Fluxes are INOUT accumulators.
 * nthreads > 1 runs pencils in parallel; flux sums keep the serial order. */
void or_solve_x(const or_dims *d, const or_grid *g, double dt, double *c,
                const double *k1, const double *u, double *W, double *E,
                int nthreads);
void or_solve_y(const or_dims *d, const or_grid *g, double dt, double *c,
                const double *k2, const double *v, double *S, double *N,
                int nthreads);
void or_solve_z(const or_dims *d, const or_grid *g, double dt, double *c,
                double *acum, const double *k3, const double *w1,
                const double *w2, double stime, const double *vs, double *D,
                double *U, int nthreads);

/* Body of F3D_time_step (mod_F3D.F90:1435-1491): u/v time interpolation,
 * dense source injection, alternating x/y sweeps, z sweep.
 * u12/v12/w12 hold both meteo snapshots (last dimension 2).
 * fluxes = {W,E,S,N,U,D} accumulators. */
void or_time_step(const or_dims *d, const or_grid *g, double dt, double time,
                  double t_its, double t_ite, int iiter, double *c,
                  double *acum, const double *s, const double *u12,
                  const double *v12, const double *w12, const double *k1,
                  const double *k2, const double *k3, const double *vs,
                  double fluxes[6], int nthreads);

/* The same body with the current winds given: u(ibs-1:ibe+1, jps:jpe,
 * kps:kpe) and v(jbs-1:jbe+1, ips:ipe, kps:kpe) as F3D_time_step holds them
 * after the time interpolation and F3D_add_radial_wind; w12 and s_time for
 * the z sweep. */
void or_time_step_uv(const or_dims *d, const or_grid *g, double dt,
                     double s_time, int iiter, double *c, double *acum,
                     const double *s, const double *u, const double *v,
                     const double *w12, const double *k1, const double *k2,
                     const double *k3, const double *vs, double fluxes[6],
                     int nthreads);

/* Current winds at s_time = (time - t_its)/(t_ite - t_its)
 * (mod_F3D.F90:1437-1439, 1450): u, v, w in the single-snapshot layouts.
 * Returns s_time. */
double or_current_winds(const or_dims *d, double time, double t_its,
                        double t_ite, const double *u12, const double *v12,
                        const double *w12, double *u, double *v, double *w);

/* Gravity current, F3D_add_radial_wind (mod_F3D.F90:978-1226).
 * p: lon, lat, start_time, end_time, c_flow_rate, k_entrain, brunt_vaisala,
 * lambda, mass_flow_rate, h_tot, input_min_radius (MY_MOD%MY_GC).
 * or_gc_state fills st = {vol_flow_rate, min_radius, radius_grav,
 * c_grav_factor, th_grav, hmin, hmax} for the given time and returns 1 when
 * the current is active (the wind is then modified and update_step set), 0
 * when the routine returns early.  lon_c(ibs:ibe), lat_c(jbs:jbe),
 * Hm1_c(jbs:jbe). */
int or_gc_state(const or_dims *d, const double p[11], double time,
                const double *lon_c, const double *lat_c, const double *Hm1_c,
                double st[7]);
/* Adds the radial wind of state st to the current u and v (layouts as in
 * or_time_step_uv); lon_p(ips:ipe), lat_p(jps:jpe), Hm1_p(jps:jpe),
 * z_c(ibs:ibe, jbs:jbe, kbs:kbe). */
void or_add_radial_wind(const or_dims *d, const double p[11],
                        const double st[7], const double *lon_c,
                        const double *lat_c, const double *lon_p,
                        const double *lat_p, const double *Hm1_p,
                        const double *Hm1_c, const double *z_c, double *u,
                        double *v);

/* phys_get_kdiffu (mod_Phys.F90:406-664) with its helpers phys_get_Rib,
 * phys_get_Fih, phys_get_Fc (:1684-1741) and grid_c2p(_2D)
 * (mod_Grid.F90:1229-1277).  kdf = {modkh, modkv, map_h} (MOD_CONSTANT 1,
 * CMAQ 2, SIMILARITY 3, RAMS 4; MAP_H_CARTESIAN 0, SPHERICAL 1); par =
 * {kh0, kv0, RAMS_CS, dlon, dlat}.  uc, vc, tvc: current corner fields
 * (ibs:ibe, jbs:jbe, kbs:kbe); pblh, mon, ust (ips:ipe, jps:jpe); z_c
 * corners; h_c (ibs:ibe, jbs:jbe).  Outputs in the reference layouts
 * k1(ips-2:ipe+2, jps:jpe, kps:kpe), k2(ips:ipe, jps-2:jpe+2, kps:kpe),
 * k3(ips:ipe, jps:jpe, kps-2:kpe+2).  Returns MY_ERR%flag. */
int or_kdiffu(const or_dims *d, const or_grid *g, const int kdf[3],
              const double par[5], const double *uc, const double *vc,
              const double *tvc, const double *pblh, const double *mon,
              const double *ust, const double *z_c, const double *h_c,
              double *k1, double *k2, double *k3);

/* grid_get_time_step (mod_Grid.F90:1026-1141) for one rank. */
void or_get_time_step(const or_dims *d, const or_grid *g, int criterion,
                      double cfl, double run_end, const double *u,
                      const double *v, const double *w, const double *k1,
                      const double *k2, const double *k3, const double *vs,
                      double *my_dt, double *gl_dt);

/* grid_get_mass_volume (mod_Grid.F90:1340-1389) and
 * grid_get_mass_boundaries (mod_Grid.F90:1461-1511). */
double or_mass_volume(const or_dims *d, const or_grid *g, const double *c);
void or_mass_boundaries(const double fluxes[6], double *ground,
                        double *lateral);

/* phys_get_vset_point (mod_Phys.F90:757-954).  Returns MY_ERR%flag
 * (0 ok, 1 bad model, 2 no convergence); *iters gets the iteration count. */
int or_vset_point(double diam, double rhop, double psi, double rhoa,
                  double visc, int model, double *vset, int *iters);
/* The same with the iteration limit maxit in place of the reference's 1000
 * (the non-convergence path, flag 2, for tests). */
int or_vset_point_n(double diam, double rhop, double psi, double rhoa,
                    double visc, int model, double *vset, int *iters, int maxit);

/* phys_get_vset (mod_Phys.F90:673-740): corner air density/temperature
 * rhoc,tc (ibs:ibe, jbs:jbe, kbs:kbe) -> my_vs (i,j,kb1h,bin), unscaled.
 * bin_cat: 1 particle, 2 aerosol (zero), 3 radionuclide.  vset_fac applies
 * to bins flagged aggregate.  Returns the flag of the LAST point solved, as
 * the reference does (mod_Phys.F90:788). */
int or_get_vset(const or_dims *d, int model, const double *rhoc,
                const double *tc, const double *diam, const double *rhop,
                const double *psi, const int *bin_cat,
                const int *is_aggregate, double vset_fac, double *vs);

/* src_solve_suzuki (mod_Src.F90:1288-1358): np points, M(nbins,np). */
void or_suzuki(int np, int nbins, double M0, double Havl, double As,
               double Ls, double zo, const double *bin_fc, double *z,
               double *M);

/* Source placement of F3D_set_source_term (mod_F3D.F90:463-542) onto the
 * dense my_s(ips:ipe,jps:jpe,kps:kpe,nbins) for a single-rank grid.
 * lon_c(ibs:ibe), lat_c(jbs:jbe), z_c(ibs:ibe,jbs:jbe,kbs:kbe). */
void or_place_source(const or_dims *d, const or_grid *g, double lonmin,
                     double latmin, double dlon, double dlat,
                     const double *lon_c, const double *lat_c,
                     const double *z_c, int np, const double *x,
                     const double *y, const double *z, const double *M,
                     double *s);

/* phys_wet_deposition (mod_Phys.F90:1358-1427) for one bin on a single-rank
 * grid.  c(ips-2:ipe+2, jps-2:jpe+2, kps-2:kpe+2) and awet(ips-2:ipe+2,
 * jps-2:jpe+2) in the reference layouts (INOUT); pre, pblh (nx, ny);
 * h_c (nx+1, ny+1); z_c (nx+1, ny+1, nz+1); dX3_p (kps-2:kpe+2). */
void or_wet_deposition(const or_dims *d, double dt, double a, double b,
                       const double *pre, const double *pblh,
                       const double *h_c, const double *z_c,
                       const double *dX3_p, double *awet, double *c);

/* phys_radionuclides (mod_Phys.F90:1216-1342): decay of the radionuclide
 * bins (bin_cat 3, species 5 Cs134 .. 9 Y90) in the air, c(...,nbins) with
 * two halos, and in the deposits acum, awet(ips-2:ipe+2, jps-2:jpe+2, nbins).
 * Returns 1 when the numbers of Sr90 and Y90 bins differ. */
int or_radionuclides(const or_dims *d, double dt, const int *bin_cat,
                     const int *bin_spe, double *c, double *acum,
                     double *awet);

/* ensemble_perturbate_variable (mod_Ensemble.F90:888-935). */
double or_perturb(int var_id, int ptype, double var, double random,
                  double range);

/* grid_build_arakawa_c, tasks 0 and 1 (mod_Grid.F90:286-676), serial
 * domain.  Arrays (caller-allocated) with their reference bounds:
 * dX1_p(-1:nx+2), dX1_b(0:nx+2), dX2_p(-1:ny+2), dX2_b(0:ny+2),
 * dX3_p(-1:nz+2), dX3_b(0:nz+2), Hm2_p(-1:ny+2); lon_c(nx+1), lat_c(ny+1),
 * X3_c(nz+1), lon_p(nx), lat_p(ny), X3_p(nz), Hm1_p(ny), Hm1_c(ny+1);
 * dhdx_p, dhdy_p, Hm3_p (nx, ny); z_c (nx+1, ny+1, nz+1) column-major; the
 * input topography hc (nx+1, ny+1).  Returns 1 for the mappings the
 * reference leaves unimplemented. */
typedef struct {
  double dlon, dlat;
  double *lon_c, *lat_c, *X3_c, *lon_p, *lat_p, *X3_p, *Hm1_p, *Hm1_c, *Hm2_p;
  double *dX1_p, *dX1_b, *dX2_p, *dX2_b, *dX3_p, *dX3_b;
  double *dhdx_p, *dhdy_p, *Hm3_p, *z_c;
} or_grid_full;
int or_build_grid(int nx, int ny, int nz, int map_h, int map_v, double lonmin,
                  double lonmax, double latmin, double latmax, double X3max,
                  const double *gl_sigma, const double *hc, or_grid_full *g);
int or_meteo_term(int nx, int ny, int nz, int map_v, double X3max, const double *X3_c,
                  const double *X3_p, const double *Hm1_p, const double *Hm2_p,
                  const double *Hm3_p, const double *dhdx_p, const double *dhdy_p,
                  const double *uc, const double *vc, const double *wc, double *u, double *v,
                  double *w, double *k1, double *k2, double *k3);

#ifdef __cplusplus
}
#endif
#endif
