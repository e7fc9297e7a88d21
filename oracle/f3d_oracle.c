/*
 * f3d_oracle.c -- CPU FP64 oracle for the FALL3D ADS time step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed
 * CPU baseline.  Each routine restates one reference routine (file:line in
 * the comment above it) with the same operation order, so that a build with
 * -O2 -ffp-contract=off reproduces the reference's IEEE FP64 arithmetic.
 * Parity against the reference binary itself is unpinned (no Fortran
 * compiler here); analytic known-answer tests pin the algorithm instead.
 */
#include "f3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPS_KT 1e-12 /* EPSILON, mod_KindType.F90:42 */
#define GI 9.81      /* mod_KindType.F90:45 */
#define VISA0 1.827e-5 /* mod_Phys.F90:67 */
#define TA0 291.15     /* mod_Phys.F90:68 */

/* ---- index helpers (0-based interior indices; halos as in the reference) */
#define NX4 (d->nx + 4)
#define NY4 (d->ny + 4)
#define NZ4 (d->nz + 4)
#define IC(i, j, k, b) \
  ((size_t)((i) + 2) + (size_t)NX4 * ((size_t)((j) + 2) + (size_t)NY4 * ((size_t)((k) + 2) + (size_t)NZ4 * (size_t)(b))))
#define IACUM(i, j, b) ((size_t)((i) + 2) + (size_t)NX4 * ((size_t)((j) + 2) + (size_t)NY4 * (size_t)(b)))
#define IU(f, j, k) ((size_t)((f) + 1) + (size_t)(d->nx + 3) * ((size_t)(j) + (size_t)d->ny * (size_t)(k)))
#define IV(f, i, k) ((size_t)((f) + 1) + (size_t)(d->ny + 3) * ((size_t)(i) + (size_t)d->nx * (size_t)(k)))
#define IW(f, i, j) ((size_t)((f) + 1) + (size_t)(d->nz + 3) * ((size_t)(i) + (size_t)d->nx * (size_t)(j)))
#define IK1(p, j, k) ((size_t)((p) + 2) + (size_t)NX4 * ((size_t)(j) + (size_t)d->ny * (size_t)(k)))
#define IK2(p, i, k) ((size_t)((p) + 2) + (size_t)NY4 * ((size_t)(i) + (size_t)d->nx * (size_t)(k)))
#define IK3(p, i, j) ((size_t)((p) + 2) + (size_t)NZ4 * ((size_t)(i) + (size_t)d->nx * (size_t)(j)))
#define IVS(i, j, f, b) \
  ((size_t)(i) + (size_t)d->nx * ((size_t)(j) + (size_t)d->ny * ((size_t)((f) + 1) + (size_t)(d->nz + 3) * (size_t)(b))))
#define IS(i, j, k, b) \
  ((size_t)(i) + (size_t)d->nx * ((size_t)(j) + (size_t)d->ny * ((size_t)(k) + (size_t)d->nz * (size_t)(b))))

static size_t n_u(const or_dims *d) { return (size_t)(d->nx + 3) * d->ny * d->nz; }
static size_t n_v(const or_dims *d) { return (size_t)(d->ny + 3) * d->nx * d->nz; }
static size_t n_w(const or_dims *d) { return (size_t)(d->nz + 3) * d->nx * d->ny; }

/* ---- limiters: mod_ADS.F90:1124-1223.  r has n+4 entries (offset 2). */
static void limiter_fn(int lim, int n, const double *c, double *r) {
  /* c, r indexed from ips-2: element p lives at [p+2] */
  for (int p = -1; p <= n; ++p) {
    double cm = c[p + 1], c0 = c[p + 2], cp = c[p + 3];
    double rv;
    if (lim == 1) { /* r_minmod :1139-1147 */
      if (fabs(cp - c0) < EPS_KT) {
        rv = 1.0;
      } else {
        double r = (c0 - cm) / (cp - c0);
        rv = fmax(0.0, fmin(1.0, r));
      }
    } else if (lim == 2) { /* r_sbee :1170-1183 */
      if (fabs(cp - c0) < EPS_KT) {
        rv = (fabs(c0 - cm) < EPS_KT) ? 0.0 : 2.0;
      } else {
        double r = (c0 - cm) / (cp - c0);
        double a = fmin(2.0 * r, 1.0), b = fmin(r, 2.0);
        rv = fmax(fmax(0.0, a), b);
      }
    } else { /* r_ospre :1206-1219 */
      if (fabs(cp - c0) < EPS_KT) {
        rv = (fabs(c0 - cm) < EPS_KT) ? 0.0 : 1.5;
      } else {
        double r = (c0 - cm) / (cp - c0);
        rv = 1.5 * (r * r + r) / (r * r + r + 1.0);
      }
    }
    r[p + 2] = rv;
  }
  r[0] = r[1];         /* r(ips-2) = r(ips-1) */
  r[n + 3] = r[n + 2]; /* r(ipe+2) = r(ipe+1) */
}

/* ---- KT_RHS: mod_ADS.F90:1057-1120 */
void or_kt_rhs(int n, int limiter, const double *c, const double *dxp,
               const double *dxb, const double *u, const double *k,
               double flux[2], double *rhs) {
  double *r = (double *)malloc(sizeof(double) * (size_t)(n + 4));
  double *cr = (double *)malloc(sizeof(double) * (size_t)(n + 3));
  double *cl = (double *)malloc(sizeof(double) * (size_t)(n + 3));
  limiter_fn(limiter, n, c, r);
  /* c_r, c_l indexed from ips-1: element p at [p+1]; c,r at [p+2] */
  for (int p = -1; p <= n; ++p) {
    cr[p + 1] = c[p + 2] - 0.5 * r[p + 2] * (c[p + 3] - c[p + 2]);
    cl[p + 1] = c[p + 1] + 0.5 * r[p + 1] * (c[p + 2] - c[p + 1]);
  }
  for (int i = 0; i < n; ++i) {
    /* u, dxb indexed from ibs-1 = ips-1: face/cell i at [i+1] */
    double ui = u[i + 1], up = u[i + 2];
    double F_ml = cl[i + 1] * ui;
    double F_mr = cr[i + 1] * ui;
    double F_pl = cl[i + 2] * up;
    double F_pr = cr[i + 2] * up;
    double F_m = 0.5 * (F_ml + F_mr) - 0.5 * fabs(ui) * (cr[i + 1] - cl[i + 1]);
    double F_p = 0.5 * (F_pl + F_pr) - 0.5 * fabs(up) * (cr[i + 2] - cl[i + 2]);
    double P_m = 0.5 * (k[i + 2] + k[i + 1]) * (c[i + 2] - c[i + 1]) / dxp[i + 1];
    double P_p = 0.5 * (k[i + 3] + k[i + 2]) * (c[i + 3] - c[i + 2]) / dxp[i + 2];
    rhs[i] = -1.0 * (F_p - F_m) / dxb[i + 1] + (P_p - P_m) / dxb[i + 1];
    if (i == 0) flux[0] = F_m + P_m;
    if (i == n - 1) flux[1] = F_p + P_p;
  }
  free(r);
  free(cr);
  free(cl);
}

/* RK4 / Euler on one pencil whose ghosts are already set (mod_ADS.F90:313-399
 * for x; identical stage arithmetic in y :506-589 and z :714-798).
 * pc: n+4 values (ghosts frozen), result written back into pc interior. */
static void pencil_march(int n, int limiter, int tm, double dt, double *pc,
                         const double *dxp, const double *dxb,
                         const double *u, const double *k, double flux[2],
                         double *work) {
  double *ki = work;              /* n   */
  double *c0 = work + n;          /* n+4 */
  double *nw = work + 2 * n + 4;  /* n+4 */
  if (tm == 1) { /* Euler: my_c = my_c + dt*ki  (:299-302) */
    or_kt_rhs(n, limiter, pc, dxp, dxb, u, k, flux, ki);
    for (int i = 0; i < n; ++i) pc[i + 2] = pc[i + 2] + dt * ki[i];
    return;
  }
  or_kt_rhs(n, limiter, pc, dxp, dxb, u, k, flux, ki);
  memcpy(c0, pc, sizeof(double) * (size_t)(n + 4));
  memcpy(nw, pc, sizeof(double) * (size_t)(n + 4));
  for (int i = 0; i < n; ++i) {
    c0[i + 2] = c0[i + 2] + 0.5 * dt * ki[i];
    nw[i + 2] = nw[i + 2] + dt * ki[i] / 6.0;
  }
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, ki);
  for (int i = 0; i < n; ++i) {
    c0[i + 2] = pc[i + 2] + 0.5 * dt * ki[i];
    nw[i + 2] = nw[i + 2] + dt * ki[i] / 3.0;
  }
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, ki);
  for (int i = 0; i < n; ++i) {
    c0[i + 2] = pc[i + 2] + dt * ki[i];
    nw[i + 2] = nw[i + 2] + dt * ki[i] / 3.0;
  }
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, ki);
  for (int i = 0; i < n; ++i) pc[i + 2] = nw[i + 2] + dt * ki[i] / 6.0;
}

/* ---- ADS_solve_1D: mod_ADS.F90:820-1053 (serial; swaps are no-ops) */
void or_ads_solve_1d(int n, int limiter, double *c, const double *dxp,
                     const double *dxb, const double *u, const double *k,
                     double dt, const double bvalue[2], double flux[2],
                     const int bcode[2]) {
  /* u, dxb from ibs-1; face 0 (ibs) at [1], face n (ibe) at [n+1] */
  double uL = u[1], uR = u[n + 1];
  if (bcode[0] == -1) {
    if (uL > 0.0) { c[1] = c[n + 1]; c[0] = c[n]; c[n + 2] = c[2]; c[n + 3] = c[3]; }
  } else if (bcode[0] == 1) {
    c[1] = 2.0 * bvalue[0] - c[2]; c[0] = c[1];
  } else if (bcode[0] == 2) {
    if (uL > 0.0) c[1] = 2.0 * bvalue[0] - c[2]; else c[1] = c[2];
    c[0] = c[1];
  }
  if (bcode[1] == -1) {
    if (uR < 0.0) { c[1] = c[n + 1]; c[0] = c[n]; c[n + 2] = c[2]; c[n + 3] = c[3]; }
  } else if (bcode[1] == 1) {
    c[n + 2] = 2.0 * bvalue[1] - c[n + 1]; c[n + 3] = c[n + 2];
  } else if (bcode[1] == 2) {
    if (uR < 0.0) c[n + 2] = 2.0 * bvalue[1] - c[n + 1]; else c[n + 2] = c[n + 1];
    c[n + 3] = c[n + 2];
  }
  double *c0 = (double *)calloc((size_t)(n + 4), sizeof(double));
  double *k1 = (double *)calloc((size_t)n, sizeof(double));
  double *k2 = (double *)calloc((size_t)n, sizeof(double));
  double *k3 = (double *)calloc((size_t)n, sizeof(double));
  double *k4 = (double *)calloc((size_t)n, sizeof(double));
  memcpy(c0, c, sizeof(double) * (size_t)(n + 4));
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, k1);
  for (int i = 0; i < n; ++i) c0[i + 2] = c[i + 2] + 0.5 * dt * k1[i];
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, k2);
  for (int i = 0; i < n; ++i) c0[i + 2] = c[i + 2] + 0.5 * dt * k2[i];
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, k3);
  for (int i = 0; i < n; ++i) c0[i + 2] = c[i + 2] + dt * k3[i];
  or_kt_rhs(n, limiter, c0, dxp, dxb, u, k, flux, k4);
  for (int i = 0; i < n; ++i)
    c[i + 2] = c[i + 2] + dt * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]) / 6.0;
  free(c0); free(k1); free(k2); free(k3); free(k4);
}

/* ---- ADS_solve_along_x: mod_ADS.F90:233-412 */
void or_solve_x(const or_dims *d, const or_grid *g, double dt, double *c,
                const double *k1, const double *u, double *W, double *E,
                int nthreads) {
  const int nx = d->nx, ny = d->ny, nz = d->nz, nb = d->nbins;
  const int npen = ny * nz;
  double *cW = (double *)malloc(sizeof(double) * (size_t)npen);
  double *cE = (double *)malloc(sizeof(double) * (size_t)npen);
  for (int b = 0; b < nb; ++b) {
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
      double *work = (double *)malloc(sizeof(double) * (size_t)(3 * nx + 8));
#pragma omp for schedule(static)
      for (int pen = 0; pen < npen; ++pen) {
        int j = pen % ny, k = pen / ny;
        double *pc = c + IC(-2, j, k, b); /* contiguous in i */
        /* freeflow dim 1 (:1239-1266), bvalue = 0 */
        if (u[IU(0, j, k)] > 0.0) pc[1] = 2.0 * 0.0 - pc[2]; else pc[1] = pc[2];
        pc[0] = pc[1];
        if (u[IU(nx, j, k)] < 0.0) pc[nx + 2] = 2.0 * 0.0 - pc[nx + 1]; else pc[nx + 2] = pc[nx + 1];
        pc[nx + 3] = pc[nx + 2];
        double flux[2] = {0.0, 0.0};
        pencil_march(nx, d->limiter, d->time_marching, dt, pc, g->dX1_p,
                     g->dX1_b, u + IU(-1, j, k), k1 + IK1(-2, j, k), flux, work);
        double area = g->dX3_b[k + 1] * g->dX2_b[j + 1];
        cW[pen] = flux[0] * area * dt;
        cE[pen] = flux[1] * area * dt;
      }
      free(work);
    }
    for (int pen = 0; pen < npen; ++pen) { /* serial order: k outer, j inner */
      *W = *W + cW[pen];
      *E = *E + cE[pen];
    }
  }
  free(cW);
  free(cE);
}

/* ---- ADS_solve_along_y: mod_ADS.F90:422-602 */
void or_solve_y(const or_dims *d, const or_grid *g, double dt, double *c,
                const double *k2, const double *v, double *S, double *N,
                int nthreads) {
  const int nx = d->nx, ny = d->ny, nz = d->nz, nb = d->nbins;
  const int npen = nx * nz;
  double *cS = (double *)malloc(sizeof(double) * (size_t)npen);
  double *cN = (double *)malloc(sizeof(double) * (size_t)npen);
  for (int b = 0; b < nb; ++b) {
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
      double *work = (double *)malloc(sizeof(double) * (size_t)(3 * ny + 8));
      double *pc = (double *)malloc(sizeof(double) * (size_t)(ny + 4));
#pragma omp for schedule(static)
      for (int pen = 0; pen < npen; ++pen) {
        int i = pen % nx, k = pen / nx;
        /* freeflow dim 2 (:1268-1295) on my_c, then the ini_c copy (:508) */
        if (v[IV(0, i, k)] > 0.0) c[IC(i, -1, k, b)] = 2.0 * 0.0 - c[IC(i, 0, k, b)];
        else c[IC(i, -1, k, b)] = c[IC(i, 0, k, b)];
        c[IC(i, -2, k, b)] = c[IC(i, -1, k, b)];
        if (v[IV(ny, i, k)] < 0.0) c[IC(i, ny, k, b)] = 2.0 * 0.0 - c[IC(i, ny - 1, k, b)];
        else c[IC(i, ny, k, b)] = c[IC(i, ny - 1, k, b)];
        c[IC(i, ny + 1, k, b)] = c[IC(i, ny, k, b)];
        for (int p = -2; p <= ny + 1; ++p) pc[p + 2] = c[IC(i, p, k, b)];
        double flux[2] = {0.0, 0.0};
        pencil_march(ny, d->limiter, d->time_marching, dt, pc, g->dX2_p,
                     g->dX2_b, v + IV(-1, i, k), k2 + IK2(-2, i, k), flux, work);
        for (int p = 0; p < ny; ++p) c[IC(i, p, k, b)] = pc[p + 2];
        double area = g->dX3_b[k + 1] * g->dX1_b[i + 1];
        cS[pen] = flux[0] * area * dt;
        cN[pen] = flux[1] * area * dt;
      }
      free(work);
      free(pc);
    }
    for (int pen = 0; pen < npen; ++pen) {
      *S = *S + cS[pen];
      *N = *N + cN[pen];
    }
  }
  free(cS);
  free(cN);
}

/* ---- ADS_solve_along_z: mod_ADS.F90:612-811 */
void or_solve_z(const or_dims *d, const or_grid *g, double dt, double *c,
                double *acum, const double *k3, const double *w1,
                const double *w2, double stime, const double *vs, double *D,
                double *U, int nthreads) {
  const int nx = d->nx, ny = d->ny, nz = d->nz, nb = d->nbins;
  const int npen = nx * ny;
  double *cD = (double *)malloc(sizeof(double) * (size_t)npen);
  double *cU = (double *)malloc(sizeof(double) * (size_t)npen);
  for (int b = 0; b < nb; ++b) {
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
      double *work = (double *)malloc(sizeof(double) * (size_t)(3 * nz + 8));
      double *pc = (double *)malloc(sizeof(double) * (size_t)(nz + 4));
      double *wp = (double *)malloc(sizeof(double) * (size_t)(nz + 3));
#pragma omp for schedule(static)
      for (int pen = 0; pen < npen; ++pen) {
        int i = pen % nx, j = pen / nx;
        /* CB%w = (1-s) w1 + s w2 - vs(i,j,:,bin)   (:667-672) */
        for (int f = -1; f <= nz + 1; ++f) {
          double wc = (1.0 - stime) * w1[IW(f, i, j)] + stime * w2[IW(f, i, j)];
          wp[f + 1] = wc - vs[IVS(i, j, f, b)];
        }
        /* freeflow dim 3 (:1297-1324) */
        if (wp[1] > 0.0) c[IC(i, j, -1, b)] = 2.0 * 0.0 - c[IC(i, j, 0, b)];
        else c[IC(i, j, -1, b)] = c[IC(i, j, 0, b)];
        c[IC(i, j, -2, b)] = c[IC(i, j, -1, b)];
        if (wp[nz + 1] < 0.0) c[IC(i, j, nz, b)] = 2.0 * 0.0 - c[IC(i, j, nz - 1, b)];
        else c[IC(i, j, nz, b)] = c[IC(i, j, nz - 1, b)];
        c[IC(i, j, nz + 1, b)] = c[IC(i, j, nz, b)];
        for (int p = -2; p <= nz + 1; ++p) pc[p + 2] = c[IC(i, j, p, b)];
        double flux[2] = {0.0, 0.0};
        pencil_march(nz, d->limiter, d->time_marching, dt, pc, g->dX3_p,
                     g->dX3_b, wp, k3 + IK3(-2, i, j), flux, work);
        for (int p = 0; p < nz; ++p) c[IC(i, j, p, b)] = pc[p + 2];
        double area = g->dX2_b[j + 1] * g->dX1_b[i + 1];
        cD[pen] = flux[0] * area * dt;
        acum[IACUM(i, j, b)] = acum[IACUM(i, j, b)] + fabs(flux[0]) * dt;
        cU[pen] = flux[1] * area * dt;
      }
      free(work);
      free(pc);
      free(wp);
    }
    for (int pen = 0; pen < npen; ++pen) { /* serial order: j outer, i inner */
      *D = *D + cD[pen];
      *U = *U + cU[pen];
    }
  }
  free(cD);
  free(cU);
}

/* ---- F3D_time_step body: mod_F3D.F90:1435-1491 */
double or_current_winds(const or_dims *d, double time, double t_its,
                        double t_ite, const double *u12, const double *v12,
                        const double *w12, double *u, double *v, double *w) {
  const size_t nu = n_u(d), nv = n_v(d), nw = n_w(d);
  double s_time = (time - t_its) / (t_ite - t_its); /* :1437 */
  for (size_t q = 0; q < nu; ++q) u[q] = (1.0 - s_time) * u12[q] + s_time * u12[q + nu];
  for (size_t q = 0; q < nv; ++q) v[q] = (1.0 - s_time) * v12[q] + s_time * v12[q + nv];
  if (w)
    for (size_t q = 0; q < nw; ++q) w[q] = (1.0 - s_time) * w12[q] + s_time * w12[q + nw];
  return s_time;
}

void or_time_step_uv(const or_dims *d, const or_grid *g, double dt,
                     double s_time, int iiter, double *c, double *acum,
                     const double *s, const double *u, const double *v,
                     const double *w12, const double *k1, const double *k2,
                     const double *k3, const double *vs, double fluxes[6],
                     int nthreads) {
  const size_t nw = n_w(d);
  /* source term (:1456-1473) */
  for (int k = 0; k < d->nz; ++k) {
    double dZ = g->dX3_p[k + 2];
    for (int j = 0; j < d->ny; ++j) {
      double dY = g->dX2_p[j + 2], Hm1 = g->Hm1_p[j], Hm2 = g->Hm2_p[j + 2];
      for (int i = 0; i < d->nx; ++i) {
        double dX = g->dX1_p[i + 2], Hm3 = g->Hm3_p[i + (size_t)d->nx * j];
        double vol = dX * dY * dZ * (Hm1 * Hm2 * Hm3);
        for (int b = 0; b < d->nbins; ++b)
          c[IC(i, j, k, b)] = c[IC(i, j, k, b)] + dt * s[IS(i, j, k, b)] / vol;
      }
    }
  }
  if (iiter % 2 == 0) {
    or_solve_x(d, g, dt, c, k1, u, &fluxes[0], &fluxes[1], nthreads);
    or_solve_y(d, g, dt, c, k2, v, &fluxes[2], &fluxes[3], nthreads);
  } else {
    or_solve_y(d, g, dt, c, k2, v, &fluxes[2], &fluxes[3], nthreads);
    or_solve_x(d, g, dt, c, k1, u, &fluxes[0], &fluxes[1], nthreads);
  }
  or_solve_z(d, g, dt, c, acum, k3, w12, w12 + nw, s_time, vs, &fluxes[5],
             &fluxes[4], nthreads);
}

void or_time_step(const or_dims *d, const or_grid *g, double dt, double time,
                  double t_its, double t_ite, int iiter, double *c,
                  double *acum, const double *s, const double *u12,
                  const double *v12, const double *w12, const double *k1,
                  const double *k2, const double *k3, const double *vs,
                  double fluxes[6], int nthreads) {
  double *u = (double *)malloc(sizeof(double) * n_u(d));
  double *v = (double *)malloc(sizeof(double) * n_v(d));
  double s_time = or_current_winds(d, time, t_its, t_ite, u12, v12, NULL, u, v, NULL);
  or_time_step_uv(d, g, dt, s_time, iiter, c, acum, s, u, v, w12, k1, k2, k3,
                  vs, fluxes, nthreads);
  free(u);
  free(v);
}

/* ---- gravity current: F3D_add_radial_wind, mod_F3D.F90:978-1226.
 * PI = 4 atan(1) and REARTH = 6356000 m (mod_KindType.F90:43-44). */
#define GC_REARTH 6356000.0

int or_gc_state(const or_dims *d, const double p[11], double time,
                const double *lon_c, const double *lat_c, const double *Hm1_c,
                double st[7]) {
  const double PI = 4.0 * atan(1.0);
  const double c_flow_rate = p[4], k_entrain = p[5], brunt_vaisala = p[6],
               lambda_grav = p[7], mass_flow_rate = p[8], h_tot = p[9];
  (void)d;
  for (int q = 0; q < 7; ++q) st[q] = 0.0;
  if (time < p[2]) return 0; /* :1026-1027 */
  if (time > p[3]) return 0;
  if (mass_flow_rate <= 0.0) return 0; /* :1031 */
  /* minimum radius from the first cell's diagonal (:1036-1045) */
  double deltax = GC_REARTH * Hm1_c[0] * (lon_c[0] - lon_c[1]) * PI / 180.0;
  double deltay = GC_REARTH * (lat_c[0] - lat_c[1]) * PI / 180.0;
  double radius = 1.5 * sqrt(deltax * deltax + deltay * deltay);
  double min_radius = radius; /* parallel_max over a single rank */
  if (p[10] > 0.0) min_radius = p[10];
  double tse = time - p[2]; /* :1049 */
  double vol_flow_rate = c_flow_rate * sqrt(k_entrain) * pow(mass_flow_rate, 0.75) /
                         pow(brunt_vaisala, 1.25);
  double c_gravr = 3.0 * lambda_grav * brunt_vaisala * vol_flow_rate / (2.0 * PI);
  double radius_grav = pow(c_gravr * (tse * tse), 0.33333);
  radius_grav = fmax(radius_grav, min_radius);
  double c_gravu = sqrt(2.0 * lambda_grav * brunt_vaisala * vol_flow_rate / (3.0 * PI));
  double c_grav_factor = 0.75 * c_gravu * sqrt(radius_grav);
  double th_grav = c_gravu / (sqrt(radius_grav) * lambda_grav * brunt_vaisala);
  double h_umbr = h_tot / 1.2;
  double hmin = fmax(h_umbr - 0.5 * th_grav, 0.5 * h_tot);
  double hmax = fmin(h_umbr + 0.5 * th_grav, h_tot);
  st[0] = vol_flow_rate;
  st[1] = min_radius;
  st[2] = radius_grav;
  st[3] = c_grav_factor;
  st[4] = th_grav;
  st[5] = hmin;
  st[6] = hmax;
  return 1;
}

void or_add_radial_wind(const or_dims *d, const double p[11],
                        const double st[7], const double *lon_c,
                        const double *lat_c, const double *lon_p,
                        const double *lat_p, const double *Hm1_p,
                        const double *Hm1_c, const double *z_c, double *u,
                        double *v) {
  const double PI = 4.0 * atan(1.0);
  const double xc = p[0], yc = p[1];
  const double min_radius = st[1], radius_grav = st[2], c_grav_factor = st[3],
               hmin = st[5], hmax = st[6];
  const size_t nxc = (size_t)d->nx + 1, nyc = (size_t)d->ny + 1;
  /* x faces (:1144-1180) */
  for (int j = 0; j < d->ny; ++j)
    for (int i = 0; i <= d->nx; ++i) {
      double deltax = GC_REARTH * Hm1_p[j] * (lon_c[i] - xc) * PI / 180.0;
      double deltay = GC_REARTH * (lat_p[j] - yc) * PI / 180.0;
      double radius = sqrt(deltax * deltax + deltay * deltay);
      if (radius > radius_grav) continue;
      double fu = (radius < 1e-3) ? 0.0 : deltax / radius / Hm1_p[j];
      radius = fmax(radius, min_radius);
      double rvel = fu * c_grav_factor / radius *
                    (1.0 + radius * radius / (3.0 * (radius_grav * radius_grav)));
      for (int k = 0; k < d->nz; ++k) {
        double zp = z_c[i + nxc * (j + nyc * k)];
        if (zp >= hmin && zp <= hmax) u[IU(i, j, k)] = u[IU(i, j, k)] + rvel;
      }
    }
  /* y faces (:1184-1214) */
  for (int j = 0; j <= d->ny; ++j)
    for (int i = 0; i < d->nx; ++i) {
      double deltax = GC_REARTH * Hm1_c[j] * (lon_p[i] - xc) * PI / 180.0;
      double deltay = GC_REARTH * (lat_c[j] - yc) * PI / 180.0;
      double radius = sqrt(deltax * deltax + deltay * deltay);
      if (radius > radius_grav) continue;
      double fu = (radius < 1e-3) ? 0.0 : deltay / radius;
      radius = fmax(radius, min_radius);
      double rvel = fu * c_grav_factor / radius *
                    (1.0 + radius * radius / (3.0 * (radius_grav * radius_grav)));
      for (int k = 0; k < d->nz; ++k) {
        double zp = z_c[i + nxc * (j + nyc * k)];
        if (zp >= hmin && zp <= hmax) v[IV(j, i, k)] = v[IV(j, i, k)] + rvel;
      }
    }
}

/* ---- phys_get_kdiffu: mod_Phys.F90:406-664 */
#define KARMAN 0.4 /* mod_KindType.F90:46 */

int or_kdiffu(const or_dims *d, const or_grid *g, const int kdf[3],
              const double par[5], const double *uc, const double *vc,
              const double *tvc, const double *pblh, const double *mon,
              const double *ust, const double *z_c, const double *h_c,
              double *k1, double *k2, double *k3) {
  const int nx = d->nx, ny = d->ny, nz = d->nz;
  const size_t NX1 = (size_t)nx + 1, NY1 = (size_t)ny + 1;
  const int modkh = kdf[0], modkv = kdf[1], map_h = kdf[2];
  const double kh0 = par[0], kv0 = par[1], rams_cs = par[2], dlon = par[3], dlat = par[4];
  const double alfa = 0.28, khf = 8000.0, rkhmin = 100.0, landac = 30.0; /* :444-447 */
  double khn0;
  if (map_h == 0) khn0 = 4000.0; /* :449-459 */
  else if (map_h == 1) khn0 = 0.036;
  else return 1;
#define UC(a, i, j, k) a[(size_t)(i) + NX1 * ((size_t)(j) + NY1 * (size_t)(k))]
#define K1(p, j, k) k1[(size_t)((p) + 2) + (size_t)(nx + 4) * ((size_t)(j) + (size_t)ny * (size_t)(k))]
#define K2(i, p, k) k2[(size_t)(i) + (size_t)nx * ((size_t)((p) + 2) + (size_t)(ny + 4) * (size_t)(k))]
#define K3(i, j, p) k3[(size_t)(i) + (size_t)nx * ((size_t)(j) + (size_t)ny * (size_t)((p) + 2))]
  /* horizontal (:474-590) */
  if (modkh == 1) {
    for (size_t q = 0; q < (size_t)(nx + 4) * ny * nz; ++q) k1[q] = kh0;
    for (size_t q = 0; q < (size_t)nx * (ny + 4) * nz; ++q) k2[q] = kh0;
  } else if (modkh == 2 || modkh == 4) {
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          double dx = g->dX1_p[i + 2] * g->Hm1_p[j];
          double dy = g->dX2_p[j + 2] * g->Hm2_p[j + 2];
          double dudx = 0.5 * (UC(uc, i + 1, j, k) - UC(uc, i, j, k) + UC(uc, i + 1, j + 1, k) - UC(uc, i, j + 1, k)) / dx;
          double dvdx = 0.5 * (UC(vc, i + 1, j, k) - UC(vc, i, j, k) + UC(vc, i + 1, j + 1, k) - UC(vc, i, j + 1, k)) / dx;
          double dudy = 0.5 * (UC(uc, i, j + 1, k) - UC(uc, i, j, k) + UC(uc, i + 1, j + 1, k) - UC(uc, i + 1, j, k)) / dy;
          double dvdy = 0.5 * (UC(vc, i, j + 1, k) - UC(vc, i, j, k) + UC(vc, i + 1, j + 1, k) - UC(vc, i + 1, j, k)) / dy;
          double kv;
          if (modkh == 2) { /* CMAQ :484-499 */
            double kht = alfa * alfa * dx * dy *
                         sqrt((dudx - dvdy) * (dudx - dvdy) + (dvdx + dudy) * (dvdx + dudy));
            double khn = khf * (khn0 / (g->Hm1_p[j] * dlon)) * (khn0 / (g->Hm2_p[j + 2] * dlat));
            if (kht < 1.0 && khn < 1.0) kv = rkhmin;
            else kv = fmax(kht * khn / (kht + khn), rkhmin);
          } else { /* RAMS :528-550 */
            double kmh = 0.075 * pow(dx * dy, 2.0 / 3.0);
            kv = rams_cs * rams_cs * dx * dy *
                 sqrt((dudy + dvdx) * (dudy + dvdx) + 2.0 * (dudx * dudx + dvdy * dvdy));
            kv = fmax(fmax(kv, kmh), rkhmin);
          }
          K1(i, j, k) = kv;
          K2(i, j, k) = kv;
        }
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        K1(-2, j, k) = K1(0, j, k);
        K1(-1, j, k) = K1(0, j, k);
        K1(nx + 1, j, k) = K1(nx - 1, j, k);
        K1(nx, j, k) = K1(nx - 1, j, k);
      }
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nx; ++i) {
        K2(i, -2, k) = K2(i, 0, k);
        K2(i, -1, k) = K2(i, 0, k);
        K2(i, ny + 1, k) = K2(i, ny - 1, k);
        K2(i, ny, k) = K2(i, ny - 1, k);
      }
  } else {
    return 1;
  }
  /* vertical (:592-662) */
  if (modkv == 1) {
    for (size_t q = 0; q < (size_t)nx * ny * (nz + 4); ++q) k3[q] = kv0;
  } else if (modkv == 3) {
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double hp = (h_c[i + NX1 * j] + h_c[i + 1 + NX1 * j] + h_c[i + NX1 * (j + 1)] +
                     h_c[i + 1 + NX1 * (j + 1)]) / 4.0;
        double pb = pblh[i + (size_t)nx * j], L = mon[i + (size_t)nx * j], us = ust[i + (size_t)nx * j];
        for (int k = 0; k < nz; ++k) {
          double zp = (UC(z_c, i, j, k) + UC(z_c, i + 1, j, k) + UC(z_c, i, j + 1, k) + UC(z_c, i + 1, j + 1, k) +
                       UC(z_c, i, j, k + 1) + UC(z_c, i + 1, j, k + 1) + UC(z_c, i, j + 1, k + 1) +
                       UC(z_c, i + 1, j + 1, k + 1)) / 8.0;
          double z = fmax(0.0, zp - hp);
          double kv;
          if (z < pb) {
            double zl = z / L, fih; /* phys_get_Fih :1702-1721 */
            if (zl < 0.0) fih = 1.0 / sqrt(1.0 - 15.0 * zl);
            else fih = 1.0 + 5.0 * zl;
            kv = KARMAN * z * us * (1.0 - z / pb) * (1.0 - z / pb) / fih;
            kv = fmax(0.0, kv);
          } else {
            double lc = 1.0 / (KARMAN * z) + 1.0 / landac;
            lc = 1.0 / lc;
            double z1 = 0.25 * (UC(z_c, i, j, k) + UC(z_c, i + 1, j, k) + UC(z_c, i, j + 1, k) + UC(z_c, i + 1, j + 1, k));
            z1 = z1 - hp;
            double z2 = 0.25 * (UC(z_c, i, j, k + 1) + UC(z_c, i + 1, j, k + 1) + UC(z_c, i, j + 1, k + 1) +
                                UC(z_c, i + 1, j + 1, k + 1));
            z2 = z2 - hp;
            double u1 = 0.25 * (UC(uc, i, j, k) + UC(uc, i + 1, j, k) + UC(uc, i, j + 1, k) + UC(uc, i + 1, j + 1, k));
            double v1 = 0.25 * (UC(vc, i, j, k) + UC(vc, i + 1, j, k) + UC(vc, i, j + 1, k) + UC(vc, i + 1, j + 1, k));
            double u2 = 0.25 * (UC(uc, i, j, k + 1) + UC(uc, i + 1, j, k + 1) + UC(uc, i, j + 1, k + 1) +
                                UC(uc, i + 1, j + 1, k + 1));
            double v2 = 0.25 * (UC(vc, i, j, k + 1) + UC(vc, i + 1, j, k + 1) + UC(vc, i, j + 1, k + 1) +
                                UC(vc, i + 1, j + 1, k + 1));
            double umod1 = sqrt(u1 * u1 + v1 * v1);
            double umod2 = sqrt(u2 * u2 + v2 * v2);
            double umod = 0.5 * (umod1 + umod2);
            double tv1 = 0.25 * (UC(tvc, i, j, k) + UC(tvc, i + 1, j, k) + UC(tvc, i, j + 1, k) + UC(tvc, i + 1, j + 1, k));
            double tv2 = 0.25 * (UC(tvc, i, j, k + 1) + UC(tvc, i + 1, j, k + 1) + UC(tvc, i, j + 1, k + 1) +
                                 UC(tvc, i + 1, j + 1, k + 1));
            /* phys_get_Rib(Tv2, Tv1, umod, z2, z1) :1684-1696 */
            double um2 = fmax(umod * umod, 1e-18);
            double Ri = GI * (z2 - z1) * (tv2 - tv1) / (um2 * 0.5 * (tv2 + tv1));
            double fc; /* phys_get_Fc :1727-1741 */
            if (Ri > 0.0) {
              fc = 1.0 + 10.0 * Ri * (1.0 + 8.0 * Ri);
              fc = 1.0 / fc;
            } else {
              fc = sqrt(1.0 - 18.0 * Ri);
            }
            kv = lc * lc * fabs((umod2 - umod1) / (z2 - z1)) * fc;
            kv = fmax(0.0, kv);
          }
          K3(i, j, k) = kv;
        }
        K3(i, j, -2) = K3(i, j, 0);
        K3(i, j, -1) = K3(i, j, 0);
        K3(i, j, nz + 1) = K3(i, j, nz - 1);
        K3(i, j, nz) = K3(i, j, nz - 1);
      }
  } else {
    return 1;
  }
#undef UC
#undef K1
#undef K2
#undef K3
  return 0;
}

/* ---- grid_get_time_step: mod_Grid.F90:1026-1141 */
void or_get_time_step(const or_dims *d, const or_grid *g, int criterion,
                      double cfl, double run_end, const double *u,
                      const double *v, const double *w, const double *k1,
                      const double *k2, const double *k3, const double *vs,
                      double *my_dt_out, double *gl_dt_out) {
  const int nx = d->nx, ny = d->ny, nz = d->nz, nb = d->nbins;
  double dt1 = 0.0, dt2 = 0.0, dt3 = 0.0;
  if (criterion == 1) {
    for (int i = 0; i < nx; ++i) {
      double dx = g->dX1_p[i + 2];
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
          double dtinv = 2.0 * k1[IK1(i, j, k)] / (dx * dx) + fabs(u[IU(i, j, k)]) / dx;
          dt1 = fmax(dt1, dtinv);
        }
    }
    for (int j = 0; j < ny; ++j) {
      double dy = g->dX2_p[j + 2];
      for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) {
          double dtinv = 2.0 * k2[IK2(j, i, k)] / (dy * dy) + fabs(v[IV(j, i, k)]) / dy;
          dt2 = fmax(dt2, dtinv);
        }
    }
    for (int k = 0; k < nz; ++k) {
      double dz = g->dX3_p[k + 2];
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          double wv = w[IW(k, i, j)], w_max = -INFINITY;
          for (int b = 0; b < nb; ++b) w_max = fmax(w_max, fabs(wv - vs[IVS(i, j, k, b)]));
          double dtinv = 2.0 * k3[IK3(k, i, j)] / (dz * dz) + w_max / dz;
          dt3 = fmax(dt3, dtinv);
        }
    }
  } else {
    for (int k = 0; k < nz; ++k) {
      double dz = g->dX3_p[k + 2];
      for (int j = 0; j < ny; ++j) {
        double dy = g->dX2_p[j + 2];
        for (int i = 0; i < nx; ++i) {
          double dx = g->dX1_p[i + 2];
          double wv = w[IW(k, i, j)], w_max = -INFINITY;
          for (int b = 0; b < nb; ++b) w_max = fmax(w_max, fabs(wv - vs[IVS(i, j, k, b)]));
          double dtinv = 2.0 * k1[IK1(i, j, k)] / (dx * dx) + fabs(u[IU(i, j, k)]) / dx +
                         2.0 * k2[IK2(j, i, k)] / (dy * dy) + fabs(v[IV(j, i, k)]) / dy +
                         2.0 * k3[IK3(k, i, j)] / (dz * dz) + w_max / dz;
          dt1 = fmax(dt1, dtinv);
        }
      }
    }
  }
  double my_dt = fmax(fmax(dt1, dt2), dt3);
  if (my_dt > 0.0) my_dt = 1.0 / my_dt;
  my_dt = cfl * my_dt;
  double dt = my_dt; /* single rank: minval of one entry */
  *my_dt_out = fmin(my_dt, run_end);
  *gl_dt_out = fmin(dt, run_end);
}

/* ---- grid_get_mass_volume: mod_Grid.F90:1340-1389 */
double or_mass_volume(const or_dims *d, const or_grid *g, const double *c) {
  double my_mass = 0.0;
  for (int k = 0; k < d->nz; ++k) {
    double dZ = g->dX3_p[k + 2];
    for (int j = 0; j < d->ny; ++j) {
      double dY = g->dX2_p[j + 2];
      for (int i = 0; i < d->nx; ++i) {
        double dX = g->dX1_p[i + 2];
        for (int b = 0; b < d->nbins; ++b)
          my_mass = my_mass + c[IC(i, j, k, b)] * dX * dY * dZ;
      }
    }
  }
  return my_mass;
}

/* ---- grid_get_mass_boundaries: mod_Grid.F90:1461-1511.
 * fluxes = {W,E,S,N,U,D} */
void or_mass_boundaries(const double fluxes[6], double *ground,
                        double *lateral) {
  *ground = fabs(fluxes[5]);
  *lateral = fabs(fluxes[0]) + fabs(fluxes[1]) + fabs(fluxes[2]) +
             fabs(fluxes[3]) + fabs(fluxes[4]);
}

/* ---- phys_get_vset_point: mod_Phys.F90:757-954 (maxit = 1000 at :794) */
int or_vset_point(double diam, double rhop, double psi, double rhoa,
                  double visc, int model, double *vset_out, int *iters) {
  return or_vset_point_n(diam, rhop, psi, rhoa, visc, model, vset_out, iters, 1000);
}

int or_vset_point_n(double diam, double rhop, double psi, double rhoa,
                    double visc, int model, double *vset_out, int *iters, int maxit) {
  const double atol = 1e-12, rtol = 1e-6;
  double cd = 1.0, vset, vold, rey;
  *iters = 0;
  switch (model) {
    case 1: /* Arastopour :800-817 */
      vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
      vold = vset;
      for (int it = 1; it <= maxit; ++it) {
        rey = rhoa * vset * diam / visc;
        if (rey <= 988.947) cd = 24.0 / rey * (1.0 + 0.15 * pow(rey, 0.687));
        else cd = 0.44;
        vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
        *iters = it;
        if (fabs(vset - vold) <= atol + rtol * fabs(vset)) { *vset_out = vset; return 0; }
        vold = vset;
      }
      break;
    case 2: /* Ganser :820-838 */
      vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
      vold = vset;
      for (int it = 1; it <= maxit; ++it) {
        rey = rhoa * vset * diam / visc;
        double rk1 = 3.0 / (1.0 + 2.0 / sqrt(psi));
        double rk2 = pow(10.0, 1.8148 * pow(-log10(psi), 0.5743));
        cd = 24.0 / (rey * rk1) * (1.0 + 0.1118 * pow(rey * rk1 * rk2, 0.6567)) +
             0.4305 * rk2 / (1.0 + 3305.0 / (rey * rk1 * rk2));
        vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
        *iters = it;
        if (fabs(vset - vold) <= atol + rtol * fabs(vset)) { *vset_out = vset; return 0; }
        vold = vset;
      }
      break;
    case 3: /* Wilson :840-853 */
      vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
      vold = vset;
      for (int it = 1; it <= maxit; ++it) {
        rey = rhoa * vset * diam / visc;
        cd = 24.0 / rey * pow(psi, -0.828) + 2.0 * sqrt(1.07 - psi);
        vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
        *iters = it;
        if (fabs(vset - vold) <= atol + rtol * fabs(vset)) { *vset_out = vset; return 0; }
        vold = vset;
      }
      break;
    case 4: { /* Dellino :855-861 */
      double d3 = diam * diam * diam;
      vset = pow(d3 * GI * rhop * rhoa * pow(psi, 1.6) / (visc * visc), 0.5206);
      vset = 1.2065 * visc * vset / (diam * rhoa);
      *vset_out = vset;
      return 0;
    }
    case 5: { /* Pfeiffer :863-887 */
      vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
      vold = vset;
      double cd100 = 0.24 * pow(psi, -0.828) + 2.0 * sqrt(1.07 - psi);
      double cd1000 = 1.0;
      double a = (cd1000 - cd100) / 900.0;
      double b = cd1000 - 1000.0 * a;
      for (int it = 1; it <= maxit; ++it) {
        rey = rhoa * vset * diam / visc;
        if (rey <= 100.0) cd = 24.0 / rey * pow(psi, -0.828) + 2.0 * sqrt(1.07 - psi);
        else if (rey > 100.0 && rey < 1000.0) cd = a * rey + b;
        else cd = cd1000;
        vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
        *iters = it;
        if (fabs(vset - vold) <= atol + rtol * fabs(vset)) { *vset_out = vset; return 0; }
        vold = vset;
      }
      break;
    }
    case 6: /* Dioguardi 2017 :889-911 */
      vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
      vold = vset;
      for (int it = 1; it <= maxit; ++it) {
        rey = rhoa * vset * diam / visc;
        cd = 24.0 * (1.0 + 0.15 * pow(rey, 0.687)) / rey + 0.42 / (1.0 + 42500.0 / pow(rey, 1.16));
        cd = 0.74533 * pow(rey, 0.146012) * cd / pow(psi, 0.5134 / pow(fmax(rey, 0.01), 0.2));
        vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
        *iters = it;
        if (fabs(vset - vold) <= atol + rtol * fabs(vset)) { *vset_out = vset; return 0; }
        vold = vset;
      }
      break;
    case 7: /* Dioguardi 2018 :913-929 */
      vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
      vold = vset;
      for (int it = 1; it <= maxit; ++it) {
        rey = rhoa * vset * diam / visc;
        cd = 24.0 / rey * (pow((1.0 - psi) / rey + 1.0, 0.25) +
                           (0.1806 * pow(rey, 0.6459)) * pow(psi, -pow(rey, 0.08))) +
             0.4251 / (1.0 + 6880.95 / rey * pow(psi, 5.03));
        vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
        *iters = it;
        if (fabs(vset - vold) <= atol + rtol * fabs(vset)) { *vset_out = vset; return 0; }
        vold = vset;
      }
      break;
    default:
      *vset_out = 0.0;
      return 1;
  }
  *vset_out = vset; /* no convergence: vset keeps its last iterate */
  return 2;
}

/* ---- phys_get_vset: mod_Phys.F90:673-740 */
int or_get_vset(const or_dims *d, int model, const double *rhoc,
                const double *tc, const double *diam, const double *rhop,
                const double *psi, const int *bin_cat,
                const int *is_aggregate, double vset_fac, double *vs) {
  const int nx = d->nx, ny = d->ny, nz = d->nz, nb = d->nbins;
  const size_t cx = (size_t)nx + 1, cy = (size_t)ny + 1;
#define ICORNER(i, j, k) ((size_t)(i) + cx * ((size_t)(j) + cy * (size_t)(k)))
  int flag = 0;
  memset(vs, 0, sizeof(double) * (size_t)nx * ny * (nz + 3) * nb);
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double rhoa = 0.25 * (rhoc[ICORNER(i, j, k)] + rhoc[ICORNER(i + 1, j, k)] +
                              rhoc[ICORNER(i + 1, j + 1, k)] + rhoc[ICORNER(i, j + 1, k)]);
        double ta = 0.25 * (tc[ICORNER(i, j, k)] + tc[ICORNER(i + 1, j, k)] +
                            tc[ICORNER(i + 1, j + 1, k)] + tc[ICORNER(i, j + 1, k)]);
        double visa = VISA0 * ((TA0 + 120.0) / (ta + 120.0)) * pow(ta / TA0, 1.5);
        for (int b = 0; b < nb; ++b) {
          if (bin_cat[b] != 2) {
            int it;
            flag = or_vset_point(diam[b], rhop[b], psi[b], rhoa, visa, model,
                                 &vs[IVS(i, j, k, b)], &it);
          }
        }
      }
  for (int b = 0; b < nb; ++b)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        vs[IVS(i, j, -1, b)] = vs[IVS(i, j, 0, b)];
        vs[IVS(i, j, nz + 1, b)] = vs[IVS(i, j, nz, b)];
      }
  for (int b = 0; b < nb; ++b)
    if (is_aggregate && is_aggregate[b])
      for (int f = -1; f <= nz + 1; ++f)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) vs[IVS(i, j, f, b)] = vset_fac * vs[IVS(i, j, f, b)];
#undef ICORNER
  return flag;
}

/* ---- src_solve_suzuki: mod_Src.F90:1288-1358 */
void or_suzuki(int np, int nbins, double M0, double Havl, double As,
               double Ls, double zo, const double *bin_fc, double *z,
               double *M) {
  double *S = (double *)malloc(sizeof(double) * (size_t)np);
  double msum = 0.0;
  double deltaz = Havl / np;
  for (int is = 1; is <= np; ++is) {
    double zz = is * deltaz;
    double z2 = fmax(1.0 - zz / Havl, 0.0);
    S[is - 1] = z2 * exp(-As * z2);
    S[is - 1] = pow(S[is - 1], Ls);
    z[is - 1] = zo + zz;
    msum = msum + S[is - 1];
  }
  for (int is = 0; is < np; ++is) S[is] = (msum > 0) ? M0 * S[is] / msum : 0.0;
  for (int is = 0; is < np; ++is)
    for (int ic = 0; ic < nbins; ++ic) M[ic + (size_t)nbins * is] = bin_fc[ic] * S[is];
  free(S);
}

/* ---- source placement of F3D_set_source_term: mod_F3D.F90:463-542 */
void or_place_source(const or_dims *d, const or_grid *g, double lonmin_g,
                     double latmin_g, double dlon_g, double dlat_g,
                     const double *lon_c, const double *lat_c,
                     const double *z_c, int np, const double *x,
                     const double *y, const double *z, const double *M,
                     double *s) {
  const int nx = d->nx, ny = d->ny, nz = d->nz, nb = d->nbins;
  const size_t cx = (size_t)nx + 1, cy = (size_t)ny + 1;
#define IZC(i, j, k) ((size_t)(i) + cx * ((size_t)(j) + cy * (size_t)(k)))
  memset(s, 0, sizeof(double) * (size_t)nx * ny * nz * nb);
  double lonmin = lon_c[0], lonmax = lon_c[nx];
  double latmin = lat_c[0], latmax = lat_c[ny];
  double glonmin = lonmin_g;
  if (glonmin >= 180.0) glonmin = glonmin - 360.0;
  double glatmin = latmin_g;
  double inv_dlon = 1.0 / dlon_g, inv_dlat = 1.0 / dlat_g;
  double *zc = (double *)malloc(sizeof(double) * (size_t)(nz + 1));
  for (int is = 0; is < np; ++is) {
    double xs = x[is], ys = y[is], zs = z[is];
    if (xs >= 180.0) xs = xs - 360.0;
    if (ys < latmin || ys >= latmax) continue;
    if (lonmin < lonmax) {
      if (xs < lonmin || xs >= lonmax) continue;
    } else {
      if (xs < lonmin && xs >= lonmax) continue;
    }
    double dla = ys - glatmin, dlo = xs - glonmin;
    if (dlo < 0) dlo = dlo + 360.0;
    int ix = 1 + (int)(dlo * inv_dlon); /* Fortran 1-based corner index */
    int iy = 1 + (int)(dla * inv_dlat);
    dla = ys - lat_c[iy - 1];
    dlo = xs - lon_c[ix - 1];
    if (dlo < 0) dlo = dlo + 360.0;
    double ss = 2.0 * dlo * inv_dlon - 1.0;
    double tt = 2.0 * dla * inv_dlat - 1.0;
    double st = ss * tt;
    double m1 = (1.0 - tt - ss + st) * 0.25;
    double m2 = (1.0 - tt + ss - st) * 0.25;
    double m3 = (1.0 + tt + ss + st) * 0.25;
    double m4 = (1.0 + tt - ss - st) * 0.25;
    for (int k = 0; k <= nz; ++k)
      zc[k] = m1 * z_c[IZC(ix - 1, iy - 1, k)] + m2 * z_c[IZC(ix, iy - 1, k)] +
              m3 * z_c[IZC(ix, iy, k)] + m4 * z_c[IZC(ix - 1, iy, k)];
    int iz = -1;
    if (zs >= zc[0] && zs < zc[nz]) {
      /* grid_get_shapez loop (mod_Grid.F90:1316-1326) */
      for (int k = 0; k < nz; ++k)
        if (zs >= zc[k] && zs <= zc[k + 1]) { iz = k; break; }
    } else if (zs < zc[0]) {
      iz = 0;
    }
    if (iz < 0) continue;
    for (int b = 0; b < nb; ++b)
      s[IS(ix - 1, iy - 1, iz, b)] = s[IS(ix - 1, iy - 1, iz, b)] + M[b + (size_t)nb * is];
  }
  free(zc);
  for (int b = 0; b < nb; ++b)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        double Hm1 = g->Hm1_p[j], Hm2 = g->Hm2_p[j + 2];
        for (int i = 0; i < nx; ++i) {
          double Hm3 = g->Hm3_p[i + (size_t)nx * j];
          s[IS(i, j, k, b)] = s[IS(i, j, k, b)] * (Hm1 * Hm2 * Hm3);
        }
      }
#undef IZC
}

/* ---- ensemble_perturbate_variable: mod_Ensemble.F90:888-935 */
double or_perturb(int var_id, int ptype, double var, double random,
                  double range) {
  double out = var, factor;
  if (ptype == 1) {
    factor = random * range / 100.0;
    out = var * (1.0 + factor);
  } else if (ptype == 2) {
    factor = random * range;
    out = var + factor;
  }
  switch (var_id) {
    case 1: case 2: case 4: case 5: case 6: case 7:
      if (out < 0.0) out = 0.0;
      break;
    case 13: case 14:
      if (out < 0.0) out = 1.0;
      break;
    default:
      break;
  }
  return out;
}

/* ---- wet deposition and radionuclide decay ------------------------------ */
void or_wet_deposition(const or_dims *d, double dt, double a, double b,
                       const double *pre, const double *pblh,
                       const double *h_c, const double *z_c,
                       const double *dX3_p, double *awet, double *c) {
  const int nx = d->nx, ny = d->ny, nz = d->nz;
  const long hx = nx + 4, hy = ny + 4;
#define HC(i, j) h_c[(i) + (long)(nx + 1) * (j)]
#define ZC(i, j, k) z_c[(i) + (long)(nx + 1) * ((j) + (long)(ny + 1) * (k))]
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      /* lambda = min(1, dt*a*pre**b)  (mod_Phys.F90:1402) */
      double lambda = dt * a * pow(pre[i + (long)nx * j], b);
      if (lambda > 1.0) lambda = 1.0;
      const double pb = pblh[i + (long)nx * j];
      const double ho = 0.25 * (HC(i, j) + HC(i + 1, j) + HC(i, j + 1) + HC(i + 1, j + 1));
      double *aw = &awet[(i + 2) + hx * (j + 2)];
      for (int k = 0; k < nz; ++k) {
        const double zp1 = 0.25 * (ZC(i, j, k) + ZC(i + 1, j, k) + ZC(i, j + 1, k) + ZC(i + 1, j + 1, k));
        const double zp2 = 0.25 * (ZC(i, j, k + 1) + ZC(i + 1, j, k + 1) + ZC(i, j + 1, k + 1) +
                                   ZC(i + 1, j + 1, k + 1));
        const double zp = 0.5 * (zp1 + zp2);
        if (ho + zp <= pb) {
          double *cc = &c[(i + 2) + hx * ((j + 2) + hy * (long)(k + 2))];
          *aw = *aw + dX3_p[k + 2] * lambda * (*cc);
          *cc = *cc * (1.0 - lambda);
        }
      }
    }
#undef HC
#undef ZC
}

static double or_decay_rate(int spe) {
  switch (spe) { /* mod_Phys.F90:79-83 */
    case 5: return 1.06e-8;   /* Cs134 */
    case 6: return 9.29e-10;  /* Cs137 */
    case 7: return 1.00e-6;   /* I131 */
    case 8: return 7.63e-10;  /* Sr90 */
    case 9: return 2.98e-6;   /* Y90 */
  }
  return -1.0;
}

int or_radionuclides(const or_dims *d, double dt, const int *bin_cat,
                     const int *bin_spe, double *c, double *acum,
                     double *awet) {
  const int nb = d->nbins;
  const long n2 = (long)(d->nx + 4) * (d->ny + 4), n3 = n2 * (d->nz + 4);
  int ny90 = 0, nsr90 = 0, shift = 0;
  for (int b = 0; b < nb; ++b) {
    if (bin_cat[b] == 3 && bin_spe[b] == 9) {
      ++ny90;
      if (ny90 == 1) shift -= b;
    }
    if (bin_cat[b] == 3 && bin_spe[b] == 8) {
      ++nsr90;
      if (nsr90 == 1) shift += b;
    }
  }
  if (ny90 != nsr90 || nb > 64) return 1;
  double fact[64];
  for (int b = 0; b < nb && b < 64; ++b) {
    fact[b] = 1.0;
    if (bin_cat[b] == 3) {
      const double kn = or_decay_rate(bin_spe[b]);
      if (kn < 0.0) return 1;
      fact[b] = exp(-kn * dt);
    }
  }
  /* in the air: bins in order; Y90 is then set from its Sr90 parent
   * (mod_Phys.F90:1303-1318) */
  for (int b = 0; b < nb; ++b) {
    if (bin_cat[b] != 3) continue;
    for (long q = 0; q < n3; ++q) {
      c[q + n3 * b] = c[q + n3 * b] * fact[b];
      if (bin_spe[b] == 9) c[q + n3 * b] = c[q + n3 * (b + shift)] * (1.0 - fact[b + shift]);
    }
  }
  /* in the deposits (mod_Phys.F90:1320-1340) */
  for (int b = 0; b < nb; ++b) {
    if (bin_cat[b] != 3) continue;
    for (long q = 0; q < n2; ++q) {
      acum[q + n2 * b] = acum[q + n2 * b] * fact[b];
      awet[q + n2 * b] = awet[q + n2 * b] * fact[b];
      if (bin_spe[b] == 9) {
        acum[q + n2 * b] = acum[q + n2 * (b + shift)] * (1.0 - fact[b + shift]);
        awet[q + n2 * b] = awet[q + n2 * (b + shift)] * (1.0 - fact[b + shift]);
      }
    }
  }
  return 0;
}

/* ---- grid_build_arakawa_c, tasks 0 and 1: mod_Grid.F90:286-676 (serial
 * domain: my_ibs = 1, my_ibe = gl_nbx, ...).  Fortran indices are kept in the
 * loops; F1(a, lo, idx) addresses element idx of an array whose first
 * element has Fortran index lo. */
#define F1(a, lo, idx) (a)[(idx) - (lo)]
int or_build_grid(int nx, int ny, int nz, int map_h, int map_v, double lonmin,
                  double lonmax, double latmin, double latmax, double X3max,
                  const double *gl_sigma, const double *hc, or_grid_full *g) {
  const int gl_nbx = nx + 1, gl_nby = ny + 1, gl_nbz = nz + 1;
  const double PI_ = 4.0 * atan(1.0), REARTH_ = 6356000.0;
  double dlon, dlat;
  /* task 0 (:326-567) */
  if (map_h == 1 && !(lonmax > lonmin))
    dlon = (360.0 + lonmax - lonmin) / (gl_nbx - 1);
  else
    dlon = (lonmax - lonmin) / (gl_nbx - 1);
  dlat = (latmax - latmin) / (gl_nby - 1);
  g->dlon = dlon;
  g->dlat = dlat;
  for (int i = 1; i <= gl_nbx; ++i) F1(g->lon_c, 1, i) = lonmin + (i - 1) * dlon;
  for (int j = 1; j <= gl_nby; ++j) F1(g->lat_c, 1, j) = latmin + (j - 1) * dlat;
  for (int k = 1; k <= gl_nbz; ++k) F1(g->X3_c, 1, k) = F1(gl_sigma, 1, k) * X3max;
  for (int i = 1; i <= nx; ++i)
    F1(g->lon_p, 1, i) = 0.5 * (F1(g->lon_c, 1, i) + F1(g->lon_c, 1, i + 1));
  for (int j = 1; j <= ny; ++j)
    F1(g->lat_p, 1, j) = 0.5 * (F1(g->lat_c, 1, j) + F1(g->lat_c, 1, j + 1));
  for (int k = 1; k <= nz; ++k)
    F1(g->X3_p, 1, k) = 0.5 * (F1(g->X3_c, 1, k) + F1(g->X3_c, 1, k + 1));
  if (map_h == 0) {
    for (int j = 1; j <= ny; ++j) F1(g->Hm1_p, 1, j) = 1.0;
    for (int j = 1; j <= gl_nby; ++j) F1(g->Hm1_c, 1, j) = 1.0;
  } else if (map_h == 1) {
    for (int j = 1; j <= ny; ++j)
      F1(g->Hm1_p, 1, j) = sin((90.0 - F1(g->lat_p, 1, j)) * PI_ / 180.0);
    for (int j = 1; j <= gl_nby; ++j)
      F1(g->Hm1_c, 1, j) = sin((90.0 - F1(g->lat_c, 1, j)) * PI_ / 180.0);
  } else {
    return 1; /* POLAR, MERCATOR: 'Mapping not implemented yet' */
  }
  for (int j = -1; j <= ny + 2; ++j) F1(g->Hm2_p, -1, j) = 1.0;
  {
    const double d1 = (map_h == 1) ? REARTH_ * dlon * PI_ / 180.0 : dlon;
    const double d2 = (map_h == 1) ? REARTH_ * dlat * PI_ / 180.0 : dlat;
    for (int i = -1; i <= nx + 2; ++i) F1(g->dX1_p, -1, i) = d1;
    for (int i = 0; i <= nx + 2; ++i) F1(g->dX1_b, 0, i) = d1;
    for (int j = -1; j <= ny + 2; ++j) F1(g->dX2_p, -1, j) = d2;
    for (int j = 0; j <= ny + 2; ++j) F1(g->dX2_b, 0, j) = d2;
  }
  /* dX3_b(kbs_1h:kbe_1h) = (0:nz+2), dX3_p(kps_2h:kpe_2h) = (-1:nz+2) */
  for (int k = 1; k <= gl_nbz - 1; ++k)
    F1(g->dX3_b, 0, k) = (F1(gl_sigma, 1, k + 1) - F1(gl_sigma, 1, k)) * X3max;
  F1(g->dX3_b, 0, 0) = F1(g->dX3_b, 0, 1);
  for (int k = gl_nbz; k <= nz + 2; ++k) F1(g->dX3_b, 0, k) = F1(g->dX3_b, 0, gl_nbz - 1);
  for (int k = 1; k <= gl_nbz - 2; ++k) {
    const double X3_p = 0.5 * (F1(gl_sigma, 1, k + 1) + F1(gl_sigma, 1, k)) * X3max;
    const double X3_p1 = 0.5 * (F1(gl_sigma, 1, k + 2) + F1(gl_sigma, 1, k + 1)) * X3max;
    F1(g->dX3_p, -1, k) = X3_p1 - X3_p;
  }
  for (int k = -1; k <= 0; ++k) F1(g->dX3_p, -1, k) = F1(g->dX3_p, -1, 1);
  for (int k = nz; k <= nz + 2; ++k) F1(g->dX3_p, -1, k) = F1(g->dX3_p, -1, nz - 1);
  if (map_h == 1) {
    for (int i = 1; i <= gl_nbx; ++i)
      if (F1(g->lon_c, 1, i) > 180.0) F1(g->lon_c, 1, i) = F1(g->lon_c, 1, i) - 360.0;
    for (int i = 1; i <= nx; ++i)
      if (F1(g->lon_p, 1, i) > 180.0) F1(g->lon_p, 1, i) = F1(g->lon_p, 1, i) - 360.0;
  }
  /* task 1 (:568-670): hc(ibs:ibe, jbs:jbe), column-major */
#define HC(i, j) hc[(size_t)((i) - 1) + (size_t)gl_nbx * (size_t)((j) - 1)]
#define P2(a, i, j) (a)[(size_t)((i) - 1) + (size_t)nx * (size_t)((j) - 1)]
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      P2(g->dhdx_p, i, j) = 0.5 * (HC(i + 1, j) + HC(i + 1, j + 1) - HC(i, j) - HC(i, j + 1)) /
                            F1(g->dX1_b, 0, i);
      P2(g->dhdy_p, i, j) = 0.5 * (-HC(i + 1, j) + HC(i + 1, j + 1) - HC(i, j) + HC(i, j + 1)) /
                            F1(g->dX2_b, 0, j);
    }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      if (map_v == 0 || map_v == 1) {
        P2(g->Hm3_p, i, j) = 1.0;
      } else if (map_v == 2) {
        const double h_p = 0.25 * (HC(i, j) + HC(i + 1, j) + HC(i + 1, j + 1) + HC(i, j + 1));
        P2(g->Hm3_p, i, j) = (X3max - h_p) / X3max;
      } else {
        return 1; /* SIGMA_EXPONENTIAL_DECAY: 'Mapping not implemented yet' */
      }
    }
  for (int j = 1; j <= gl_nby; ++j)
    for (int i = 1; i <= gl_nbx; ++i) {
      const double h = HC(i, j);
      for (int k = 1; k <= gl_nbz; ++k) {
        double z;
        if (map_v == 0) z = F1(g->X3_c, 1, k);
        else if (map_v == 1) z = F1(g->X3_c, 1, k) + h;
        else z = F1(g->X3_c, 1, k) * (X3max - h) / X3max + h;
        g->z_c[(size_t)(i - 1) + (size_t)gl_nbx * ((size_t)(j - 1) + (size_t)gl_nby * (size_t)(k - 1))] = z;
      }
    }
#undef HC
#undef P2
  return 0;
}
#undef F1

/* ---- the meteo term of the step (serial domain: my_ibs = 1, my_ibe = nx+1,
 * my_ips = 1, my_ipe = nx, likewise j and k).  Loops keep the reference's
 * Fortran indices; each array is addressed by its own lower bound.
 *
 *   grid_get_stagered_velocity   mod_Grid.F90:685-752
 *   grid_get_scaled_velocity     mod_Grid.F90:761-870
 *   grid_get_scaled_variables    mod_Grid.F90:879-1017, the k1/k2/k3 part
 *
 * uc, vc, wc: corner winds (ibs:ibe, jbs:jbe, kbs:kbe), ground level already
 * zeroed by the caller (mod_F3D.F90:676-683).  Outputs u (ibs-1:ibe+1,
 * jps:jpe, kps:kpe), v (ips:ipe, jbs-1:jbe+1, kps:kpe), w (ips:ipe, jps:jpe,
 * kbs-1:kbe+1).  k1 (ips-2:ipe+2, jps:jpe, kps:kpe), k2 (ips:ipe,
 * jps-2:jpe+2, kps:kpe), k3 (ips:ipe, jps:jpe, kps-2:kpe+2) are scaled in
 * place.  Grid arrays: Hm1_p (jps:jpe), Hm2_p (jps-2:jpe+2), Hm3_p, dhdx_p,
 * dhdy_p (ips:ipe, jps:jpe), X3_c (kbs:kbe), X3_p (kps:kpe).  map_v: 0
 * Cartesian, 1 sigma without decay, 2 sigma with linear decay.  Returns 1
 * for any other mapping (the reference's 'Mapping not implemented yet' /
 * 'Incorrect vertical mapping'), 0 otherwise.  The serial domain has no
 * neighbours, so the domain_swap_* halo exchanges do nothing. */
int or_meteo_term(int nx, int ny, int nz, int map_v, double X3max, const double *X3_c,
                  const double *X3_p, const double *Hm1_p, const double *Hm2_p,
                  const double *Hm3_p, const double *dhdx_p, const double *dhdy_p,
                  const double *uc, const double *vc, const double *wc, double *u, double *v,
                  double *w, double *k1, double *k2, double *k3) {
  const long NBX = nx + 1, NBY = ny + 1;
#define CRN(a, i, j, k) (a)[((i) - 1) + NBX * (((j) - 1) + NBY * (long)((k) - 1))]
#define UF(i, j, k) u[(i) + (long)(nx + 3) * (((j) - 1) + (long)ny * ((k) - 1))]
#define VF(i, j, k) v[((i) - 1) + (long)nx * ((j) + (long)(ny + 3) * ((k) - 1))]
#define WF(i, j, k) w[((i) - 1) + (long)nx * (((j) - 1) + (long)ny * (k))]
#define K1(i, j, k) k1[((i) + 1) + (long)(nx + 4) * (((j) - 1) + (long)ny * ((k) - 1))]
#define K2(i, j, k) k2[((i) - 1) + (long)nx * (((j) + 1) + (long)(ny + 4) * ((k) - 1))]
#define K3(i, j, k) k3[((i) - 1) + (long)nx * (((j) - 1) + (long)ny * ((k) + 1))]
#define P2(a, i, j) (a)[((i) - 1) + (long)nx * ((j) - 1)]
  if (map_v < 0 || map_v > 2) return 1;
  /* staggered u: faces i = 1..nx+1, one halo each side */
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx + 1; ++i)
        UF(i, j, k) = 0.25 * (CRN(uc, i, j, k) + CRN(uc, i, j + 1, k) + CRN(uc, i, j, k + 1) +
                              CRN(uc, i, j + 1, k + 1));
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      UF(0, j, k) = UF(1, j, k);
      UF(nx + 2, j, k) = UF(nx + 1, j, k);
    }
  /* staggered v */
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i)
      for (int j = 1; j <= ny + 1; ++j)
        VF(i, j, k) = 0.25 * (CRN(vc, i, j, k) + CRN(vc, i + 1, j, k) + CRN(vc, i, j, k + 1) +
                              CRN(vc, i + 1, j, k + 1));
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) {
      VF(i, 0, k) = VF(i, 1, k);
      VF(i, ny + 2, k) = VF(i, ny + 1, k);
    }
  /* staggered w */
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 1; k <= nz + 1; ++k)
        WF(i, j, k) = 0.25 * (CRN(wc, i, j, k) + CRN(wc, i + 1, j, k) + CRN(wc, i, j + 1, k) +
                              CRN(wc, i + 1, j + 1, k));
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      WF(i, j, 0) = WF(i, j, 1);
      WF(i, j, nz + 2) = WF(i, j, nz + 1);
    }
  /* scaled u and v */
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const double Hm1 = Hm1_p[j - 1];
      for (int i = 0; i <= nx + 2; ++i) UF(i, j, k) = UF(i, j, k) / Hm1;
    }
  for (int k = 1; k <= nz; ++k)
    for (int j = 0; j <= ny + 2; ++j) {
      const double Hm2 = 0.5 * (Hm2_p[j + 1] + Hm2_p[j]); /* Hm2_p(j) + Hm2_p(j-1) */
      for (int i = 1; i <= nx; ++i) VF(i, j, k) = VF(i, j, k) / Hm2;
    }
  /* scaled w: the terrain correction */
  if (map_v != 0) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double Hm3 = P2(Hm3_p, i, j);
        for (int k = 1; k <= nz + 1; ++k) {
          double hx = P2(dhdx_p, i, j), hy = P2(dhdy_p, i, j);
          if (map_v == 2) {
            const double hz = 1.0 - X3_c[k - 1] / X3max;
            hx = hx * hz;
            hy = hy * hz;
          }
          const double uw = 0.25 * (CRN(uc, i, j, k) + CRN(uc, i + 1, j, k) + CRN(uc, i, j + 1, k) +
                                    CRN(uc, i + 1, j + 1, k));
          const double vw = 0.25 * (CRN(vc, i, j, k) + CRN(vc, i + 1, j, k) + CRN(vc, i, j + 1, k) +
                                    CRN(vc, i + 1, j + 1, k));
          WF(i, j, k) = (WF(i, j, k) - hx * uw - hy * vw) / Hm3;
        }
      }
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        WF(i, j, 0) = WF(i, j, 1);
        WF(i, j, nz + 2) = WF(i, j, nz + 1);
      }
  }
  /* scaled k3 (mass points), then its two halos each side */
  if (map_v != 0)
    for (int k = 1; k <= nz; ++k) {
      const double hz = (map_v == 2) ? 1.0 - X3_p[k - 1] / X3max : 1.0;
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          const double Hm3 = P2(Hm3_p, i, j);
          double hx = P2(dhdx_p, i, j), hy = P2(dhdy_p, i, j);
          if (map_v == 2) {
            hx = hx * hz;
            hy = hy * hz;
          }
          K3(i, j, k) = (K3(i, j, k) + hx * hx * K1(i, j, k) + hy * hy * K2(i, j, k)) / (Hm3 * Hm3);
        }
    }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      K3(i, j, -1) = K3(i, j, 1);
      K3(i, j, 0) = K3(i, j, 1);
      K3(i, j, nz + 2) = K3(i, j, nz);
      K3(i, j, nz + 1) = K3(i, j, nz);
    }
  /* scaled k1 and k2 */
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const double Hm1 = Hm1_p[j - 1];
      for (int i = -1; i <= nx + 2; ++i) K1(i, j, k) = K1(i, j, k) / (Hm1 * Hm1);
    }
  for (int k = 1; k <= nz; ++k)
    for (int j = -1; j <= ny + 2; ++j) {
      const double Hm2 = Hm2_p[j + 1];
      for (int i = 1; i <= nx; ++i) K2(i, j, k) = K2(i, j, k) / (Hm2 * Hm2);
    }
#undef CRN
#undef UF
#undef VF
#undef WF
#undef K1
#undef K2
#undef K3
#undef P2
  return 0;
}
