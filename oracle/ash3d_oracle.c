/*
 * ash3d_oracle.c -- CPU restatement of Ash3d's per-time-step transport path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); see
 * ash3d_oracle.h.  Every routine cites the reference file:line it restates.
 * Compiled with -O3 -fno-fast-math -ffp-contract=off so that each Fortran
 * expression rounds exactly as written (left-to-right, one rounding per
 * operation, no fused multiply-add).
 */
#include "ash3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- index helpers for the Fortran layouts (1-based, ghosts at -1,0) ---- */
#define NXG(s) ((s)->nx + 4)
#define NYG(s) ((s)->ny + 4)
#define NZG(s) ((s)->nz + 4)

static inline size_t i3(const orc_state *s, int i, int j, int k) {
  return (size_t)(i + 1) + (size_t)NXG(s) * ((size_t)(j + 1) + (size_t)NYG(s) * (size_t)(k + 1));
}
static inline size_t c5(const orc_state *s, int i, int j, int k, int n, int t) {
  return i3(s, i, j, k) + (size_t)NXG(s) * NYG(s) * NZG(s) * ((size_t)(n - 1) + (size_t)s->ns * t);
}
static inline size_t v4(const orc_state *s, int i, int j, int k, int n) {
  return i3(s, i, j, k) + (size_t)NXG(s) * NYG(s) * NZG(s) * (size_t)(n - 1);
}
static inline size_t k3(const orc_state *s, int i, int j, int k) { /* (0:nx+1,0:ny+1,0:nz+1) */
  return (size_t)i + (size_t)(s->nx + 2) * ((size_t)j + (size_t)(s->ny + 2) * (size_t)k);
}
static inline size_t oyz(const orc_state *s, int j, int k, int n) {
  return (size_t)(j + 1) + (size_t)NYG(s) * ((size_t)(k + 1) + (size_t)NZG(s) * (size_t)(n - 1));
}
static inline size_t oxz(const orc_state *s, int i, int k, int n) {
  return (size_t)(i + 1) + (size_t)NXG(s) * ((size_t)(k + 1) + (size_t)NZG(s) * (size_t)(n - 1));
}
static inline size_t oxy(const orc_state *s, int i, int j, int n) {
  return (size_t)(i + 1) + (size_t)NXG(s) * ((size_t)(j + 1) + (size_t)NYG(s) * (size_t)(n - 1));
}
static inline size_t dep(const orc_state *s, int i, int j, int n) {
  return (size_t)(i - 1) + (size_t)s->nx * ((size_t)(j - 1) + (size_t)s->ny * (size_t)(n - 1));
}

/* Fortran MAX/MIN of two reals (no NaNs reach these). */
static inline size_t d2(const orc_state *s, int i, int j) { /* (-1:nx+2,-1:ny+2) */
  return (size_t)(i + 1) + (size_t)(s->nx + 4) * (size_t)(j + 1);
}
static inline double fmx(double a, double b) { return a > b ? a : b; }
static inline double fmn(double a, double b) { return a < b ? a : b; }

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

/* ======================================================================== */
/* Set_BC(bc_code), src/Set_BC.f90:15-126                                   */
/* ======================================================================== */
int orc_set_bc(orc_state *s, int code) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, ns = s->ns;
  double *c = s->concen;
  if (code == 1) {
    /* velocities: zero-order extrapolation (periodic wrap in x), :44-70 */
    for (int k = -1; k <= nz + 2; k++)
      for (int j = -1; j <= ny + 2; j++) {
        if (s->periodic) {
          s->vx[i3(s, -1, j, k)] = s->vx[i3(s, nx - 1, j, k)];
          s->vx[i3(s, 0, j, k)] = s->vx[i3(s, nx, j, k)];
          s->vx[i3(s, nx + 1, j, k)] = s->vx[i3(s, 1, j, k)];
          s->vx[i3(s, nx + 2, j, k)] = s->vx[i3(s, 2, j, k)];
        } else {
          s->vx[i3(s, -1, j, k)] = s->vx[i3(s, 1, j, k)];
          s->vx[i3(s, 0, j, k)] = s->vx[i3(s, 1, j, k)];
          s->vx[i3(s, nx + 1, j, k)] = s->vx[i3(s, nx, j, k)];
          s->vx[i3(s, nx + 2, j, k)] = s->vx[i3(s, nx, j, k)];
        }
      }
    for (int k = -1; k <= nz + 2; k++)
      for (int i = -1; i <= nx + 2; i++) {
        s->vy[i3(s, i, -1, k)] = s->vy[i3(s, i, 1, k)];
        s->vy[i3(s, i, 0, k)] = s->vy[i3(s, i, 1, k)];
        s->vy[i3(s, i, ny + 1, k)] = s->vy[i3(s, i, ny, k)];
        s->vy[i3(s, i, ny + 2, k)] = s->vy[i3(s, i, ny, k)];
      }
    for (int j = -1; j <= ny + 2; j++)
      for (int i = -1; i <= nx + 2; i++) {
        s->vz[i3(s, i, j, -1)] = s->vz[i3(s, i, j, 1)];
        s->vz[i3(s, i, j, 0)] = s->vz[i3(s, i, j, 1)];
        s->vz[i3(s, i, j, nz + 1)] = s->vz[i3(s, i, j, nz)];
        s->vz[i3(s, i, j, nz + 2)] = s->vz[i3(s, i, j, nz)];
      }
    for (int n = 1; n <= ns; n++)
      for (int j = -1; j <= ny + 2; j++)
        for (int i = -1; i <= nx + 2; i++) {
          s->vf[v4(s, i, j, -1, n)] = s->vf[v4(s, i, j, 1, n)];
          s->vf[v4(s, i, j, 0, n)] = s->vf[v4(s, i, j, 1, n)];
          s->vf[v4(s, i, j, nz + 1, n)] = s->vf[v4(s, i, j, nz, n)];
          s->vf[v4(s, i, j, nz + 2, n)] = s->vf[v4(s, i, j, nz, n)];
        }
    /* concentrations: zero all ghost shells of ts0, then periodic x, :77-91 */
    for (int n = 1; n <= ns; n++) {
      for (int k = -1; k <= nz + 2; k++)
        for (int j = -1; j <= ny + 2; j++) {
          c[c5(s, -1, j, k, n, 0)] = 0.0; c[c5(s, 0, j, k, n, 0)] = 0.0;
          c[c5(s, nx + 1, j, k, n, 0)] = 0.0; c[c5(s, nx + 2, j, k, n, 0)] = 0.0;
        }
      for (int k = -1; k <= nz + 2; k++)
        for (int i = -1; i <= nx + 2; i++) {
          c[c5(s, i, -1, k, n, 0)] = 0.0; c[c5(s, i, 0, k, n, 0)] = 0.0;
          c[c5(s, i, ny + 1, k, n, 0)] = 0.0; c[c5(s, i, ny + 2, k, n, 0)] = 0.0;
        }
      for (int j = -1; j <= ny + 2; j++)
        for (int i = -1; i <= nx + 2; i++) {
          c[c5(s, i, j, -1, n, 0)] = 0.0; c[c5(s, i, j, 0, n, 0)] = 0.0;
          c[c5(s, i, j, nz + 1, n, 0)] = 0.0; c[c5(s, i, j, nz + 2, n, 0)] = 0.0;
        }
      if (s->periodic)
        for (int k = -1; k <= nz + 2; k++)
          for (int j = -1; j <= ny + 2; j++) {
            c[c5(s, -1, j, k, n, 0)] = c[c5(s, nx - 1, j, k, n, 0)];
            c[c5(s, 0, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
            c[c5(s, nx + 1, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
            c[c5(s, nx + 2, j, k, n, 0)] = c[c5(s, 2, j, k, n, 0)];
          }
    }
    return 0;
  } else if (code == 2) {
    /* Neumann mirror of the concentration ghosts, :98-118 */
    for (int n = 1; n <= ns; n++) {
      for (int k = -1; k <= nz + 2; k++)
        for (int j = -1; j <= ny + 2; j++) {
          c[c5(s, -1, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
          c[c5(s, 0, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
          c[c5(s, nx + 1, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
          c[c5(s, nx + 2, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
          if (s->periodic) {
            c[c5(s, -1, j, k, n, 0)] = c[c5(s, nx - 1, j, k, n, 0)];
            c[c5(s, 0, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
            c[c5(s, nx + 1, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
            c[c5(s, nx + 2, j, k, n, 0)] = c[c5(s, 2, j, k, n, 0)];
          }
        }
      for (int k = -1; k <= nz + 2; k++)
        for (int i = -1; i <= nx + 2; i++) {
          c[c5(s, i, -1, k, n, 0)] = c[c5(s, i, 1, k, n, 0)];
          c[c5(s, i, 0, k, n, 0)] = c[c5(s, i, 1, k, n, 0)];
          c[c5(s, i, ny + 1, k, n, 0)] = c[c5(s, i, ny, k, n, 0)];
          c[c5(s, i, ny + 2, k, n, 0)] = c[c5(s, i, ny, k, n, 0)];
        }
      for (int j = -1; j <= ny + 2; j++)
        for (int i = -1; i <= nx + 2; i++) {
          c[c5(s, i, j, -1, n, 0)] = c[c5(s, i, j, 1, n, 0)];
          c[c5(s, i, j, 0, n, 0)] = c[c5(s, i, j, 1, n, 0)];
          c[c5(s, i, j, nz + 1, n, 0)] = c[c5(s, i, j, nz, n, 0)];
          c[c5(s, i, j, nz + 2, n, 0)] = c[c5(s, i, j, nz, n, 0)];
        }
    }
    return 0;
  }
  return 1; /* "ERROR BC code not recognized", :119-123 */
}

/* ======================================================================== */
/* One DCU row: the body shared by advect_x/y/z                              */
/* src/AdvectionHorz_DCU.f90:153-281 (identical in :485-533 and              */
/* src/AdvectionVert_DCU.f90:183-298).  All arrays are indexed -1..len+2     */
/* through pointers offset by one element.  The topography term (:251-257)   */
/* is added when topo is set (ZScaling_ID 2, DelDonD_cc of :163-166 in       */
/* r->deld); for ZScaling_ID 0/1 DelDonD_cc is 0 and the term is not        */
/* restated.                                                                */
/* ======================================================================== */
typedef struct {
  double *q, *vel, *sig, *kap, *dtv, *usig, *dq, *fss, *fsl, *fsr, *upd, *deld;
  double *mem;
} row_scratch;

static void row_alloc(row_scratch *r, int len) {
  size_t m = (size_t)len + 4;
  r->mem = (double *)calloc(12 * m, sizeof(double));
  double *p = r->mem;
  r->q = p + 1; p += m;  r->vel = p + 1; p += m; r->sig = p + 1; p += m;
  r->kap = p + 1; p += m; r->dtv = p + 1; p += m; r->usig = p + 1; p += m;
  r->dq = p + 1; p += m;  r->fss = p + 1; p += m; r->fsl = p + 1; p += m;
  r->fsr = p + 1; p += m; r->upd = p + 1; p += m; r->deld = p + 1;
}

static void dcu_row(const orc_state *s, row_scratch *r, int len, int rmin, int rmax, int topo) {
  const double dt = s->dt, eps = s->eps_thresh;
  double *q = r->q, *vel = r->vel, *sig = r->sig, *kap = r->kap;
  double *dtv = r->dtv, *usig = r->usig, *dq = r->dq, *fss = r->fss;
  double *fsl = r->fsl, *fsr = r->fsr, *upd = r->upd;
  for (int i = rmin - 2; i <= rmax + 2; i++) dtv[i] = dt / kap[i];           /* :155 */
  for (int i = -1; i <= len + 2; i++) usig[i] = 0.0;                        /* :159 */
  for (int I = rmin - 1; I <= rmax + 1; I++)                                 /* :160 */
    usig[I] = 0.5 * (vel[I - 1] + vel[I]) * sig[I];
  for (int I = rmin - 1; I <= rmax + 2; I++) dq[I] = q[I] - q[I - 1];       /* :168 */
  for (int I = rmin - 1; I <= rmax + 2; I++) { fsl[I] = 0.0; fsr[I] = 0.0; fss[I] = 0.0; }
  if (s->limiter != ORC_LIM_NONE) {
    for (int I = rmin; I <= rmax + 1; I++) {                                  /* :179-231 */
      if (!s->nocycle && fabs(dq[I]) <= eps) continue;
      double ldq;
      if (s->limiter == ORC_LIM_LAXWEN) {
        ldq = dq[I];
      } else {
        double dqu = (usig[I] > 0.0) ? dq[I - 1] : dq[I + 1];
        double theta;
        if (fabs(dqu) > 3.0 * fabs(dq[I]) || fabs(dq[I]) < eps)
          theta = copysign(3.0, dqu * dq[I]);
        else
          theta = dqu / dq[I];
        switch (s->limiter) {
          case ORC_LIM_BW: ldq = dqu; break;
          case ORC_LIM_FROMM: ldq = dq[I] * (0.5 * (1.0 + theta)); break;
          case ORC_LIM_MINMOD: ldq = dq[I] * fmx(0.0, fmn(1.0, theta)); break;
          case ORC_LIM_MC:
            ldq = dq[I] * fmx(0.0, fmn(fmn((1.0 + theta) / 2.0, 2.0), 2.0 * theta));
            break;
          case ORC_LIM_SUPERBEE:
          default:
            ldq = dq[I] * fmx(fmx(0.0, fmn(1.0, 2.0 * theta)), fmn(2.0, theta));
            break;
        }
      }
      double aus = fabs(usig[I]);
      fss[I] = 0.5 * aus * (1.0 - dtv[I] * aus) * ldq;                       /* :230 */
    }
  }
  for (int I = rmin - 1; I <= rmax + 1; I++) {                                /* :238-259 */
    fsr[I] = fmx(0.0, usig[I]) * dq[I];
    fsl[I] = fmn(0.0, usig[I]) * dq[I];
    double divu_p = fmx(0.0, usig[I]) - fmx(0.0, usig[I - 1]);
    double divu_m = fmn(0.0, usig[I + 1]) - fmn(0.0, usig[I]);
    fsr[I] = fsr[I] + q[I] * divu_m;
    fsl[I] = fsl[I] + q[I - 1] * divu_p;
    if (topo) {                                                                 /* :251-257 */
      const double *dd = r->deld;
      fsr[I] = fsr[I] + 0.5 * vel[I] * (sig[I] + sig[I + 1]) * q[I] * dd[I];
      fsl[I] = fsl[I] - 0.5 * vel[I - 1] * (sig[I - 1] + sig[I]) * q[I - 1] * dd[I - 1];
    }
  }
  for (int i = rmin - 1; i <= rmax + 1; i++)                                  /* :264-281 */
    upd[i] = -(dtv[i] * (fsl[i + 1] + fsr[i] + fss[i + 1] - fss[i]));
}

static void zero_level(orc_state *s, int t) {
  size_t lev = (size_t)NXG(s) * NYG(s) * NZG(s) * s->ns;
  memset(s->concen + lev * t, 0, lev * sizeof(double));
}

static void copy_back(orc_state *s) { /* ts0(1:nx,1:ny,1:nz,:) = ts1(...) */
  for (int n = 1; n <= s->ns; n++)
    for (int k = 1; k <= s->nz; k++)
      for (int j = 1; j <= s->ny; j++)
        memcpy(&s->concen[c5(s, 1, j, k, n, 0)], &s->concen[c5(s, 1, j, k, n, 1)],
               (size_t)s->nx * sizeof(double));
}

static int max3(int a, int b, int c) { int m = a > b ? a : b; return m > c ? m : c; }

/* advect_x, src/AdvectionHorz_DCU.f90:68-305 */
void orc_advect_x(orc_state *s) {
  orc_set_bc(s, 1);                                                           /* :115 */
  const int rmin = s->imin, rmax = s->imax, nx = s->nx;
  const int topo = s->use_topo && s->zscaling_id == 2;
  zero_level(s, 1);                                                           /* :122 */
  const int nth = orc_get_threads();
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
#pragma omp parallel num_threads(nth)
    {
      row_scratch r; row_alloc(&r, nx);
#pragma omp for collapse(2) schedule(static)
      for (int k = s->kmin; k <= s->kmax; k++)
        for (int j = s->jmin; j <= s->jmax; j++) {
          for (int i = rmin - 2; i <= rmax + 2; i++) {                        /* :143-146 */
            r.q[i] = s->concen[c5(s, i, j, k, n, 0)];
            r.vel[i] = s->vx[i3(s, i, j, k)];
            r.sig[i] = s->sig_nx[i3(s, i, j, k)];
            r.kap[i] = s->kappa[i3(s, i, j, k)];
          }
          if (topo)                                                           /* :163-166 */
            for (int i = rmin - 2; i <= rmax + 2; i++)
              r.deld[i] = (i >= rmin - 1 && i <= rmax + 1) ? s->deldx[d2(s, i, j)] : 0.0;
          dcu_row(s, &r, nx, rmin, rmax, topo);
          for (int i = rmin; i <= rmax; i++)                                  /* :285-287 */
            s->concen[c5(s, i, j, k, n, 1)] = s->concen[c5(s, i, j, k, n, 0)] + r.upd[i];
          if (rmin == 1 && !s->periodic) s->outflow_yz1[oyz(s, j, k, n)] += r.upd[0];
          if (rmax == nx && !s->periodic) s->outflow_yz2[oyz(s, j, k, n)] += r.upd[nx + 1];
        }
      free(r.mem);
    }
  }
  copy_back(s);                                                               /* :302-303 */
}

/* advect_y, src/AdvectionHorz_DCU.f90:322-556 */
void orc_advect_y(orc_state *s) {
  orc_set_bc(s, 1);
  const int rmin = s->jmin, rmax = s->jmax, ny = s->ny;
  const int topo = s->use_topo && s->zscaling_id == 2;
  zero_level(s, 1);
  const int nth = orc_get_threads();
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
#pragma omp parallel num_threads(nth)
    {
      row_scratch r; row_alloc(&r, ny);
#pragma omp for collapse(2) schedule(static)
      for (int k = s->kmin; k <= s->kmax; k++)
        for (int i = s->imin; i <= s->imax; i++) {
          for (int j = rmin - 2; j <= rmax + 2; j++) {
            r.q[j] = s->concen[c5(s, i, j, k, n, 0)];
            r.vel[j] = s->vy[i3(s, i, j, k)];
            r.sig[j] = s->sig_ny[i3(s, i, j, k)];
            r.kap[j] = s->kappa[i3(s, i, j, k)];
          }
          if (topo)                                                           /* :414-417 */
            for (int j = rmin - 2; j <= rmax + 2; j++)
              r.deld[j] = (j >= rmin - 1 && j <= rmax + 1) ? s->deldy[d2(s, i, j)] : 0.0;
          dcu_row(s, &r, ny, rmin, rmax, topo);
          for (int j = rmin; j <= rmax; j++)
            s->concen[c5(s, i, j, k, n, 1)] = s->concen[c5(s, i, j, k, n, 0)] + r.upd[j];
          if (rmin == 1) s->outflow_xz1[oxz(s, i, k, n)] += r.upd[0];          /* :540-545 */
          if (rmax == ny) s->outflow_xz2[oxz(s, i, k, n)] += r.upd[ny + 1];
        }
      free(r.mem);
    }
  }
  copy_back(s);
}

/* advect_z, src/AdvectionVert_DCU.f90:100-323 */
void orc_advect_z(orc_state *s) {
  orc_set_bc(s, 1);
  const int rmin = s->kmin, rmax = s->kmax, nz = s->nz;
  const int ncells = rmax - rmin + 1;
  zero_level(s, 1);
  const int nth = orc_get_threads();
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
#pragma omp parallel num_threads(nth)
    {
      row_scratch r; row_alloc(&r, max3(nz, ncells + 1, 1));
#pragma omp for collapse(2) schedule(static)
      for (int j = s->jmin; j <= s->jmax; j++)
        for (int i = s->imin; i <= s->imax; i++) {
          for (int k = rmin - 2; k <= rmax + 2; k++) {                        /* :171-176 */
            r.q[k] = s->concen[c5(s, i, j, k, n, 0)];
            r.vel[k] = s->vz[i3(s, i, j, k)] + s->vh[i3(s, i, j, k)] + s->vf[v4(s, i, j, k, n)];
            r.sig[k] = s->sig_nz[i3(s, i, j, k)];
            r.kap[k] = s->kappa[i3(s, i, j, k)];
          }
          dcu_row(s, &r, nz, rmin, rmax, 0);
          for (int k = rmin; k <= rmax; k++)
            s->concen[c5(s, i, j, k, n, 1)] = s->concen[c5(s, i, j, k, n, 0)] + r.upd[k];
          if (rmin == 1) s->outflow_xy1[oxy(s, i, j, n)] += r.upd[0];          /* :306-308 */
          /* :309-311 uses update_cc(ncells+1), which equals rmax+1 only when
           * kmin == 1 (the top-outflow index quirk is kept). */
          if (rmax == nz) s->outflow_xy2[oxy(s, i, j, n)] += r.upd[ncells + 1];
        }
      free(r.mem);
    }
  }
  copy_back(s);
  for (int n = 1; n <= s->ns; n++)                                            /* :321 */
    for (int j = 1; j <= s->ny; j++)
      for (int i = 1; i <= s->nx; i++)
        s->deposit[dep(s, i, j, n)] = s->outflow_xy1[oxy(s, i, j, n)];
}

/* get_minmax_index, src/Calc_Mesh.f90:432-542.  The per-plane maxval()s are
 * gathered in one pass (a max does not depend on the visiting order). */
int orc_get_minmax_index(orc_state *s, int ivent, int jvent, int kvent) {
  const double th = s->cloudcon_grid_thresh;
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  double *pi = (double *)malloc(sizeof(double) * (size_t)(nx + ny + nz + 3));
  double *pj = pi + nx + 1, *pk = pj + ny + 1;
  for (int i = 0; i <= nx; i++) pi[i] = -HUGE_VAL;
  for (int j = 0; j <= ny; j++) pj[j] = -HUGE_VAL;
  for (int k = 0; k <= nz; k++) pk[k] = -HUGE_VAL;
  for (int n = 1; n <= s->ns; n++)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          double v = s->concen[c5(s, i, j, k, n, 0)];
          if (v > pi[i]) pi[i] = v;
          if (v > pj[j]) pj[j] = v;
          if (v > pk[k]) pk[k] = v;
        }
  s->imin = 1; s->imax = nx;
  for (int i = 2; i <= ivent - 1; i++) { if (pi[i] < th) s->imin = i; else break; }
  for (int i = nx; i >= s->imin + 2; i--) { if (pi[i] < th) s->imax = i; else break; }
  if (s->periodic && (s->imin == 1 || s->imax == nx)) { s->imin = 1; s->imax = nx; }
  s->jmin = 1; s->jmax = ny;
  for (int j = 2; j <= jvent - 1; j++) { if (pj[j] < th) s->jmin = j; else break; }
  for (int j = ny; j >= s->jmin + 2; j--) { if (pj[j] < th) s->jmax = j; else break; }
  s->kmin = 1; s->kmax = nz;
  for (int k = 2; k <= kvent - 1; k++) { if (pk[k] < th) s->kmin = k; else break; }
  for (int k = nz; k >= s->kmin + 2; k--) { if (pk[k] < th) s->kmax = k; else break; }
  free(pi);
  if (s->kmax < s->kmin) return 1;
  if (s->imax - s->imin < 2) { s->imax = (s->imax + 1 < nx) ? s->imax + 1 : nx; s->imin = s->imax - 2; }
  if (s->jmax - s->jmin < 2) { s->jmax = (s->jmax + 1 < ny) ? s->jmax + 1 : ny; s->jmin = s->jmax - 2; }
  if (s->kmax - s->kmin < 2) { s->kmax = (s->kmax + 1 < nz) ? s->kmax + 1 : nz; s->kmin = s->kmax - 2; }
  return 0;
}

/* AdvectHorz(itoggle), src/AdvectionHorz.f90:47-85 */
int orc_advect_horz(orc_state *s, int itoggle, int ivent, int jvent, int kvent) {
  if (s->fast_subgrid) {
    if (orc_get_minmax_index(s, ivent, jvent, kvent)) return 1;
  } else {
    s->imin = 1; s->imax = s->nx; s->jmin = 1; s->jmax = s->ny; s->kmin = 1; s->kmax = s->nz;
  }
  if (itoggle % 2 == 0) { orc_advect_y(s); orc_advect_x(s); }
  else { orc_advect_x(s); orc_advect_y(s); }
  return 0;
}

/* AdvectVert, src/AdvectionVert_DCU.f90:64-82 */
void orc_advect_vert(orc_state *s) { orc_advect_z(s); }  /* advect_sigma == advect_z */

/* Calc_Vmod_Topo, src/Topography.f90:2138-2166 (every i, j, k of vh_pd). */
void orc_calc_vmod_topo(orc_state *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int k = -1; k <= nz + 2; k++)
    for (int j = -1; j <= ny + 2; j++)
      for (int i = -1; i <= nx + 2; i++) {
        const size_t m = i3(s, i, j, k);
        if (!s->use_topo || s->zscaling_id == 0) {
          s->vh[m] = 0.0;
        } else {
          const double g = s->vx[m] * s->dhdx[d2(s, i, j)] + s->vy[m] * s->dhdy[d2(s, i, j)];
          if (s->zscaling_id == 1) s->vh[m] = -1.0 * g;
          else s->vh[m] = (s->s_cc[k + 1] / s->ztop - 1.0) * g;
        }
      }
}

/* ======================================================================== */
/* Explicit diffusion, src/Diffusion.F90:266-650                             */
/* ======================================================================== */
/* One explicit row: q,kap indexed rmin-1..rmax+1, sig 1..; kk the
 * diffusivity along the row (indexed like q).  :335-377 */
static void diff_row(double dt, int rmin, int rmax, const double *q, const double *kap,
                     const double *sig, const double *kk, double *upd) {
  /* ds_I/k_ds_I at interfaces rmin..rmax+1 */
  for (int l = rmin; l <= rmax; l++) {
    double dsR = 2.0 * sig[l + 1] / (kap[l] + kap[l + 1]);
    double kdsR = 0.5 * (kk[l] + kk[l + 1]) * dsR;
    double dsL = 2.0 * sig[l] / (kap[l - 1] + kap[l]);
    double kdsL = 0.5 * (kk[l - 1] + kk[l]) * dsL;
    double dqR = q[l + 1] - q[l];
    double dqL = q[l] - q[l - 1];
    double LF = dt * kdsR * dqR * (sig[l + 1] / kap[l]);
    double RF = -(dt * kdsL * dqL * (sig[l] / kap[l]));
    upd[l] = LF + RF;
  }
}

static void neumann_x(orc_state *s) { /* :317-327 */
  const int nx = s->nx;
  double *c = s->concen;
  for (int n = 1; n <= s->ns; n++)
    for (int k = -1; k <= s->nz + 2; k++)
      for (int j = -1; j <= s->ny + 2; j++) {
        c[c5(s, -1, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
        c[c5(s, 0, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
        c[c5(s, nx + 1, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
        c[c5(s, nx + 2, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
        if (s->periodic) {
          c[c5(s, -1, j, k, n, 0)] = c[c5(s, nx - 1, j, k, n, 0)];
          c[c5(s, 0, j, k, n, 0)] = c[c5(s, nx, j, k, n, 0)];
          c[c5(s, nx + 1, j, k, n, 0)] = c[c5(s, 1, j, k, n, 0)];
          c[c5(s, nx + 2, j, k, n, 0)] = c[c5(s, 2, j, k, n, 0)];
        }
      }
}
static void neumann_y(orc_state *s) { /* :457-460 */
  const int ny = s->ny;
  double *c = s->concen;
  for (int n = 1; n <= s->ns; n++)
    for (int k = -1; k <= s->nz + 2; k++)
      for (int i = -1; i <= s->nx + 2; i++) {
        c[c5(s, i, -1, k, n, 0)] = c[c5(s, i, 1, k, n, 0)];
        c[c5(s, i, 0, k, n, 0)] = c[c5(s, i, 1, k, n, 0)];
        c[c5(s, i, ny + 1, k, n, 0)] = c[c5(s, i, ny, k, n, 0)];
        c[c5(s, i, ny + 2, k, n, 0)] = c[c5(s, i, ny, k, n, 0)];
      }
}
static void neumann_z(orc_state *s) { /* :587-590 */
  const int nz = s->nz;
  double *c = s->concen;
  for (int n = 1; n <= s->ns; n++)
    for (int j = -1; j <= s->ny + 2; j++)
      for (int i = -1; i <= s->nx + 2; i++) {
        c[c5(s, i, j, -1, n, 0)] = c[c5(s, i, j, 1, n, 0)];
        c[c5(s, i, j, 0, n, 0)] = c[c5(s, i, j, 1, n, 0)];
        c[c5(s, i, j, nz + 1, n, 0)] = c[c5(s, i, j, nz, n, 0)];
        c[c5(s, i, j, nz + 2, n, 0)] = c[c5(s, i, j, nz, n, 0)];
      }
}

typedef struct { double *q, *kap, *sig, *kk, *upd, *mem; } drow;
static void drow_alloc(drow *r, int len) {
  size_t m = (size_t)len + 4;
  r->mem = (double *)calloc(5 * m, sizeof(double));
  r->q = r->mem + 1; r->kap = r->q + m; r->sig = r->kap + m; r->kk = r->sig + m; r->upd = r->kk + m;
}

void orc_diff_x(orc_state *s) { /* :266-388 */
  const int rmin = s->imin, rmax = s->imax;
  zero_level(s, 1);
  neumann_x(s);
  drow r; drow_alloc(&r, s->nx);
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
    for (int k = s->kmin; k <= s->kmax; k++)
      for (int j = s->jmin; j <= s->jmax; j++) {
        for (int i = rmin - 1; i <= rmax + 1; i++) {
          r.q[i] = s->concen[c5(s, i, j, k, n, 0)];
          r.kap[i] = s->kappa[i3(s, i, j, k)];
          r.kk[i] = s->kx[k3(s, i, j, k)];
          r.sig[i] = s->sig_nx[i3(s, i, j, k)];
        }
        diff_row(s->dt, rmin, rmax, r.q, r.kap, r.sig, r.kk, r.upd);
        for (int i = rmin; i <= rmax; i++)
          s->concen[c5(s, i, j, k, n, 1)] = s->concen[c5(s, i, j, k, n, 0)] + r.upd[i];
      }
  }
  free(r.mem);
  copy_back(s);
}

void orc_diff_y(orc_state *s) { /* :406-518 */
  const int rmin = s->jmin, rmax = s->jmax;
  zero_level(s, 1);
  neumann_y(s);
  drow r; drow_alloc(&r, s->ny);
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
    for (int k = s->kmin; k <= s->kmax; k++)
      for (int i = s->imin; i <= s->imax; i++) {
        for (int j = rmin - 1; j <= rmax + 1; j++) {
          r.q[j] = s->concen[c5(s, i, j, k, n, 0)];
          r.kap[j] = s->kappa[i3(s, i, j, k)];
          r.kk[j] = s->ky[k3(s, i, j, k)];
          r.sig[j] = s->sig_ny[i3(s, i, j, k)];
        }
        diff_row(s->dt, rmin, rmax, r.q, r.kap, r.sig, r.kk, r.upd);
        for (int j = rmin; j <= rmax; j++)
          s->concen[c5(s, i, j, k, n, 1)] = s->concen[c5(s, i, j, k, n, 0)] + r.upd[j];
      }
  }
  free(r.mem);
  copy_back(s);
}

void orc_diff_z(orc_state *s) { /* :536-650 */
  const int rmin = s->kmin, rmax = s->kmax;
  zero_level(s, 1);
  neumann_z(s);
  drow r; drow_alloc(&r, s->nz);
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
    for (int j = s->jmin; j <= s->jmax; j++)
      for (int i = s->imin; i <= s->imax; i++) {
        for (int k = rmin - 1; k <= rmax + 1; k++) {
          r.q[k] = s->concen[c5(s, i, j, k, n, 0)];
          r.kap[k] = s->kappa[i3(s, i, j, k)];
          r.kk[k] = s->kz[k3(s, i, j, k)];
          r.sig[k] = s->sig_nz[i3(s, i, j, k)];
        }
        diff_row(s->dt, rmin, rmax, r.q, r.kap, r.sig, r.kk, r.upd);
        for (int k = rmin; k <= rmax; k++)
          s->concen[c5(s, i, j, k, n, 1)] = s->concen[c5(s, i, j, k, n, 0)] + r.upd[k];
      }
  }
  free(r.mem);
  copy_back(s);
}

/* ======================================================================== */
/* LAPACK dgtsv restatement (NRHS = 1).                                      */
/* Published algorithm of reference LAPACK's DGTSV: for i = 1..n-1 eliminate */
/* the subdiagonal with partial pivoting between rows i and i+1 (the         */
/* interchange stores the second superdiagonal in DL), then back-substitute. */
/* Arrays are 0-based here: dl[0..n-2], d[0..n-1], du[0..n-2], b[0..n-1].     */
/* ======================================================================== */
int orc_dgtsv(int n, double *dl, double *d, double *du, double *b) {
  if (n < 0) return -1;
  if (n == 0) return 0;
  for (int i = 0; i < n - 2; i++) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        d[i + 1] = d[i + 1] - fact * du[i];
        b[i + 1] = b[i + 1] - fact * b[i];
      } else {
        return i + 1;
      }
      dl[i] = 0.0;
    } else {
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      double temp = d[i + 1];
      d[i + 1] = du[i] - fact * temp;
      dl[i] = du[i + 1];
      du[i + 1] = -fact * dl[i];
      du[i] = temp;
      temp = b[i];
      b[i] = b[i + 1];
      b[i + 1] = temp - fact * b[i + 1];
    }
  }
  if (n > 1) {
    int i = n - 2;
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        d[i + 1] = d[i + 1] - fact * du[i];
        b[i + 1] = b[i + 1] - fact * b[i];
      } else {
        return i + 1;
      }
    } else {
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      double temp = d[i + 1];
      d[i + 1] = du[i] - fact * temp;
      du[i] = temp;
      temp = b[i];
      b[i] = b[i + 1];
      b[i + 1] = temp - fact * b[i + 1];
    }
  }
  if (d[n - 1] == 0.0) return n;
  b[n - 1] = b[n - 1] / d[n - 1];
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
  for (int i = n - 3; i >= 0; i--)
    b[i] = (b[i] - du[i] * b[i + 1] - dl[i] * b[i + 2]) / d[i];
  return 0;
}

/* ======================================================================== */
/* Crank-Nicolson diffusion, src/Diffusion.F90:671-1428                      */
/* ======================================================================== */
typedef struct { double *q, *kap, *sig, *kk, *DL, *D, *DU, *B, *mem; } cnrow;
static void cnrow_alloc(cnrow *r, int len) {
  size_t m = (size_t)len + 4;
  r->mem = (double *)calloc(8 * m, sizeof(double));
  r->q = r->mem + 1; r->kap = r->q + m; r->sig = r->kap + m; r->kk = r->sig + m;
  r->DL = r->kk + m; r->D = r->DL + m; r->DU = r->D + m; r->B = r->DU + m;
}

/* Builds and solves one line (q,kap,kk indexed rmin-1..rmax+1; sig rmin..rmax+1);
 * the solution is left in r->B[0..ncells-1].  :791-890 */
static void cn_line(double dt, double imp, int rmin, int rmax, cnrow *r) {
  const int ncells = rmax - rmin + 1;
  const double *q = r->q, *kap = r->kap, *sig = r->sig, *kk = r->kk;
  double *DL = r->DL, *D = r->D, *DU = r->DU, *B = r->B;
  for (int l = 1; l <= ncells; l++) {
    const int c = rmin - 1 + l;   /* cell index */
    const int IL = c, IR = c + 1; /* interface indices */
    double vavgL = 0.5 * (kap[IL - 1] + kap[IL]);
    double kavgL = 0.5 * (kk[IL - 1] + kk[IL]);
    double dsL = sig[IL] / vavgL;
    double kdsL = kavgL * dsL;
    double vavgR = 0.5 * (kap[IR - 1] + kap[IR]);
    double kavgR = 0.5 * (kk[IR - 1] + kk[IR]);
    double dsR = sig[IR] / vavgR;
    double kdsR = kavgR * dsR;
    double LeftFac = dt * kdsL * sig[IL] / kap[c];
    double RightFac = dt * kdsR * sig[IR] / kap[c];
    double CenterFac = LeftFac + RightFac;
    if (l == 1) {
      D[0] = 1.0 + imp * CenterFac - imp * LeftFac;
      DU[0] = -(imp * RightFac);
      double bcl = q[rmin];
      B[0] = (1.0 - imp) * LeftFac * bcl + (1.0 - (1.0 - imp) * CenterFac) * q[c] +
             (1.0 - imp) * RightFac * q[c + 1];
    } else if (l < ncells) {
      DL[l - 2] = -(imp * LeftFac);
      D[l - 1] = 1.0 + imp * CenterFac;
      DU[l - 1] = -(imp * RightFac);
      B[l - 1] = (1.0 - imp) * LeftFac * q[c - 1] + (1.0 - (1.0 - imp) * CenterFac) * q[c] +
                 (1.0 - imp) * RightFac * q[c + 1];
    } else {
      DL[l - 2] = -(imp * LeftFac);
      D[l - 1] = 1.0 + imp * CenterFac - imp * RightFac;
      double bcr = q[rmin - 1 + ncells];
      B[l - 1] = (1.0 - imp) * LeftFac * q[c - 1] + (1.0 - (1.0 - imp) * CenterFac) * q[c] +
                 (1.0 - imp) * RightFac * bcr;
    }
  }
  (void)orc_dgtsv(ncells, DL, D, DU, B); /* INFO is ignored, :881-890 */
}

void orc_diffcn_x(orc_state *s) { /* :671-911 */
  const int rmin = s->imin, rmax = s->imax, ncells = rmax - rmin + 1;
  zero_level(s, 1);
  neumann_x(s);
  if (ncells <= 1) return;
  cnrow r; cnrow_alloc(&r, s->nx);
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
    for (int k = s->kmin; k <= s->kmax; k++)
      for (int j = s->jmin; j <= s->jmax; j++) {
        for (int i = rmin - 1; i <= rmax + 1; i++) {
          r.q[i] = s->concen[c5(s, i, j, k, n, 0)];
          r.kap[i] = s->kappa[i3(s, i, j, k)];
          r.kk[i] = s->kx[k3(s, i, j, k)];
          r.sig[i] = s->sig_nx[i3(s, i, j, k)];
        }
        cn_line(s->dt, s->imp_fac, rmin, rmax, &r);
        for (int l = 0; l < ncells; l++) s->concen[c5(s, rmin + l, j, k, n, 1)] = r.B[l];
      }
  }
  free(r.mem);
  copy_back(s);
}

void orc_diffcn_y(orc_state *s) { /* :932-1167 */
  const int rmin = s->jmin, rmax = s->jmax, ncells = rmax - rmin + 1;
  zero_level(s, 1);
  neumann_y(s);
  if (ncells <= 1) return;
  cnrow r; cnrow_alloc(&r, s->ny);
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
    for (int k = s->kmin; k <= s->kmax; k++)
      for (int i = s->imin; i <= s->imax; i++) {
        for (int j = rmin - 1; j <= rmax + 1; j++) {
          r.q[j] = s->concen[c5(s, i, j, k, n, 0)];
          r.kap[j] = s->kappa[i3(s, i, j, k)];
          r.kk[j] = s->ky[k3(s, i, j, k)];
          r.sig[j] = s->sig_ny[i3(s, i, j, k)];
        }
        cn_line(s->dt, s->imp_fac, rmin, rmax, &r);
        for (int l = 0; l < ncells; l++) s->concen[c5(s, i, rmin + l, k, n, 1)] = r.B[l];
      }
  }
  free(r.mem);
  copy_back(s);
}

void orc_diffcn_z(orc_state *s) { /* :1188-1428 */
  const int rmin = s->kmin, rmax = s->kmax, ncells = rmax - rmin + 1;
  zero_level(s, 1);
  neumann_z(s);
  if (ncells <= 1) return;
  cnrow r; cnrow_alloc(&r, s->nz);
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) continue;
    for (int j = s->jmin; j <= s->jmax; j++)
      for (int i = s->imin; i <= s->imax; i++) {
        for (int k = rmin - 1; k <= rmax + 1; k++) {
          r.q[k] = s->concen[c5(s, i, j, k, n, 0)];
          r.kap[k] = s->kappa[i3(s, i, j, k)];
          r.kk[k] = s->kz[k3(s, i, j, k)];
          r.sig[k] = s->sig_nz[i3(s, i, j, k)];
        }
        cn_line(s->dt, s->imp_fac, rmin, rmax, &r);
        for (int l = 0; l < ncells; l++) s->concen[c5(s, i, j, rmin + l, n, 1)] = r.B[l];
      }
  }
  free(r.mem);
  copy_back(s);
}

/* DiffuseHorz(i), src/Diffusion.F90:151-216 */
void orc_diffuse_horz(orc_state *s, int itime) {
  if (s->fast_subgrid) {
    s->imin = s->imin - 1 > 1 ? s->imin - 1 : 1;
    s->imax = s->imax + 1 < s->nx ? s->imax + 1 : s->nx;
    s->jmin = s->jmin - 1 > 1 ? s->jmin - 1 : 1;
    s->jmax = s->jmax + 1 < s->ny ? s->jmax + 1 : s->ny;
    s->kmin = s->kmin - 1 > 1 ? s->kmin - 1 : 1;
    s->kmax = s->kmax + 1 < s->nz ? s->kmax + 1 : s->nz;
  } else {
    s->imin = 1; s->imax = s->nx; s->jmin = 1; s->jmax = s->ny; s->kmin = 1; s->kmax = s->nz;
  }
  if (s->use_cn) {
    if (itime % 2 == 0) { orc_diffcn_x(s); orc_diffcn_y(s); }
    else { orc_diffcn_y(s); orc_diffcn_x(s); }
  } else {
    if (itime % 2 == 0) { orc_diff_x(s); orc_diff_y(s); }
    else { orc_diff_y(s); orc_diff_x(s); }
  }
}

/* DiffuseVert, src/Diffusion.F90:232-247 */
void orc_diffuse_vert(orc_state *s) {
  if (s->use_cn) orc_diffcn_z(s); else orc_diff_z(s);
}

/* ======================================================================== */
/* Adjust_DT(.false.), src/Adjust_dt.f90:19-339                              */
/* ======================================================================== */
void orc_adjust_dt(orc_state *s, double time, double next_write_time, double simtime,
                   double *dt_out) {
  double v[3];
  orc_cfl_maxima(s, v);
  orc_dt_from_maxima(s, v, s->n_gs_aloft, time, next_write_time, simtime, dt_out);
}

/* src/Adjust_dt.f90:136-173: the three maxima (projected grids: max|vx|, max|vy|
 * before the division by dx, dy). */
void orc_cfl_maxima(orc_state *s, double out3[3]) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, ns = s->ns;
  double vxmax_dx = 0.0, vymax_dy = 0.0, vzmax_dz = 0.0;
  if (!s->latlon) {                                                           /* :137-146 */
    double vxmax = 0.0, vymax = 0.0;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          double a = fabs(s->vx[i3(s, i, j, k)]);
          double b = fabs(s->vy[i3(s, i, j, k)]);
          if (a > vxmax) vxmax = a;
          if (b > vymax) vymax = b;
        }
    vxmax_dx = vxmax;   /* divided by dx, dy in orc_dt_from_maxima */
    vymax_dy = vymax;
  }
  for (int i = 1; i <= nx; i++)                                               /* :147-173 */
    for (int j = 1; j <= ny; j++)
      for (int k = 1; k <= nz; k++) {
        if (s->latlon) {
          double minsig = fmn(s->sig_nx[i3(s, i, j, k)], s->sig_nx[i3(s, i + 1, j, k)]);
          double tmp1 = fabs(s->vx[i3(s, i, j, k)]) * minsig / s->kappa[i3(s, i, j, k)];
          if (tmp1 > vxmax_dx) vxmax_dx = tmp1;
          minsig = fmn(s->sig_ny[i3(s, i, j, k)], s->sig_ny[i3(s, i, j + 1, k)]);
          double tmp2 = fabs(s->vy[i3(s, i, j, k)]) * minsig / s->kappa[i3(s, i, j, k)];
          if (tmp2 > vymax_dy) vymax_dy = tmp2;
        }
        double vfmax = 0.0;
        for (int n = 1; n <= ns; n++) {
          double a = fabs(s->vf[v4(s, i, j, k, n)]);
          if (n == 1 || a > vfmax) vfmax = a;
        }
        double tmp3 = (fabs(s->vz[i3(s, i, j, k)]) + vfmax) / s->dz_vec[k + 1];
        if (tmp3 > vzmax_dz) vzmax_dz = tmp3;
      }
  out3[0] = vxmax_dx; out3[1] = vymax_dy; out3[2] = vzmax_dz;
}

/* Adjust_DT(mesostep=.true.), the FAST_DT branch of src/Adjust_dt.f90:96-135:
 * the maxima over the FP32 met step (vx_sp, vy_sp, vz_sp: (nx,ny,nz), m/s)
 * and vf_meso_next_step_sp (per_grain: ns values, the real(Tephra_v_s,sp)
 * that Read_NextMesoStep puts in every cell; else (nx,ny,nz,ns)).  Projected
 * grids: real(maxval(abs(vx_sp)))*MPS_2_KMPHR, divided by dx in
 * orc_dt_from_maxima as the non-meso branch is. */
void orc_cfl_maxima_meso(orc_state *s, const float *vx_sp, const float *vy_sp, const float *vz_sp,
                         const float *vf_sp, int per_grain, double out3[3]) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, ns = s->ns;
  const size_t n3 = (size_t)nx * ny * nz;
  double vxmax_dx = 0.0, vymax_dy = 0.0, vzmax_dz = 0.0;
  if (!s->latlon) {                                                           /* :99-108 */
    float ax = 0.0f, ay = 0.0f;  /* maxval over (1:nx,1:ny,1:nz), column-major */
    for (size_t m = 0; m < n3; m++) {
      if (m == 0 || fabsf(vx_sp[m]) > ax) ax = fabsf(vx_sp[m]);
      if (m == 0 || fabsf(vy_sp[m]) > ay) ay = fabsf(vy_sp[m]);
    }
    double vxmax = (double)ax;
    vxmax = vxmax * 3.6;
    double vymax = (double)ay;
    vymax = vymax * 3.6;
    vxmax_dx = vxmax;   /* divided by dx, dy in orc_dt_from_maxima */
    vymax_dy = vymax;
  }
  for (int i = 1; i <= nx; i++)                                               /* :112-134 */
    for (int j = 1; j <= ny; j++)
      for (int k = 1; k <= nz; k++) {
        const size_t m = (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (k - 1));
        if (s->latlon) {
          double minsig = fmn(s->sig_nx[i3(s, i, j, k)], s->sig_nx[i3(s, i + 1, j, k)]);
          double tmp1 = (double)fabsf(vx_sp[m]) * 3.6 * minsig / s->kappa[i3(s, i, j, k)];
          if (tmp1 > vxmax_dx) vxmax_dx = tmp1;
          minsig = fmn(s->sig_ny[i3(s, i, j, k)], s->sig_ny[i3(s, i, j + 1, k)]);
          double tmp2 = (double)fabsf(vy_sp[m]) * 3.6 * minsig / s->kappa[i3(s, i, j, k)];
          if (tmp2 > vymax_dy) vymax_dy = tmp2;
        }
        float vfmax = 0.0f;
        for (int n = 1; n <= ns; n++) {
          const float a = fabsf(per_grain ? vf_sp[n - 1] : vf_sp[m + n3 * (size_t)(n - 1)]);
          if (n == 1 || a > vfmax) vfmax = a;
        }
        const float sum = fabsf(vz_sp[m]) + vfmax;   /* FP32 sum before widening */
        double tmp3 = (double)sum * 3.6 / s->dz_vec[k + 1];
        if (tmp3 > vzmax_dz) vzmax_dz = tmp3;
      }
  out3[0] = vxmax_dx; out3[1] = vymax_dy; out3[2] = vzmax_dz;
}

/* The FAST_DT step dt, src/MesoInterpolater.f90:250-258. */
double orc_fast_dt(orc_state *s, double dt_meso_last, double dt_meso_next, double interval_frac,
                   double time, double next_write_time, double simtime) {
  double dt = dt_meso_last + (dt_meso_next - dt_meso_last) * interval_frac;
  if (((next_write_time - time) > s->eps_small) && (next_write_time - time < dt))
    dt = next_write_time - time;
  if (time + dt > simtime) dt = simtime - time;
  s->dt = dt;
  return dt;
}

/* src/Adjust_dt.f90:137-146 (division by dx, dy) and :176-332. */
void orc_dt_from_maxima(orc_state *s, const double v3[3], int n_gs_aloft, double time,
                        double next_write_time, double simtime, double *dt_out) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  double vxmax_dx = v3[0], vymax_dy = v3[1], vzmax_dz = v3[2];
  if (!s->latlon) {
    vxmax_dx = vxmax_dx / s->dx;
    vymax_dy = vymax_dy / s->dy;
  }
  if (n_gs_aloft == 0) vzmax_dz = 0.0;                                        /* :176 */
  double time_advect = 1.0 / fmx(fmx(vxmax_dx, vymax_dy), vzmax_dz);          /* :179 */
  if (s->use_diffusion) {                                                      /* :184-287 */
    if (!s->have_dt_diffus) {
      double td = s->dt_max;
      for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++)
          for (int k = 1; k <= nz; k++) {
            double kap = s->kappa[i3(s, i, j, k)];
            double minsig = fmn(s->sig_nx[i3(s, i, j, k)], s->sig_nx[i3(s, i + 1, j, k)]);
            double r1 = kap / minsig;
            double tmp1 = (r1 * r1) / s->kx[k3(s, i, j, k)];
            minsig = fmn(s->sig_ny[i3(s, i, j, k)], s->sig_ny[i3(s, i, j + 1, k)]);
            double r2 = kap / minsig;
            double tmp2 = (r2 * r2) / s->ky[k3(s, i, j, k)];
            minsig = fmn(s->sig_nz[i3(s, i, j, k)], s->sig_nz[i3(s, i, j, k + 1)]);
            double r3 = kap / minsig;
            double tmp3b = (r3 * r3) / s->kz[k3(s, i, j, k)];
            double tmp4 = tmp1 + tmp2 + tmp3b;
            if (td > tmp4) td = tmp4;
          }
      td = s->use_cn ? td * s->imp_dt_fac : td * 0.5;
      s->time_diffuse = td;
      s->have_dt_diffus = 1;
    }
  } else {
    s->time_diffuse = s->dt_max;
  }
  double dt_tmp = fmn(time_advect, s->time_diffuse);                          /* :290-319 */
  double dt;
  if (dt_tmp < s->dt_min) dt = s->dt_min;
  else if (dt_tmp > s->dt_max) dt = s->dt_max;
  else dt = fmn(1.0, s->cfl) * dt_tmp;
  long long fac = (long long)(dt / s->dt_min);                                /* :321-323 */
  dt = s->dt_min * (double)fac;
  if ((next_write_time - time) > s->eps_small && (next_write_time - time) < dt)
    dt = next_write_time - time;                                              /* :325-327 */
  if (time + dt > simtime) dt = simtime - time;                               /* :329-332 */
  s->dt = dt;
  if (dt_out) *dt_out = dt;
}

/* ======================================================================== */
/* TimeStepTotals sums, src/TimeStepTotals.f90:57-66;                        */
/* Calc_AshVol_Aloft/Deposit/Outflow, src/Output_Vars.f90:1255-1459.          */
/* gfortran's SUM over an array section accumulates in array-element order.  */
/* ======================================================================== */
void orc_timestep_totals(orc_state *s, double out[4]) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, ns = s->ns;
  const double rho = s->magma_density, km3 = 1.0e9;
  double aloft = 0.0, depv = 0.0, outv = 0.0;
  for (int n = 1; n <= ns; n++) {
    double m = 0.0;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
          m = m + s->concen[c5(s, i, j, k, n, 0)] * s->kappa[i3(s, i, j, k)];
    s->mass_aloft[n - 1] = m;
  }
  for (int n = 1; n <= ns; n++) aloft = aloft + s->mass_aloft[n - 1] / rho / km3;
  for (int n = 1; n <= ns; n++) {
    double m = 0.0;
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++)
        m = m + s->deposit[dep(s, i, j, n)] * s->kappa[i3(s, i, j, 0)];
    depv = depv + m / rho / km3;
  }
  for (int n = 1; n <= ns; n++) {
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, s5 = 0.0;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) s1 = s1 + s->outflow_yz1[oyz(s, j, k, n)] * s->kappa[i3(s, 0, j, k)];
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) s2 = s2 + s->outflow_yz2[oyz(s, j, k, n)] * s->kappa[i3(s, nx + 1, j, k)];
    for (int k = 1; k <= nz; k++)
      for (int i = 1; i <= nx; i++) s3 = s3 + s->outflow_xz1[oxz(s, i, k, n)] * s->kappa[i3(s, i, 0, k)];
    for (int k = 1; k <= nz; k++)
      for (int i = 1; i <= nx; i++) s4 = s4 + s->outflow_xz2[oxz(s, i, k, n)] * s->kappa[i3(s, i, ny + 1, k)];
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) s5 = s5 + s->outflow_xy2[oxy(s, i, j, n)] * s->kappa[i3(s, i, j, nz + 1)];
    outv = outv + (s1 + s2 + s3 + s4 + s5) / rho / km3;
  }
  out[0] = aloft; out[1] = depv; out[2] = outv; out[3] = aloft + depv + outv;
}

/* ======================================================================== */
/* Step pieces from the main loop, src/Ash3d.F90:376-431                     */
/* ======================================================================== */
void orc_step_prologue(orc_state *s) {
  size_t lev = (size_t)NXG(s) * NYG(s) * NZG(s) * s->ns;
  memcpy(s->concen, s->concen + lev, lev * sizeof(double));
  memset(s->concen + lev, 0, lev * sizeof(double));
}

void orc_add_source(orc_state *s, int ivent, int jvent, const double *flux, double dt) {
  for (int n = 1; n <= s->ns; n++)
    for (int k = 1; k <= s->nz + 1; k++)
      s->concen[c5(s, ivent, jvent, k, n, 0)] =
          s->concen[c5(s, ivent, jvent, k, n, 0)] + dt * flux[(size_t)(k - 1) + (size_t)(s->nz + 1) * (n - 1)];
}

void orc_vprofiles(orc_state *s, int npts, const int32_t *i_pts, const int32_t *j_pts, double thresh,
                   double *out, int32_t *written) {
  for (int p = 0; p < npts; p++) {
    const int i = i_pts[p], j = j_pts[p];
    double total = 0.0;                       /* sum(concen(i,j,1:nz,1:ns,ts1)), k fastest */
    for (int n = 1; n <= s->ns; n++)
      for (int k = 1; k <= s->nz; k++) total = total + s->concen[c5(s, i, j, k, n, 1)];
    written[p] = !(total < thresh);
    if (!written[p]) continue;                /* :1350 */
    for (int k = 1; k <= s->nz; k++) {
      double sum = 0.0;
      for (int n = 1; n <= s->ns; n++) sum = sum + s->concen[c5(s, i, j, k, n, 1)];
      out[(size_t)(k - 1) + (size_t)s->nz * p] = sum * 1.0e6 / 1.0e9;
    }
  }
}

void orc_add_umbrella_winds(orc_state *s, int ibase, int itop, int i0, int i1, int j0, int j1,
                            const double *uvx, const double *uvy) {
  const int ni = i1 - i0 + 1;
  for (int k = ibase; k <= itop; k++)
    for (int j = j0; j <= j1; j++)
      for (int i = i0; i <= i1; i++) {
        const size_t m = (size_t)(i - i0) + (size_t)ni * (j - j0);
        s->vx[i3(s, i, j, k)] = s->vx[i3(s, i, j, k)] + uvx[m];
        s->vy[i3(s, i, j, k)] = s->vy[i3(s, i, j, k)] + uvy[m];
      }
}

void orc_add_source_umbrella(orc_state *s, int ivent, int jvent, int ibase, int itop,
                             const double *stencil, const double *flux, double dt) {
  const int nz = s->nz;
  for (int k = ibase; k <= itop; k++)                              /* :448-453 */
    for (int n = 1; n <= s->ns; n++) {
      double avg = 0.0;                                            /* AvgCon_Umbrella */
      for (int i = 1; i <= 3; i++)
        for (int j = 1; j <= 3; j++)
          avg = avg + s->concen[c5(s, ivent - 2 + i, jvent - 2 + j, k, n, 0)] *
                          stencil[(i - 1) + 3 * (j - 1) + 9 * (k - 1)];
      for (int i = 1; i <= 3; i++)
        for (int j = 1; j <= 3; j++) s->concen[c5(s, ivent - 2 + i, jvent - 2 + j, k, n, 0)] = avg;
    }
  for (int n = 1; n <= s->ns; n++)                                 /* :455-458 */
    for (int k = 1; k <= nz + 1; k++)
      for (int j = 1; j <= 3; j++)
        for (int i = 1; i <= 3; i++) {
          const size_t a = c5(s, ivent - 2 + i, jvent - 2 + j, k, n, 0);
          s->concen[a] = s->concen[a] +
                         dt * flux[(i - 1) + 3 * (j - 1) + 9 * ((size_t)(k - 1) + (size_t)(nz + 1) * (n - 1))];
        }
}

void orc_interp_winds(orc_state *s, const float *vx_last, const float *vx_next,
                      const float *vy_last, const float *vy_next,
                      const float *vz_last, const float *vz_next, double frac) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t m = (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (k - 1));
        float dx_ = vx_next[m] - vx_last[m];
        float dy_ = vy_next[m] - vy_last[m];
        float dz_ = vz_next[m] - vz_last[m];
        s->vx[i3(s, i, j, k)] = ((double)vx_last[m] + (double)dx_ * frac) * 3.6;
        s->vy[i3(s, i, j, k)] = ((double)vy_last[m] + (double)dy_ * frac) * 3.6;
        s->vz[i3(s, i, j, k)] = ((double)vz_last[m] + (double)dz_ * frac) * 3.6;
      }
}

void orc_prune_gs(orc_state *s, double airborne_thresh) {
  int naloft = 0;
  for (int n = 0; n < s->ns; n++) {
    if (s->is_aloft[n] && s->mass_aloft[n] < airborne_thresh) s->is_aloft[n] = 0;
    else naloft++;
  }
  s->n_gs_aloft = naloft;
}

/* ======================================================================== */
/* Discrete adjoint of the transport step (no counterpart in the reference). */
/*                                                                          */
/* Each sweep is piecewise linear in the concentration: with the limiter    */
/* branches fixed by the state the sweep was applied to, the limited slope   */
/* ldq is a*dq + b*dqu (a, b constants of the branch), so the sweep is a     */
/* linear map J(c) and these routines apply its transpose J(c)^T to lam (the */
/* adjoint of the sweep's output), in place.  They are written as the        */
/* reverse of the forward statements (hand reverse mode): the forward state  */
/* must be in concen(:,:,:,:,ts0) (the sweep's input), the box must be the   */
/* full grid (the subgrid box depends on the state), and lam has the shape   */
/* of one concentration level (ghosts ignored, left zero).  Ghost values     */
/* written by Set_BC(1) are zero (their adjoint is dropped) except x-        */
/* periodic wraps, whose adjoint goes back to the wrapped cells; Neumann     */
/* ghosts of the diffusion sweeps go back to the edge cells.  Grains that    */
/* are not aloft are zeroed by every sweep, so their adjoint is zero.        */
/* ======================================================================== */

/* Coefficients of the frozen limiter branch: d(ldq) = a*d(dq) + b*d(dqu).    */
/* Ties between branches follow the forward fmx/fmn selection.               */
void orc_lim_coef(int lim, double dq, double dqu, double eps, double *a, double *b) {
  if (lim == ORC_LIM_LAXWEN) { *a = 1.0; *b = 0.0; return; }
  if (lim == ORC_LIM_BW) { *a = 0.0; *b = 1.0; return; }
  const int clamp = fabs(dqu) > 3.0 * fabs(dq) || fabs(dq) < eps;
  const double th = clamp ? copysign(3.0, dqu * dq) : dqu / dq;
  double phi, dphi;
  switch (lim) {
    case ORC_LIM_FROMM:
      phi = 0.5 * (1.0 + th); dphi = 0.5; break;
    case ORC_LIM_MINMOD: {
      double m = fmn(1.0, th), dm = (1.0 < th) ? 0.0 : 1.0;
      phi = fmx(0.0, m); dphi = (0.0 > m) ? 0.0 : dm; break;
    }
    case ORC_LIM_MC: {
      double m1 = fmn((1.0 + th) / 2.0, 2.0), dm1 = ((1.0 + th) / 2.0 < 2.0) ? 0.5 : 0.0;
      double m2 = fmn(m1, 2.0 * th), dm2 = (m1 < 2.0 * th) ? dm1 : 2.0;
      phi = fmx(0.0, m2); dphi = (0.0 > m2) ? 0.0 : dm2; break;
    }
    case ORC_LIM_SUPERBEE:
    default: {
      double m1 = fmn(1.0, 2.0 * th), dm1 = (1.0 < 2.0 * th) ? 0.0 : 2.0;
      double a1 = fmx(0.0, m1), da1 = (0.0 > m1) ? 0.0 : dm1;
      double m2 = fmn(2.0, th), dm2 = (2.0 < th) ? 0.0 : 1.0;
      phi = fmx(a1, m2); dphi = (a1 > m2) ? da1 : dm2; break;
    }
  }
  if (clamp) dphi = 0.0;
  *a = phi - th * dphi;
  *b = dphi;
}

/* Reverse of dcu_row: lu[i] (i = rmin-1..rmax+1) is the adjoint of upd[i];
 * adds the adjoint of q[i] (i = rmin-2..rmax+2) into lq.  r->q, vel, sig,
 * kap hold the forward row. */
static void adj_dcu_row(const orc_state *s, row_scratch *r, int len, int rmin, int rmax,
                        const double *lu, double *lq) {
  const double dt = s->dt, eps = s->eps_thresh;
  double *q = r->q, *vel = r->vel, *sig = r->sig, *kap = r->kap;
  double *dtv = r->dtv, *usig = r->usig, *dq = r->dq;
  double *lfsl = r->fsl, *lfsr = r->fsr, *lfss = r->fss, *ldq = r->upd;  /* reused as adjoints */
  for (int i = rmin - 2; i <= rmax + 2; i++) dtv[i] = dt / kap[i];
  for (int i = -1; i <= len + 2; i++) usig[i] = 0.0;
  for (int I = rmin - 1; I <= rmax + 1; I++) usig[I] = 0.5 * (vel[I - 1] + vel[I]) * sig[I];
  for (int I = rmin - 1; I <= rmax + 2; I++) dq[I] = q[I] - q[I - 1];
  for (int I = rmin - 1; I <= rmax + 2; I++) { lfsl[I] = 0.0; lfsr[I] = 0.0; lfss[I] = 0.0; ldq[I] = 0.0; }
  /* upd[i] = -(dtv[i]*(fsl[i+1] + fsr[i] + fss[i+1] - fss[i])) */
  for (int i = rmin - 1; i <= rmax + 1; i++) {
    const double t = -(dtv[i] * lu[i]);
    lfsl[i + 1] += t; lfsr[i] += t; lfss[i + 1] += t; lfss[i] -= t;
  }
  /* fsr[I] = max(0,u)dq[I] + q[I]divu_m; fsl[I] = min(0,u)dq[I] + q[I-1]divu_p */
  for (int I = rmin - 1; I <= rmax + 1; I++) {
    const double divu_p = fmx(0.0, usig[I]) - fmx(0.0, usig[I - 1]);
    const double divu_m = fmn(0.0, usig[I + 1]) - fmn(0.0, usig[I]);
    ldq[I] += fmx(0.0, usig[I]) * lfsr[I] + fmn(0.0, usig[I]) * lfsl[I];
    lq[I] += divu_m * lfsr[I];
    lq[I - 1] += divu_p * lfsl[I];
  }
  /* fss[I] = w*(a*dq[I] + b*dqu) */
  if (s->limiter != ORC_LIM_NONE) {
    for (int I = rmin; I <= rmax + 1; I++) {
      if (!s->nocycle && fabs(dq[I]) <= eps) continue;
      const int up = usig[I] > 0.0 ? I - 1 : I + 1;
      double a, b;
      orc_lim_coef(s->limiter, dq[I], dq[up], eps, &a, &b);
      const double aus = fabs(usig[I]);
      const double w = 0.5 * aus * (1.0 - dtv[I] * aus);
      ldq[I] += w * a * lfss[I];
      ldq[up] += w * b * lfss[I];
    }
  }
  /* dq[I] = q[I] - q[I-1] */
  for (int I = rmin - 1; I <= rmax + 2; I++) { lq[I] += ldq[I]; lq[I - 1] -= ldq[I]; }
}

static size_t lv(const orc_state *s, int i, int j, int k, int n) { return c5(s, i, j, k, n, 0); }

void orc_adj_advect_x(orc_state *s, double *lam) {
  orc_set_bc(s, 1);
  const int rmin = s->imin, rmax = s->imax, nx = s->nx;
  const int nth = orc_get_threads();
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) {
      for (int k = 1; k <= s->nz; k++) for (int j = 1; j <= s->ny; j++) for (int i = 1; i <= nx; i++)
        lam[lv(s, i, j, k, n)] = 0.0;
      continue;
    }
#pragma omp parallel num_threads(nth)
    {
      row_scratch r; row_alloc(&r, nx);
      double *lu = (double *)calloc(nx + 6, sizeof(double)) + 2;
      double *lq = (double *)calloc(nx + 6, sizeof(double)) + 2;
#pragma omp for collapse(2) schedule(static)
      for (int k = s->kmin; k <= s->kmax; k++)
        for (int j = s->jmin; j <= s->jmax; j++) {
          for (int i = rmin - 2; i <= rmax + 2; i++) {
            r.q[i] = s->concen[c5(s, i, j, k, n, 0)];
            r.vel[i] = s->vx[i3(s, i, j, k)];
            r.sig[i] = s->sig_nx[i3(s, i, j, k)];
            r.kap[i] = s->kappa[i3(s, i, j, k)];
            lq[i] = 0.0;
          }
          lu[rmin - 1] = 0.0; lu[rmax + 1] = 0.0;  /* outflows are not observed */
          for (int i = rmin; i <= rmax; i++) lu[i] = lam[lv(s, i, j, k, n)];
          adj_dcu_row(s, &r, nx, rmin, rmax, lu, lq);
          for (int i = rmin; i <= rmax; i++) lq[i] += lu[i];  /* out = q + upd */
          if (s->periodic) {  /* Set_BC(1) wraps */
            lq[nx - 1] += lq[-1]; lq[nx] += lq[0]; lq[1] += lq[nx + 1]; lq[2] += lq[nx + 2];
          }
          for (int i = 1; i <= nx; i++) lam[lv(s, i, j, k, n)] = lq[i];
        }
      free(r.mem); free(lu - 2); free(lq - 2);
    }
  }
}

void orc_adj_advect_y(orc_state *s, double *lam) {
  orc_set_bc(s, 1);
  const int rmin = s->jmin, rmax = s->jmax, ny = s->ny;
  const int nth = orc_get_threads();
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) {
      for (int k = 1; k <= s->nz; k++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= s->nx; i++)
        lam[lv(s, i, j, k, n)] = 0.0;
      continue;
    }
#pragma omp parallel num_threads(nth)
    {
      row_scratch r; row_alloc(&r, ny);
      double *lu = (double *)calloc(ny + 6, sizeof(double)) + 2;
      double *lq = (double *)calloc(ny + 6, sizeof(double)) + 2;
#pragma omp for collapse(2) schedule(static)
      for (int k = s->kmin; k <= s->kmax; k++)
        for (int i = s->imin; i <= s->imax; i++) {
          for (int j = rmin - 2; j <= rmax + 2; j++) {
            r.q[j] = s->concen[c5(s, i, j, k, n, 0)];
            r.vel[j] = s->vy[i3(s, i, j, k)];
            r.sig[j] = s->sig_ny[i3(s, i, j, k)];
            r.kap[j] = s->kappa[i3(s, i, j, k)];
            lq[j] = 0.0;
          }
          lu[rmin - 1] = 0.0; lu[rmax + 1] = 0.0;
          for (int j = rmin; j <= rmax; j++) lu[j] = lam[lv(s, i, j, k, n)];
          adj_dcu_row(s, &r, ny, rmin, rmax, lu, lq);
          for (int j = rmin; j <= rmax; j++) lq[j] += lu[j];
          for (int j = 1; j <= ny; j++) lam[lv(s, i, j, k, n)] = lq[j];
        }
      free(r.mem); free(lu - 2); free(lq - 2);
    }
  }
}

/* lam_dep: adjoint of DepositGranularity = outflow_xy1 (nx,ny,ns), which
 * accumulates upd(0) of every z column (src/AdvectionVert_DCU.f90:306-308,321);
 * NULL for none. */
void orc_adj_advect_z(orc_state *s, double *lam, const double *lam_dep) {
  orc_set_bc(s, 1);
  const int rmin = s->kmin, rmax = s->kmax, nz = s->nz;
  const int nth = orc_get_threads();
  for (int n = 1; n <= s->ns; n++) {
    if (!s->is_aloft[n - 1]) {
      for (int k = 1; k <= nz; k++) for (int j = 1; j <= s->ny; j++) for (int i = 1; i <= s->nx; i++)
        lam[lv(s, i, j, k, n)] = 0.0;
      continue;
    }
#pragma omp parallel num_threads(nth)
    {
      row_scratch r; row_alloc(&r, nz);
      double *lu = (double *)calloc(nz + 6, sizeof(double)) + 2;
      double *lq = (double *)calloc(nz + 6, sizeof(double)) + 2;
#pragma omp for collapse(2) schedule(static)
      for (int j = s->jmin; j <= s->jmax; j++)
        for (int i = s->imin; i <= s->imax; i++) {
          for (int k = rmin - 2; k <= rmax + 2; k++) {
            r.q[k] = s->concen[c5(s, i, j, k, n, 0)];
            r.vel[k] = s->vz[i3(s, i, j, k)] + s->vh[i3(s, i, j, k)] + s->vf[v4(s, i, j, k, n)];
            r.sig[k] = s->sig_nz[i3(s, i, j, k)];
            r.kap[k] = s->kappa[i3(s, i, j, k)];
            lq[k] = 0.0;
          }
          lu[rmin - 1] = (lam_dep && rmin == 1) ? lam_dep[dep(s, i, j, n)] : 0.0;
          lu[rmax + 1] = 0.0;
          for (int k = rmin; k <= rmax; k++) lu[k] = lam[lv(s, i, j, k, n)];
          adj_dcu_row(s, &r, nz, rmin, rmax, lu, lq);
          for (int k = rmin; k <= rmax; k++) lq[k] += lu[k];
          for (int k = 1; k <= nz; k++) lam[lv(s, i, j, k, n)] = lq[k];
        }
      free(r.mem); free(lu - 2); free(lq - 2);
    }
  }
}

/* Explicit diffusion: out[l] = q[l] + cR_l (q[l+1]-q[l]) - cL_l (q[l]-q[l-1])
 * with cR_l = dt*kdsR*(sig[l+1]/kap[l]), cL_l = dt*kdsL*(sig[l]/kap[l]) and
 * Neumann ghosts (periodic in x). */
static void adj_diff_row(double dt, int n, int periodic, const double *kap, const double *sig,
                         const double *kk, const double *lo, double *lq) {
  for (int l = 0; l <= n + 1; l++) lq[l] = 0.0;
  for (int l = 1; l <= n; l++) {
    const double dsR = 2.0 * sig[l + 1] / (kap[l] + kap[l + 1]);
    const double kdsR = 0.5 * (kk[l] + kk[l + 1]) * dsR;
    const double dsL = 2.0 * sig[l] / (kap[l - 1] + kap[l]);
    const double kdsL = 0.5 * (kk[l - 1] + kk[l]) * dsL;
    const double cR = dt * kdsR * (sig[l + 1] / kap[l]);
    const double cL = dt * kdsL * (sig[l] / kap[l]);
    lq[l] += lo[l] - cR * lo[l] - cL * lo[l];
    lq[l + 1] += cR * lo[l];
    lq[l - 1] += cL * lo[l];
  }
  if (periodic) { lq[n] += lq[0]; lq[1] += lq[n + 1]; }
  else { lq[1] += lq[0]; lq[n] += lq[n + 1]; }
}

static void adj_diff_dir(orc_state *s, double *lam, int dir) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int n = dir == 0 ? nx : dir == 1 ? ny : nz;
  const int na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
  double *buf = (double *)calloc(6 * (size_t)(n + 4), sizeof(double));
  double *kap = buf + 1, *sig = kap + (n + 4), *kk = sig + (n + 4), *lo = kk + (n + 4), *lq = lo + (n + 4);
  for (int g = 1; g <= s->ns; g++)
    for (int b = 1; b <= nb; b++)
      for (int a = 1; a <= na; a++) {
        for (int l = 0; l <= n + 1; l++) {
          const int i = dir == 0 ? l : a, j = dir == 1 ? l : (dir == 0 ? a : b), k = dir == 2 ? l : b;
          kap[l] = s->kappa[i3(s, i, j, k)];
          sig[l] = (dir == 0 ? s->sig_nx : dir == 1 ? s->sig_ny : s->sig_nz)[i3(s, i, j, k)];
          kk[l] = (dir == 0 ? s->kx : dir == 1 ? s->ky : s->kz)[k3(s, i, j, k)];
          lo[l] = (l >= 1 && l <= n && s->is_aloft[g - 1]) ? lam[lv(s, i, j, k, g)] : 0.0;
        }
        adj_diff_row(s->dt, n, dir == 0 && s->periodic, kap, sig, kk, lo, lq);
        for (int l = 1; l <= n; l++) {
          const int i = dir == 0 ? l : a, j = dir == 1 ? l : (dir == 0 ? a : b), k = dir == 2 ? l : b;
          lam[lv(s, i, j, k, g)] = lq[l];
        }
      }
  free(buf);
}

/* Crank-Nicolson: out = M^-1 N q with M = (DL, D, DU) and N the explicit
 * half (Neumann rows).  Adjoint: solve M^T y = lam (dgtsv on the transposed
 * diagonals), then lam_q = N^T y. */
static void adj_cn_dir(orc_state *s, double *lam, int dir) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int n = dir == 0 ? nx : dir == 1 ? ny : nz;
  if (n <= 1) return;  /* the forward sweep leaves ts0 unchanged (:770) */
  const int na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
  const double dt = s->dt, imp = s->imp_fac;
  double *buf = (double *)calloc(12 * (size_t)(n + 4), sizeof(double));
  double *kap = buf + 1, *sig = kap + (n + 4), *kk = sig + (n + 4);
  double *DL = kk + (n + 4), *D = DL + (n + 4), *DU = D + (n + 4);
  double *CL = DU + (n + 4), *CC = CL + (n + 4), *CR = CC + (n + 4), *y = CR + (n + 4);
  double *lq = y + (n + 4);
  for (int g = 1; g <= s->ns; g++)
    for (int b = 1; b <= nb; b++)
      for (int a = 1; a <= na; a++) {
        for (int l = 0; l <= n + 1; l++) {
          const int i = dir == 0 ? l : a, j = dir == 1 ? l : (dir == 0 ? a : b), k = dir == 2 ? l : b;
          kap[l] = s->kappa[i3(s, i, j, k)];
          sig[l] = (dir == 0 ? s->sig_nx : dir == 1 ? s->sig_ny : s->sig_nz)[i3(s, i, j, k)];
          kk[l] = (dir == 0 ? s->kx : dir == 1 ? s->ky : s->kz)[k3(s, i, j, k)];
        }
        for (int l = 1; l <= n; l++) {
          const double vavgL = 0.5 * (kap[l - 1] + kap[l]), kavgL = 0.5 * (kk[l - 1] + kk[l]);
          const double kdsL = kavgL * (sig[l] / vavgL);
          const double vavgR = 0.5 * (kap[l] + kap[l + 1]), kavgR = 0.5 * (kk[l] + kk[l + 1]);
          const double kdsR = kavgR * (sig[l + 1] / vavgR);
          const double Lf = dt * kdsL * sig[l] / kap[l], Rf = dt * kdsR * sig[l + 1] / kap[l];
          const double Cf = Lf + Rf;
          const int r = l - 1;
          D[r] = 1.0 + imp * Cf - (l == 1 ? imp * Lf : 0.0) - (l == n ? imp * Rf : 0.0);
          if (l < n) DU[r] = -(imp * Rf);   /* M(r, r+1) */
          if (l > 1) DL[r - 1] = -(imp * Lf);  /* M(r, r-1) */
          CL[r] = (1.0 - imp) * Lf; CC[r] = 1.0 - (1.0 - imp) * Cf; CR[r] = (1.0 - imp) * Rf;
        }
        for (int l = 1; l <= n; l++) {
          const int i = dir == 0 ? l : a, j = dir == 1 ? l : (dir == 0 ? a : b), k = dir == 2 ? l : b;
          y[l - 1] = s->is_aloft[g - 1] ? lam[lv(s, i, j, k, g)] : 0.0;
        }
        /* M^T: sub-diagonal DU, super-diagonal DL (dgtsv overwrites copies) */
        {
          double *dl2 = (double *)malloc(sizeof(double) * 3 * (size_t)n);
          double *d2 = dl2 + n, *du2 = d2 + n;
          for (int r = 0; r < n - 1; r++) { dl2[r] = DU[r]; du2[r] = DL[r]; }
          for (int r = 0; r < n; r++) d2[r] = D[r];
          (void)orc_dgtsv(n, dl2, d2, du2, y);
          free(dl2);
        }
        /* N: row 0 = (CL0+CC0) q0 + CR0 q1; row n-1 = CL q(n-2) + (CC+CR) q(n-1) */
        for (int r = 0; r < n; r++) lq[r] = 0.0;
        for (int r = 0; r < n; r++) {
          const int rm = r > 0 ? r - 1 : 0, rp = r < n - 1 ? r + 1 : n - 1;
          lq[rm] += CL[r] * y[r];
          lq[r] += CC[r] * y[r];
          lq[rp] += CR[r] * y[r];
        }
        for (int l = 1; l <= n; l++) {
          const int i = dir == 0 ? l : a, j = dir == 1 ? l : (dir == 0 ? a : b), k = dir == 2 ? l : b;
          lam[lv(s, i, j, k, g)] = s->is_aloft[g - 1] ? lq[l - 1] : 0.0;
        }
      }
  free(buf);
}

void orc_adj_diffuse_horz(orc_state *s, double *lam, int itime) {
  /* forward: even x then y, odd y then x (src/Diffusion.F90:186-214) */
  const int first = (itime % 2 == 0) ? 1 : 0, second = 1 - first;  /* reverse order */
  if (s->use_cn) { adj_cn_dir(s, lam, first); adj_cn_dir(s, lam, second); }
  else { adj_diff_dir(s, lam, first); adj_diff_dir(s, lam, second); }
}

void orc_adj_diffuse_vert(orc_state *s, double *lam) {
  if (s->use_cn) adj_cn_dir(s, lam, 2); else adj_diff_dir(s, lam, 2);
}

/* ======================================================================== */
/* Output products of Gen_Output_Vars (src/Output_Vars.f90:1192-1240):       */
/* ConcentrationCalculator (:1026-1123), AshThicknessCalculator (:855-895),  */
/* CloudAreaCalculator (:1138-1177) and the arrival-time marks (:1226-1236). */
/* 2-D arrays are (nx,ny), i fastest; z_cc holds z_cc_pd(1:nz).              */
/* areas = {CloudArea, DepositAreaCovered, CloudLoadArea(1:5)}.              */
/* ======================================================================== */
void orc_output_vars(orc_state *s, const double *z_cc, double cloudcon_thresh,
                     double cloudload_thresh, double depo_thresh, double deposit_density,
                     double time, double *cloud_load, double *max_height, double *min_height,
                     double *max_conc, int32_t *mask_cloud, double *dep_thick, int32_t *mask_dep,
                     double *cloud_arrival, double *dep_arrival, double *areas) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, ns = s->ns;
  const double *dz = s->dz_vec + 1; /* dz[k] = dz_vec_pd(k) */
  double *tc = (double *)calloc((size_t)nz + 1, sizeof(double));
  /* AshThicknessCalculator */
  double dep_area = 0.0;
  for (int i = 1; i <= nx; i++)
    for (int j = 1; j <= ny; j++) {
      const size_t o = (size_t)(i - 1) + (size_t)nx * (j - 1);
      double sg = 0.0;
      for (int n = 1; n <= ns; n++) sg = sg + s->deposit[dep(s, i, j, n)];
      dep_thick[o] = sg * dz[1] / 1.0e6 / deposit_density * 1.0e3;
      mask_dep[o] = dep_thick[o] > depo_thresh;
      if (mask_dep[o]) dep_area = dep_area + s->sig_nz[i3(s, i, j, 1)];
    }
  /* ConcentrationCalculator */
  for (int i = 1; i <= nx; i++)
    for (int j = 1; j <= ny; j++) {
      const size_t o = (size_t)(i - 1) + (size_t)nx * (j - 1);
      cloud_load[o] = 0.0; max_conc[o] = 0.0; max_height[o] = 0.0; min_height[o] = 100.0;
      mask_cloud[o] = 0;
    }
  double cloud_area = 0.0;
  if (ns > 0)
    for (int i = s->imin; i <= s->imax; i++)
      for (int j = s->jmin; j <= s->jmax; j++) {
        const size_t o = (size_t)(i - 1) + (size_t)nx * (j - 1);
        for (int k = 1; k <= nz; k++) {
          double sg = 0.0;
          for (int n = 1; n <= ns; n++) sg = sg + s->concen[c5(s, i, j, k, n, 0)];
          cloud_load[o] = cloud_load[o] + sg * dz[k] / 1.0e3;
          tc[k] = sg;
          if (tc[k] >= cloudcon_thresh) max_height[o] = z_cc[k - 1] + 0.5 * dz[k];
        }
        for (int k = nz; k >= 1; k--)
          if (tc[k] <= cloudcon_thresh) min_height[o] = z_cc[k - 1] - 0.5 * dz[k];
        double mx = tc[1];
        for (int k = 2; k <= nz; k++) mx = fmx(mx, tc[k]);
        mask_cloud[o] = cloud_load[o] >= cloudload_thresh;
        if (mask_cloud[o]) {
          if (min_height[o] < 0.0 && max_height[o] > 0.0) min_height[o] = 0.0;
          min_height[o] = fmn(max_height[o], min_height[o]);
          cloud_area = cloud_area + s->sig_nz[i3(s, i, j, 1)];
          max_conc[o] = mx * 1.0e6 / 1.0e9;
        } else {
          cloud_load[o] = 0.0; max_conc[o] = 0.0; max_height[o] = 0.0; min_height[o] = 0.0;
        }
      }
  /* CloudAreaCalculator */
  static const double load_val[5] = {0.24, 1.0, 2.0, 4.0, 6.0};
  double la[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (ns > 0)
    for (int i = s->imin; i <= s->imax; i++)
      for (int j = s->jmin; j <= s->jmax; j++) {
        const double cell = s->sig_nz[i3(s, i, j, 1)];
        const size_t o = (size_t)(i - 1) + (size_t)nx * (j - 1);
        for (int k = 0; k < 5; k++)
          if (cloud_load[o] > load_val[k]) la[k] = la[k] + cell;
      }
  /* arrival times */
  for (size_t o = 0; o < (size_t)nx * ny; o++) {
    if (mask_dep[o] && dep_arrival[o] < 0.0) dep_arrival[o] = time;
    if (mask_cloud[o] && cloud_arrival[o] < 0.0) cloud_arrival[o] = time;
  }
  areas[0] = cloud_area;
  areas[1] = dep_area;
  for (int k = 0; k < 5; k++) areas[2 + k] = la[k];
  free(tc);
}
