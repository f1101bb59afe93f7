// k_advect.cu -- limited-upwind (DCU) advection sweeps on the device.
//
// Restates the row algorithm of advect_x / advect_y (src/AdvectionHorz_DCU.f90
// :68-305 / :322-556) and advect_z (src/AdvectionVert_DCU.f90:100-323):
// interface flux areas usig = 0.5*(v_{I-1}+v_I)*sigma_I, slopes dq, the
// limited second-order flux fss (superbee and the other LIM_* choices), the
// first-order fluctuations fs_r/fs_l with the divergence correction, and
// update = -dt/kappa*(fs_l(I+1)+fs_r(I)+fss(I+1)-fss(I)).  Every expression
// keeps the reference's operation order; the library is compiled with
// --fmad=false so that each product and sum rounds on its own, as the CPU
// build does, and divisions are IEEE (div.rn).
//
// Mapping: a CTA owns a tile of TL cells along the sweep (2 of them overlap
// the neighbouring tiles, so that the outflow cells 0 and n+1 get computed)
// and, for the y and z sweeps, 32 consecutive i (coalesced).  Rows are staged
// in shared memory with the 2-cell limiter halo, ghost values generated on
// load.  All grains of a row are processed by the same CTA so the flux areas
// (grain independent for x and y) are computed once.
#include "a3g_internal.cuh"

namespace a3g {

// Limited second-order flux at one interface, src/AdvectionHorz_DCU.f90:179-231.
template <int LIM>
__device__ __forceinline__ double dcu_fss(double dqm, double dq, double dqp, double us,
                                          double dtv, double eps, int nocycle) {
  if (LIM == A3G_LIM_NONE) return 0.0;
  if (!nocycle && fabs(dq) <= eps) return 0.0;
  double ldq;
  if (LIM == A3G_LIM_LAXWEN) {
    ldq = dq;
  } else {
    const double dqu = (us > 0.0) ? dqm : dqp;
    double theta;
    if (fabs(dqu) > 3.0 * fabs(dq) || fabs(dq) < eps)
      theta = copysign(3.0, dqu * dq);
    else
      theta = dqu / dq;
    if (LIM == A3G_LIM_BW) ldq = dqu;
    else if (LIM == A3G_LIM_FROMM) ldq = dq * (0.5 * (1.0 + theta));
    else if (LIM == A3G_LIM_MINMOD) ldq = dq * fmx(0.0, fmn(1.0, theta));
    else if (LIM == A3G_LIM_MC) ldq = dq * fmx(0.0, fmn(fmn((1.0 + theta) / 2.0, 2.0), 2.0 * theta));
    else ldq = dq * fmx(fmx(0.0, fmn(1.0, 2.0 * theta)), fmn(2.0, theta));
  }
  const double aus = fabs(us);
  return 0.5 * aus * (1.0 - dtv * aus) * ldq;
}

// First-order fluctuations with the divergence correction, :238-249.
__device__ __forceinline__ void dcu_fluct(double qm, double q, double dq, double usm,
                                          double us, double usp, double &fsr, double &fsl) {
  fsr = fmx(0.0, us) * dq;
  fsl = fmn(0.0, us) * dq;
  const double divu_p = fmx(0.0, us) - fmx(0.0, usm);
  const double divu_m = fmn(0.0, usp) - fmn(0.0, us);
  fsr = fsr + q * divu_m;
  fsl = fsl + qm * divu_p;
}

// ---------------------------------------------------------------------------
// x sweep: one CTA = one (j,k) row segment of TX computed cells.
// ---------------------------------------------------------------------------
template <int LIM, int TX>
__global__ void __launch_bounds__(TX) k_advect_x(Layout L, Box box, int periodic, int nocycle,
                                                 double eps, const double *__restrict__ cin,
                                                 double *__restrict__ cout,
                                                 const double *__restrict__ vx, Geo3 sig, Geo3 kap,
                                                 const int32_t *__restrict__ aloft,
                                                 DevScalars *sc, double *__restrict__ out1,
                                                 double *__restrict__ out2) {
  __shared__ double s_q[TX + 4];    // cells cA-2 .. cA+TX+1
  __shared__ double s_us[TX + 3];   // interfaces cA-1 .. cA+TX+1
  __shared__ double s_fss[TX + 1];  // interfaces cA .. cA+TX
  __shared__ double s_fsl[TX + 1];
  const int nx = L.nx;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  const int t0 = 1 + blockIdx.x * (TX - 2);
  const int cA = t0 - 1;
  const int tid = threadIdx.x;
  const int c = cA + tid;
  const bool own = tid >= 1 && tid <= TX - 2 && c >= 1 && c <= nx;
  const int rmin = box.imin, rmax = box.imax;
  const bool row_active = j >= box.jmin && j <= box.jmax && k >= box.kmin && k <= box.kmax;
  const long rowoff = L.cell(1, j, k);  // offset of cell (1,j,k) in a grain slab

  if (!row_active) {
    if (own)
      for (int g = 0; g < L.ns; g++) cout[(long)g * L.PG + rowoff + (c - 1)] = 0.0;
    return;
  }
  const double dt = sc->dt;
  // flux areas (grain independent), :159-162
  const double *vrow = vx + rowoff;
  for (int m = tid; m < TX + 3; m += TX) {
    const int I = cA - 1 + m;
    double u = 0.0;
    if (I >= rmin - 1 && I <= rmax + 1) {
      int ia = I - 1, ib = I;
      if (periodic) {
        ia = ia < 1 ? ia + nx : (ia > nx ? ia - nx : ia);
        ib = ib < 1 ? ib + nx : (ib > nx ? ib - nx : ib);
      } else {
        ia = ia < 1 ? 1 : (ia > nx ? nx : ia);
        ib = ib < 1 ? 1 : (ib > nx ? nx : ib);
      }
      u = 0.5 * (vrow[ia - 1] + vrow[ib - 1]) * sig.at(I, j, k);
    }
    s_us[m] = u;
  }
  // dt/kappa for this thread's cell (also the fss interface I=c), :155
  const bool c_in = c >= rmin - 2 && c <= rmax + 2;
  const double dtv_c = c_in ? dt / kap.at(c, j, k) : 0.0;
  const int cx = cA + TX;  // extra interface handled by tid 0
  const double dtv_x = (tid == 0 && cx >= rmin - 2 && cx <= rmax + 2) ? dt / kap.at(cx, j, k) : 0.0;
  const bool out_lo = (tid == 0 && c == 0 && rmin == 1 && !periodic);
  const bool out_hi = (c == nx + 1 && rmax == nx && !periodic && t0 <= nx && nx <= t0 + TX - 3);

  for (int g = 0; g < L.ns; g++) {
    const long goff = (long)g * L.PG + rowoff;
    if (!aloft[g]) {
      if (own) cout[goff + (c - 1)] = 0.0;
      continue;
    }
    __syncthreads();  // smem reuse across grains (and s_us ready on the first pass)
    const double *qrow = cin + goff;
    for (int m = tid; m < TX + 4; m += TX) {
      const int cc = cA - 2 + m;
      double v = 0.0;
      if (cc >= rmin - 2 && cc <= rmax + 2) {
        if (cc >= 1 && cc <= nx) v = qrow[cc - 1];
        else if (periodic) v = qrow[(cc < 1 ? cc + nx : cc - nx) - 1];
      }
      s_q[m] = v;
    }
    __syncthreads();
    // interface I = c (index tid in s_fss/s_fsl); s_q index of cell x is x-(cA-2)
    double fsr_c = 0.0;
    {
      const int I = c;
      const double qm2 = s_q[tid], qm = s_q[tid + 1], q = s_q[tid + 2], qp = s_q[tid + 3];
      const double dqm = qm - qm2, dq = q - qm, dqp = qp - q;
      const double us = s_us[tid + 1];
      double fss = 0.0, fsl = 0.0;
      if (I >= rmin && I <= rmax + 1) fss = dcu_fss<LIM>(dqm, dq, dqp, us, dtv_c, eps, nocycle);
      if (I >= rmin - 1 && I <= rmax + 1) dcu_fluct(qm, q, dq, s_us[tid], us, s_us[tid + 2], fsr_c, fsl);
      s_fss[tid] = fss;
      s_fsl[tid] = fsl;
    }
    if (tid == 0) {
      const int I = cx;
      const int b = TX;
      const double qm2 = s_q[b], qm = s_q[b + 1], q = s_q[b + 2], qp = s_q[b + 3];
      const double dqm = qm - qm2, dq = q - qm, dqp = qp - q;
      const double us = s_us[b + 1];
      double fss = 0.0, fsl = 0.0, fsr = 0.0;
      if (I >= rmin && I <= rmax + 1) fss = dcu_fss<LIM>(dqm, dq, dqp, us, dtv_x, eps, nocycle);
      if (I >= rmin - 1 && I <= rmax + 1) dcu_fluct(qm, q, dq, s_us[b], us, s_us[b + 2], fsr, fsl);
      s_fss[b] = fss;
      s_fsl[b] = fsl;
    }
    __syncthreads();
    // update of cell c, :264-281
    const double upd = -(dtv_c * (s_fsl[tid + 1] + fsr_c + s_fss[tid + 1] - s_fss[tid]));
    if (own) {
      const bool in_box = c >= rmin && c <= rmax;
      cout[goff + (c - 1)] = in_box ? s_q[tid + 2] + upd : 0.0;
    }
    if (out_lo) out1[(long)g * L.ny * L.nz + (long)(k - 1) * L.ny + (j - 1)] += upd;
    if (out_hi) out2[(long)g * L.ny * L.nz + (long)(k - 1) * L.ny + (j - 1)] += upd;
  }
}

// ---------------------------------------------------------------------------
// y and z sweeps: CTA = 32 lanes along i x TL cells along the sweep.
// DIR 1: sweep along j, blockIdx.z = k-1.  DIR 2: sweep along k, blockIdx.z = j-1.
// ---------------------------------------------------------------------------
template <int DIR, int LIM, int TL, int BY>
__global__ void __launch_bounds__(32 * BY) k_advect_yz(Layout L, Box box, int nocycle, double eps,
                                                       const double *__restrict__ cin,
                                                       double *__restrict__ cout,
                                                       const double *__restrict__ vel, Geo4 vf,
                                                       Geo3 sig, Geo3 kap,
                                                       const int32_t *__restrict__ aloft,
                                                       DevScalars *sc, double *__restrict__ out1,
                                                       double *__restrict__ out2) {
  constexpr int M = TL / BY;  // cells per thread
  __shared__ double s_q[TL + 4][32];
  __shared__ double s_us[TL + 3][32];
  __shared__ double s_fss[TL + 1][32];
  __shared__ double s_fsl[TL + 1][32];
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + lane + 1;
  const int o = blockIdx.z + 1;
  const int n = (DIR == 1) ? L.ny : L.nz;
  const int t0 = 1 + blockIdx.y * (TL - 2);
  const int cA = t0 - 1;
  const int rmin = (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  const bool lane_ok = i <= L.nx;
  const bool lane_active = lane_ok && i >= box.imin && i <= box.imax &&
                           ((DIR == 1) ? (o >= box.kmin && o <= box.kmax)
                                       : (o >= box.jmin && o <= box.jmax));
  const long sstride = (DIR == 1) ? L.P : L.PY;  // stride along the sweep
  const long base = (DIR == 1) ? L.cell(i, 1, o) : L.cell(i, o, 1);
  const long oplane = (DIR == 1) ? (long)(o - 1) * L.nx + (i - 1) : (long)(o - 1) * L.nx + (i - 1);
  const long oslab = (DIR == 1) ? (long)L.nx * L.nz : (long)L.nx * L.ny;
  const double dt = sc->dt;

  // geometry per cell of this thread (grain independent)
  auto geo_sig = [&](int I) { return (DIR == 1) ? sig.at(i, I, o) : sig.at(i, o, I); };
  auto geo_kap = [&](int cc) { return (DIR == 1) ? kap.at(i, cc, o) : kap.at(i, o, cc); };
  double dtv[M + 1];
#pragma unroll
  for (int m = 0; m <= M; m++) {
    const int cc = cA + ty + BY * m;
    dtv[m] = (lane_active && cc >= rmin - 2 && cc <= rmax + 2 && (m < M || ty == 0)) ? dt / geo_kap(cc) : 0.0;
  }
  // top-outflow cell: ny+1 for y; update_cc(ncells+1) for z (:309-311), which
  // is nz+1 only when kmin == 1.  The tile whose own cells contain it adds it.
  const int ctop = (DIR == 2) ? ncells + 1 : rmax + 1;
  const int hc = (ctop == n + 1) ? n : ctop;
  const bool top_here = (rmax == n) && (t0 <= hc && hc <= t0 + TL - 3) && (ctop >= rmin - 1);
  if (DIR == 2 && rmax == n && ctop < rmin - 1 && lane_active && blockIdx.y == 0 && ty == 0)
    raise_error(sc, A3G_ERR_UNSUPPORTED, 311);

  // velocity at cell cc with the edge extrapolation of Set_BC(1) (:55-70)
  auto vel_at = [&](int cc, int g) {
    const int cl = cc < 1 ? 1 : (cc > n ? n : cc);
    double v = vel[base + (long)(cl - 1) * sstride];
    if (DIR == 2) v = v + vf.at(i, o, cl, g);
    return v;
  };

  for (int g = 0; g < L.ns; g++) {
    const long goff = (long)g * L.PG + base;
    if (!aloft[g]) {  // uniform over the CTA
      if (lane_ok) {
#pragma unroll
        for (int m = 0; m < M; m++) {
          const int cc = cA + ty + BY * m;
          if (cc >= t0 && cc <= t0 + TL - 3 && cc <= n) cout[goff + (long)(cc - 1) * sstride] = 0.0;
        }
      }
      continue;
    }
    __syncthreads();
    // flux areas (:160-162; AdvectionVert :190-192 where vf enters per grain)
    for (int m = ty; m < TL + 3; m += BY) {
      const int I = cA - 1 + m;
      double u = 0.0;
      if (lane_active && I >= rmin - 1 && I <= rmax + 1)
        u = 0.5 * (vel_at(I - 1, g) + vel_at(I, g)) * geo_sig(I);
      s_us[m][lane] = u;
    }
    for (int m = ty; m < TL + 4; m += BY) {
      const int cc = cA - 2 + m;
      double v = 0.0;
      if (lane_active && cc >= rmin - 2 && cc <= rmax + 2 && cc >= 1 && cc <= n)
        v = cin[goff + (long)(cc - 1) * sstride];
      s_q[m][lane] = v;
    }
    __syncthreads();
    double fsr_r[M];
#pragma unroll
    for (int m = 0; m <= M; m++) {
      if (m == M && ty != 0) break;
      const int t = ty + BY * m;  // local interface index (I = cA + t)
      const int I = cA + t;
      const double qm2 = s_q[t][lane], qm = s_q[t + 1][lane], q = s_q[t + 2][lane],
                   qp = s_q[t + 3][lane];
      const double dqm = qm - qm2, dq = q - qm, dqp = qp - q;
      const double us = s_us[t + 1][lane];
      double fss = 0.0, fsl = 0.0, fsr = 0.0;
      if (I >= rmin && I <= rmax + 1) fss = dcu_fss<LIM>(dqm, dq, dqp, us, dtv[m], eps, nocycle);
      if (I >= rmin - 1 && I <= rmax + 1) dcu_fluct(qm, q, dq, s_us[t][lane], us, s_us[t + 2][lane], fsr, fsl);
      s_fss[t][lane] = fss;
      s_fsl[t][lane] = fsl;
      if (m < M) fsr_r[m] = fsr;
    }
    __syncthreads();
    if (!lane_ok) continue;
#pragma unroll
    for (int m = 0; m < M; m++) {
      const int t = ty + BY * m;
      const int cc = cA + t;
      const double upd = -(dtv[m] * (s_fsl[t + 1][lane] + fsr_r[m] + s_fss[t + 1][lane] - s_fss[t][lane]));
      if (cc >= t0 && cc <= t0 + TL - 3 && cc <= n) {
        const bool in_box = lane_active && cc >= rmin && cc <= rmax;
        cout[goff + (long)(cc - 1) * sstride] = in_box ? s_q[t + 2][lane] + upd : 0.0;
      }
      if (lane_active && cc == 0 && rmin == 1) out1[(long)g * oslab + oplane] += upd;
      if (lane_active && cc == ctop && top_here) out2[(long)g * oslab + oplane] += upd;
    }
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int LIM>
static void launch_x_lim(a3g_ctx *ctx) {
  constexpr int TX = 128;
  const Layout &L = ctx->L;
  dim3 grid((L.nx + TX - 3) / (TX - 2), L.ny, L.nz);
  k_advect_x<LIM, TX><<<grid, TX, 0, ctx->stream>>>(
      L, ctx->box, ctx->grid.periodic, ctx->prm.nocycle, ctx->prm.eps_thresh, ctx->c0, ctx->c1,
      ctx->vx, ctx->snx, ctx->kappa, ctx->aloft, ctx->sc, ctx->out_yz1, ctx->out_yz2);
}

template <int DIR, int LIM>
static void launch_yz_lim(a3g_ctx *ctx) {
  constexpr int TL = 32, BY = 8;
  const Layout &L = ctx->L;
  const int n = (DIR == 1) ? L.ny : L.nz;
  dim3 grid((L.nx + 31) / 32, (n + TL - 3) / (TL - 2), (DIR == 1) ? L.nz : L.ny);
  dim3 block(32, BY);
  k_advect_yz<DIR, LIM, TL, BY><<<grid, block, 0, ctx->stream>>>(
      L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ctx->c0, ctx->c1,
      (DIR == 1) ? ctx->vy : ctx->vz, ctx->vf, (DIR == 1) ? ctx->sny : ctx->snz, ctx->kappa,
      ctx->aloft, ctx->sc, (DIR == 1) ? ctx->out_xz1 : ctx->out_xy1,
      (DIR == 1) ? ctx->out_xz2 : ctx->out_xy2);
}

#define A3G_LIM_SWITCH(FN, ...)                                      \
  switch (ctx->prm.limiter) {                                        \
    case A3G_LIM_NONE: FN<__VA_ARGS__ A3G_LIM_NONE>(ctx); break;     \
    case A3G_LIM_LAXWEN: FN<__VA_ARGS__ A3G_LIM_LAXWEN>(ctx); break; \
    case A3G_LIM_BW: FN<__VA_ARGS__ A3G_LIM_BW>(ctx); break;         \
    case A3G_LIM_FROMM: FN<__VA_ARGS__ A3G_LIM_FROMM>(ctx); break;   \
    case A3G_LIM_MINMOD: FN<__VA_ARGS__ A3G_LIM_MINMOD>(ctx); break; \
    case A3G_LIM_MC: FN<__VA_ARGS__ A3G_LIM_MC>(ctx); break;         \
    default: FN<__VA_ARGS__ A3G_LIM_SUPERBEE>(ctx); break;           \
  }

int launch_advect_x(a3g_ctx *ctx) {
  tbegin(ctx, A3G_K_ADVECT_X);
  A3G_LIM_SWITCH(launch_x_lim, )
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  return A3G_OK;
}
int launch_advect_y(a3g_ctx *ctx) {
  tbegin(ctx, A3G_K_ADVECT_Y);
  A3G_LIM_SWITCH(launch_yz_lim, 1, )
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  return A3G_OK;
}
int launch_advect_z(a3g_ctx *ctx) {
  tbegin(ctx, A3G_K_ADVECT_Z);
  A3G_LIM_SWITCH(launch_yz_lim, 2, )
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  return A3G_OK;
}

}  // namespace a3g
