// k_advect.cu -- dt/kappa of the step and the discrete adjoint of the advection
// sweeps.  The forward sweeps are in k_advect.cuh.
#include "k_advect.cuh"

namespace a3g {

// dt/kappa of the current step on the compressed kappa layout (the reference
// forms dt_vol_cc = dt/kap_cc in every row, :155; the quotient is the same).
__global__ void k_dtv(const double *__restrict__ kap, long n, const DevScalars *__restrict__ sc,
                      double *__restrict__ dtv) {
  const double dt = sc->dt;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    dtv[t] = dt / kap[t];
}

int refresh_dtv(a3g_ctx *ctx) {
  // recomputed whenever the step's dt may have changed
  if (ctx->dtv_valid && ctx->dtv_stamp == ctx->dt_stamp) return A3G_OK;
  const long n = (long)ctx->kappa_len;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  tbegin(ctx, A3G_K_OTHER);
  k_dtv<<<blocks, 256, 0, ctx->stream>>>(ctx->kappa.p, n, ctx->sc, const_cast<double *>(ctx->dtv.p));
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  ctx->dtv_valid = true;
  ctx->dtv_stamp = ctx->dt_stamp;
  return A3G_OK;
}

// ===========================================================================
// Discrete adjoint of one advection sweep (no counterpart in the reference).
//
// With the limiter branches fixed by the sweep's input state q, the limited
// slope is ldq = a*dq + b*dqu, so the sweep is linear; this kernel applies
// its transpose to lam (the adjoint of the sweep's output).  It is a gather:
// one thread per cell-grain, lanes along x in every direction (coalesced),
// each thread re-deriving the four interfaces m-1..m+2 that its cell feeds
// (limiter branch, flux-area terms) from q, winds and geometry.  With t(i) =
// -dt/kappa(i)*lam_u(i) (lam_u = lam inside the line, the deposit adjoint
// at the z bottom outflow, 0 at the other outflows):
//   lam_fsr(I) = t(I), lam_fsl(I) = t(I-1), lam_fss(I) = t(I-1) - t(I)
//   e(J) = 0.5|us|(1 - dtv|us|) * lam_fss(J)       (active fss interfaces)
//   lam_dq(I) = max(0,us)lam_fsr(I) + min(0,us)lam_fsl(I) + a(I)e(I)
//               + b(I+1)e(I+1) [us(I+1) > 0] + b(I-1)e(I-1) [us(I-1) <= 0]
//   lam_q(m)  = lam(m) + divu_m(m)lam_fsr(m) + divu_p(m+1)lam_fsl(m+1)
//               + lam_dq(m) - lam_dq(m+1)
// Ghost cells of Set_BC(1) are zero (their adjoint is dropped) except x-
// periodic wraps, whose adjoint is added back to the wrapped cells.  Full box
// only (the subgrid box depends on the state).
// ===========================================================================

// d(ldq) = a*d(dq) + b*d(dqu) on the branch the forward limiter takes.
template <int LIM>
__device__ __forceinline__ void lim_coef(double dq, double dqu, double eps, double &a, double &b) {
  if (LIM == A3G_LIM_LAXWEN) { a = 1.0; b = 0.0; return; }
  if (LIM == A3G_LIM_BW) { a = 0.0; b = 1.0; return; }
  const bool clamp = fabs(dqu) > 3.0 * fabs(dq) || fabs(dq) < eps;
  const double th = clamp ? copysign(3.0, dqu * dq) : div_rn(dqu, dq);
  double phi, dphi;
  if (LIM == A3G_LIM_FROMM) {
    phi = 0.5 * (1.0 + th); dphi = 0.5;
  } else if (LIM == A3G_LIM_MINMOD) {
    const double m = fmn(1.0, th), dm = (1.0 < th) ? 0.0 : 1.0;
    phi = fmx(0.0, m); dphi = (0.0 > m) ? 0.0 : dm;
  } else if (LIM == A3G_LIM_MC) {
    const double m1 = fmn((1.0 + th) / 2.0, 2.0), dm1 = ((1.0 + th) / 2.0 < 2.0) ? 0.5 : 0.0;
    const double m2 = fmn(m1, 2.0 * th), dm2 = (m1 < 2.0 * th) ? dm1 : 2.0;
    phi = fmx(0.0, m2); dphi = (0.0 > m2) ? 0.0 : dm2;
  } else {  // superbee
    const double m1 = fmn(1.0, 2.0 * th), dm1 = (1.0 < 2.0 * th) ? 0.0 : 2.0;
    const double a1 = fmx(0.0, m1), da1 = (0.0 > m1) ? 0.0 : dm1;
    const double m2 = fmn(2.0, th), dm2 = (2.0 < th) ? 0.0 : 1.0;
    phi = fmx(a1, m2); dphi = (a1 > m2) ? da1 : dm2;
  }
  if (clamp) dphi = 0.0;
  a = phi - th * dphi;
  b = dphi;
}

template <int DIR, int LIM, bool PER>
__global__ void __launch_bounds__(256) k_adj_advect(Layout L, int nocycle, double eps,
                                                    const double *__restrict__ cq,
                                                    const double *__restrict__ lin,
                                                    double *__restrict__ lout,
                                                    const double *__restrict__ vel, Geo4 vf, Geo3 sig,
                                                    Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                    const double *__restrict__ lam_lo) {
  const int i = blockIdx.x * 32 + threadIdx.x + 1;
  const int j = blockIdx.y * 8 + threadIdx.y + 1;
  const int k = (int)(blockIdx.z % L.nz) + 1;
  const int g = (int)(blockIdx.z / L.nz);
  if (i > L.nx || j > L.ny) return;
  const long cell = L.cell(i, j, k);
  const long gb = (long)g * L.PG;
  if (!aloft[g]) {
    lout[gb + cell] = 0.0;
    return;
  }
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int m = (DIR == 0) ? i : (DIR == 1) ? j : k;
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? L.P : L.PY;
  const long lb = cell - (long)(m - 1) * st;  // sweep index 1 of this line
  const int la = (DIR == 0) ? j : i, lo_ = (DIR == 2) ? j : k;
  const LineGeo gsig = line_of<DIR>(sig, la, lo_);
  const LineGeo gdtv = line_of<DIR>(dtvt, la, lo_);
  const double *pq = cq + gb + lb;
  const double *pl = lin + gb + lb;
  const double *pv = vel + lb;
  const double *pvf = vf.p + (long)(i + 1) * vf.si + (long)(j + 1) * vf.sj + (long)g * vf.sg;
  auto wrap = [&](int c) { return c < 1 ? c + n : (c > n ? c - n : c); };
  auto Q = [&](int c) -> double {
    if (c < -1 || c > n + 2) return 0.0;
    if (c >= 1 && c <= n) return pq[(long)(c - 1) * st];
    return PER ? pq[(long)(wrap(c) - 1) * st] : 0.0;
  };
  auto V = [&](int c) -> double {
    const int cl = PER ? wrap(c) : (c < 1 ? 1 : (c > n ? n : c));
    double v = pv[(long)(cl - 1) * st];
    if (DIR == 2) v = v + pvf[(long)(cl + 1) * vf.sk];
    return v;
  };
  auto US = [&](int I) -> double {  // usig(I), zero outside [0, n+1]
    if (I < 0 || I > n + 1) return 0.0;
    return 0.5 * (V(I - 1) + V(I)) * gsig.at(I);
  };
  auto T = [&](int c) -> double {  // t(c) = -dtv(c)*lam_u(c)
    if (c < 0 || c > n + 1) return 0.0;
    double lu = 0.0;
    if (c >= 1 && c <= n) lu = pl[(long)(c - 1) * st];
    else if (c == 0 && lam_lo) lu = lam_lo[(long)g * L.nx * L.ny + (long)(j - 1) * L.nx + (i - 1)];
    return -(gdtv.at(c) * lu);
  };
  auto DQ = [&](int I) -> double { return (I < 0 || I > n + 2) ? 0.0 : Q(I) - Q(I - 1); };
  // lam_q at sweep index c (an interior cell or a ghost)
  auto lam_at = [&](int c) -> double {
    double us[6], tt[5], dq[6];
#pragma unroll
    for (int d = 0; d < 6; d++) us[d] = US(c - 2 + d);  // us(c-2 .. c+3)
#pragma unroll
    for (int d = 0; d < 5; d++) tt[d] = T(c - 2 + d);   // t(c-2 .. c+2)
#pragma unroll
    for (int d = 0; d < 6; d++) dq[d] = DQ(c - 2 + d);  // dq(c-2 .. c+3)
    // interfaces J = c-1 .. c+2 (index r = J-c+1): a*e, b*e, upwind side
    double ea[4], eb[4];
    bool up[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int J = c - 1 + r;
      const double u = us[r + 1];
      up[r] = u > 0.0;
      ea[r] = 0.0;
      eb[r] = 0.0;
      if (LIM != A3G_LIM_NONE && J >= 1 && J <= n + 1) {
        const double dqJ = dq[r + 1];
        if (nocycle || !(fabs(dqJ) <= eps)) {
          const double aus = fabs(u);
          const double w = 0.5 * aus * (1.0 - gdtv.at(J) * aus);
          const double e = w * (tt[r] - tt[r + 1]);  // t(J-1) - t(J)
          double a, b;
          lim_coef<LIM>(dqJ, up[r] ? dq[r] : dq[r + 2], eps, a, b);
          ea[r] = a * e;
          eb[r] = b * e;
        }
      }
    }
    // lam_dq(c) (r = 1) and lam_dq(c+1) (r = 2)
    double ldq[2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int I = c + s, r = 1 + s;
      double v = 0.0;
      if (I >= 0 && I <= n + 2) {
        const double u = us[r + 1];
        const double lfsr = tt[r + 1];                          // t(I)
        const double lfsl = (I <= n + 1) ? tt[r] : 0.0;         // t(I-1)
        v = dmx(0.0, u) * lfsr + dmn(0.0, u) * lfsl + ea[r];
        if (up[r + 1]) v = v + eb[r + 1];
        if (!up[r - 1]) v = v + eb[r - 1];
      }
      ldq[s] = v;
    }
    double lam = (c >= 1 && c <= n) ? pl[(long)(c - 1) * st] : 0.0;
    if (c >= 0 && c <= n + 1) {  // divu_m(c)*lam_fsr(c)
      const double divm = dmn(0.0, us[3]) - dmn(0.0, us[2]);
      lam = lam + divm * tt[2];
    }
    if (c + 1 >= 0 && c + 1 <= n + 1) {  // divu_p(c+1)*lam_fsl(c+1)
      const double divp = dmx(0.0, us[3]) - dmx(0.0, us[2]);
      lam = lam + divp * tt[2];
    }
    return lam + ldq[0] - ldq[1];
  };
  double lam = lam_at(m);
  if (PER) {
    if (m <= 2) lam = lam + lam_at(m + n);
    if (m >= n - 1) lam = lam + lam_at(m - n);
  }
  lout[gb + cell] = lam;
}

// Block form of k_adj_advect: a thread takes V consecutive cells of a line
// and forms each of the V+3 interfaces they read (c0-1 .. c0+V+1) once,
// instead of the four a cell-per-thread gather forms for every cell; the
// expressions and their order are lam_at's, so the results are the same
// bits.  Not x-periodic (the wrapped ghosts stay with the gather kernel).
// DIR 0: lanes are consecutive blocks along i; DIR 1, 2: lanes along i.
template <int DIR, int LIM, int V, bool CK>
__device__ __forceinline__ void adj_block_body(const Layout &L, int nocycle, double eps, int n, int c0, long st,
                                               const double *__restrict__ pq, const double *__restrict__ pl,
                                               double *__restrict__ po, const double *__restrict__ pv,
                                               const double *__restrict__ pvf, long vfs, const LineGeo &gsig,
                                               const LineGeo &gdtv, double lam_lo0) {
  auto Q = [&](int c) -> double {
    if (CK && (c < 1 || c > n)) return 0.0;
    return pq[(long)(c - 1) * st];
  };
  auto VV = [&](int c) -> double {
    const int cl = CK ? (c < 1 ? 1 : (c > n ? n : c)) : c;
    double v = pv[(long)(cl - 1) * st];
    if (DIR == 2) v = v + pvf[(long)(cl + 1) * vfs];
    return v;
  };
  auto T = [&](int c) -> double {  // t(c) = -dtv(c)*lam_u(c)
    if (CK && (c < 0 || c > n + 1)) return 0.0;
    double lu = 0.0;
    if (!CK || (c >= 1 && c <= n)) lu = pl[(long)(c - 1) * st];
    else if (c == 0 && DIR == 2) lu = lam_lo0;
    return -(gdtv.at(c) * lu);
  };
  // window: q(c0-3 .. c0+V+2), vel(c0-3 .. c0+V+2), t(c0-2 .. c0+V+1)
  double q[V + 6], vv[V + 6], tt[V + 4];
#pragma unroll
  for (int m = 0; m < V + 6; m++) {
    q[m] = Q(c0 - 3 + m);
    vv[m] = VV(c0 - 3 + m);
  }
#pragma unroll
  for (int m = 0; m < V + 4; m++) tt[m] = T(c0 - 2 + m);
  // dq(c0-2 .. c0+V+2): dq(I) = q(I) - q(I-1), zero outside [0, n+2]
  double dq[V + 5];
#pragma unroll
  for (int m = 0; m < V + 5; m++) {
    const int I = c0 - 2 + m;
    dq[m] = (CK && (I < 0 || I > n + 2)) ? 0.0 : q[m + 1] - q[m];
  }
  // interfaces J = c0-1+r, r = 0 .. V+2: usig, upwind side, a*e, b*e
  double us[V + 3], ea[V + 3], eb[V + 3];
  bool up[V + 3];
#pragma unroll
  for (int r = 0; r < V + 3; r++) {
    const int J = c0 - 1 + r;
    const double u = (CK && (J < 0 || J > n + 1)) ? 0.0 : 0.5 * (vv[r + 1] + vv[r + 2]) * gsig.at(J);
    us[r] = u;
    up[r] = u > 0.0;
    ea[r] = 0.0;
    eb[r] = 0.0;
    if (LIM != A3G_LIM_NONE && (!CK || (J >= 1 && J <= n + 1))) {
      const double dqJ = dq[r + 1];
      if (nocycle || !(fabs(dqJ) <= eps)) {
        const double aus = fabs(u);
        const double w = 0.5 * aus * (1.0 - gdtv.at(J) * aus);
        const double e = w * (tt[r] - tt[r + 1]);  // t(J-1) - t(J)
        double a, b;
        lim_coef<LIM>(dqJ, up[r] ? dq[r] : dq[r + 2], eps, a, b);
        ea[r] = a * e;
        eb[r] = b * e;
      }
    }
  }
#pragma unroll
  for (int v = 0; v < V; v++) {
    const int c = c0 + v;
    if (CK && c > n) break;
    double ldq[2];
#pragma unroll
    for (int s2 = 0; s2 < 2; s2++) {
      const int I = c + s2, r = v + 1 + s2;
      double val = 0.0;
      if (!CK || (I >= 0 && I <= n + 2)) {
        const double u = us[r];
        const double lfsr = tt[v + 2 + s2];                              // t(I)
        const double lfsl = (!CK || I <= n + 1) ? tt[v + 1 + s2] : 0.0;  // t(I-1)
        val = dmx(0.0, u) * lfsr + dmn(0.0, u) * lfsl + ea[r];
        if (up[r + 1]) val = val + eb[r + 1];
        if (!up[r - 1]) val = val + eb[r - 1];
      }
      ldq[s2] = val;
    }
    double lam = pl[(long)(c - 1) * st];
    const double divm = dmn(0.0, us[v + 2]) - dmn(0.0, us[v + 1]);
    lam = lam + divm * tt[v + 2];
    const double divp = dmx(0.0, us[v + 2]) - dmx(0.0, us[v + 1]);
    lam = lam + divp * tt[v + 2];
    po[(long)(c - 1) * st] = lam + ldq[0] - ldq[1];
  }
}

template <int DIR, int LIM, int V>
__global__ void __launch_bounds__(128) k_adj_advect_blk(Layout L, int nocycle, double eps, int nblk,
                                                        const double *__restrict__ cq,
                                                        const double *__restrict__ lin,
                                                        double *__restrict__ lout,
                                                        const double *__restrict__ vel, Geo4 vf, Geo3 sig,
                                                        Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                        const double *__restrict__ lam_lo) {
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  int a, o, blk, g;  // lane index (i or j), other index, block, grain (k_advect_block's mapping)
  if (DIR == 0) {
    blk = blockIdx.x * 32 + threadIdx.x;
    a = blockIdx.y * 4 + threadIdx.y + 1;  // j
    o = (int)(blockIdx.z % L.nz) + 1;      // k
    g = (int)(blockIdx.z / L.nz);
    if (blk >= nblk || a > L.ny) return;
  } else {
    a = blockIdx.x * 32 + threadIdx.x + 1;  // i
    const int w = blockIdx.y * 4 + threadIdx.y;
    blk = w % nblk;
    o = w / nblk + 1;
    g = blockIdx.z;
    const int nother = (DIR == 1) ? L.nz : L.ny;
    if (a > L.nx || o > nother) return;
  }
  const int c0 = 1 + blk * V;
  const long base = (DIR == 0) ? L.cell(1, a, o) : (DIR == 1) ? L.cell(a, 1, o) : L.cell(a, o, 1);
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? L.P : L.PY;
  const long gb = (long)g * L.PG;
  double *po = lout + gb + base;
  if (!aloft[g]) {
    for (int v = 0; v < V; v++)
      if (c0 + v <= n) po[(long)(c0 + v - 1) * st] = 0.0;
    return;
  }
  const int i = (DIR == 0) ? 1 : a, j = (DIR == 1) ? 1 : (DIR == 0 ? a : o);
  const LineGeo gsig = line_of<DIR>(sig, a, o);
  const LineGeo gdtv = line_of<DIR>(dtvt, a, o);
  const double *pvf = vf.p + (long)(i + 1) * vf.si + (long)(j + 1) * vf.sj + (long)g * vf.sg;
  const double lam_lo0 = (DIR == 2 && lam_lo && c0 <= 2) ? lam_lo[(long)g * L.nx * L.ny + (long)(j - 1) * L.nx + (i - 1)]
                                                         : 0.0;
  const bool fast = c0 - 3 >= 1 && c0 + V + 2 <= n;
  if (fast)
    adj_block_body<DIR, LIM, V, false>(L, nocycle, eps, n, c0, st, cq + gb + base, lin + gb + base, po, vel + base,
                                       pvf, vf.sk, gsig, gdtv, lam_lo0);
  else
    adj_block_body<DIR, LIM, V, true>(L, nocycle, eps, n, c0, st, cq + gb + base, lin + gb + base, po, vel + base,
                                      pvf, vf.sk, gsig, gdtv, lam_lo0);
}

template <int DIR, int LIM>
static void launch_adj_dir_lim(a3g_ctx *ctx, const double *cq, const double *lin, double *lout,
                               const double *lam_lo) {
  const Layout &L = ctx->L;
  dim3 grid((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz * L.ns);
  const bool per = (DIR == 0) && ctx->grid.periodic;
  const double *vel = (DIR == 0) ? ctx->vx : (DIR == 1) ? ctx->vy : ctx->vz;
  const Geo3 &sig = (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz;
  if (per) {
    k_adj_advect<DIR, LIM, true><<<grid, dim3(32, 8), 0, ctx->stream>>>(
        L, ctx->prm.nocycle, ctx->prm.eps_thresh, cq, lin, lout, vel, ctx->vf, sig, ctx->dtv, ctx->aloft,
        lam_lo);
  } else if (ctx->adj_gather) {
    k_adj_advect<DIR, LIM, false><<<grid, dim3(32, 8), 0, ctx->stream>>>(
        L, ctx->prm.nocycle, ctx->prm.eps_thresh, cq, lin, lout, vel, ctx->vf, sig, ctx->dtv, ctx->aloft,
        lam_lo);
  } else {
    constexpr int V = 4;
    const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
    const int nblk = (n + V - 1) / V;
    dim3 gb;
    if (DIR == 0) gb = dim3((nblk + 31) / 32, (L.ny + 3) / 4, L.nz * L.ns);
    else gb = dim3((L.nx + 31) / 32, (nblk * ((DIR == 1) ? L.nz : L.ny) + 3) / 4, L.ns);
    k_adj_advect_blk<DIR, LIM, V><<<gb, dim3(32, 4), 0, ctx->stream>>>(
        L, ctx->prm.nocycle, ctx->prm.eps_thresh, nblk, cq, lin, lout, vel, ctx->vf, sig, ctx->dtv, ctx->aloft,
        lam_lo);
  }
}

template <int DIR>
static void launch_adj_dir(a3g_ctx *ctx, const double *cq, const double *lin, double *lout,
                           const double *lam_lo) {
  switch (ctx->prm.limiter) {
    case A3G_LIM_NONE: launch_adj_dir_lim<DIR, A3G_LIM_NONE>(ctx, cq, lin, lout, lam_lo); break;
    case A3G_LIM_LAXWEN: launch_adj_dir_lim<DIR, A3G_LIM_LAXWEN>(ctx, cq, lin, lout, lam_lo); break;
    case A3G_LIM_BW: launch_adj_dir_lim<DIR, A3G_LIM_BW>(ctx, cq, lin, lout, lam_lo); break;
    case A3G_LIM_FROMM: launch_adj_dir_lim<DIR, A3G_LIM_FROMM>(ctx, cq, lin, lout, lam_lo); break;
    case A3G_LIM_MINMOD: launch_adj_dir_lim<DIR, A3G_LIM_MINMOD>(ctx, cq, lin, lout, lam_lo); break;
    case A3G_LIM_MC: launch_adj_dir_lim<DIR, A3G_LIM_MC>(ctx, cq, lin, lout, lam_lo); break;
    default: launch_adj_dir_lim<DIR, A3G_LIM_SUPERBEE>(ctx, cq, lin, lout, lam_lo); break;
  }
}

// lam_out <- J(cq)^T lam_in for the advection sweep along dir (0 x, 1 y, 2 z).
int launch_adj_advect(a3g_ctx *ctx, int dir, const double *cq, const double *lin, double *lout,
                      const double *lam_lo) {
  int rc = refresh_dtv(ctx);
  if (rc) return rc;
  tbegin(ctx, A3G_K_ADJOINT);
  if (dir == 0) launch_adj_dir<0>(ctx, cq, lin, lout, nullptr);
  else if (dir == 1) launch_adj_dir<1>(ctx, cq, lin, lout, nullptr);
  else launch_adj_dir<2>(ctx, cq, lin, lout, lam_lo);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// ===========================================================================
// Tangent-linear of one advection sweep (no counterpart in the reference).
//
// The same linear map k_adj_advect transposes: with the limiter branches
// fixed by the sweep's input state q (lim_coef: ldq = a*dq + b*dqu), a
// perturbation d of the input goes to
//   d_fss(I) = cf(I)*(a(I)*dd(I) + b(I)*dd_u(I))   (active fss interfaces)
//   d_fsr(I) = max(0,us)*dd(I) + d(I)*divu_m(I),  d_fsl(I) = min(0,us)*dd(I) + d(I-1)*divu_p(I)
//   d_out(m) = d(m) - dt/kappa(m)*(d_fsl(m+1) + d_fsr(m) + d_fss(m+1) - d_fss(m))
// with dd = the perturbation's slopes and Set_BC(1) ghosts (zero, x-periodic
// wrap).  The z sweep adds the perturbation of the bottom outflow (the
// deposit) to dep.  One thread per cell-grain, full box.
// ===========================================================================
template <int DIR, int LIM, bool PER>
__global__ void __launch_bounds__(256) k_tl_advect(Layout L, int nocycle, double eps,
                                                   const double *__restrict__ cq,
                                                   const double *__restrict__ din,
                                                   double *__restrict__ dout,
                                                   const double *__restrict__ vel, Geo4 vf, Geo3 sig,
                                                   Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                   double *__restrict__ dep) {
  const int i = blockIdx.x * 32 + threadIdx.x + 1;
  const int j = blockIdx.y * 8 + threadIdx.y + 1;
  const int k = (int)(blockIdx.z % L.nz) + 1;
  const int g = (int)(blockIdx.z / L.nz);
  if (i > L.nx || j > L.ny) return;
  const long cell = L.cell(i, j, k);
  const long gb = (long)g * L.PG;
  if (!aloft[g]) {
    dout[gb + cell] = 0.0;
    return;
  }
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int m = (DIR == 0) ? i : (DIR == 1) ? j : k;
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? L.P : L.PY;
  const long lb = cell - (long)(m - 1) * st;
  const int la = (DIR == 0) ? j : i, lo_ = (DIR == 2) ? j : k;
  const LineGeo gsig = line_of<DIR>(sig, la, lo_);
  const LineGeo gdtv = line_of<DIR>(dtvt, la, lo_);
  const double *pq = cq + gb + lb;
  const double *pd = din + gb + lb;
  const double *pv = vel + lb;
  const double *pvf = vf.p + (long)(i + 1) * vf.si + (long)(j + 1) * vf.sj + (long)g * vf.sg;
  auto wrap = [&](int c) { return c < 1 ? c + n : (c > n ? c - n : c); };
  auto ghosted = [&](const double *p, int c) -> double {
    if (c < -1 || c > n + 2) return 0.0;
    if (c >= 1 && c <= n) return p[(long)(c - 1) * st];
    return PER ? p[(long)(wrap(c) - 1) * st] : 0.0;
  };
  auto V = [&](int c) -> double {
    const int cl = PER ? wrap(c) : (c < 1 ? 1 : (c > n ? n : c));
    double v = pv[(long)(cl - 1) * st];
    if (DIR == 2) v = v + pvf[(long)(cl + 1) * vf.sk];
    return v;
  };
  auto US = [&](int I) -> double {  // usig(I), zero outside [0, n+1]
    if (I < 0 || I > n + 1) return 0.0;
    return 0.5 * (V(I - 1) + V(I)) * gsig.at(I);
  };
  // d_fss, d_fsr, d_fsl of interface I
  auto iface = [&](int I, double &dfss, double &dfsr, double &dfsl) {
    const double us = US(I), usm = US(I - 1), usp = US(I + 1);
    dfss = 0.0;
    dfsr = 0.0;
    dfsl = 0.0;
    if (I < 0 || I > n + 1) return;
    const double qm2 = ghosted(pq, I - 2), qm1 = ghosted(pq, I - 1), q0 = ghosted(pq, I), qp1 = ghosted(pq, I + 1);
    const double dm2 = ghosted(pd, I - 2), dm1 = ghosted(pd, I - 1), d0 = ghosted(pd, I), dp1 = ghosted(pd, I + 1);
    const double dq = q0 - qm1, ddq = d0 - dm1;
    const bool up = us > 0.0;
    if (LIM != A3G_LIM_NONE && I >= 1 && (nocycle || !(fabs(dq) <= eps))) {
      const double dqu = up ? qm1 - qm2 : qp1 - q0;
      const double ddqu = up ? dm1 - dm2 : dp1 - d0;
      double a, b;
      lim_coef<LIM>(dq, dqu, eps, a, b);
      const double aus = fabs(us);
      const double cf = 0.5 * aus * (1.0 - gdtv.at(I) * aus);
      dfss = cf * (a * ddq + b * ddqu);
    }
    const double divm = fmn(0.0, usp) - fmn(0.0, us);
    const double divp = fmx(0.0, us) - fmx(0.0, usm);
    dfsr = fmx(0.0, us) * ddq + d0 * divm;
    dfsl = fmn(0.0, us) * ddq + dm1 * divp;
  };
  double fssL, fsrL, fslL, fssR, fsrR, fslR;
  iface(m, fssL, fsrL, fslL);
  iface(m + 1, fssR, fsrR, fslR);
  const double dupd = -(gdtv.at(m) * (fslR + fsrL + fssR - fssL));
  dout[gb + cell] = pd[(long)(m - 1) * st] + dupd;
  if (DIR == 2 && dep && m == 1) {  // cell 0 (the bottom outflow): interfaces 0 and 1, fss(0) = 0
    double fss0, fsr0, fsl0;
    iface(0, fss0, fsr0, fsl0);
    const double d0upd = -(gdtv.at(0) * (fslL + fsr0 + fssL - 0.0));
    dep[(long)g * L.nx * L.ny + (long)(j - 1) * L.nx + (i - 1)] += d0upd;
  }
}

template <int DIR, int LIM>
static void launch_tl_dir_lim(a3g_ctx *ctx, const double *cq, const double *din, double *dout, double *dep) {
  const Layout &L = ctx->L;
  dim3 grid((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz * L.ns);
  const bool per = (DIR == 0) && ctx->grid.periodic;
  const double *vel = (DIR == 0) ? ctx->vx : (DIR == 1) ? ctx->vy : ctx->vz;
  const Geo3 &sig = (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz;
  if (per)
    k_tl_advect<DIR, LIM, true><<<grid, dim3(32, 8), 0, ctx->stream>>>(
        L, ctx->prm.nocycle, ctx->prm.eps_thresh, cq, din, dout, vel, ctx->vf, sig, ctx->dtv, ctx->aloft, dep);
  else
    k_tl_advect<DIR, LIM, false><<<grid, dim3(32, 8), 0, ctx->stream>>>(
        L, ctx->prm.nocycle, ctx->prm.eps_thresh, cq, din, dout, vel, ctx->vf, sig, ctx->dtv, ctx->aloft, dep);
}

template <int DIR>
static void launch_tl_dir(a3g_ctx *ctx, const double *cq, const double *din, double *dout, double *dep) {
  switch (ctx->prm.limiter) {
    case A3G_LIM_NONE: launch_tl_dir_lim<DIR, A3G_LIM_NONE>(ctx, cq, din, dout, dep); break;
    case A3G_LIM_LAXWEN: launch_tl_dir_lim<DIR, A3G_LIM_LAXWEN>(ctx, cq, din, dout, dep); break;
    case A3G_LIM_BW: launch_tl_dir_lim<DIR, A3G_LIM_BW>(ctx, cq, din, dout, dep); break;
    case A3G_LIM_FROMM: launch_tl_dir_lim<DIR, A3G_LIM_FROMM>(ctx, cq, din, dout, dep); break;
    case A3G_LIM_MINMOD: launch_tl_dir_lim<DIR, A3G_LIM_MINMOD>(ctx, cq, din, dout, dep); break;
    case A3G_LIM_MC: launch_tl_dir_lim<DIR, A3G_LIM_MC>(ctx, cq, din, dout, dep); break;
    default: launch_tl_dir_lim<DIR, A3G_LIM_SUPERBEE>(ctx, cq, din, dout, dep); break;
  }
}

// dout <- J(cq) din for the advection sweep along dir; dep (z only, may be
// null) gains the perturbation of the bottom outflow.
int launch_tl_advect(a3g_ctx *ctx, int dir, const double *cq, const double *din, double *dout, double *dep) {
  int rc = refresh_dtv(ctx);
  if (rc) return rc;
  tbegin(ctx, A3G_K_ADJOINT);
  if (dir == 0) launch_tl_dir<0>(ctx, cq, din, dout, nullptr);
  else if (dir == 1) launch_tl_dir<1>(ctx, cq, din, dout, nullptr);
  else launch_tl_dir<2>(ctx, cq, din, dout, dep);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

}  // namespace a3g
