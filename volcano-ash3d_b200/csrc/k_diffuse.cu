// k_diffuse.cu -- explicit and Crank-Nicolson diffusion sweeps on the device.
//
// Explicit: diff_x/diff_y/diff_z, src/Diffusion.F90:266-650 (LeVeque eq. 4.11)
//   update(l) = dt*k_ds(l+1)*dq(l+1)*(sig(l+1)/kap(l)) - dt*k_ds(l)*dq(l)*(sig(l)/kap(l))
//   with k_ds = 0.5*(k_{l-1}+k_l) * 2*sig/(kap_{l-1}+kap_l) and Neumann ghosts
//   (periodic in x).  One thread per cell, all grains in a loop: the
//   grain-independent products dt*k_ds and sig/kap are formed once.
//
// Crank-Nicolson: diffCN_x/y/z, src/Diffusion.F90:671-1428 (eq. 4.13), each
// line solved by LAPACK dgtsv in the reference.  The matrices are strictly
// diagonally dominant (D >= 1, off-diagonals -Imp_fac*L <= 0), so dgtsv's
// partial pivoting never interchanges rows on them and its elimination
// reduces to: fact = DL(i)/D'(i); D'(i+1) = D(i+1) - fact*DU(i);
// B'(i+1) = B(i+1) - fact*B'(i); then x(n) = B'(n)/D'(n),
// x(i) = (B'(i) - DU(i)*x(i+1))/D'(i).  The factorisation (fact, D', DU) and
// the right-hand-side weights depend only on geometry, diffusivity and dt, so
// a per-step table holds them once per distinct line geometry (a projected
// grid has one per k) and the solve kernel runs one thread per (line, grain).
// A line that would need a row interchange (or a zero pivot) raises
// A3G_ERR_PIVOT instead of silently diverging from dgtsv.
#include "a3g_internal.cuh"
#include "exact_div.cuh"

namespace a3g {

// ---------------------------------------------------------------------------
// explicit diffusion
// ---------------------------------------------------------------------------
template <int DIR>
__global__ void __launch_bounds__(256) k_diff(Layout L, Box box, int periodic,
                                              const double *__restrict__ cin,
                                              double *__restrict__ cout, Geo3 sig, Geo3 kap,
                                              Geo3 kk, const int32_t *__restrict__ aloft,
                                              const DevScalars *__restrict__ sc) {
  const int i = blockIdx.x * 32 + threadIdx.x + 1;
  const int j = blockIdx.y * 8 + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > L.nx || j > L.ny) return;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int l = (DIR == 0) ? i : (DIR == 1) ? j : k;
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  const bool active = i >= box.imin && i <= box.imax && j >= box.jmin && j <= box.jmax &&
                      k >= box.kmin && k <= box.kmax;
  const long cell = L.cell(i, j, k);
  if (!active) {
    for (int g = 0; g < L.ns; g++) cout[(long)g * L.PG + cell] = 0.0;
    return;
  }
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? L.P : L.PY;
  auto G = [&](const Geo3 &a, int m) {
    return (DIR == 0) ? a.at(m, j, k) : (DIR == 1) ? a.at(i, m, k) : a.at(i, j, m);
  };
  const double dt = sc->dt;
  // interface l+1 (right) and l (left), :351-360
  const double dsR = 2.0 * G(sig, l + 1) / (G(kap, l) + G(kap, l + 1));
  const double kdsR = 0.5 * (G(kk, l) + G(kk, l + 1)) * dsR;
  const double dsL = 2.0 * G(sig, l) / (G(kap, l - 1) + G(kap, l));
  const double kdsL = 0.5 * (G(kk, l - 1) + G(kk, l)) * dsL;
  const double aR = dt * kdsR, aL = dt * kdsL;
  const double sR = G(sig, l + 1) / G(kap, l), sL = G(sig, l) / G(kap, l);
  // neighbour offsets with the Neumann (or periodic x) ghosts, :317-327
  long offL = -st, offR = st;
  bool selfL = false, selfR = false;
  if (l - 1 < 1) {
    if (DIR == 0 && periodic) offL = (long)(n - 1);
    else selfL = true;
  }
  if (l + 1 > n) {
    if (DIR == 0 && periodic) offR = -(long)(n - 1);
    else selfR = true;
  }
  for (int g = 0; g < L.ns; g++) {
    const long a = (long)g * L.PG + cell;
    if (!aloft[g]) { cout[a] = 0.0; continue; }
    const double q = cin[a];
    const double qL = selfL ? q : cin[a + offL];
    const double qR = selfR ? q : cin[a + offR];
    const double LF = aR * (qR - q) * sR;
    const double RF = -(aL * (q - qL) * sL);
    cout[a] = (l >= rmin && l <= rmax) ? q + (LF + RF) : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Crank-Nicolson line tables
// ---------------------------------------------------------------------------
// Table fields, stored [field][position][line] so that neighbouring lines
// (neighbouring threads) read neighbouring words.
// CN_RDP holds RN(1/D'), so that the back substitution's quotients can be
// formed by exact_div.cuh's certified path.
enum { CN_FACT = 0, CN_DP = 1, CN_DU = 2, CN_CL = 3, CN_CC = 4, CN_CR = 5, CN_RDP = 6, CN_NF = 7 };

struct LineMap {  // distinct-line indexing for one sweep direction
  int na, nb;     // extents of the two fixed indices (a fastest)
  int da, db;     // 1 if the coefficients vary with a / b
  int U;          // number of distinct lines
  __device__ __forceinline__ int u(int a, int b) const {
    return (da ? a - 1 : 0) + (da ? na : 1) * (db ? b - 1 : 0);
  }
};

template <int DIR>
__global__ void k_cn_table(Layout L, Box box, double imp, LineMap map, Geo3 sig, Geo3 kap, Geo3 kk,
                           DevScalars *sc, double *__restrict__ tab) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= map.U) return;
  // representative fixed indices of this distinct line
  const int amin = (DIR == 0) ? box.jmin : box.imin;
  const int bmin = (DIR == 2) ? box.jmin : box.kmin;
  const int na1 = map.da ? map.na : 1;
  const int a = map.da ? (u % na1) + 1 : amin;
  const int b = map.db ? (u / na1) + 1 : bmin;
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  auto G = [&](const Geo3 &g3, int m) {
    return (DIR == 0) ? g3.at(m, a, b) : (DIR == 1) ? g3.at(a, m, b) : g3.at(a, b, m);
  };
  const double dt = sc->dt;
  const long U = map.U;
  double dp_prev = 0.0, du_prev = 0.0;
  for (int l = 1; l <= ncells; l++) {
    const int c = rmin - 1 + l;
    // :794-801 and :809-811
    const double vavgL = 0.5 * (G(kap, c - 1) + G(kap, c));
    const double kavgL = 0.5 * (G(kk, c - 1) + G(kk, c));
    const double dsL = G(sig, c) / vavgL;
    const double kdsL = kavgL * dsL;
    const double vavgR = 0.5 * (G(kap, c) + G(kap, c + 1));
    const double kavgR = 0.5 * (G(kk, c) + G(kk, c + 1));
    const double dsR = G(sig, c + 1) / vavgR;
    const double kdsR = kavgR * dsR;
    const double Lf = dt * kdsL * G(sig, c) / G(kap, c);
    const double Rf = dt * kdsR * G(sig, c + 1) / G(kap, c);
    const double Cf = Lf + Rf;
    double D, DU = 0.0;
    if (l == 1) {
      D = 1.0 + imp * Cf - imp * Lf;
      DU = -(imp * Rf);
    } else if (l < ncells) {
      D = 1.0 + imp * Cf;
      DU = -(imp * Rf);
    } else {
      D = 1.0 + imp * Cf - imp * Rf;
    }
    double fact = 0.0, Dp = D;
    if (l > 1) {
      const double DL = -(imp * Lf);  // DL_d(l-1)
      if (!(fabs(dp_prev) >= fabs(DL)) || dp_prev == 0.0) raise_error(sc, A3G_ERR_PIVOT, l);
      fact = DL / dp_prev;
      Dp = D - fact * du_prev;
    }
    const long o = (long)(l - 1) * U + u;
    const long F = (long)ncells * U;
    tab[CN_FACT * F + o] = fact;
    tab[CN_DP * F + o] = Dp;
    tab[CN_DU * F + o] = DU;
    tab[CN_CL * F + o] = (1.0 - imp) * Lf;
    tab[CN_CC * F + o] = 1.0 - (1.0 - imp) * Cf;
    tab[CN_CR * F + o] = (1.0 - imp) * Rf;
    tab[CN_RDP * F + o] = 1.0 / Dp;
    dp_prev = Dp;
    du_prev = DU;
  }
  if (dp_prev == 0.0) raise_error(sc, A3G_ERR_PIVOT, ncells);
}

// Solve of one line (a, b) of grain g from the table.  The eliminated
// right-hand side B' is written to the output line and read back by the back
// substitution, which prefetches PF entries ahead (the loads cannot move
// above the stores to the same line on their own).
template <int DIR>
__device__ __forceinline__ void cn_line(const Layout &L, const Box &box, const LineMap &map,
                                        const double *__restrict__ cin, double *__restrict__ cout,
                                        const double *__restrict__ tab,
                                        const int32_t *__restrict__ aloft, int a, int b, int g) {
  constexpr int PF = 4;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  bool active;
  long base, st;
  if (DIR == 0) {
    active = a >= box.jmin && a <= box.jmax && b >= box.kmin && b <= box.kmax;
    base = L.cell(1, a, b); st = 1;
  } else if (DIR == 1) {
    active = a >= box.imin && a <= box.imax && b >= box.kmin && b <= box.kmax;
    base = L.cell(a, 1, b); st = L.P;
  } else {
    active = a >= box.imin && a <= box.imax && b >= box.jmin && b <= box.jmax;
    base = L.cell(a, b, 1); st = L.PY;
  }
  base += (long)g * L.PG;
  const double *q = cin + base;
  double *x = cout + base;
  if (!active || !aloft[g]) {
    for (int c = 1; c <= n; c++) x[(long)(c - 1) * st] = 0.0;
    return;
  }
  for (int c = 1; c < rmin; c++) x[(long)(c - 1) * st] = 0.0;
  for (int c = rmax + 1; c <= n; c++) x[(long)(c - 1) * st] = 0.0;
  const long U = map.U;
  const long F = (long)ncells * U;
  const double *t = tab + map.u(a, b);
  const double *qq = q + (long)(rmin - 1) * st;  // cell rmin
  double *xx = x + (long)(rmin - 1) * st;
  // forward elimination with the right-hand side built on the fly, :813-851
  double qm = qq[0];  // BC_left_t0 = q(rmin)
  double qc = qm;
  double bp = 0.0;
#pragma unroll 4
  for (int l = 0; l < ncells; l++) {
    const double qp = (l + 1 < ncells) ? qq[(long)(l + 1) * st] : qc;  // BC_right_t0 = q(rmax)
    const long o = (long)l * U;
    const double B = t[CN_CL * F + o] * qm + t[CN_CC * F + o] * qc + t[CN_CR * F + o] * qp;
    bp = (l == 0) ? B : B - t[CN_FACT * F + o] * bp;
    xx[(long)l * st] = bp;
    qm = qc;
    qc = qp;
  }
  // back substitution with a PF-deep prefetch of B'
  double ring[PF];
#pragma unroll
  for (int p = 0; p < PF; p++) ring[p] = (ncells - 1 - p >= 0) ? xx[(long)(ncells - 1 - p) * st] : 0.0;
  double xn = 0.0;
  for (int l0 = ncells - 1; l0 >= 0; l0 -= PF) {
#pragma unroll
    for (int p = 0; p < PF; p++) {
      const int l = l0 - p;
      if (l >= 0) {
        const double b2 = ring[p];
        const int lp = l - PF;  // refill this slot for the next round
        ring[p] = (lp >= 0) ? xx[(long)lp * st] : 0.0;
        const long o = (long)l * U;
        const double num = (l == ncells - 1) ? b2 : b2 - t[CN_DU * F + o] * xn;
        const double v = div_rn_rcp(num, t[CN_DP * F + o], t[CN_RDP * F + o]);
        xx[(long)l * st] = v;
        xn = v;
      }
    }
  }
}

// Solve kernel: one thread per line (a, b, grain), lines enumerated with a
// fastest so that a warp holds neighbouring lines (neighbouring i for y and
// z lines: coalesced; neighbouring rows for x lines).
template <int DIR>
__global__ void __launch_bounds__(128) k_cn_solve(Layout L, Box box, LineMap map,
                                                  const double *__restrict__ cin,
                                                  double *__restrict__ cout,
                                                  const double *__restrict__ tab,
                                                  const int32_t *__restrict__ aloft) {
  const int na = (DIR == 0) ? L.ny : L.nx;
  const int nb = (DIR == 2) ? L.ny : L.nz;
  const long nlines = (long)na * nb * L.ns;
  const long w = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (w >= nlines) return;
  const int a = (int)(w % na) + 1;
  const long r = w / na;
  const int b = (int)(r % nb) + 1;
  const int g = (int)(r / nb);
  cn_line<DIR>(L, box, map, cin, cout, tab, aloft, a, b, g);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int DIR>
static int launch_diff_dir(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const Geo3 &sig = (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz;
  const Geo3 &kk = (DIR == 0) ? ctx->kx : (DIR == 1) ? ctx->ky : ctx->kz;
  dim3 grid((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz);
  tbegin(ctx, A3G_K_DIFF_X + DIR);
  k_diff<DIR><<<grid, dim3(32, 8), 0, ctx->stream>>>(L, ctx->box, ctx->grid.periodic, ctx->c0,
                                                     ctx->c1, sig, ctx->kappa, kk, ctx->aloft,
                                                     ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  return A3G_OK;
}

int launch_diff_x(a3g_ctx *ctx) { return launch_diff_dir<0>(ctx); }
int launch_diff_y(a3g_ctx *ctx) { return launch_diff_dir<1>(ctx); }
int launch_diff_z(a3g_ctx *ctx) { return launch_diff_dir<2>(ctx); }

static inline bool varies(const Geo3 &g, int idx) {  // idx 0:i 1:j 2:k
  return (idx == 0 ? g.si : idx == 1 ? g.sj : g.sk) != 0;
}

size_t cn_table_doubles(const a3g_ctx *ctx, int dir) {
  const Layout &L = ctx->L;
  const Geo3 &sig = (dir == 0) ? ctx->snx : (dir == 1) ? ctx->sny : ctx->snz;
  const Geo3 &kk = (dir == 0) ? ctx->kx : (dir == 1) ? ctx->ky : ctx->kz;
  const int ia = (dir == 0) ? 1 : 0, ib = (dir == 2) ? 1 : 2;
  const int na = (dir == 0) ? L.ny : L.nx, nb = (dir == 2) ? L.ny : L.nz;
  const bool da = varies(ctx->kappa, ia) || varies(sig, ia) || varies(kk, ia);
  const bool db = varies(ctx->kappa, ib) || varies(sig, ib) || varies(kk, ib);
  const size_t n = (dir == 0) ? L.nx : (dir == 1) ? L.ny : L.nz;
  return (size_t)CN_NF * n * (size_t)(da ? na : 1) * (size_t)(db ? nb : 1);
}

template <int DIR>
static int launch_cn_dir(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const Box &box = ctx->box;
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  if (rmax - rmin + 1 <= 1) {
    // :770 skips the solve and the copy-back; ts1 stays zero.
    ctx->ts1_zeroed = true;
    return A3G_OK;
  }
  const Geo3 &sig = (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz;
  const Geo3 &kk = (DIR == 0) ? ctx->kx : (DIR == 1) ? ctx->ky : ctx->kz;
  const int ia = (DIR == 0) ? 1 : 0, ib = (DIR == 2) ? 1 : 2;
  LineMap map;
  map.na = (DIR == 0) ? L.ny : L.nx;
  map.nb = (DIR == 2) ? L.ny : L.nz;
  map.da = varies(ctx->kappa, ia) || varies(sig, ia) || varies(kk, ia);
  map.db = varies(ctx->kappa, ib) || varies(sig, ib) || varies(kk, ib);
  map.U = (map.da ? map.na : 1) * (map.db ? map.nb : 1);
  tbegin(ctx, A3G_K_CN_TABLE);
  k_cn_table<DIR><<<(map.U + 127) / 128, 128, 0, ctx->stream>>>(L, box, ctx->prm.imp_fac, map, sig,
                                                                ctx->kappa, kk, ctx->sc, ctx->cn_buf);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  const long nlines = (long)map.na * map.nb * L.ns;
  tbegin(ctx, A3G_K_CN_SOLVE_X + DIR);
  k_cn_solve<DIR><<<(unsigned)((nlines + 127) / 128), 128, 0, ctx->stream>>>(
      L, box, map, ctx->c0, ctx->c1, ctx->cn_buf, ctx->aloft);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  ctx->ts1_zeroed = false;
  return A3G_OK;
}

int launch_diffcn_x(a3g_ctx *ctx) { return launch_cn_dir<0>(ctx); }
int launch_diffcn_y(a3g_ctx *ctx) { return launch_cn_dir<1>(ctx); }
int launch_diffcn_z(a3g_ctx *ctx) { return launch_cn_dir<2>(ctx); }

}  // namespace a3g
