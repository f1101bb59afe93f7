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
#include "tma.cuh"

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

// Constant runs.  Along a line whose geometry and diffusivity do not change
// (every x line of a lon/lat grid, every line of a projected grid with
// uniform spacing) the interior rows of the matrix are identical, and the
// elimination factors of dgtsv settle to a fixed point after a few rows, so
// the table rows become bit-identical.  Per distinct line the table keeps the
// run [lo, hi] of identical rows that ends at the last interior row
// (hi = ncells-2): row lo is stored, rows lo+1..hi are not, and readers take
// them from registers.  The values are the same bits either way.  The run
// bounds follow the CN_NF fields: [2][U] doubles holding lo and hi.
struct CnRun {
  int lo, hi;
  double v[CN_NF];
};

__device__ __forceinline__ void cn_load_run(const double *__restrict__ t, long F, long U,
                                            const double *__restrict__ runs, long u, CnRun &R) {
  R.lo = (int)runs[u];
  R.hi = (int)runs[U + u];
#pragma unroll
  for (int f = 0; f < CN_NF; f++) R.v[f] = t[f * F + (long)R.lo * U];
}

// Field f of row l: from the run registers inside (lo, hi], else from the table.
__device__ __forceinline__ double cn_coef(const double *__restrict__ t, long F, long U, const CnRun &R,
                                          int f, int l) {
  return (l > R.lo && l <= R.hi) ? R.v[f] : t[f * F + (long)l * U];
}

struct LineMap {  // distinct-line indexing for one sweep direction
  int na, nb;     // extents of the two fixed indices (a fastest)
  int da, db;     // 1 if the coefficients vary with a / b
  int U;          // number of distinct lines
  __host__ __device__ __forceinline__ int u(int a, int b) const {
    return (da ? a - 1 : 0) + (da ? na : 1) * (db ? b - 1 : 0);
  }
};

__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}

// Only the x tables (read by the warp-tiled x solve) leave their final run
// unstored; the y and z tables are written in full, because their solves
// read every row.
template <int DIR>
__global__ void k_cn_table(Layout L, Box box, double imp, LineMap map, Geo3 sig, Geo3 kap, Geo3 kk,
                           DevScalars *sc, const double *__restrict__ cstate, double *__restrict__ tab) {
  constexpr bool COMPRESS = (DIR == 0);
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= map.U) return;
  if (cstate[3 + DIR] != 0.0) return;  // the table already holds this dt's factors
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
  const long F = (long)ncells * U;
  auto put = [&](int l, const double *v) {
#pragma unroll
    for (int f = 0; f < CN_NF; f++) tab[f * F + (long)l * U + u] = v[f];
  };
  double dp_prev = 0.0, du_prev = 0.0;
  double rv[CN_NF];   // first row of the current run
  int s = 0;          // index of that row
  bool cont = false;  // row l-1 repeated row l-2
  double pin[8];      // inputs of row l-1
  for (int l = 0; l < ncells - 1; l++) {
    const int c = rmin + l;
    const double in[8] = {G(kap, c - 1), G(kap, c), G(kap, c + 1), G(kk, c - 1),
                          G(kk, c),      G(kk, c + 1), G(sig, c),   G(sig, c + 1)};
    bool same_in = l >= 2;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      if (l >= 2) same_in = same_in && same_bits(in[e], pin[e]);
      pin[e] = in[e];
    }
    // an interior row with the inputs and the carried (D', DU) of its
    // predecessor repeats it: nothing to compute or store
    if (cont && same_in) {
      if (!COMPRESS) put(l, rv);
      continue;
    }
    // :794-801 and :809-811
    const double vavgL = 0.5 * (in[0] + in[1]);
    const double kavgL = 0.5 * (in[3] + in[4]);
    const double dsL = in[6] / vavgL;
    const double kdsL = kavgL * dsL;
    const double vavgR = 0.5 * (in[1] + in[2]);
    const double kavgR = 0.5 * (in[4] + in[5]);
    const double dsR = in[7] / vavgR;
    const double kdsR = kavgR * dsR;
    const double Lf = dt * kdsL * in[6] / in[1];
    const double Rf = dt * kdsR * in[7] / in[1];
    const double Cf = Lf + Rf;
    double D, DU = 0.0;
    if (l == 0) {
      D = 1.0 + imp * Cf - imp * Lf;
      DU = -(imp * Rf);
    } else {
      D = 1.0 + imp * Cf;
      DU = -(imp * Rf);
    }
    double fact = 0.0, Dp = D;
    if (l > 0) {
      const double DL = -(imp * Lf);  // DL_d(l-1)
      if (!(fabs(dp_prev) >= fabs(DL)) || dp_prev == 0.0) raise_error(sc, A3G_ERR_PIVOT, l + 1);
      fact = DL / dp_prev;
      Dp = D - fact * du_prev;
    }
    const double v[CN_NF] = {fact, Dp, DU, (1.0 - imp) * Lf, 1.0 - (1.0 - imp) * Cf, (1.0 - imp) * Rf,
                             1.0 / Dp};
    bool same = l >= 1;
#pragma unroll
    for (int f = 0; f < CN_NF; f++) same = same && same_bits(v[f], rv[f]);
    cont = same;
    dp_prev = Dp;
    du_prev = DU;
    if (same) {
      if (!COMPRESS) put(l, rv);
      continue;
    }
    if (COMPRESS)
      for (int m = s + 1; m < l; m++) put(m, rv);  // materialise the finished run
    put(l, v);
#pragma unroll
    for (int f = 0; f < CN_NF; f++) rv[f] = v[f];
    s = l;
  }
  // last row (always distinct: DU = 0); the run ending at ncells-2 stays unstored
  {
    const int l = ncells - 1;
    const int c = rmin + l;
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
    const double D = 1.0 + imp * Cf - imp * Rf;
    const double DL = -(imp * Lf);
    if (!(fabs(dp_prev) >= fabs(DL)) || dp_prev == 0.0) raise_error(sc, A3G_ERR_PIVOT, l + 1);
    const double fact = DL / dp_prev;
    const double Dp = D - fact * du_prev;
    if (Dp == 0.0) raise_error(sc, A3G_ERR_PIVOT, ncells);
    const double v[CN_NF] = {fact, Dp, 0.0, (1.0 - imp) * Lf, 1.0 - (1.0 - imp) * Cf, (1.0 - imp) * Rf,
                             1.0 / Dp};
    put(l, v);
    double *runs = tab + CN_NF * F;
    runs[u] = (double)s;
    runs[U + u] = (double)(ncells - 2);
  }
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
  const long u = map.u(a, b);
  const double *t = tab + u;
  CnRun R;
  if (DIR == 0) cn_load_run(t, F, U, tab + CN_NF * F, u, R);
  auto co = [&](int f, int l) {  // the y and z tables are stored in full
    return (DIR == 0) ? cn_coef(t, F, U, R, f, l) : t[f * F + (long)l * U];
  };
  const double *qq = q + (long)(rmin - 1) * st;  // cell rmin
  double *xx = x + (long)(rmin - 1) * st;
  // forward elimination with the right-hand side built on the fly, :813-851
  double qm = qq[0];  // BC_left_t0 = q(rmin)
  double qc = qm;
  double bp = 0.0;
#pragma unroll 4
  for (int l = 0; l < ncells; l++) {
    const double qp = (l + 1 < ncells) ? qq[(long)(l + 1) * st] : qc;  // BC_right_t0 = q(rmax)
    const double B = co(CN_CL, l) * qm + co(CN_CC, l) * qc +
                     co(CN_CR, l) * qp;
    bp = (l == 0) ? B : B - co(CN_FACT, l) * bp;
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
        const double num = (l == ncells - 1) ? b2 : b2 - co(CN_DU, l) * xn;
        const double v = div_rn_rcp(num, co(CN_DP, l), co(CN_RDP, l));
        xx[(long)l * st] = v;
        xn = v;
      }
    }
  }
}

// y and z lines, GC grains of one line per thread: the factor-table row is
// the same for every grain, so its loads are shared, and the GC recurrences
// are independent chains the scheduler interleaves.  Same operations per
// grain as cn_line.
template <int DIR, int GC>
__device__ __forceinline__ void cn_line_gc(const Layout &L, const Box &box, const LineMap &map,
                                           const double *__restrict__ cin, double *__restrict__ cout,
                                           const double *__restrict__ tab,
                                           const int32_t *__restrict__ aloft, int a, int b, int g0) {
  constexpr int PF = 4;
  const int n = (DIR == 1) ? L.ny : L.nz;
  const int rmin = (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  bool active;
  long base, st;
  if (DIR == 1) {
    active = a >= box.imin && a <= box.imax && b >= box.kmin && b <= box.kmax;
    base = L.cell(a, 1, b); st = L.P;
  } else {
    active = a >= box.imin && a <= box.imax && b >= box.jmin && b <= box.jmax;
    base = L.cell(a, b, 1); st = L.PY;
  }
  const double *q[GC];
  double *x[GC];
  bool on[GC], any = false;
#pragma unroll
  for (int u = 0; u < GC; u++) {
    const int g = g0 + u < L.ns ? g0 + u : L.ns - 1;
    q[u] = cin + base + (long)g * L.PG;
    x[u] = cout + base + (long)g * L.PG;
    on[u] = g0 + u < L.ns && active && aloft[g] != 0;
    any = any || on[u];
    if (g0 + u < L.ns && !on[u])
      for (int c = 1; c <= n; c++) x[u][(long)(c - 1) * st] = 0.0;
    else if (on[u]) {
      for (int c = 1; c < rmin; c++) x[u][(long)(c - 1) * st] = 0.0;
      for (int c = rmax + 1; c <= n; c++) x[u][(long)(c - 1) * st] = 0.0;
    }
  }
  if (!any) return;
  const long U = map.U;
  const long F = (long)ncells * U;
  const double *t = tab + map.u(a, b);
  auto co = [&](int f, int l) { return t[f * F + (long)l * U]; };
  const long off = (long)(rmin - 1) * st;
  // forward elimination with the right-hand side built on the fly, :813-851
  double qm[GC], qc[GC], bp[GC];
#pragma unroll
  for (int u = 0; u < GC; u++) {
    qm[u] = on[u] ? q[u][off] : 0.0;  // BC_left_t0 = q(rmin)
    qc[u] = qm[u];
    bp[u] = 0.0;
  }
#pragma unroll 4
  for (int l = 0; l < ncells; l++) {
    const double cl = co(CN_CL, l), cc = co(CN_CC, l), cr = co(CN_CR, l), fa = co(CN_FACT, l);
#pragma unroll
    for (int u = 0; u < GC; u++) {
      const double qp = (l + 1 < ncells) ? (on[u] ? q[u][off + (long)(l + 1) * st] : 0.0) : qc[u];
      const double B = cl * qm[u] + cc * qc[u] + cr * qp;
      bp[u] = (l == 0) ? B : B - fa * bp[u];
      if (on[u]) x[u][off + (long)l * st] = bp[u];
      qm[u] = qc[u];
      qc[u] = qp;
    }
  }
  // back substitution with a PF-deep prefetch of B'
  double ring[GC][PF];
#pragma unroll
  for (int u = 0; u < GC; u++)
#pragma unroll
    for (int p = 0; p < PF; p++)
      ring[u][p] = (on[u] && ncells - 1 - p >= 0) ? x[u][off + (long)(ncells - 1 - p) * st] : 0.0;
  double xn[GC];
#pragma unroll
  for (int u = 0; u < GC; u++) xn[u] = 0.0;
  for (int l0 = ncells - 1; l0 >= 0; l0 -= PF) {
#pragma unroll
    for (int p = 0; p < PF; p++) {
      const int l = l0 - p;
      if (l >= 0) {
        const int lp = l - PF;
        const double du = co(CN_DU, l), dp = co(CN_DP, l), rd = co(CN_RDP, l);
#pragma unroll
        for (int u = 0; u < GC; u++) {
          const double b2 = ring[u][p];
          ring[u][p] = (on[u] && lp >= 0) ? x[u][off + (long)lp * st] : 0.0;
          const double num = (l == ncells - 1) ? b2 : b2 - du * xn[u];
          const double v = div_rn_rcp(num, dp, rd);
          if (on[u]) x[u][off + (long)l * st] = v;
          xn[u] = v;
        }
      }
    }
  }
}

template <int DIR, int GC>
__device__ __forceinline__ void cn_solve_gc_thread(const Layout &L, const Box &box, const LineMap &map,
                                                   const double *__restrict__ cin,
                                                   double *__restrict__ cout,
                                                   const double *__restrict__ tab,
                                                   const int32_t *__restrict__ aloft) {
  const int na = L.nx;
  const int nb = (DIR == 2) ? L.ny : L.nz;
  const int ngr = (L.ns + GC - 1) / GC;
  const long nlines = (long)na * nb * ngr;
  const long w = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (w >= nlines) return;
  const int a = (int)(w % na) + 1;
  const long r = w / na;
  const int b = (int)(r % nb) + 1;
  const int gg = (int)(r / nb);
  cn_line_gc<DIR, GC>(L, box, map, cin, cout, tab, aloft, a, b, gg * GC);
}

// z lines: unconstrained registers (64-96, no spills) measured fastest; an
// 8-blocks-per-SM bound slowed the C2 z solve 1.29 -> 1.37 ms on B200.
template <int DIR, int GC>
__global__ void __launch_bounds__(128) k_cn_solve_gc(Layout L, Box box, LineMap map,
                                                     const double *__restrict__ cin,
                                                     double *__restrict__ cout,
                                                     const double *__restrict__ tab,
                                                     const int32_t *__restrict__ aloft) {
  cn_solve_gc_thread<DIR, GC>(L, box, map, cin, cout, tab, aloft);
}

// y lines: 12 blocks of 128 per SM (at most 40 registers, some spilled to
// L1) hide the strided dependent loads better (C2 1.76 -> 1.62 ms on B200).
template <int GC>
__global__ void __launch_bounds__(128, 12) k_cn_solve_gc_y(Layout L, Box box, LineMap map,
                                                           const double *__restrict__ cin,
                                                           double *__restrict__ cout,
                                                           const double *__restrict__ tab,
                                                           const int32_t *__restrict__ aloft) {
  cn_solve_gc_thread<1, GC>(L, box, map, cin, cout, tab, aloft);
}

template <int DIR, int GC>
static void launch_cn_solve_gc(a3g_ctx *ctx, const LineMap &map, const double *tab) {
  const Layout &L = ctx->L;
  const long n = (long)map.na * map.nb * ((L.ns + GC - 1) / GC);
  const unsigned grid = (unsigned)((n + 127) / 128);
  if constexpr (DIR == 1)
    k_cn_solve_gc_y<GC><<<grid, 128, 0, ctx->stream>>>(L, ctx->box, map, ctx->c0, ctx->c1, tab, ctx->aloft);
  else
    k_cn_solve_gc<DIR, GC><<<grid, 128, 0, ctx->stream>>>(L, ctx->box, map, ctx->c0, ctx->c1, tab, ctx->aloft);
}

// Solve kernel: one thread per line (a, b, grain), lines enumerated with a
// fastest so that a warp holds neighbouring lines (neighbouring i for y and
// z lines: coalesced loads and stores).
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

// x lines, warp-tiled.  A warp owns 32 consecutive x rows (row r =
// (g*nz + k-1)*ny + j-1 starts at r*P) and walks them in chunks of 32 cells
// through a shared-memory tile: every global load and store of the
// concentration is a coalesced 256-byte row segment, and each lane then runs
// its own row's recurrence out of the tile.
//   pass 1 (forward): the elimination of B' over the whole row, keeping only
//     B' at the last cell of every chunk (a checkpoint, parked in the output
//     row at that cell);
//   pass 2 (backward, last chunk first): reload the chunk, recompute its B'
//     from the checkpoint of the previous chunk (same operations, same bits),
//     back-substitute, store the chunk.
// Against writing B' out and reading it back this moves one read of the
// input in place of a write and a read of B'.
constexpr int XT_WARPS = 4;
constexpr int XT_S = 35;  // tile row stride in doubles: 34 columns, odd stride

__global__ void __launch_bounds__(128, 5) k_cn_solve_xt(Layout L, Box box, LineMap map,
                                                     const double *__restrict__ cin,
                                                     double *__restrict__ cout,
                                                     const double *__restrict__ tab,
                                                     const int32_t *__restrict__ aloft) {
  __shared__ double sh[XT_WARPS][32 * XT_S];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *tile = sh[w];
  const long nrows = (long)L.ny * L.nz * L.ns;
  const long r0 = ((long)blockIdx.x * XT_WARPS + w) * 32;
  if (r0 >= nrows) return;  // uniform over the warp
  const long r = r0 + lane;
  const bool valid = r < nrows;
  const long rc = valid ? r : nrows - 1;
  const int j = (int)(rc % L.ny) + 1;
  const long t1 = rc / L.ny;
  const int k = (int)(t1 % L.nz) + 1;
  const int g = (int)(t1 / L.nz);
  const bool active =
      valid && j >= box.jmin && j <= box.jmax && k >= box.kmin && k <= box.kmax && aloft[g] != 0;
  const unsigned amask = __ballot_sync(0xffffffffu, active);
  const int nvalid = (int)((nrows - r0) < 32 ? (nrows - r0) : 32);
  const int rmin = box.imin, rmax = box.imax;
  const int ncells = rmax - rmin + 1;
  const long P = L.P;
  if (valid) {  // cells outside [rmin, rmax] (FAST_SUBGRID box)
    double *xr = cout + r * P;
    for (int c = 1; c < rmin; c++) xr[c - 1] = 0.0;
    for (int c = rmax + 1; c <= L.nx; c++) xr[c - 1] = 0.0;
  }
  const double *q0 = cin + r0 * P + (rmin - 1);  // row r0, cell rmin
  double *x0 = cout + r0 * P + (rmin - 1);
  const double *qown = q0 + (long)lane * P;
  double *xown = x0 + (long)lane * P;
  const long U = map.U;
  const long F = (long)ncells * U;
  const long u = map.u(j, k);
  const double *t = tab + u;
  CnRun R;
  cn_load_run(t, F, U, tab + CN_NF * F, u, R);
  double *tr = tile + lane * XT_S;  // this lane's row of the tile
  const int nch = (ncells + 31) >> 5;

  // tile columns: 0 = cell l0-1, 1..32 = cells l0..l0+31, 33 = cell l0+32
  auto load_tile = [&](int l0, int cnt) {
#pragma unroll
    for (int h = 0; h < 32; h += 8) {
      double v[8];
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int row = h + e;
        v[e] = (row < nvalid && lane < cnt) ? q0[(long)row * P + l0 + lane] : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 8; e++) tile[(h + e) * XT_S + 1 + lane] = v[e];
    }
    tr[0] = (valid && l0 > 0) ? qown[l0 - 1] : 0.0;
    tr[33] = (valid && l0 + 32 < ncells) ? qown[l0 + 32] : 0.0;
    __syncwarp();
  };

  // A chunk whose rows all lie inside every lane's constant run (rows
  // lo_w+1 .. ncells-2, lo_w the warp's largest lo) takes its coefficients
  // from registers with no per-row test: the fast path.
  int lo_w = R.lo;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lo_w = max(lo_w, __shfl_xor_sync(0xffffffffu, lo_w, o));
  auto fast_chunk = [&](int l0, int cnt) { return cnt == 32 && l0 > lo_w && l0 + 31 <= ncells - 2; };
  const double fCL = R.v[CN_CL], fCC = R.v[CN_CC], fCR = R.v[CN_CR], fFA = R.v[CN_FACT];
  const double fDU = R.v[CN_DU], fDP = R.v[CN_DP], fRD = R.v[CN_RDP];

  // pass 1: forward elimination, checkpoints only (:813-851 and dgtsv)
  double qm = 0.0, qc = 0.0, bp = 0.0;
  for (int ch = 0; ch < nch; ch++) {
    const int l0 = ch << 5;
    const int cnt = (ncells - l0) < 32 ? (ncells - l0) : 32;
    load_tile(l0, cnt);
    if (ch == 0) {
      qm = tr[1];  // BC_left_t0 = q(rmin)
      qc = qm;
    }
    if (fast_chunk(l0, cnt)) {  // rows l0..l0+31 < ncells-1: qp always from the tile
#pragma unroll 8
      for (int c = 0; c < 32; c++) {
        const double qp = tr[c + 2];
        const double B = fCL * qm + fCC * qc + fCR * qp;
        bp = B - fFA * bp;
        qm = qc;
        qc = qp;
      }
      if (valid && ch + 1 < nch) xown[l0 + 31] = bp;
      __syncwarp();
      continue;
    }
    for (int c = 0; c < cnt; c++) {
      const int l = l0 + c;
      const double qp = (l + 1 < ncells) ? tr[c + 2] : qc;  // BC_right_t0 = q(rmax)
      const double B = cn_coef(t, F, U, R, CN_CL, l) * qm + cn_coef(t, F, U, R, CN_CC, l) * qc +
                       cn_coef(t, F, U, R, CN_CR, l) * qp;
      bp = (l == 0) ? B : B - cn_coef(t, F, U, R, CN_FACT, l) * bp;
      qm = qc;
      qc = qp;
    }
    if (valid && ch + 1 < nch) xown[l0 + 31] = bp;  // checkpoint B'(l0+31)
    __syncwarp();
  }

  // pass 2: per chunk, last first: recompute B', back-substitute, store
  double xn = 0.0;
  for (int ch = nch - 1; ch >= 0; ch--) {
    const int l0 = ch << 5;
    const int cnt = (ncells - l0) < 32 ? (ncells - l0) : 32;
    load_tile(l0, cnt);
    double bq = (valid && ch > 0) ? xown[l0 - 1] : 0.0;
    double qm2 = (ch == 0) ? tr[1] : tr[0];
    double qc2 = tr[1];
    if (fast_chunk(l0, cnt)) {
#pragma unroll 8
      for (int c = 0; c < 32; c++) {
        const double qp = tr[c + 2];
        const double B = fCL * qm2 + fCC * qc2 + fCR * qp;
        bq = B - fFA * bq;
        tr[c + 1] = bq;
        qm2 = qc2;
        qc2 = qp;
      }
#pragma unroll 8
      for (int c = 31; c >= 0; c--) {
        const double num = tr[c + 1] - fDU * xn;
        const double v = div_rn_rcp(num, fDP, fRD);
        tr[c + 1] = v;
        xn = v;
      }
    } else {
    for (int c = 0; c < cnt; c++) {
      const int l = l0 + c;
      const double qp = (l + 1 < ncells) ? tr[c + 2] : qc2;
      const double B = cn_coef(t, F, U, R, CN_CL, l) * qm2 + cn_coef(t, F, U, R, CN_CC, l) * qc2 +
                       cn_coef(t, F, U, R, CN_CR, l) * qp;
      bq = (l == 0) ? B : B - cn_coef(t, F, U, R, CN_FACT, l) * bq;
      tr[c + 1] = bq;
      qm2 = qc2;
      qc2 = qp;
    }
    for (int c = cnt - 1; c >= 0; c--) {
      const int l = l0 + c;
      const double b2 = tr[c + 1];
      const double num = (l == ncells - 1) ? b2 : b2 - cn_coef(t, F, U, R, CN_DU, l) * xn;
      const double v = div_rn_rcp(num, cn_coef(t, F, U, R, CN_DP, l), cn_coef(t, F, U, R, CN_RDP, l));
      tr[c + 1] = v;
      xn = v;
    }
    }
    __syncwarp();
#pragma unroll 8
    for (int row = 0; row < 32; row++) {
      if (row < nvalid && lane < cnt)
        x0[(long)row * P + l0 + lane] = ((amask >> row) & 1u) ? tile[row * XT_S + 1 + lane] : 0.0;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// x lines, warp-tiled, with TMA tiles.  The walk of k_cn_solve_xt (a warp
// owns 32 consecutive x rows, chunks of 32 cells, checkpoints of B' in pass
// 1, recompute and back substitution in pass 2; the same operations and the
// same bits), but each chunk's tile arrives by one tensor load of 36 cells x
// 32 rows (the rows of a level are a 2-D array of pitch P) into a dense
// staging buffer, one chunk ahead: the lanes copy it into the odd-stride
// tile (conflict-free per-lane rows), and the next chunk's load then runs
// while they work through the current one.  The load starts on the even
// cell at or before the chunk's left neighbour (the 16-byte rule for the
// innermost coordinate); cells outside the level read as zero.
// Chunks are loaded in the order the two passes use them (0 .. nch-1, then
// nch-2 .. 0): the last chunk of pass 1 is still in the tile for pass 2.
// ---------------------------------------------------------------------------
constexpr int ZT_BAR_BYTES = 128;  // barriers ahead of the tiles (keeps tiles 128-byte aligned)
constexpr int XT2_WARPS = 2;
constexpr int XT2_DENSE = 32 * XT2_COLS;             // doubles of the staging buffer
constexpr int XT2_WARP_D = XT2_DENSE + 32 * XT_S;    // staging buffer + tile
static_assert((XT2_DENSE * 8) % 128 == 0 && (XT2_WARP_D * 8) % 128 == 0, "128-byte aligned buffers");

__global__ void __launch_bounds__(32 * XT2_WARPS) k_cn_solve_xt2(const __grid_constant__ CUtensorMap trow,
                                                                Layout L, Box box, LineMap map,
                                                                const double *__restrict__ cin,
                                                                double *__restrict__ cout,
                                                                const double *__restrict__ tab,
                                                                const int32_t *__restrict__ aloft,
                                                                DevScalars *sc) {
  extern __shared__ __align__(128) unsigned char x2_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t *bar = reinterpret_cast<uint64_t *>(x2_smem) + w;
  double *dense = reinterpret_cast<double *>(x2_smem + ZT_BAR_BYTES) + (long)w * XT2_WARP_D;
  double *tile = dense + XT2_DENSE;
  const long nrows = (long)L.ny * L.nz * L.ns;
  const long r0 = ((long)blockIdx.x * XT2_WARPS + w) * 32;
  if (r0 >= nrows) return;  // uniform over the warp
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  __syncwarp();
  const long r = r0 + lane;
  const bool valid = r < nrows;
  const long rc = valid ? r : nrows - 1;
  const int j = (int)(rc % L.ny) + 1;
  const long t1 = rc / L.ny;
  const int k = (int)(t1 % L.nz) + 1;
  const int g = (int)(t1 / L.nz);
  const bool active =
      valid && j >= box.jmin && j <= box.jmax && k >= box.kmin && k <= box.kmax && aloft[g] != 0;
  const unsigned amask = __ballot_sync(0xffffffffu, active);
  const int nvalid = (int)((nrows - r0) < 32 ? (nrows - r0) : 32);
  const int rmin = box.imin, rmax = box.imax;
  const int ncells = rmax - rmin + 1;
  const long P = L.P;
  if (valid) {  // cells outside [rmin, rmax] (FAST_SUBGRID box)
    double *xr = cout + r * P;
    for (int c = 1; c < rmin; c++) xr[c - 1] = 0.0;
    for (int c = rmax + 1; c <= L.nx; c++) xr[c - 1] = 0.0;
  }
  double *x0 = cout + r0 * P + (rmin - 1);
  double *xown = x0 + (long)lane * P;
  const long U = map.U;
  const long F = (long)ncells * U;
  const long u = map.u(j, k);
  const double *t = tab + u;
  CnRun R;
  cn_load_run(t, F, U, tab + CN_NF * F, u, R);
  double *tr = tile + lane * XT_S;  // this lane's row of the tile
  const int nch = (ncells + 31) >> 5;
  const int nload = 2 * nch - 1;  // chunks 0 .. nch-1, then nch-2 .. 0
  auto chunk_of = [&](int p) { return p < nch ? p : 2 * nch - 2 - p; };
  // tile columns: 0 = cell l0-1, 1..32 = cells l0..l0+31, 33 = cell l0+32;
  // cell l0-1 is line position l0-1, 0-based x = rmin + l0 - 2
  auto issue = [&](int p) {
    if (lane == 0) {
      const int xa = rmin + (chunk_of(p) << 5) - 2;
      mbar_arrive_expect_tx(bar, XT2_DENSE * 8);
      tma_load_2d(dense, &trow, bar, xa & ~1, (int)r0);
    }
  };
  uint32_t phase = 0u;
  bool ok = true;
  // waits for load p, copies it into the tile, then starts load p+1
  auto next_tile = [&](int p) {
    if (!mbar_wait(bar, phase)) {
      ok = false;
      return;
    }
    phase ^= 1u;
    const int off = (rmin + (chunk_of(p) << 5) - 2) & 1;
#pragma unroll 8
    for (int row = 0; row < 32; row++) tile[row * XT_S + lane] = dense[row * XT2_COLS + off + lane];
    tr[32] = dense[lane * XT2_COLS + off + 32];
    tr[33] = dense[lane * XT2_COLS + off + 33];
    __syncwarp();
    if (p + 1 < nload) issue(p + 1);
  };

  int lo_w = R.lo;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lo_w = max(lo_w, __shfl_xor_sync(0xffffffffu, lo_w, o));
  auto fast_chunk = [&](int l0, int cnt) { return cnt == 32 && l0 > lo_w && l0 + 31 <= ncells - 2; };
  const double fCL = R.v[CN_CL], fCC = R.v[CN_CC], fCR = R.v[CN_CR], fFA = R.v[CN_FACT];
  const double fDU = R.v[CN_DU], fDP = R.v[CN_DP], fRD = R.v[CN_RDP];

  // pass 1: forward elimination, checkpoints only (:813-851 and dgtsv)
  double qm = 0.0, qc = 0.0, bp = 0.0;
  issue(0);
  for (int ch = 0; ch < nch; ch++) {
    const int l0 = ch << 5;
    const int cnt = (ncells - l0) < 32 ? (ncells - l0) : 32;
    next_tile(ch);
    if (!ok) break;
    if (ch == 0) {
      qm = tr[1];  // BC_left_t0 = q(rmin)
      qc = qm;
    }
    if (fast_chunk(l0, cnt)) {  // rows l0..l0+31 < ncells-1: qp always from the tile
#pragma unroll 8
      for (int c = 0; c < 32; c++) {
        const double qp = tr[c + 2];
        const double B = fCL * qm + fCC * qc + fCR * qp;
        bp = B - fFA * bp;
        qm = qc;
        qc = qp;
      }
    } else {
      for (int c = 0; c < cnt; c++) {
        const int l = l0 + c;
        const double qp = (l + 1 < ncells) ? tr[c + 2] : qc;  // BC_right_t0 = q(rmax)
        const double B = cn_coef(t, F, U, R, CN_CL, l) * qm + cn_coef(t, F, U, R, CN_CC, l) * qc +
                         cn_coef(t, F, U, R, CN_CR, l) * qp;
        bp = (l == 0) ? B : B - cn_coef(t, F, U, R, CN_FACT, l) * bp;
        qm = qc;
        qc = qp;
      }
    }
    if (valid && ch + 1 < nch) xown[l0 + 31] = bp;  // checkpoint B'(l0+31)
    if (ch + 1 < nch) __syncwarp();  // the last chunk stays in the tile for pass 2
  }

  // pass 2: per chunk, last first: recompute B', back-substitute, store
  double xn = 0.0;
  for (int ch = nch - 1; ch >= 0 && ok; ch--) {
    const int l0 = ch << 5;
    const int cnt = (ncells - l0) < 32 ? (ncells - l0) : 32;
    if (ch != nch - 1) {
      next_tile(2 * nch - 2 - ch);
      if (!ok) break;
    }
    double bq = (valid && ch > 0) ? xown[l0 - 1] : 0.0;
    double qm2 = (ch == 0) ? tr[1] : tr[0];
    double qc2 = tr[1];
    if (fast_chunk(l0, cnt)) {
#pragma unroll 8
      for (int c = 0; c < 32; c++) {
        const double qp = tr[c + 2];
        const double B = fCL * qm2 + fCC * qc2 + fCR * qp;
        bq = B - fFA * bq;
        tr[c + 1] = bq;
        qm2 = qc2;
        qc2 = qp;
      }
#pragma unroll 8
      for (int c = 31; c >= 0; c--) {
        const double num = tr[c + 1] - fDU * xn;
        const double v = div_rn_rcp(num, fDP, fRD);
        tr[c + 1] = v;
        xn = v;
      }
    } else {
      for (int c = 0; c < cnt; c++) {
        const int l = l0 + c;
        const double qp = (l + 1 < ncells) ? tr[c + 2] : qc2;
        const double B = cn_coef(t, F, U, R, CN_CL, l) * qm2 + cn_coef(t, F, U, R, CN_CC, l) * qc2 +
                         cn_coef(t, F, U, R, CN_CR, l) * qp;
        bq = (l == 0) ? B : B - cn_coef(t, F, U, R, CN_FACT, l) * bq;
        tr[c + 1] = bq;
        qm2 = qc2;
        qc2 = qp;
      }
      for (int c = cnt - 1; c >= 0; c--) {
        const int l = l0 + c;
        const double b2 = tr[c + 1];
        const double num = (l == ncells - 1) ? b2 : b2 - cn_coef(t, F, U, R, CN_DU, l) * xn;
        const double v = div_rn_rcp(num, cn_coef(t, F, U, R, CN_DP, l), cn_coef(t, F, U, R, CN_RDP, l));
        tr[c + 1] = v;
        xn = v;
      }
    }
    __syncwarp();
#pragma unroll 8
    for (int row = 0; row < 32; row++) {
      if (row < nvalid && lane < cnt)
        x0[(long)row * P + l0 + lane] = ((amask >> row) & 1u) ? tile[row * XT_S + 1 + lane] : 0.0;
    }
    __syncwarp();
  }
  if (!ok && lane == 0) raise_error(sc, A3G_ERR_TIMEOUT, 5);
}

// ---------------------------------------------------------------------------
// z lines through TMA column tiles.  A warp owns the 32 z lines of 32
// consecutive i at one (j, grain): one tensor load brings the whole tile
// (32 i x nz levels, tile[k][lane]) into shared memory, each lane runs its
// line's elimination and back substitution in place (the same operations as
// cn_line, so the same bits), and one tensor store writes the tile back.  The
// level is read once and written once, with no B' round trip through global
// memory, and the copies run asynchronously to the other warps' arithmetic.
// The factor-table rows of the tile's line (the same for its 32 lines: the
// coefficients do not vary along i) are staged in shared memory by the warp,
// so the recurrences read only shared memory.  Warps are persistent and take
// contiguous runs of tiles (neighbouring i, then j), which share table rows.
// ---------------------------------------------------------------------------

// doubles of shared memory per warp: the tile and the staged table rows,
// rounded up to 128 bytes so that every warp's tile stays aligned
__host__ __device__ __forceinline__ long zt_warp_doubles(int nz) {
  return (32L * nz + CN_NF * (long)nz + 15) / 16 * 16;
}

__global__ void __launch_bounds__(64, 8) k_cn_solve_zt(const __grid_constant__ CUtensorMap tin,
                                                    const __grid_constant__ CUtensorMap tout, Layout L,
                                                    Box box, LineMap map, const double *__restrict__ tab,
                                                    const int32_t *__restrict__ aloft, DevScalars *sc,
                                                    int wpb) {
  extern __shared__ __align__(128) unsigned char zt_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nz = L.nz;
  uint64_t *bar = reinterpret_cast<uint64_t *>(zt_smem) + wid;
  double *tile = reinterpret_cast<double *>(zt_smem + ZT_BAR_BYTES) + (long)wid * zt_warp_doubles(nz);
  double *stab = tile + 32L * nz;  // staged table: field f, row l at stab[f*nz + l]
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
    prefetch_tensormap(&tin);
    prefetch_tensormap(&tout);
  }
  __syncwarp();
  const int nti = (L.nx + 31) >> 5;
  const long ntiles = (long)nti * L.ny * L.ns;
  const long nwarps = (long)gridDim.x * wpb;
  const long per = (ntiles + nwarps - 1) / nwarps;
  const long t0 = ((long)blockIdx.x * wpb + wid) * per;
  const long t1 = t0 + per < ntiles ? t0 + per : ntiles;
  const int rmin = box.kmin, rmax = box.kmax;
  const int ncells = rmax - rmin + 1;
  const long U = map.U;
  const long F = (long)ncells * U;
  const uint32_t tile_bytes = 32u * (uint32_t)nz * 8u;
  uint32_t phase = 0;
  int staged = -1;            // the line index u whose rows stab holds
  double *col = tile + lane;  // this lane's line: level k (1-based) at col[(k-1)*32]
  for (long t = t0; t < t1; t++) {
    const int it = (int)(t % nti);
    const long r = t / nti;
    const int j = (int)(r % L.ny) + 1;
    const int g = (int)(r / L.ny);
    const int i = (it << 5) + lane + 1;
    const bool act = i <= L.nx && i >= box.imin && i <= box.imax && j >= box.jmin && j <= box.jmax &&
                     aloft[g] != 0;
    const bool any = __any_sync(0xffffffffu, act);
    // the previous tile's store must have read the buffer before it is refilled
    if (lane == 0) bulk_wait_read0();
    __syncwarp();
    if (any) {
      if (lane == 0) {
        mbar_arrive_expect_tx(bar, tile_bytes);
        tma_load_4d(tile, &tin, bar, it << 5, j - 1, 0, g);
      }
      const int u = map.u(1, j);  // the coefficients do not vary along i (map.da == 0)
      if (u != staged) {          // stage the rows while the tile is in flight
        const double *tl = tab + u;
        for (int l = lane; l < ncells; l += 32)
#pragma unroll
          for (int f = 0; f < CN_NF; f++) stab[f * nz + l] = tl[f * F + (long)l * U];
        staged = u;
      }
      if (!mbar_wait(bar, phase)) {
        if (lane == 0) {
          raise_error(sc, A3G_ERR_TIMEOUT, 2);
          bulk_wait0();
        }
        return;
      }
      phase ^= 1u;
      __syncwarp();
    }
    if (act) {
      auto co = [&](int f, int l) { return stab[f * nz + l]; };
      double *xx = col + (long)(rmin - 1) * 32;  // row l at xx[l*32]
      // forward elimination with the right-hand side built on the fly, :813-851
      // (ncells >= 2: a single-row line is skipped before the launch; the
      // first and last rows are taken out of the loops, which then need no
      // per-row boundary tests)
      double qm = xx[0];  // BC_left_t0 = q(rmin)
      double qc = qm;
      double bp;
      {
        const double qp = xx[32];
        bp = co(CN_CL, 0) * qm + co(CN_CC, 0) * qc + co(CN_CR, 0) * qp;
        xx[0] = bp;
        qm = qc;
        qc = qp;
      }
#pragma unroll 4
      for (int l = 1; l < ncells - 1; l++) {
        const double qp = xx[(l + 1) * 32];
        const double B = co(CN_CL, l) * qm + co(CN_CC, l) * qc + co(CN_CR, l) * qp;
        bp = B - co(CN_FACT, l) * bp;
        xx[l * 32] = bp;
        qm = qc;
        qc = qp;
      }
      {
        const int l = ncells - 1;
        const double qp = qc;  // BC_right_t0 = q(rmax)
        const double B = co(CN_CL, l) * qm + co(CN_CC, l) * qc + co(CN_CR, l) * qp;
        bp = B - co(CN_FACT, l) * bp;
        xx[l * 32] = bp;
      }
      // back substitution
      double xn = div_rn_rcp(xx[(ncells - 1) * 32], co(CN_DP, ncells - 1), co(CN_RDP, ncells - 1));
      xx[(ncells - 1) * 32] = xn;
#pragma unroll 4
      for (int l = ncells - 2; l >= 0; l--) {
        const double num = xx[l * 32] - co(CN_DU, l) * xn;
        const double v = div_rn_rcp(num, co(CN_DP, l), co(CN_RDP, l));
        xx[l * 32] = v;
        xn = v;
      }
      for (int k = 1; k < rmin; k++) col[(k - 1) * 32] = 0.0;  // outside the box
      for (int k = rmax + 1; k <= nz; k++) col[(k - 1) * 32] = 0.0;
    } else {
      for (int k = 1; k <= nz; k++) col[(k - 1) * 32] = 0.0;  // the reference leaves zeros
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_4d(&tout, tile, it << 5, j - 1, 0, g);
      bulk_commit();
    }
  }
  if (lane == 0) bulk_wait0();
}

// ---------------------------------------------------------------------------
// y lines through TMA chunk tiles.  A warp owns the 32 y lines of 32
// consecutive i at one (k, grain) and walks them in chunks of YT_CH cells;
// each chunk arrives by one tensor load as a tile of YT_CH + 2 rows (the
// cell before the chunk and the cell after it included; row r holds line
// position l0 - 1 + r), tile[r][lane].  Two buffers per warp: the next
// chunk's load is in flight while the lanes work on the current one.
//   pass 1 (forward): the elimination of B' over the whole line, keeping only
//     B' at the last cell of every chunk (a checkpoint, parked in the output
//     line at that cell, which the chunk's own store overwrites later);
//   pass 2 (backward, last chunk first, which pass 1 left in its buffer):
//     recompute the chunk's B' from the previous chunk's checkpoint (same
//     operations, same bits), back-substitute in place, and store the chunk
//     with one tensor store.
// The arithmetic is cn_line's, operation for operation.  Each chunk's
// factor-table rows (the same for the warp's 32 lines) are staged in shared
// memory while its tile is in flight.  Warps take contiguous runs of line
// groups (neighbouring i, then k), which share table rows.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(64, 10) k_cn_solve_yt(const __grid_constant__ CUtensorMap tin,
                                                    const __grid_constant__ CUtensorMap tout, Layout L,
                                                    Box box, LineMap map, double *__restrict__ cout,
                                                    const double *__restrict__ tab,
                                                    const int32_t *__restrict__ aloft, DevScalars *sc,
                                                    int wpb) {
  extern __shared__ __align__(128) unsigned char yt_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int BUF = 32 * YT_ROWS;  // doubles per buffer (a multiple of 16: 128-byte aligned buffers)
  uint64_t *bar = reinterpret_cast<uint64_t *>(yt_smem) + 2 * wid;
  double *wbase = reinterpret_cast<double *>(yt_smem + ZT_BAR_BYTES) + (long)wid * (2 * BUF + CN_NF * 32);
  auto buf = [&](int bi) { return wbase + (bi ? BUF : 0); };
  double *stab = wbase + 2 * BUF;  // staged table of the chunk: field f, row c at stab[f*32 + c]
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
    prefetch_tensormap(&tin);
    prefetch_tensormap(&tout);
  }
  __syncwarp();
  const int nti = (L.nx + 31) >> 5;
  const long ngroups = (long)nti * L.nz * L.ns;
  const long nwarps = (long)gridDim.x * wpb;
  const long per = (ngroups + nwarps - 1) / nwarps;
  const long t0 = ((long)blockIdx.x * wpb + wid) * per;
  const long t1 = t0 + per < ngroups ? t0 + per : ngroups;
  const int rmin = box.jmin, rmax = box.jmax;
  const int ncells = rmax - rmin + 1;
  const int nch = (ncells + YT_CH - 1) / YT_CH;
  const long U = map.U;
  const long F = (long)ncells * U;
  const uint32_t tile_bytes = 32u * YT_ROWS * 8u;
  uint32_t ph = 0u;  // bit b: the parity of buffer b's barrier
  for (long t = t0; t < t1; t++) {
    const int it = (int)(t % nti);
    const long r = t / nti;
    const int k = (int)(r % L.nz) + 1;
    const int g = (int)(r / L.nz);
    const int i = (it << 5) + lane + 1;
    const bool act = i <= L.nx && i >= box.imin && i <= box.imax && k >= box.kmin && k <= box.kmax &&
                     aloft[g] != 0;
    const bool any = __any_sync(0xffffffffu, act);
    double *xg = cout + (long)g * L.PG + (long)(k - 1) * L.PY + (i - 1);  // cell (i, 1, k) of this lane
    if (!any) {  // the reference leaves zeros
      if (i <= L.nx)
        for (int j = 1; j <= L.ny; j++) xg[(long)(j - 1) * L.P] = 0.0;
      continue;
    }
    if (i <= L.nx) {  // cells that no chunk store covers: outside [rmin, rmin + nch*YT_CH)
      for (int j = 1; j < rmin; j++) xg[(long)(j - 1) * L.P] = 0.0;
      for (int j = rmin + nch * YT_CH; j <= L.ny; j++) xg[(long)(j - 1) * L.P] = 0.0;
    }
    auto issue = [&](int bi, int ch) {  // tensor load of chunk ch into buffer bi
      if (lane == 0) {
        bulk_wait_read0();  // a store from this buffer must have read it first
        mbar_arrive_expect_tx(&bar[bi], tile_bytes);
        tma_load_4d(buf(bi), &tin, &bar[bi], it << 5, rmin - 2 + ch * YT_CH, k - 1, g);
      }
    };
    bool ok = true;
    auto wait = [&](int bi) {
      ok = mbar_wait(&bar[bi], (ph >> bi) & 1u);
      ph ^= 1u << bi;
    };
    const double *tl = tab + map.u(1, k);  // the coefficients do not vary along i (map.da == 0)
    auto stage = [&](int l0, int nf) {      // fields 0..nf-1 of the chunk's rows into stab
      const int l = l0 + lane;
      if (lane < YT_CH && l < ncells)
        for (int f = 0; f < nf; f++) stab[f * 32 + lane] = tl[f * F + (long)l * U];
    };
    auto co = [&](int f, int c) { return stab[f * 32 + c]; };
    // pass 1: forward elimination, checkpoints only (:813-851 and dgtsv)
    double qm = 0.0, qc = 0.0, bp = 0.0;
    issue(0, 0);
    for (int ch = 0; ch < nch && ok; ch++) {
      const int bi = ch & 1;
      if (ch + 1 < nch) issue(bi ^ 1, ch + 1);
      const int l0 = ch * YT_CH;
      stage(l0, CN_CR + 1);  // FACT, DP, DU, CL, CC, CR
      wait(bi);
      if (!ok) break;
      __syncwarp();
      const double *T = buf(bi) + lane;
      const int cnt = (ncells - l0) < YT_CH ? (ncells - l0) : YT_CH;
      if (act) {
        if (ch == 0) {
          qm = T[32];  // BC_left_t0 = q(rmin)
          qc = qm;
        }
        if (ch > 0 && l0 + YT_CH <= ncells - 1) {  // interior chunk: rows 1 .. ncells-2 only
#pragma unroll
          for (int c = 0; c < YT_CH; c++) {
            const double qp = T[(c + 2) * 32];
            const double B = co(CN_CL, c) * qm + co(CN_CC, c) * qc + co(CN_CR, c) * qp;
            bp = B - co(CN_FACT, c) * bp;
            qm = qc;
            qc = qp;
          }
        } else {
#pragma unroll 4
          for (int c = 0; c < cnt; c++) {
            const int l = l0 + c;
            const double qp = (l + 1 < ncells) ? T[(c + 2) * 32] : qc;  // BC_right_t0 = q(rmax)
            const double B = co(CN_CL, c) * qm + co(CN_CC, c) * qc + co(CN_CR, c) * qp;
            bp = (l == 0) ? B : B - co(CN_FACT, c) * bp;
            qm = qc;
            qc = qp;
          }
        }
        if (ch + 1 < nch) xg[(long)(rmin + l0 + YT_CH - 2) * L.P] = bp;  // checkpoint B'(l0+YT_CH-1)
      }
      __syncwarp();
    }
    fence_proxy_async_all();  // the checkpoints land before any store of this line's chunks
    // pass 2: per chunk, last first: recompute B', back-substitute, store
    double xn = 0.0;
    for (int ch = nch - 1; ch >= 0 && ok; ch--) {
      const int bi = ch & 1;
      if (ch - 1 >= 0) issue(bi ^ 1, ch - 1);
      const int l0 = ch * YT_CH;
      stage(l0, CN_NF);
      if (ch != nch - 1) {
        wait(bi);
        if (!ok) break;
      }
      __syncwarp();
      double *T = buf(bi) + lane;
      const int cnt = (ncells - l0) < YT_CH ? (ncells - l0) : YT_CH;
      if (act) {
        double bq = ch > 0 ? xg[(long)(rmin + l0 - 2) * L.P] : 0.0;
        double qm2 = (ch == 0) ? T[32] : T[0];
        double qc2 = T[32];
        if (ch > 0 && l0 + YT_CH <= ncells - 1) {  // interior chunk: rows 1 .. ncells-2 only
#pragma unroll
          for (int c = 0; c < YT_CH; c++) {
            const double qp = T[(c + 2) * 32];
            const double B = co(CN_CL, c) * qm2 + co(CN_CC, c) * qc2 + co(CN_CR, c) * qp;
            bq = B - co(CN_FACT, c) * bq;
            T[(c + 1) * 32] = bq;
            qm2 = qc2;
            qc2 = qp;
          }
#pragma unroll
          for (int c = YT_CH - 1; c >= 0; c--) {
            const double num = T[(c + 1) * 32] - co(CN_DU, c) * xn;
            const double v = div_rn_rcp(num, co(CN_DP, c), co(CN_RDP, c));
            T[(c + 1) * 32] = v;
            xn = v;
          }
        } else {
#pragma unroll 4
          for (int c = 0; c < cnt; c++) {
            const int l = l0 + c;
            const double qp = (l + 1 < ncells) ? T[(c + 2) * 32] : qc2;
            const double B = co(CN_CL, c) * qm2 + co(CN_CC, c) * qc2 + co(CN_CR, c) * qp;
            bq = (l == 0) ? B : B - co(CN_FACT, c) * bq;
            T[(c + 1) * 32] = bq;
            qm2 = qc2;
            qc2 = qp;
          }
#pragma unroll 4
          for (int c = cnt - 1; c >= 0; c--) {
            const int l = l0 + c;
            const double b2 = T[(c + 1) * 32];
            const double num = (l == ncells - 1) ? b2 : b2 - co(CN_DU, c) * xn;
            const double v = div_rn_rcp(num, co(CN_DP, c), co(CN_RDP, c));
            T[(c + 1) * 32] = v;
            xn = v;
          }
        }
        for (int c = cnt; c < YT_CH; c++) T[(c + 1) * 32] = 0.0;  // beyond rmax
      } else {
        for (int c = 0; c < YT_CH; c++) T[(c + 1) * 32] = 0.0;  // the reference leaves zeros
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        tma_store_4d(&tout, buf(bi) + 32, it << 5, rmin - 1 + l0, k - 1, g);
        bulk_commit();
      }
    }
    if (!ok) {
      if (lane == 0) {
        raise_error(sc, A3G_ERR_TIMEOUT, 1);
        bulk_wait0();
      }
      return;
    }
  }
  if (lane == 0) bulk_wait0();
}

// ---------------------------------------------------------------------------
// TMA tensor maps over the concentration levels
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

// Looked up once per process; the initialisation of a function-local static
// is thread-safe, and contexts may make their first launches from several
// host threads at once (concurrent ensemble members).
static EncodeTiledFn encode_tiled_fn() {
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
    return nullptr;
  }();
  return fn;
}

// A level as a 4-D tensor (i, j, k, grain) of doubles with the device
// layout's pitches (a wind array: the same with one grain); the box is one
// tile of the given kind (TmapKind).
bool tensor_map(a3g_ctx *ctx, const double *p, int kind, CUtensorMap *out) {
  for (const TmapEntry &e : ctx->tmaps)
    if (e.p == p && e.kind == kind) {
      *out = e.map;
      return true;
    }
  EncodeTiledFn enc = encode_tiled_fn();
  if (!enc) return false;
  const Layout &L = ctx->L;
  const bool wind = kind == TM_ADV_VY || kind == TM_ADV_VZ || kind == TM_ADV_VX;
  const cuuint64_t dims[4] = {(cuuint64_t)L.nx, (cuuint64_t)L.ny, (cuuint64_t)L.nz,
                              (cuuint64_t)(wind ? 1 : L.ns)};
  const cuuint64_t strides[3] = {(cuuint64_t)L.P * 8, (cuuint64_t)L.PY * 8, (cuuint64_t)L.PG * 8};
  cuuint32_t box[4] = {32, 1, 1, 1};
  cuuint32_t rank = 4;
  // the rows of a level form a 2-D array: row r = (g*nz + k-1)*ny + j-1 at r*P
  const cuuint64_t rdims[2] = {(cuuint64_t)L.nx, (cuuint64_t)L.ny * L.nz * L.ns};
  if (kind == TM_XROWS) {
    rank = 2;
    box[0] = XT2_COLS;
    box[1] = 32;
  } else if (kind == TM_COLUMN) {
    if (L.nz > 256) return false;
    box[2] = (cuuint32_t)L.nz;
  } else if (kind == TM_YCHUNK_IN) {
    box[1] = YT_ROWS;
  } else if (kind == TM_YCHUNK_OUT) {
    box[1] = YT_CH;
  } else if (kind == TM_ADV_QY || kind == TM_ADV_VY) {
    box[1] = ACH;

  } else if (kind == TM_ADV_QZ || kind == TM_ADV_VZ) {
    box[2] = ACH;
  } else if (kind == TM_ADV_QX1 || kind == TM_ADV_VX) {
  } else if (kind == TM_ADV_QX2) {
    if (L.ns < 2) return false;
    box[3] = 2;
  } else {
    return false;
  }
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  TmapEntry e;
  e.p = p;
  e.kind = kind;
  if (enc(&e.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, const_cast<double *>(p), rank == 2 ? rdims : dims,
          strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  // a step uses about 17 (two levels alternating under each tile shape, and
  // the wind arrays); the adjoint's stage levels add more
  if (ctx->tmaps.size() >= 64) ctx->tmaps.erase(ctx->tmaps.begin());
  ctx->tmaps.push_back(e);
  *out = e.map;
  return true;
}

// Launches the z solve through column tiles; false when the shape is outside
// what the tiles cover (the caller takes the per-thread kernel).
static bool launch_cn_solve_zt(a3g_ctx *ctx, const LineMap &map, const double *tab) {
  const Layout &L = ctx->L;
  if (L.nz > 256 || map.da) return false;
  CUtensorMap tin, tout;
  if (!tensor_map(ctx, ctx->c0, TM_COLUMN, &tin) || !tensor_map(ctx, ctx->c1, TM_COLUMN, &tout)) return false;
  const int wpb = L.nz <= 128 ? 2 : 1;
  const size_t smem = ZT_BAR_BYTES + (size_t)wpb * zt_warp_doubles(L.nz) * sizeof(double);
  if (ctx->tma_grid[0] == 0) {
    // the opt-in maximum, so that contexts of any nz can share the attribute
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess ||
        (size_t)optin < smem ||
        cudaFuncSetAttribute(k_cn_solve_zt, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess ||
        cudaFuncSetAttribute(k_cn_solve_zt, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return false;
    int per_sm = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cn_solve_zt, 32 * wpb, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess || per_sm < 1)
      return false;
    ctx->tma_grid[0] = per_sm * nsm;
  }
  const long ntiles = (long)((L.nx + 31) / 32) * L.ny * L.ns;
  const long need = (ntiles + wpb - 1) / wpb;
  const int grid = (int)(need < ctx->tma_grid[0] ? need : ctx->tma_grid[0]);
  k_cn_solve_zt<<<grid, 32 * wpb, smem, ctx->stream>>>(tin, tout, L, ctx->box, map, tab, ctx->aloft, ctx->sc,
                                                       wpb);
  return true;
}

// Launches the y solve through chunk tiles; false when the maps cannot be
// made (the caller takes the per-thread kernel).
static bool launch_cn_solve_yt(a3g_ctx *ctx, const LineMap &map, const double *tab) {
  const Layout &L = ctx->L;
  if (map.da) return false;
  CUtensorMap tin, tout;
  if (!tensor_map(ctx, ctx->c0, TM_YCHUNK_IN, &tin) || !tensor_map(ctx, ctx->c1, TM_YCHUNK_OUT, &tout))
    return false;
  const int wpb = 2;
  const size_t smem = ZT_BAR_BYTES + (size_t)wpb * (2 * 32 * YT_ROWS + CN_NF * 32) * sizeof(double);
  if (ctx->tma_grid[1] == 0) {
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess ||
        (size_t)optin < smem ||
        cudaFuncSetAttribute(k_cn_solve_yt, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess ||
        cudaFuncSetAttribute(k_cn_solve_yt, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return false;
    int per_sm = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cn_solve_yt, 32 * wpb, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess || per_sm < 1)
      return false;
    ctx->tma_grid[1] = per_sm * nsm;
  }
  const long ngroups = (long)((L.nx + 31) / 32) * L.nz * L.ns;
  const long need = (ngroups + wpb - 1) / wpb;
  const int grid = (int)(need < ctx->tma_grid[1] ? need : ctx->tma_grid[1]);
  k_cn_solve_yt<<<grid, 32 * wpb, smem, ctx->stream>>>(tin, tout, L, ctx->box, map, ctx->c1, tab, ctx->aloft,
                                                       ctx->sc, wpb);
  return true;
}

// Launches the x solve through TMA tiles; false when the map cannot be made.
static bool launch_cn_solve_xt2(a3g_ctx *ctx, const LineMap &map, const double *tab) {
  const Layout &L = ctx->L;
  CUtensorMap trow;
  if (!tensor_map(ctx, ctx->c0, TM_XROWS, &trow)) return false;
  const size_t smem = ZT_BAR_BYTES + (size_t)XT2_WARPS * XT2_WARP_D * sizeof(double);
  if (ctx->tma_grid[2] == 0) {
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess ||
        (size_t)optin < smem ||
        cudaFuncSetAttribute(k_cn_solve_xt2, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess)
      return false;
    ctx->tma_grid[2] = 1;
  }
  const long nwarps = ((long)L.ny * L.nz * L.ns + 31) / 32;
  k_cn_solve_xt2<<<(unsigned)((nwarps + XT2_WARPS - 1) / XT2_WARPS), 32 * XT2_WARPS, smem, ctx->stream>>>(
      trow, L, ctx->box, map, ctx->c0, ctx->c1, tab, ctx->aloft, ctx->sc);
  return true;
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
  const size_t U = (size_t)(da ? na : 1) * (size_t)(db ? nb : 1);
  return (size_t)CN_NF * n * U + 2 * U;
}

// Decides on the device whether direction dir's table can be kept: the host
// allows it (same box, geometry and diffusivity as when it was built) and
// the step's dt equals the table's.
__global__ void k_cn_check(const DevScalars *__restrict__ sc, double *__restrict__ st, int dir, int may) {
  const double dt = sc->dt;
  const bool keep = may && st[dir] == dt;
  st[3 + dir] = keep ? 1.0 : 0.0;
  st[dir] = dt;
}

static inline bool same_box(const Box &a, const Box &b) {
  return a.imin == b.imin && a.imax == b.imax && a.jmin == b.jmin && a.jmax == b.jmax && a.kmin == b.kmin &&
         a.kmax == b.kmax;
}

// The factor table of direction DIR for the step's dt: built by k_cn_table,
// or kept from the previous build when nothing it depends on has changed.
template <int DIR>
static int cn_table(a3g_ctx *ctx, const LineMap &map, const Geo3 &sig, const Geo3 &kk) {
  const bool may = ctx->cn_valid[DIR] && same_box(ctx->cn_box[DIR], ctx->box);
  k_cn_check<<<1, 1, 0, ctx->stream>>>(ctx->sc, ctx->cn_state, DIR, may ? 1 : 0);
  A3G_LAUNCH_CHECK(ctx);
  k_cn_table<DIR><<<(map.U + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ctx->box, ctx->prm.imp_fac, map, sig,
                                                                ctx->kappa, kk, ctx->sc, ctx->cn_state,
                                                                ctx->cn_tab[DIR]);
  A3G_LAUNCH_CHECK(ctx);
  ctx->cn_valid[DIR] = true;
  ctx->cn_box[DIR] = ctx->box;
  return A3G_OK;
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
  int rc = cn_table<DIR>(ctx, map, sig, kk);
  tend(ctx);
  if (rc) return rc;
  const double *tab = ctx->cn_tab[DIR];
  const long nlines = (long)map.na * map.nb * L.ns;
  tbegin(ctx, A3G_K_CN_SOLVE_X + DIR);
  if (DIR == 0 && ctx->tune_cn_x == 2 && launch_cn_solve_xt2(ctx, map, tab)) {
    // tiles through TMA
  } else if (DIR == 0 && ctx->tune_cn_x == 0) {
    const long nwarps = (nlines + 31) / 32;
    k_cn_solve_xt<<<(unsigned)((nwarps + XT_WARPS - 1) / XT_WARPS), 32 * XT_WARPS, 0, ctx->stream>>>(
        L, box, map, ctx->c0, ctx->c1, tab, ctx->aloft);
  } else if (DIR == 2 && ctx->tune_cn_yz == 3 && launch_cn_solve_zt(ctx, map, tab)) {
    // column tiles through TMA
  } else if (DIR == 1 && ctx->tune_cn_yz == 3 && launch_cn_solve_yt(ctx, map, tab)) {
    // chunk tiles through TMA
  } else if (DIR != 0 && (ctx->tune_cn_yz == 1 || ctx->tune_cn_yz == 3) && L.ns >= 2) {
    launch_cn_solve_gc<DIR == 0 ? 1 : DIR, 2>(ctx, map, tab);
  } else if (DIR != 0 && ctx->tune_cn_yz == 2 && L.ns >= 2) {
    launch_cn_solve_gc<DIR == 0 ? 1 : DIR, 4>(ctx, map, tab);
  } else {
    k_cn_solve<DIR><<<(unsigned)((nlines + 127) / 128), 128, 0, ctx->stream>>>(
        L, box, map, ctx->c0, ctx->c1, tab, ctx->aloft);
  }
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  swap_levels(ctx);
  ctx->ts1_zeroed = false;
  return A3G_OK;
}

int launch_diffcn_x(a3g_ctx *ctx) { return launch_cn_dir<0>(ctx); }
int launch_diffcn_y(a3g_ctx *ctx) { return launch_cn_dir<1>(ctx); }
int launch_diffcn_z(a3g_ctx *ctx) { return launch_cn_dir<2>(ctx); }

// ===========================================================================
// Discrete adjoint of the diffusion sweeps (no counterpart in the reference).
// Both sweeps are linear; full box only.
// ===========================================================================
// Explicit: out(l) = q(l) + cR(l)(q(l+1)-q(l)) - cL(l)(q(l)-q(l-1)) with the
// Neumann ghosts (periodic in x); the transpose gathers, per cell m,
//   lam_q(m) = lam(m)(1 - cR(m) - cL(m)) + cR(m-1)lam(m-1) + cL(m+1)lam(m+1)
// and folds the ghost terms back: cL(1)lam(1) into cell 1 and cR(n)lam(n)
// into cell n (Neumann), or into cells n and 1 (periodic).
template <int DIR>
__global__ void __launch_bounds__(256) k_adj_diff(Layout L, int periodic, const double *__restrict__ lin,
                                                  double *__restrict__ lout, Geo3 sig, Geo3 kap, Geo3 kk,
                                                  const int32_t *__restrict__ aloft,
                                                  const DevScalars *__restrict__ sc) {
  const int i = blockIdx.x * 32 + threadIdx.x + 1;
  const int j = blockIdx.y * 8 + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > L.nx || j > L.ny) return;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int l = (DIR == 0) ? i : (DIR == 1) ? j : k;
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? L.P : L.PY;
  const long cell = L.cell(i, j, k);
  auto G = [&](const Geo3 &a, int m) {
    return (DIR == 0) ? a.at(m, j, k) : (DIR == 1) ? a.at(i, m, k) : a.at(i, j, m);
  };
  const double dt = sc->dt;
  auto cR = [&](int m) {
    const double dsR = 2.0 * G(sig, m + 1) / (G(kap, m) + G(kap, m + 1));
    return dt * (0.5 * (G(kk, m) + G(kk, m + 1)) * dsR) * (G(sig, m + 1) / G(kap, m));
  };
  auto cL = [&](int m) {
    const double dsL = 2.0 * G(sig, m) / (G(kap, m - 1) + G(kap, m));
    return dt * (0.5 * (G(kk, m - 1) + G(kk, m)) * dsL) * (G(sig, m) / G(kap, m));
  };
  const bool per = DIR == 0 && periodic;
  const double cRl = cR(l), cLl = cL(l);
  const double cRm = (l > 1) ? cR(l - 1) : 0.0, cLp = (l < n) ? cL(l + 1) : 0.0;
  const double cRn = (l == 1 && per) ? cR(n) : 0.0, cL1 = (l == n && per) ? cL(1) : 0.0;
  for (int g = 0; g < L.ns; g++) {
    const long a = (long)g * L.PG + cell;
    if (!aloft[g]) { lout[a] = 0.0; continue; }
    const double lm = lin[a];
    double v = lm - cRl * lm - cLl * lm;
    if (l > 1) v = v + cRm * lin[a - st];
    if (l < n) v = v + cLp * lin[a + st];
    if (!per) {
      if (l == 1) v = v + cLl * lm;
      if (l == n) v = v + cRl * lm;
    } else {
      if (l == 1) v = v + cRn * lin[a + (long)(n - 1) * st];
      if (l == n) v = v + cL1 * lin[a - (long)(n - 1) * st];
    }
    lout[a] = v;
  }
}

// Crank-Nicolson: out = M^-1 N q.  With dgtsv's factors M = L U (L unit
// lower with multipliers fact(r), U upper with D'(r), DU(r)), the adjoint
// solves U^T z = lam (forward), L^T y = z (backward), then applies N^T:
//   lam_q(r) = CC(r)y(r) + CR(r-1)y(r-1) + CL(r+1)y(r+1)
// plus CL(0)y(0) in row 0 and CR(n-1)y(n-1) in the last row (the Neumann
// columns of N).  One thread per line; z is parked in the output line.
template <int DIR>
__global__ void __launch_bounds__(128) k_adj_cn(Layout L, LineMap map, const double *__restrict__ lin,
                                                double *__restrict__ lout, const double *__restrict__ tab,
                                                const int32_t *__restrict__ aloft) {
  const int na = (DIR == 0) ? L.ny : L.nx;
  const int nb = (DIR == 2) ? L.ny : L.nz;
  const long nlines = (long)na * nb * L.ns;
  const long w = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (w >= nlines) return;
  const int a = (int)(w % na) + 1;
  const long r0 = w / na;
  const int b = (int)(r0 % nb) + 1;
  const int g = (int)(r0 / nb);
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  long base, st;
  if (DIR == 0) { base = L.cell(1, a, b); st = 1; }
  else if (DIR == 1) { base = L.cell(a, 1, b); st = L.P; }
  else { base = L.cell(a, b, 1); st = L.PY; }
  base += (long)g * L.PG;
  const double *li = lin + base;
  double *lo = lout + base;
  if (!aloft[g]) {
    for (int r = 0; r < n; r++) lo[(long)r * st] = 0.0;
    return;
  }
  const long U = map.U;
  const long F = (long)n * U;
  const long u = map.u(a, b);
  const double *t = tab + u;
  CnRun R;
  if (DIR == 0) cn_load_run(t, F, U, tab + CN_NF * F, u, R);
  auto co = [&](int f, int l) { return (DIR == 0) ? cn_coef(t, F, U, R, f, l) : t[f * F + (long)l * U]; };
  // U^T z = lam
  double zp = 0.0;
  for (int r = 0; r < n; r++) {
    const double rhs = (r == 0) ? li[0] : li[(long)r * st] - co(CN_DU, r - 1) * zp;
    zp = rhs / co(CN_DP, r);
    lo[(long)r * st] = zp;
  }
  // L^T y = z, with lam_q(r+1) emitted as soon as y(r) is known
  double y2 = 0.0;                 // y(r+2)
  double y1 = lo[(long)(n - 1) * st];  // y(n-1) = z(n-1)
  for (int r = n - 2; r >= -1; r--) {
    double y0 = 0.0;
    if (r >= 0) y0 = lo[(long)r * st] - co(CN_FACT, r + 1) * y1;
    const int q = r + 1;  // finished row
    double v = co(CN_CC, q) * y1;
    if (q > 0) v = v + co(CN_CR, q - 1) * y0;
    if (q < n - 1) v = v + co(CN_CL, q + 1) * y2;
    if (q == 0) v = v + co(CN_CL, 0) * y1;
    if (q == n - 1) v = v + co(CN_CR, n - 1) * y1;
    lo[(long)q * st] = v;
    y2 = y1;
    y1 = y0;
  }
}

template <int DIR>
static int launch_adj_diff_dir(a3g_ctx *ctx, const double *lin, double *lout) {
  const Layout &L = ctx->L;
  const Geo3 &sig = (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz;
  const Geo3 &kk = (DIR == 0) ? ctx->kx : (DIR == 1) ? ctx->ky : ctx->kz;
  dim3 grid((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz);
  tbegin(ctx, A3G_K_ADJOINT);
  k_adj_diff<DIR><<<grid, dim3(32, 8), 0, ctx->stream>>>(L, ctx->grid.periodic, lin, lout, sig, ctx->kappa,
                                                         kk, ctx->aloft, ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

template <int DIR>
static int launch_adj_cn_dir(a3g_ctx *ctx, const double *lin, double *lout) {
  const Layout &L = ctx->L;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  if (n <= 1) {  // the forward sweep leaves ts0 unchanged (:770)
    A3G_CUDA(cudaMemcpyAsync(lout, lin, sizeof(double) * L.PG * L.ns, cudaMemcpyDeviceToDevice,
                             ctx->stream));
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
  tbegin(ctx, A3G_K_ADJOINT);
  int rc = cn_table<DIR>(ctx, map, sig, kk);
  if (rc) return rc;
  const long nlines = (long)map.na * map.nb * L.ns;
  k_adj_cn<DIR><<<(unsigned)((nlines + 127) / 128), 128, 0, ctx->stream>>>(L, map, lin, lout, ctx->cn_tab[DIR],
                                                                           ctx->aloft);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// lam_out <- D^T lam_in for the diffusion sweep along dir (explicit or CN
// as the context is configured).  Full box.
int launch_adj_diffuse(a3g_ctx *ctx, int dir, const double *lin, double *lout) {
  if (ctx->prm.use_cn) {
    if (dir == 0) return launch_adj_cn_dir<0>(ctx, lin, lout);
    if (dir == 1) return launch_adj_cn_dir<1>(ctx, lin, lout);
    return launch_adj_cn_dir<2>(ctx, lin, lout);
  }
  if (dir == 0) return launch_adj_diff_dir<0>(ctx, lin, lout);
  if (dir == 1) return launch_adj_diff_dir<1>(ctx, lin, lout);
  return launch_adj_diff_dir<2>(ctx, lin, lout);
}

}  // namespace a3g
