#pragma once
// k_advect.cuh -- the forward advection sweeps (kernels and launch
// templates), shared by k_advect_x.cu, k_advect_y.cu and k_advect_z.cu, which
// instantiate one direction each, and by k_advect.cu (dt/kappa, adjoint).
//
// limited-upwind (DCU) advection sweeps on the device.
//
// Restates the row algorithm of advect_x / advect_y (src/AdvectionHorz_DCU.f90
// :68-305 / :322-556) and advect_z (src/AdvectionVert_DCU.f90:100-323):
// interface flux areas usig = 0.5*(v_{I-1}+v_I)*sigma_I, slopes dq, the
// limited second-order flux fss (superbee and the other LIM_* choices), the
// first-order fluctuations fs_r/fs_l with the divergence correction, and
// update = -dt/kappa*(fs_l(I+1)+fs_r(I)+fss(I+1)-fss(I)).  Every expression
// keeps the reference's operation order; the library is compiled with
// --fmad=false so that each product and sum rounds on its own, as the CPU
// build does, and divisions are IEEE (div.rn).  Terms that do not depend on
// the grain (flux areas, dt/kappa, 0.5|u|(1-dt/kappa|u|), the divergence
// corrections) are formed once per interface and shared by the grains a
// thread carries, which leaves each grain with one division (the limiter's
// theta) and about 25 other FP64 operations per cell.
//
// Mapping: a thread owns one line (a row along i, or a column along j or k)
// of GC grains and marches along a segment of it with a sliding register
// window (q, dq, fluxes); ghost values are generated at the line ends.  The
// y and z sweeps put neighbouring i on neighbouring lanes (coalesced); the x
// sweep puts neighbouring rows on lanes and relies on L1 to serve the four
// steps that share a 32-byte sector.  No shared memory, no barriers; the
// interior of a segment runs a branch-free step.
// Cells outside the active box and grains not aloft are written as zero: the
// zero-then-copy-back of the reference (AdvectionHorz_DCU.f90:122,302-303).
#include "a3g_internal.cuh"
#include "exact_div.cuh"
#include "tma.cuh"

#include <cstring>

namespace a3g {

// Fortran MAX/MIN of two reals as one FP64 min/max instruction.  For the
// non-NaN operands of this path they return the same value as the
// reference; at most the sign of an exact zero can differ, which no later
// operation of the sweep can turn into a different non-zero value.
__device__ __forceinline__ double dmx(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double dmn(double a, double b) { return fmin(a, b); }

// Limited slope of one interface (src/AdvectionHorz_DCU.f90:179-226); *skip
// is set when the reference "cycle"s on |dq| <= EPS_THRESH (fss stays 0).
template <int LIM>
__device__ __forceinline__ double dcu_ldq(double dqm, double dq, double dqp, bool upw_left,
                                          double eps, int nocycle, bool &skip) {
  skip = false;
  if (!nocycle && fabs(dq) <= eps) {
    skip = true;
    return 0.0;
  }
  if (LIM == A3G_LIM_LAXWEN) return dq;
  const double dqu = upw_left ? dqm : dqp;
  double theta;
  if (fabs(dqu) > 3.0 * fabs(dq) || fabs(dq) < eps)
    theta = copysign(3.0, dqu * dq);
  else
    theta = div_rn(dqu, dq);  // == dqu/dq, see exact_div.cuh
  if (LIM == A3G_LIM_BW) return dqu;
  if (LIM == A3G_LIM_FROMM) return dq * (0.5 * (1.0 + theta));
  if (LIM == A3G_LIM_MINMOD) return dq * dmx(0.0, dmn(1.0, theta));
  if (LIM == A3G_LIM_MC) return dq * dmx(0.0, dmn(dmn((1.0 + theta) / 2.0, 2.0), 2.0 * theta));
  return dq * dmx(dmx(0.0, dmn(1.0, 2.0 * theta)), dmn(2.0, theta));
}

// Grain-independent quantities of one interface.
struct Iface {
  double usp, usm;      // max(0,usig), min(0,usig)
  double divp, divm;    // divu_p, divu_m (:245-246)
  double cf;            // 0.5*|usig|*(1 - dt_vol(I)*|usig|)  (:227-230)
  bool up;              // usig > 0 (upwind on the left)
  bool fss_ok, fs_ok;   // I in [rmin, rmax+1] / [rmin-1, rmax+1]
};

__device__ __forceinline__ Iface make_iface(double us_m, double us, double us_p, double dtv, bool fss_ok,
                                            bool fs_ok) {
  Iface f;
  f.usp = dmx(0.0, us);
  f.usm = dmn(0.0, us);
  f.divp = dmx(0.0, us) - dmx(0.0, us_m);
  f.divm = dmn(0.0, us_p) - dmn(0.0, us);
  const double aus = fabs(us);
  f.cf = 0.5 * aus * (1.0 - dtv * aus);
  f.up = us > 0.0;
  f.fss_ok = fss_ok;
  f.fs_ok = fs_ok;
  return f;
}

// fss, fs_r, fs_l of one interface for one grain (:179-249).
template <int LIM>
__device__ __forceinline__ void iface_grain(const Iface &f, double dqm, double dq, double dqp, double qm,
                                            double q, double eps, int nocycle, double &fss, double &fsr,
                                            double &fsl) {
  fss = 0.0;
  if (LIM != A3G_LIM_NONE && f.fss_ok) {
    bool skip;
    const double ldq = dcu_ldq<LIM>(dqm, dq, dqp, f.up, eps, nocycle, skip);
    if (!skip) fss = f.cf * ldq;
  }
  if (f.fs_ok) {
    fsr = f.usp * dq;
    fsl = f.usm * dq;
    fsr = fsr + q * f.divm;
    fsl = fsl + qm * f.divp;
  } else {
    fsr = 0.0;
    fsl = 0.0;
  }
}

// update of a cell from its two interfaces (:264-281)
__device__ __forceinline__ double cell_update(double dtv, double fsl_r, double fsr_l, double fss_r,
                                              double fss_l) {
  return -(dtv * (fsl_r + fsr_l + fss_r - fss_l));
}

// ---------------------------------------------------------------------------
// Marching sweep.  DIR 0: along i (lanes j, other index k); DIR 1: along j
// (lanes i, other k); DIR 2: along k (lanes i, other j).  Block (32, 4):
// threadIdx.x the lane, threadIdx.y the other index.  blockIdx.x = lane block
// * ngroups + grain group (the groups of one region run together and share
// the wind loads through L2); blockIdx.z = segment along the sweep.
// For DIR 0 the lanes are rows: each load touches one 32-byte sector per row,
// which serves the next three steps from L1.
// ---------------------------------------------------------------------------
struct LineGeo {        // a ghosted geometry line: value at sweep index c is p[(c+1)*s]
  const double *p;
  long s;
  __device__ __forceinline__ double at(int c) const { return p[(long)(c + 1) * s]; }
};

template <int DIR>
__device__ __forceinline__ LineGeo line_of(const Geo3 &g, int a, int o) {
  LineGeo r;
  if (DIR == 0) { r.p = g.p + (long)(a + 1) * g.sj + (long)(o + 1) * g.sk; r.s = g.si; }
  else if (DIR == 1) { r.p = g.p + (long)(a + 1) * g.si + (long)(o + 1) * g.sk; r.s = g.sj; }
  else { r.p = g.p + (long)(a + 1) * g.si + (long)(o + 1) * g.sj; r.s = g.sk; }
  return r;
}

// stride of a broadcast geometry array along sweep direction DIR (0: constant along the line)
template <int DIR>
inline long along(const Geo3 &g) { return DIR == 0 ? g.si : DIR == 1 ? g.sj : g.sk; }

struct CkT { static constexpr bool value = true; };     // step with range checks
struct FastT { static constexpr bool value = false; };  // interior step

template <int DIR, int LIM, int GC, bool PER, bool TOPO>
__global__ void __launch_bounds__(128, 1) k_advect_march(Layout L, Box box, int nocycle, double eps, int seg,
                                                      int ngroups, const double *__restrict__ cin,
                                                      double *__restrict__ cout,
                                                      const double *__restrict__ vel,
                                                      const double *__restrict__ vghost,
                                                      const double *__restrict__ deld, Geo4 vf, Geo3 sig,
                                                      Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                      DevScalars *sc, double *__restrict__ out1,
                                                      double *__restrict__ out2) {
  // flux areas are grain independent except in z (settling speed per grain)
  constexpr int NU = (DIR == 2) ? GC : 1;
  const int gg = blockIdx.x % ngroups;
  const int a = (blockIdx.x / ngroups) * 32 + threadIdx.x + 1;   // lane index
  const int o = blockIdx.y * 4 + threadIdx.y + 1;                // other index
  const int na = (DIR == 0) ? L.ny : L.nx;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int nother = (DIR == 2) ? L.ny : L.nz;
  if (a > na || o > nother) return;  // no barriers below
  const int g0 = gg * GC;
  const int s0 = 1 + blockIdx.z * seg;
  const int s1 = min(n, s0 + seg - 1);
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? L.P : L.PY;
  const long base = (DIR == 0) ? L.cell(1, a, o) : (DIR == 1) ? L.cell(a, 1, o) : L.cell(a, o, 1);
  bool lane_active;
  if (DIR == 0) lane_active = a >= box.jmin && a <= box.jmax && o >= box.kmin && o <= box.kmax;
  else if (DIR == 1) lane_active = a >= box.imin && a <= box.imax && o >= box.kmin && o <= box.kmax;
  else lane_active = a >= box.imin && a <= box.imax && o >= box.jmin && o <= box.jmax;
  bool gval[GC], gal[GC];
  const double *pq[GC];
  double *po[GC];
  const double *pvf[GC];
  bool any = false;
#pragma unroll
  for (int q = 0; q < GC; q++) {
    const int g = g0 + q;
    gval[q] = g < L.ns;
    gal[q] = gval[q] && lane_active && aloft[g] != 0;
    pq[q] = cin + (long)(gval[q] ? g : 0) * L.PG + base;
    po[q] = cout + (long)(gval[q] ? g : 0) * L.PG + base;
    // vf line of this grain at sweep index c: pvf[q][(c+1)*vf.sk] (z only)
    pvf[q] = vf.p + (long)(a + 1) * vf.si + (long)(o + 1) * vf.sj + (long)(gval[q] ? g : 0) * vf.sg;
    any = any || gal[q];
  }
  if (!any) {  // nothing to advect here: the reference leaves zeros
#pragma unroll
    for (int q = 0; q < GC; q++)
      if (gval[q])
        for (int c = s0; c <= s1; c++) po[q][(long)(c - 1) * st] = 0.0;
    return;
  }
  const LineGeo gsig = line_of<DIR>(sig, a, o);
  const LineGeo gdtv = line_of<DIR>(dtvt, a, o);  // dt/kappa of this step
  const double *pv = vel + base;
  const double *pvg = vghost + base;  // ghost levels of z: plain vz (no vh)
  // DelDonD_cc(c) of this line (ZScaling_ID 2, :163-166; 0 outside
  // rmin-1..rmax+1): x row (j = a) at (c+1) + (a+1)*(nx+4), y column (i = a)
  // at (a+1) + (c+1)*(nx+4)
  const long dst = (DIR == 0) ? 1 : (long)(L.nx + 4);
  const double *pd = TOPO ? ((DIR == 0) ? deld + 1 + (long)(a + 1) * (L.nx + 4) : deld + (a + 1) + (L.nx + 4))
                          : nullptr;
  // top-outflow cell: n+1 for x and y; update_cc(ncells+1) for z (:309-311)
  const int ctop = (DIR == 2) ? ncells + 1 : rmax + 1;
  if (DIR == 2 && rmax == n && ctop < rmin - 1) raise_error(sc, A3G_ERR_UNSUPPORTED, 311);
  const bool out_lo = !PER && rmin == 1;
  const bool out_hi = !PER && rmax == n;
  const int cs = (s0 == 1 && out_lo) ? 0 : s0;
  const int ce = (s1 == n && out_hi) ? n + 1 : s1;
  const long oo_base = (long)(o - 1) * na + (a - 1);
  const long oslab = (long)na * nother;

  // ghost-aware loads (Set_BC(1): zero concentration, edge or periodic winds)
  auto wrap = [&](int c) { return c < 1 ? c + n : (c > n ? c - n : c); };
  auto qload = [&](int q, int c) -> double {
    if (c < rmin - 2 || c > rmax + 2) return 0.0;
    if (c >= 1 && c <= n) return pq[q][(long)(c - 1) * st];
    if (PER) return pq[q][(long)(wrap(c) - 1) * st];
    return 0.0;
  };
  auto vload = [&](int c) -> double {
    const int cl = PER ? wrap(c) : (c < 1 ? 1 : (c > n ? n : c));
    const double *src = (DIR == 2 && (c < 1 || c > n)) ? pvg : pv;
    return src[(long)(cl - 1) * st];
  };
  auto dload = [&](int c) -> double {
    return (c >= rmin - 1 && c <= rmax + 1) ? pd[(long)c * dst] : 0.0;
  };
  auto vfload = [&](int q, int c) -> double {
    const int cl = c < 1 ? 1 : (c > n ? n : c);
    return pvf[q][(long)(cl + 1) * vf.sk];
  };
  auto fs_ok = [&](int I) { return I >= rmin - 1 && I <= rmax + 1; };
  auto fss_ok = [&](int I) { return I >= rmin && I <= rmax + 1; };

  // ---- prologue at cell cs: interface cs, window q(cs), q(cs+1) ----------
  double q0[GC], q1[GC], d0[GC], d1[GC], fss0[GC], fsr0[GC];
  double usA[NU], usB[NU], vB[NU];  // us(c), us(c+1), vel(c+1) (+vf for z)
  double dtv0 = gdtv.at(cs);
  // topography term T(c) = 0.5*vel(c)*(sig(c)+sig(c+1))*q(c)*DelDonD(c) of
  // :251-257 (fs_r(I) += T(I), fs_l(I) -= T(I-1)): tp = T(c) per grain,
  // sB = sig(c+1) unmasked
  double tp[GC], sB = 0.0;
  {
    const double vm2 = vload(cs - 2), vm1 = vload(cs - 1), v0 = vload(cs), v1 = vload(cs + 1);
    const double sm1 = fs_ok(cs - 1) ? gsig.at(cs - 1) : 0.0;
    const double s0_ = fs_ok(cs) ? gsig.at(cs) : 0.0;
    const double s1_ = fs_ok(cs + 1) ? gsig.at(cs + 1) : 0.0;
    double usm1[NU];
#pragma unroll
    for (int u = 0; u < NU; u++) {
      double va = vm2, vb = vm1, vc = v0, vd = v1;
      if (DIR == 2) {
        va = va + vfload(u, cs - 2);
        vb = vb + vfload(u, cs - 1);
        vc = vc + vfload(u, cs);
        vd = vd + vfload(u, cs + 1);
      }
      usm1[u] = fs_ok(cs - 1) ? 0.5 * (va + vb) * sm1 : 0.0;
      usA[u] = fs_ok(cs) ? 0.5 * (vb + vc) * s0_ : 0.0;
      usB[u] = fs_ok(cs + 1) ? 0.5 * (vc + vd) * s1_ : 0.0;
      vB[u] = vd;
    }
#pragma unroll
    for (int q = 0; q < GC; q++) {
      const int u = (DIR == 2) ? q : 0;
      const double qm2 = qload(q, cs - 2), qm1 = qload(q, cs - 1);
      q0[q] = qload(q, cs);
      q1[q] = qload(q, cs + 1);
      const double dm = qm1 - qm2;
      d0[q] = q0[q] - qm1;
      d1[q] = q1[q] - q0[q];
      const Iface f = make_iface(usm1[u], usA[u], usB[u], dtv0, fss_ok(cs), fs_ok(cs));
      double fsl_unused;
      iface_grain<LIM>(f, dm, d0[q], d1[q], qm1, q0[q], eps, nocycle, fss0[q], fsr0[q], fsl_unused);
      if (TOPO) {
        const double t0 = (((0.5 * v0) * (gsig.at(cs) + gsig.at(cs + 1))) * q0[q]) * dload(cs);
        if (fs_ok(cs)) fsr0[q] = fsr0[q] + t0;
        tp[q] = t0;
      }
    }
    if (TOPO) sB = gsig.at(cs + 1);
  }

  // ---- one march step: interface c+1 and the update of cell c -------------
  // The values at the leading edge (q(c+2), vel(c+2), sigma(c+2), vf(c+2),
  // dt/kappa(c+1)) are passed in, so that the interior loop can load them
  // PF steps ahead.
  auto step = [&](int c, auto checked, const double *q2v, double vn, double sI2raw, double dtv1,
                  const double *vf2) {
    constexpr bool CK = decltype(checked)::value;
    const int I = c + 1;
    const bool fsok2 = CK ? fs_ok(c + 2) : true;
    const bool fsok1 = CK ? fs_ok(I) : true;
    const bool fssok1 = CK ? fss_ok(I) : true;
    const double sI2 = fsok2 ? sI2raw : 0.0;
    const bool own = CK ? (c >= s0 && c <= s1) : true;
    const bool inbox = CK ? (c >= rmin && c <= rmax) : true;
    const double vc1 = vB[0];                     // vel(c+1) (x, y)
    const double dcur = TOPO ? dload(I) : 0.0;    // DelDonD(c+1)
    Iface f[NU];
#pragma unroll
    for (int u = 0; u < NU; u++) {
      double vnq = vn;
      if (DIR == 2) vnq = vnq + vf2[u];
      const double usC = fsok2 ? 0.5 * (vB[u] + vnq) * sI2 : 0.0;
      vB[u] = vnq;
      f[u] = make_iface(usA[u], usB[u], usC, dtv1, fssok1, fsok1);
      usA[u] = usB[u];
      usB[u] = usC;
    }
#pragma unroll
    for (int q = 0; q < GC; q++) {
      const double q2 = q2v[q];
      const double d2 = q2 - q1[q];
      double fss1, fsr1, fsl1;
      iface_grain<LIM>(f[(DIR == 2) ? q : 0], d0[q], d1[q], d2, q0[q], q1[q], eps, nocycle, fss1, fsr1,
                       fsl1);
      if (TOPO) {
        const double t1 = (((0.5 * vc1) * (sB + sI2raw)) * q1[q]) * dcur;
        if (fsok1) {
          fsr1 = fsr1 + t1;
          fsl1 = fsl1 - tp[q];
        }
        tp[q] = t1;
      }
      const double upd = cell_update(dtv0, fsl1, fsr0[q], fss1, fss0[q]);
      if (gval[q]) {
        if (own) po[q][(long)(c - 1) * st] = (gal[q] && inbox) ? q0[q] + upd : 0.0;
        if (gal[q]) {
          if (CK && out_lo && c == 0) out1[(long)(g0 + q) * oslab + oo_base] += upd;
          if (out_hi && c == ctop) out2[(long)(g0 + q) * oslab + oo_base] += upd;
        }
      }
      fss0[q] = fss1;
      fsr0[q] = fsr1;
      q0[q] = q1[q];
      q1[q] = q2;
      d0[q] = d1[q];
      d1[q] = d2;
    }
    dtv0 = dtv1;
    if (TOPO) sB = sI2raw;
  };
  auto checked_step = [&](int c) {
    double q2v[GC], vf2[NU];
#pragma unroll
    for (int q = 0; q < GC; q++) q2v[q] = qload(q, c + 2);
#pragma unroll
    for (int u = 0; u < NU; u++) vf2[u] = (DIR == 2) ? vfload(u, c + 2) : 0.0;
    // unmasked for the topography term (sigma is ghosted to n+2)
    const double sraw = (TOPO ? (c + 2 <= n + 2) : fs_ok(c + 2)) ? gsig.at(c + 2) : 0.0;
    step(c, CkT{}, q2v, vload(c + 2), sraw, gdtv.at(c + 1), vf2);
  };
  // cells whose step needs no range checks: c >= rmin, c+2 <= min(n, rmax+1)
  int fa = max(cs, max(rmin, s0)), fb = min(ce, min(rmax - 1, n - 2));
  if (fb < fa) { fa = ce + 1; fb = ce; }
  int c = cs;
  for (; c < fa; c++) checked_step(c);
  if (fa <= fb) {
    // interior: leading-edge values come from a PF-deep ring loaded ahead;
    // loads stay inside the fast range (position <= fb+2 for q, vel, sigma,
    // vf; <= fb+1 for dt/kappa)
    constexpr int PF = 4;
    double rq[PF][GC], rv[PF], rs[PF], rd[PF], rf[PF][NU];
    auto fill = [&](int r, int cc) {  // leading-edge values of step cc into slot r
      const bool okq = cc + 2 <= fb + 2;
#pragma unroll
      for (int q = 0; q < GC; q++) rq[r][q] = okq ? pq[q][(long)(cc + 1) * st] : 0.0;
      rv[r] = okq ? pv[(long)(cc + 1) * st] : 0.0;
      rs[r] = okq ? gsig.at(cc + 2) : 0.0;
      rd[r] = okq ? gdtv.at(cc + 1) : 0.0;
#pragma unroll
      for (int u = 0; u < NU; u++) rf[r][u] = (DIR == 2 && okq) ? pvf[u][(long)(cc + 3) * vf.sk] : 0.0;
    };
#pragma unroll
    for (int r = 0; r < PF; r++) fill(r, fa + r);
    for (; c + PF - 1 <= fb; c += PF) {
#pragma unroll
      for (int r = 0; r < PF; r++) {
        double q2v[GC], vf2[NU];
#pragma unroll
        for (int q = 0; q < GC; q++) q2v[q] = rq[r][q];
#pragma unroll
        for (int u = 0; u < NU; u++) vf2[u] = rf[r][u];
        const double vn = rv[r], sr = rs[r], dd = rd[r];
        fill(r, c + r + PF);
        step(c + r, FastT{}, q2v, vn, sr, dd, vf2);
      }
    }
    // tail of the interior (fewer than PF steps); c - fa is a multiple of PF
#pragma unroll
    for (int r = 0; r < PF; r++) {
      if (c + r <= fb) {
        double q2v[GC], vf2[NU];
#pragma unroll
        for (int q = 0; q < GC; q++) q2v[q] = rq[r][q];
#pragma unroll
        for (int u = 0; u < NU; u++) vf2[u] = rf[r][u];
        step(c + r, FastT{}, q2v, rv[r], rs[r], rd[r], vf2);
      }
    }
    c = fb + 1;
  }
  for (; c <= ce; c++) checked_step(c);
}

// ---------------------------------------------------------------------------
// Block sweep: a thread computes V consecutive cells of one line for one
// grain with every input of the block loaded up front (q and the winds on
// cells c0-2 .. c0+V+1).  The V+1 interfaces of the block are independent
// straight-line code, which gives the scheduler V+1 limiter chains to
// interleave.  The limiter is written with selects (no divergent branches):
// the quotient is formed for every interface from safe operands and then
// selected.
// DIR 0: lanes are consecutive blocks along i of one row (contiguous memory,
// vector loads); DIR 1/2: lanes are consecutive i (coalesced).
// ---------------------------------------------------------------------------
template <int LIM>
__device__ __forceinline__ double fss_select(double dqm, double dq, double dqp, bool up, double cf,
                                             bool fss_ok, double eps, int nocycle) {
  if (LIM == A3G_LIM_NONE) return 0.0;
  const double adq = fabs(dq);
  const bool skip = (!nocycle && adq <= eps) || !fss_ok;  // :183 "cycle" (fss stays 0)
  double ldq;
  if (LIM == A3G_LIM_LAXWEN) {
    ldq = dq;
  } else {
    const double dqu = up ? dqm : dqp;
    const bool clamp = fabs(dqu) > 3.0 * adq || adq < eps;
    const bool use_div = !(skip || clamp);
    const double th = div_rn(use_div ? dqu : 1.0, use_div ? dq : 1.0);
    const double theta = clamp ? copysign(3.0, dqu * dq) : th;
    if (LIM == A3G_LIM_BW) ldq = dqu;
    else if (LIM == A3G_LIM_FROMM) ldq = dq * (0.5 * (1.0 + theta));
    else if (LIM == A3G_LIM_MINMOD) ldq = dq * dmx(0.0, dmn(1.0, theta));
    else if (LIM == A3G_LIM_MC) ldq = dq * dmx(0.0, dmn(dmn((1.0 + theta) / 2.0, 2.0), 2.0 * theta));
    else ldq = dq * dmx(dmx(0.0, dmn(1.0, 2.0 * theta)), dmn(2.0, theta));
  }
  return skip ? 0.0 : cf * ldq;
}

template <int DIR, int LIM, int V, bool PER, bool CK, bool LC>
__device__ __forceinline__ void block_body(const Layout &L, const Box &box, int nocycle, double eps,
                                           const double *__restrict__ line, double *__restrict__ oline,
                                           long st, const double *__restrict__ pv,
                                           const double *__restrict__ pvg, const double *pvf,
                                           long vfs, const LineGeo &gsig, const LineGeo &gdtv, int c0,
                                           int n, bool lane_active, bool al, double *o1, double *o2,
                                           DevScalars *sc) {
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  const bool out_lo = !PER && rmin == 1;
  const bool out_hi = !PER && rmax == n;
  const int ctop = (DIR == 2) ? ncells + 1 : rmax + 1;
  auto wrap = [&](int c) { return c < 1 ? c + n : (c > n ? c - n : c); };
  // window w[m] = q(c0-2+m), vw[m] = vel(c0-2+m) (+vf for z), m = 0..V+3
  double w[V + 4], vw[V + 4];
  if (!CK && DIR == 0) {
    const double2 *p2 = reinterpret_cast<const double2 *>(line + (c0 - 3));
    const double2 *v2 = reinterpret_cast<const double2 *>(pv + (c0 - 3));
#pragma unroll
    for (int m = 0; m < (V + 4) / 2; m++) {
      const double2 a = p2[m], b = v2[m];
      w[2 * m] = a.x; w[2 * m + 1] = a.y;
      vw[2 * m] = b.x; vw[2 * m + 1] = b.y;
    }
  } else {
#pragma unroll
    for (int m = 0; m < V + 4; m++) {
      const int c = c0 - 2 + m;
      if (CK) {
        double q = 0.0;
        if (c >= rmin - 2 && c <= rmax + 2) {
          if (c >= 1 && c <= n) q = line[(long)(c - 1) * st];
          else if (PER) q = line[(long)(wrap(c) - 1) * st];
        }
        w[m] = q;
        const int cl = PER ? wrap(c) : (c < 1 ? 1 : (c > n ? n : c));
        vw[m] = ((DIR == 2 && (c < 1 || c > n)) ? pvg : pv)[(long)(cl - 1) * st];
      } else {
        w[m] = line[(long)(c - 1) * st];
        vw[m] = pv[(long)(c - 1) * st];
      }
    }
  }
  // LC: sigma, dt/kappa and (z) the fall speed do not vary along the line
  // (zero broadcast stride), so one load of each serves every index
  const double sig_c = LC ? gsig.p[0] : 0.0, dtv_c = LC ? gdtv.p[0] : 0.0;
  if (DIR == 2) {
    const double vf_c = LC ? pvf[0] : 0.0;
#pragma unroll
    for (int m = 0; m < V + 4; m++) {
      const int c = c0 - 2 + m;
      const int cl = CK ? (c < 1 ? 1 : (c > n ? n : c)) : c;
      vw[m] = vw[m] + (LC ? vf_c : pvf[(long)(cl + 1) * vfs]);
    }
  }
  auto fs_ok = [&](int I) { return !CK || (I >= rmin - 1 && I <= rmax + 1); };
  auto fss_ok = [&](int I) { return !CK || (I >= rmin && I <= rmax + 1); };
  // flux areas us(I), I = c0-1 .. c0+V+1  (us index u = I - (c0-1))
  double us[V + 3];
#pragma unroll
  for (int u = 0; u < V + 3; u++) {
    const int I = c0 - 1 + u;
    us[u] = fs_ok(I) ? 0.5 * (vw[u] + vw[u + 1]) * (LC ? sig_c : gsig.at(I)) : 0.0;
  }
  double dtv[V + 1];
#pragma unroll
  for (int m = 0; m <= V; m++) dtv[m] = LC ? dtv_c : gdtv.at(c0 + m);
  // interfaces I = c0+m, m = 0..V
  double fss[V + 1], fsr[V + 1], fsl[V + 1];
#pragma unroll
  for (int m = 0; m <= V; m++) {
    const int I = c0 + m;
    const Iface f = make_iface(us[m], us[m + 1], us[m + 2], dtv[m], fss_ok(I), fs_ok(I));
    const double dqm = w[m + 1] - w[m], dq = w[m + 2] - w[m + 1], dqp = w[m + 3] - w[m + 2];
    fss[m] = fss_select<LIM>(dqm, dq, dqp, f.up, f.cf, f.fss_ok, eps, nocycle);
    if (f.fs_ok) {
      fsr[m] = f.usp * dq;
      fsl[m] = f.usm * dq;
      fsr[m] = fsr[m] + w[m + 2] * f.divm;
      fsl[m] = fsl[m] + w[m + 1] * f.divp;
    } else {
      fsr[m] = 0.0;
      fsl[m] = 0.0;
    }
  }
  double outv[V];
#pragma unroll
  for (int v = 0; v < V; v++) {
    const int c = c0 + v;
    const double upd = cell_update(dtv[v], fsl[v + 1], fsr[v], fss[v + 1], fss[v]);
    const bool inbox = !CK || (c >= rmin && c <= rmax);
    outv[v] = (al && inbox) ? w[v + 2] + upd : 0.0;
    if (CK && al && out_hi && c == n) {  // cell n+1 (x, y; z when kmin == 1)
      const double updh = cell_update(dtv[v + 1], 0.0, fsr[v + 1], 0.0, fss[v + 1]);
      if (ctop == n + 1) *o2 += updh;
    }
    if (al && out_hi && c == ctop && c <= n) *o2 += upd;  // z quirk: ctop inside the column
  }
  if (CK && al && out_lo && c0 == 1) {
    // cell 0 from interfaces 0 and 1; fss(0) = 0 since rmin = 1
    const double us_m1 = 0.0;  // interface -1 is outside [rmin-1, rmax+1]
    const double dtv0 = LC ? dtv_c : gdtv.at(0);
    const Iface f0 = make_iface(us_m1, us[0], us[1], dtv0, false, true);
    const double dq0 = w[1] - w[0];
    const double fsr0 = f0.usp * dq0 + w[1] * f0.divm;
    const double upd0 = cell_update(dtv0, fsl[0], fsr0, fss[0], 0.0);
    *o1 += upd0;
  }
  if (DIR == 2 && CK && out_hi && ctop < rmin - 1) raise_error(sc, A3G_ERR_UNSUPPORTED, 311);
  // store own cells
  if (!CK && DIR == 0) {
    double2 *po = reinterpret_cast<double2 *>(oline + (c0 - 1));
#pragma unroll
    for (int v = 0; v < V / 2; v++) po[v] = make_double2(outv[2 * v], outv[2 * v + 1]);
  } else {
#pragma unroll
    for (int v = 0; v < V; v++) {
      const int c = c0 + v;
      if (!CK || c <= n) oline[(long)(c - 1) * st] = outv[v];
    }
  }
}

template <int DIR, int LIM, int V, bool PER, bool LC>
// 7 blocks of 128 per SM (at most 72 registers, a few spilled to L1): more
// warps in flight beat the spills (C2 z sweep 2.15 -> 1.81 ms on B200)
__global__ void __launch_bounds__(128, 7) k_advect_block(Layout L, Box box, int nocycle, double eps, int nblk,
                                                      const double *__restrict__ cin,
                                                      double *__restrict__ cout,
                                                      const double *__restrict__ vel,
                                                      const double *__restrict__ vghost, Geo4 vf, Geo3 sig,
                                                      Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                      DevScalars *sc, double *__restrict__ out1,
                                                      double *__restrict__ out2) {
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  int a, o, blk, g;  // lane index (i or j), other index, block, grain
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
  bool lane_active;
  if (DIR == 0) lane_active = a >= box.jmin && a <= box.jmax && o >= box.kmin && o <= box.kmax;
  else if (DIR == 1) lane_active = a >= box.imin && a <= box.imax && o >= box.kmin && o <= box.kmax;
  else lane_active = a >= box.imin && a <= box.imax && o >= box.jmin && o <= box.jmax;
  const bool al = lane_active && aloft[g] != 0;
  double *oline = cout + (long)g * L.PG + base;
  if (!al) {  // the reference leaves zeros
    for (int v = 0; v < V; v++)
      if (c0 + v <= n) oline[(long)(c0 + v - 1) * st] = 0.0;
    return;
  }
  const double *line = cin + (long)g * L.PG + base;
  const double *pv = vel + base;
  const double *pvg = vghost + base;
  const double *pvf = vf.p + (long)(((DIR == 0) ? 0 : a) + 1) * vf.si +
                      (long)(((DIR == 2) ? o : 0) + 1) * vf.sj + (long)g * vf.sg;
  const LineGeo gsig = line_of<DIR>(sig, a, o);
  const LineGeo gdtv = line_of<DIR>(dtvt, a, o);
  const int rmin = (DIR == 0) ? box.imin : (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 0) ? box.imax : (DIR == 1) ? box.jmax : box.kmax;
  const long na = (DIR == 0) ? L.ny : L.nx;
  const long nother = (DIR == 2) ? L.ny : L.nz;
  const long oo = (long)g * na * nother + (long)(o - 1) * na + (a - 1);
  const bool fast = c0 >= 3 && c0 >= rmin && c0 + V <= rmax && c0 + V <= n - 1;
  if (fast)
    block_body<DIR, LIM, V, PER, false, LC>(L, box, nocycle, eps, line, oline, st, pv, pvg, pvf, vf.sk, gsig, gdtv,
                                        c0, n, lane_active, al, out1 + oo, out2 + oo, sc);
  else
    block_body<DIR, LIM, V, PER, true, LC>(L, box, nocycle, eps, line, oline, st, pv, pvg, pvf, vf.sk, gsig, gdtv,
                                       c0, n, lane_active, al, out1 + oo, out2 + oo, sc);
}

// ---------------------------------------------------------------------------
// Warp-tiled x sweep.  A warp owns 32 x rows (row r = (g*nz + k-1)*ny + j-1
// starts at r*P; its winds at (r mod ny*nz)*P) and marches them side by side,
// one lane per row, over the whole row.  The leading-edge values of each
// step (q and the wind at cell c+2) come from shared-memory tiles of XA_TW
// columns that the warp fills with coalesced row segments, and the updated
// cells go out through a third tile the same way, so no lane touches global
// memory row-wise in the interior.  The arithmetic of a step is the march's
// (make_iface, iface_grain, cell_update in the same order), so the results
// are the same bits.  No lane returns early: lanes of rows past the end, of
// rows outside the box or of grains not aloft take part in the tile traffic
// and write zeros (or nothing past the last row).
// ---------------------------------------------------------------------------
constexpr int XA_TW = 16;        // tile width (cells)
constexpr int XA_S = XA_TW + 1;  // tile row stride (odd: conflict-free per-lane reads)
constexpr int XA_WARPS = 2;

template <int LIM, bool PER>
__global__ void __launch_bounds__(32 * XA_WARPS) k_advect_xt(Layout L, Box box, int nocycle, double eps,
                                                           const double *__restrict__ cin,
                                                           double *__restrict__ cout,
                                                           const double *__restrict__ vel, Geo3 sig,
                                                           Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                           double *__restrict__ out1,
                                                           double *__restrict__ out2) {
  __shared__ double tq[XA_WARPS][32 * XA_S], tv[XA_WARPS][32 * XA_S], to[XA_WARPS][32 * XA_S];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long nrows = (long)L.ny * L.nz * L.ns;
  const long r0 = ((long)blockIdx.x * XA_WARPS + w) * 32;
  if (r0 >= nrows) return;  // uniform over the warp
  double *const sq = tq[w], *const sv = tv[w], *const so = to[w];
  const long plane = (long)L.ny * L.nz;
  const long r = r0 + lane;
  const bool valid = r < nrows;
  const long rc = valid ? r : nrows - 1;
  const int j = (int)(rc % L.ny) + 1;
  const int k = (int)((rc / L.ny) % L.nz) + 1;
  const int g = (int)(rc / plane);
  const int n = L.nx;
  const int rmin = box.imin, rmax = box.imax;
  const bool lane_active = j >= box.jmin && j <= box.jmax && k >= box.kmin && k <= box.kmax;
  const bool al = valid && lane_active && aloft[g] != 0;
  const long P = L.P;
  const double *pq = cin + rc * P;          // own row
  const double *pv = vel + (rc % plane) * P;
  const LineGeo gsig = line_of<0>(sig, j, k);
  const LineGeo gdtv = line_of<0>(dtvt, j, k);
  const bool out_lo = !PER && rmin == 1;
  const bool out_hi = !PER && rmax == n;
  const int ctop = rmax + 1;
  const long oo = (long)g * L.ny * L.nz + (long)(k - 1) * L.ny + (j - 1);
  auto wrap = [&](int c) { return c < 1 ? c + n : (c > n ? c - n : c); };
  // ghost-aware values of cell c of a row (Set_BC(1): zero concentration,
  // edge or periodic winds); cells beyond the reach of any step give 0
  auto qval = [&](const double *row, int c) -> double {
    if (c < rmin - 2 || c > rmax + 2 || c < -1 || c > n + 2) return 0.0;
    if (c >= 1 && c <= n) return row[c - 1];
    return PER ? row[wrap(c) - 1] : 0.0;
  };
  auto vval = [&](const double *row, int c) -> double {
    if (c < -1 || c > n + 2) return 0.0;
    const int cl = PER ? wrap(c) : (c < 1 ? 1 : (c > n ? n : c));
    return row[cl - 1];
  };
  // tile of cells t0 .. t0+XA_TW-1 for the warp's 32 rows
  auto load_tiles = [&](int t0) {
#pragma unroll 4
    for (int it = 0; it < 32 * XA_TW / 32; it++) {
      const int row = it * (32 / XA_TW) + lane / XA_TW, col = lane % XA_TW;
      const long rr = r0 + row;
      double a = 0.0, b = 0.0;
      if (rr < nrows) {
        a = qval(cin + rr * P, t0 + col);
        b = vval(vel + (rr % plane) * P, t0 + col);
      }
      sq[row * XA_S + col] = a;
      sv[row * XA_S + col] = b;
    }
    __syncwarp();
  };
  // output tile of cells o0 .. o0+XA_TW-1 (only cells 1..n are stored)
  auto flush = [&](int o0) {
    __syncwarp();
#pragma unroll 4
    for (int it = 0; it < 32 * XA_TW / 32; it++) {
      const int row = it * (32 / XA_TW) + lane / XA_TW, col = lane % XA_TW;
      const long rr = r0 + row;
      const int c = o0 + col;
      if (rr < nrows && c >= 1 && c <= n) cout[rr * P + (c - 1)] = so[row * XA_S + col];
    }
    __syncwarp();
  };
  auto fs_ok = [&](int I) { return I >= rmin - 1 && I <= rmax + 1; };
  auto fss_ok = [&](int I) { return I >= rmin && I <= rmax + 1; };
  const int cs = out_lo ? 0 : 1;
  const int ce = out_hi ? n + 1 : n;

  // ---- prologue at cell cs: interface cs, window q(cs), q(cs+1) ----
  double q0, q1, d0, d1, fss0, fsr0, usA, usB, vB;
  double dtv0 = gdtv.at(cs);
  {
    const double vm2 = vval(pv, cs - 2), vm1 = vval(pv, cs - 1), v0 = vval(pv, cs), v1 = vval(pv, cs + 1);
    const double sm1 = fs_ok(cs - 1) ? gsig.at(cs - 1) : 0.0;
    const double s0_ = fs_ok(cs) ? gsig.at(cs) : 0.0;
    const double s1_ = fs_ok(cs + 1) ? gsig.at(cs + 1) : 0.0;
    const double usm1 = fs_ok(cs - 1) ? 0.5 * (vm2 + vm1) * sm1 : 0.0;
    usA = fs_ok(cs) ? 0.5 * (vm1 + v0) * s0_ : 0.0;
    usB = fs_ok(cs + 1) ? 0.5 * (v0 + v1) * s1_ : 0.0;
    vB = v1;
    const double qm2 = qval(pq, cs - 2), qm1 = qval(pq, cs - 1);
    q0 = qval(pq, cs);
    q1 = qval(pq, cs + 1);
    const double dm = qm1 - qm2;
    d0 = q0 - qm1;
    d1 = q1 - q0;
    const Iface f = make_iface(usm1, usA, usB, dtv0, fss_ok(cs), fs_ok(cs));
    double fsl_unused;
    iface_grain<LIM>(f, dm, d0, d1, qm1, q0, eps, nocycle, fss0, fsr0, fsl_unused);
  }
  // steps that need no range checks: c >= rmin, c+2 <= min(n, rmax+1)
  const int fa = max(cs, rmin), fb = min(ce, min(rmax - 1, n - 2));
  int t0 = cs + 2;  // q/vel tile holds cells t0 .. t0+XA_TW-1 (the c+2 of steps c)
  load_tiles(t0);
  int o0 = 1;       // output tile holds cells o0 .. o0+XA_TW-1
  for (int c = cs; c <= ce; c++) {
    if (c + 2 >= t0 + XA_TW) {  // uniform: every lane is at the same c
      t0 += XA_TW;
      __syncwarp();
      load_tiles(t0);
    }
    const int ti = lane * XA_S + (c + 2 - t0);
    const double q2 = sq[ti], vn = sv[ti];
    const int I = c + 1;
    const bool fast = c >= fa && c <= fb;
    const bool fsok2 = fast || fs_ok(c + 2);
    const double sI2 = fsok2 ? gsig.at(c + 2) : 0.0;
    const double dtv1 = gdtv.at(I);
    const double usC = fsok2 ? 0.5 * (vB + vn) * sI2 : 0.0;
    vB = vn;
    const Iface f = make_iface(usA, usB, usC, dtv1, fast || fss_ok(I), fast || fs_ok(I));
    usA = usB;
    usB = usC;
    const double d2 = q2 - q1;
    double fss1, fsr1, fsl1;
    iface_grain<LIM>(f, d0, d1, d2, q0, q1, eps, nocycle, fss1, fsr1, fsl1);
    const double upd = cell_update(dtv0, fsl1, fsr0, fss1, fss0);
    if (c >= 1 && c <= n) {
      const bool inbox = c >= rmin && c <= rmax;
      so[lane * XA_S + (c - o0)] = (al && inbox) ? q0 + upd : 0.0;
      if (c == o0 + XA_TW - 1 || c == n) {
        flush(o0);
        o0 += XA_TW;
      }
    }
    if (al) {
      if (out_lo && c == 0) out1[oo] += upd;
      if (out_hi && c == ctop) out2[oo] += upd;
    }
    fss0 = fss1;
    fsr0 = fsr1;
    q0 = q1;
    q1 = q2;
    d0 = d1;
    d1 = d2;
    dtv0 = dtv1;
  }
}

template <int LIM>
static void launch_advect_xt(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const long nrows = (long)L.ny * L.nz * L.ns;
  const long nwarps = (nrows + 31) / 32;
  const unsigned blocks = (unsigned)((nwarps + XA_WARPS - 1) / XA_WARPS);
  if (ctx->grid.periodic)
    k_advect_xt<LIM, true><<<blocks, 32 * XA_WARPS, 0, ctx->stream>>>(
        L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ctx->c0, ctx->c1, ctx->vx, ctx->snx, ctx->dtv,
        ctx->aloft, ctx->out_yz1, ctx->out_yz2);
  else
    k_advect_xt<LIM, false><<<blocks, 32 * XA_WARPS, 0, ctx->stream>>>(
        L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ctx->c0, ctx->c1, ctx->vx, ctx->snx, ctx->dtv,
        ctx->aloft, ctx->out_yz1, ctx->out_yz2);
}

// ---------------------------------------------------------------------------
// Warp-row x sweep.  A warp owns one x row (j, k) and a group of GC grains and
// walks the row in chunks of 32 cells with the lanes along i, so every global
// load and store is a coalesced row segment.  Lane l of the chunk starting at
// cell b loads cell i = b + l, forms the flux area us(i), and computes the
// fluxes of interface I = i - 1 (which needs q(I-2..I+1), us(I-1..I+1): the
// cells behind it come from per-warp shared-memory rings of 64 entries); it
// then updates cell c = I - 1 from interface I (its own) and interface c
// (lane l-1's, through the same rings).  Each interface is computed once, in
// the march's expressions (make_iface, iface_grain, cell_update), so the
// results are the same bits.  Nothing is carried in registers between
// chunks, which keeps the register count and the L1 traffic low.
// With TMA, the loads of the interior chunks (the ones without range checks)
// arrive by tensor copies instead: the warp's GC grains and the wind of the
// chunk, one chunk ahead, into one of two staging buffers, so that the
// lanes no longer wait on global loads there.  Same arithmetic, same bits.
// ---------------------------------------------------------------------------
constexpr int XW_WARPS = 4;

template <int LIM, int GC, bool PER, bool LC, bool TMA>
__global__ void __launch_bounds__(32 * XW_WARPS, 6) k_advect_xw(const __grid_constant__ CUtensorMap tq,
                                                          const __grid_constant__ CUtensorMap tv, Layout L,
                                                          Box box, int nocycle, double eps,
                                                          int ngroups, const double *__restrict__ cin,
                                                          double *__restrict__ cout,
                                                          const double *__restrict__ vel, Geo3 sig, Geo3 dtvt,
                                                          const int32_t *__restrict__ aloft, DevScalars *sc,
                                                          double *__restrict__ out1, double *__restrict__ out2) {
  __shared__ __align__(128) double s_st[TMA ? XW_WARPS : 1][2][(GC + 1) * 32];  // staged q (GC grains), v
  __shared__ __align__(8) uint64_t s_bar[XW_WARPS][2];
  __shared__ double s_q[XW_WARPS][GC][64];
  __shared__ double s_fss[XW_WARPS][GC][64];
  __shared__ double s_fsr[XW_WARPS][GC][64];
  __shared__ double s_v[XW_WARPS][64];
  __shared__ double s_u[XW_WARPS][64];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long w = (long)blockIdx.x * XW_WARPS + wid;
  if (w >= (long)L.ny * L.nz * ngroups) return;  // whole warps only; no block barrier below
  const int j = (int)(w % L.ny) + 1;
  const int k = (int)((w / L.ny) % L.nz) + 1;
  const int g0 = (int)(w / ((long)L.ny * L.nz)) * GC;
  const int n = L.nx;
  const int rmin = box.imin, rmax = box.imax;
  const bool row_active = j >= box.jmin && j <= box.jmax && k >= box.kmin && k <= box.kmax;
  const long base = L.cell(1, j, k);
  bool gval[GC], gal[GC];
  const double *pq[GC];
  double *po[GC];
  bool any = false;
#pragma unroll
  for (int q = 0; q < GC; q++) {
    const int g = g0 + q;
    gval[q] = g < L.ns;
    gal[q] = gval[q] && row_active && aloft[g] != 0;
    pq[q] = cin + (long)(gval[q] ? g : 0) * L.PG + base;
    po[q] = cout + (long)(gval[q] ? g : 0) * L.PG + base;
    any = any || gal[q];
  }
  if (!any) {  // the reference leaves zeros
#pragma unroll
    for (int q = 0; q < GC; q++)
      if (gval[q])
        for (int c = 1 + lane; c <= n; c += 32) po[q][c - 1] = 0.0;
    return;
  }
  const LineGeo gsig = line_of<0>(sig, j, k);
  const LineGeo gdtv = line_of<0>(dtvt, j, k);
  // LC: sigma and dt/kappa do not vary along the row (zero broadcast stride)
  const double sig_c = LC ? gsig.p[0] : 0.0, dtv_c = LC ? gdtv.p[0] : 0.0;
  const double *pv = vel + base;
  const bool out_lo = !PER && rmin == 1;
  const bool out_hi = !PER && rmax == n;
  const long oo = (long)(k - 1) * L.ny + (j - 1);
  const long oslab = (long)L.ny * L.nz;
  auto wrap = [&](int c) { return c < 1 ? c + n : (c > n ? c - n : c); };
  auto fs_ok = [&](int I) { return I >= rmin - 1 && I <= rmax + 1; };
  auto fss_ok = [&](int I) { return I >= rmin && I <= rmax + 1; };
  // ring slots of the chunk before the first (cells -4..-2): zero
#pragma unroll
  for (int q = 0; q < GC; q++) {
    s_q[wid][q][32 + lane] = 0.0;
    s_fss[wid][q][32 + lane] = 0.0;
    s_fsr[wid][q][32 + lane] = 0.0;
  }
  s_v[wid][32 + lane] = 0.0;
  s_u[wid][32 + lane] = 0.0;
  // chunk t covers loads i = 32t - 1 + lane and updates cells c = i - 2.  A
  // chunk whose loads all lie in [max(rmin+2, 1), min(n, rmax+1)] needs no
  // range check (its cells are inside the box, its interfaces and flux
  // areas inside [rmin, rmax+1], no ghost or outflow cell); the others take
  // the checked body.
  const int ilo = max(rmin + 2, 1), ihi = min(n, rmax + 1);
  auto chunk = [&](int t, auto checked, const double *stg) {
    constexpr bool CK = decltype(checked)::value;
    __syncwarp();
    const int i = 32 * t - 1 + lane;
    const int sl = (32 * t + lane) & 63;
    const int sl1 = (sl + 63) & 63, sl2 = (sl + 62) & 63, sl3 = (sl + 61) & 63;
    double qi[GC];
#pragma unroll
    for (int q = 0; q < GC; q++) {
      double v = 0.0;
      if (!CK) {
        v = TMA ? stg[q * 32 + lane] : pq[q][i - 1];
      } else if (i >= rmin - 2 && i <= rmax + 2) {  // ghost cells of Set_BC(1): zero, or wrapped
        if (i >= 1 && i <= n) v = pq[q][i - 1];
        else if (PER) v = pq[q][wrap(i) - 1];
      }
      qi[q] = v;
      s_q[wid][q][sl] = v;
    }
    double vi = 0.0;  // vel(i) is read by us(i) and us(i+1) only
    if (!CK) vi = TMA ? stg[GC * 32 + lane] : pv[i - 1];
    else if (i >= rmin - 2 && i <= rmax + 1) vi = pv[(PER ? wrap(i) : (i < 1 ? 1 : (i > n ? n : i))) - 1];
    s_v[wid][sl] = vi;
    __syncwarp();
    const double usi = (!CK || fs_ok(i)) ? 0.5 * (s_v[wid][sl1] + vi) * (LC ? sig_c : gsig.at(i)) : 0.0;
    s_u[wid][sl] = usi;
    __syncwarp();
    const int I = i - 1;
    const double dtvI = (!CK || (I >= -1 && I <= n + 2)) ? (LC ? dtv_c : gdtv.at(I)) : 0.0;
    const Iface f = make_iface(s_u[wid][sl2], s_u[wid][sl1], usi, dtvI, !CK || fss_ok(I), !CK || fs_ok(I));
    double qm[GC], fsl[GC], fss[GC];
#pragma unroll
    for (int q = 0; q < GC; q++) {
      const double q3 = s_q[wid][q][sl3], q2 = s_q[wid][q][sl2], q1 = s_q[wid][q][sl1];
      double fsr;
      iface_grain<LIM>(f, q2 - q3, q1 - q2, qi[q] - q1, q2, q1, eps, nocycle, fss[q], fsr, fsl[q]);
      qm[q] = q2;
      s_fss[wid][q][sl] = fss[q];
      s_fsr[wid][q][sl] = fsr;
    }
    __syncwarp();
    const int c = I - 1;
    if (!CK || (c >= 0 && c <= n + 1)) {
      const double dtvc = LC ? dtv_c : gdtv.at(c);
      const bool inbox = !CK || (c >= rmin && c <= rmax);
#pragma unroll
      for (int q = 0; q < GC; q++) {
        const double upd = cell_update(dtvc, fsl[q], s_fsr[wid][q][sl1], fss[q], s_fss[wid][q][sl1]);
        if (gval[q]) {
          if (!CK || (c >= 1 && c <= n)) po[q][c - 1] = (gal[q] && inbox) ? qm[q] + upd : 0.0;
          if (CK && gal[q]) {
            if (out_lo && c == 0) out1[(long)(g0 + q) * oslab + oo] += upd;
            if (out_hi && c == rmax + 1) out2[(long)(g0 + q) * oslab + oo] += upd;
          }
        }
      }
    }
  };
  // the interior chunks form the run tf0..tf1
  const int tf0 = (ilo + 32) / 32, tf1 = ihi >= 30 ? (ihi - 30) / 32 : -1;
  uint32_t ph = 0u;  // bit b: the parity of staging buffer b's barrier
  auto issue = [&](int t) {  // chunk t's loads i = 32t-1 .. 32t+30 (x from 32t-2 >= 0, even)
    const int bi = (t - tf0) & 1;
    if (lane == 0) {
      mbar_arrive_expect_tx(&s_bar[wid][bi], (GC + 1) * 32 * 8);
      tma_load_4d(s_st[wid][bi], &tq, &s_bar[wid][bi], 32 * t - 2, j - 1, k - 1, g0);
      tma_load_4d(s_st[wid][bi] + GC * 32, &tv, &s_bar[wid][bi], 32 * t - 2, j - 1, k - 1, 0);
    }
  };
  if (TMA) {
    if (lane == 0) {
      mbar_init(&s_bar[wid][0], 1);
      mbar_init(&s_bar[wid][1], 1);
      mbar_init_fence();
    }
    __syncwarp();
    if (tf0 <= tf1) issue(tf0);
  }
  for (int t = 0; 32 * t - 3 <= n + 1; t++) {
    if (t >= tf0 && t <= tf1) {
      if (TMA) {
        const int bi = (t - tf0) & 1;
        if (t + 1 <= tf1) issue(t + 1);
        if (!mbar_wait(&s_bar[wid][bi], (ph >> bi) & 1u)) {
          if (lane == 0) raise_error(sc, A3G_ERR_TIMEOUT, 4);
          return;
        }
        ph ^= 1u << bi;
        chunk(t, FastT{}, s_st[wid][bi]);
      } else {
        chunk(t, FastT{}, nullptr);
      }
    } else {
      chunk(t, CkT{}, nullptr);
    }
  }
}

template <int LIM>
static void launch_advect_xw(a3g_ctx *ctx, bool tma) {
  const Layout &L = ctx->L;
  const int gc = (L.ns >= 2) ? 2 : 1;
  const int ngroups = (L.ns + gc - 1) / gc;
  const long nwarps = (long)L.ny * L.nz * ngroups;
  const unsigned blocks = (unsigned)((nwarps + XW_WARPS - 1) / XW_WARPS);
  const bool lc = along<0>(ctx->snx) == 0 && along<0>(ctx->dtv) == 0;
  CUtensorMap tq, tv;
  std::memset(&tq, 0, sizeof(tq));
  std::memset(&tv, 0, sizeof(tv));
  if (tma && !(tensor_map(ctx, ctx->c0, gc == 2 ? TM_ADV_QX2 : TM_ADV_QX1, &tq) &&
               tensor_map(ctx, ctx->vx, TM_ADV_VX, &tv)))
    tma = false;
#define A3G_XW(GC_, PER_, LC_)                                                                              \
  if (tma)                                                                                                   \
    k_advect_xw<LIM, GC_, PER_, LC_, true><<<blocks, 32 * XW_WARPS, 0, ctx->stream>>>(                      \
        tq, tv, L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ngroups, ctx->c0, ctx->c1, ctx->vx,      \
        ctx->snx, ctx->dtv, ctx->aloft, ctx->sc, ctx->out_yz1, ctx->out_yz2);                                \
  else                                                                                                       \
    k_advect_xw<LIM, GC_, PER_, LC_, false><<<blocks, 32 * XW_WARPS, 0, ctx->stream>>>(                     \
        tq, tv, L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ngroups, ctx->c0, ctx->c1, ctx->vx,      \
        ctx->snx, ctx->dtv, ctx->aloft, ctx->sc, ctx->out_yz1, ctx->out_yz2)
#define A3G_XW_LC(GC_, PER_) \
  if (lc) { A3G_XW(GC_, PER_, true); } else { A3G_XW(GC_, PER_, false); }
  if (gc == 2) {
    if (ctx->grid.periodic) { A3G_XW_LC(2, true); } else { A3G_XW_LC(2, false); }
  } else {
    if (ctx->grid.periodic) { A3G_XW_LC(1, true); } else { A3G_XW_LC(1, false); }
  }
#undef A3G_XW_LC
#undef A3G_XW
}

// the vertical wind of the z sweep: vz + vh once terrain is bound
static inline const double *dir_vel(a3g_ctx *ctx, int dir) {
  return (dir == 0) ? ctx->vx : (dir == 1) ? ctx->vy : (ctx->topo_on ? ctx->vzh : ctx->vz);
}
static inline const double *dir_vghost(a3g_ctx *ctx, int dir) {
  return (dir == 0) ? ctx->vx : (dir == 1) ? ctx->vy : ctx->vz;
}

// ---------------------------------------------------------------------------
// Column march for the y and z sweeps (DIR 1, 2): one thread per line and
// grain, lanes along i (every load and store a coalesced 256-byte row
// segment), marching the whole line with a rolling window so that each
// interface is formed once (the block kernel forms V+1 interfaces for V
// cells and loads a V+4 window).  Offsets along the line are 32-bit strides
// from per-line base pointers, the grain's fall speed is loaded once when it
// is the same in every cell (VFC), and the interior of the line runs without
// range checks.  The arithmetic of every interface and cell is block_body's
// (make_iface, fss_select, the fs_r/fs_l order, cell_update), so the results
// are the same bits.  Not periodic (only x can be), no ZScaling_ID 2 terms.
// ---------------------------------------------------------------------------
template <int DIR, int LIM, bool VFC>
__global__ void __launch_bounds__(128, 5) k_advect_col(Layout L, Box box, int nocycle, double eps,
                                                    const double *__restrict__ cin,
                                                    double *__restrict__ cout,
                                                    const double *__restrict__ vel,
                                                    const double *__restrict__ vghost, Geo4 vf, Geo3 sig,
                                                    Geo3 dtvt, const int32_t *__restrict__ aloft,
                                                    DevScalars *sc, double *__restrict__ out1,
                                                    double *__restrict__ out2) {
  static_assert(DIR == 1 || DIR == 2, "lanes along i: y and z sweeps only");
  const int a = blockIdx.x * 32 + threadIdx.x + 1;  // i
  const int o = blockIdx.y * 4 + threadIdx.y + 1;   // k (y sweep) or j (z sweep)
  const int g = blockIdx.z;
  const int nother = (DIR == 1) ? L.nz : L.ny;
  if (a > L.nx || o > nother) return;  // no barriers below
  const int n = (DIR == 1) ? L.ny : L.nz;
  const int rmin = (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  const int st = (DIR == 1) ? (int)L.P : (int)L.PY;
  const long base = (DIR == 1) ? L.cell(a, 1, o) : L.cell(a, o, 1);
  const bool lane_active = (DIR == 1) ? (a >= box.imin && a <= box.imax && o >= box.kmin && o <= box.kmax)
                                      : (a >= box.imin && a <= box.imax && o >= box.jmin && o <= box.jmax);
  const bool al = lane_active && aloft[g] != 0;
  double *po = cout + (long)g * L.PG + base;
  if (!al) {  // the reference leaves zeros
    for (int c = 1; c <= n; c++) po[(c - 1) * st] = 0.0;
    return;
  }
  const double *pq = cin + (long)g * L.PG + base;
  const double *pv = vel + base;
  const double *pvg = vghost + base;
  const LineGeo gsig = line_of<DIR>(sig, a, o);
  const LineGeo gdtv = line_of<DIR>(dtvt, a, o);
  // fall speed of this grain along the line (z only): vf(c) at pvf[(c+1)*vfs]
  const double *pvf = vf.p + (long)(a + 1) * vf.si + (long)(((DIR == 2) ? o : 0) + 1) * vf.sj + (long)g * vf.sg;
  const long vfs = vf.sk;
  const double vf0 = (DIR == 2 && VFC) ? pvf[0] : 0.0;
  const bool out_lo = rmin == 1;
  const bool out_hi = rmax == n;
  const int ctop = (DIR == 2) ? ncells + 1 : rmax + 1;  // update_cc(ncells+1) for z (:309-311)
  if (DIR == 2 && out_hi && ctop < rmin - 1) raise_error(sc, A3G_ERR_UNSUPPORTED, 311);
  const long na = L.nx;
  const long oo = (long)g * na * nother + (long)(o - 1) * na + (a - 1);
  auto fs_ok = [&](int I) { return I >= rmin - 1 && I <= rmax + 1; };
  auto fss_ok = [&](int I) { return I >= rmin && I <= rmax + 1; };
  // ghost-aware loads (Set_BC(1): zero concentration, edge winds; the z
  // ghost levels read the plain vertical wind)
  auto qload = [&](int c) -> double {
    return (c >= rmin - 2 && c <= rmax + 2 && c >= 1 && c <= n) ? pq[(c - 1) * st] : 0.0;
  };
  auto vload = [&](int c) -> double {
    const int cl = c < 1 ? 1 : (c > n ? n : c);
    double v = ((DIR == 2 && (c < 1 || c > n)) ? pvg : pv)[(cl - 1) * st];
    if (DIR == 2) v = v + (VFC ? vf0 : pvf[(long)(cl + 1) * vfs]);
    return v;
  };
  const int cs = out_lo ? 0 : 1;
  const int ce = out_hi ? n + 1 : n;
  // ---- interface cs and the window at cs ----------------------------------
  double q0 = qload(cs), q1 = qload(cs + 1);
  double d0 = q0 - qload(cs - 1), d1 = q1 - q0;
  double usA, usB, vB, dtv0 = gdtv.at(cs), fss0, fsr0;
  {
    const double vm2 = vload(cs - 2), vm1 = vload(cs - 1), v0 = vload(cs);
    vB = vload(cs + 1);
    const double usm1 = fs_ok(cs - 1) ? 0.5 * (vm2 + vm1) * gsig.at(cs - 1) : 0.0;
    usA = fs_ok(cs) ? 0.5 * (vm1 + v0) * gsig.at(cs) : 0.0;
    usB = fs_ok(cs + 1) ? 0.5 * (v0 + vB) * gsig.at(cs + 1) : 0.0;
    const double qm1 = qload(cs - 1);
    const double dm = qm1 - qload(cs - 2);
    const Iface f = make_iface(usm1, usA, usB, dtv0, fss_ok(cs), fs_ok(cs));
    fss0 = fss_select<LIM>(dm, d0, d1, f.up, f.cf, f.fss_ok, eps, nocycle);
    fsr0 = f.fs_ok ? (f.usp * d0) + q0 * f.divm : 0.0;
  }
  // ---- one step: interface c+1 and the update of cell c --------------------
  auto step = [&](int c, auto checked, double q2, double vn, double s2, double dtv1) {
    constexpr bool CK = decltype(checked)::value;
    const int I = c + 1;
    const bool fsok2 = !CK || fs_ok(c + 2);
    const double usC = fsok2 ? 0.5 * (vB + vn) * s2 : 0.0;
    vB = vn;
    const Iface f = make_iface(usA, usB, usC, dtv1, !CK || fss_ok(I), !CK || fs_ok(I));
    usA = usB;
    usB = usC;
    const double d2 = q2 - q1;
    const double fss1 = fss_select<LIM>(d0, d1, d2, f.up, f.cf, f.fss_ok, eps, nocycle);
    double fsr1 = 0.0, fsl1 = 0.0;
    if (f.fs_ok) {
      fsr1 = f.usp * d1;
      fsl1 = f.usm * d1;
      fsr1 = fsr1 + q1 * f.divm;
      fsl1 = fsl1 + q0 * f.divp;
    }
    const double upd = cell_update(dtv0, fsl1, fsr0, fss1, fss0);
    if (!CK || (c >= 1 && c <= n)) {
      const bool inbox = !CK || (c >= rmin && c <= rmax);
      po[(c - 1) * st] = inbox ? q0 + upd : 0.0;
    }
    if (CK && out_lo && c == 0) out1[oo] += upd;
    if (out_hi && c == ctop) out2[oo] += upd;
    fss0 = fss1;
    fsr0 = fsr1;
    q0 = q1;
    q1 = q2;
    d0 = d1;
    d1 = d2;
    dtv0 = dtv1;
  };
  auto checked_step = [&](int c) {
    step(c, CkT{}, qload(c + 2), vload(c + 2), fs_ok(c + 2) ? gsig.at(c + 2) : 0.0, gdtv.at(c + 1));
  };
  // steps without range checks: c >= rmin, c+2 <= min(n, rmax+1)
  int fa = max(cs, rmin), fb = min(n - 2, rmax - 1);
  if (fb < fa) { fa = ce + 1; fb = ce; }
  int c = cs;
  for (; c < fa; c++) checked_step(c);
  if (fa <= fb) {
    const double *qn = pq + (fa + 1) * st;   // q(c+2)
    const double *vn = pv + (fa + 1) * st;   // vel(c+2)
    const double *sn = gsig.p + (long)(fa + 3) * gsig.s;   // sigma(c+2)
    const double *dn = gdtv.p + (long)(fa + 2) * gdtv.s;   // dt/kappa(c+1)
    const double *fn = pvf + (long)(fa + 3) * vfs;         // vf(c+2)
    const int ss = (int)gsig.s, ds = (int)gdtv.s, fs = (int)vfs;
#pragma unroll 4
    for (; c <= fb; c++) {
      double v = *vn;
      if (DIR == 2) v = v + (VFC ? vf0 : *fn);
      step(c, FastT{}, *qn, v, *sn, *dn);
      qn += st;
      vn += st;
      sn += ss;
      dn += ds;
      if (DIR == 2 && !VFC) fn += fs;
    }
  }
  for (; c <= ce; c++) checked_step(c);
}

template <int DIR, int LIM>
static void launch_col(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const int nother = (DIR == 1) ? L.nz : L.ny;
  dim3 grid((L.nx + 31) / 32, (nother + 3) / 4, L.ns);
  const bool vfc = ctx->vf.si == 0 && ctx->vf.sj == 0 && ctx->vf.sk == 0;
#define A3G_COL(VFC_)                                                                                     \
  k_advect_col<DIR, LIM, VFC_><<<grid, dim3(32, 4), 0, ctx->stream>>>(                                  \
      L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ctx->c0, ctx->c1, dir_vel(ctx, DIR),           \
      dir_vghost(ctx, DIR), ctx->vf, (DIR == 1) ? ctx->sny : ctx->snz, ctx->dtv, ctx->aloft, ctx->sc,    \
      (DIR == 1) ? ctx->out_xz1 : ctx->out_xy1, (DIR == 1) ? ctx->out_xz2 : ctx->out_xy2)
  if (DIR == 2 && !vfc) A3G_COL(false); else A3G_COL(true);
#undef A3G_COL
}

// ---------------------------------------------------------------------------
// Column march fed by TMA chunks (y and z sweeps).  The march of k_advect_col
// -- one warp per 32 lines of 32 consecutive i at one (other index, grain),
// each interface formed once, the same step() arithmetic and so the same bits
// -- but the interior steps read the concentration and the wind of cell c+2
// from shared memory: chunks of ACH cells of both arrive by two tensor loads
// into one of two buffers per warp, the next chunk in flight while the lanes
// march through the current one, and the geometry of the chunk's cells
// (sigma, dt/kappa: the same for the warp's lines) is staged beside them.
// The prologue and the few checked steps at the line ends keep the global
// loads of k_advect_col.  Warps are ordered grain-fastest, so the grains of a
// tile run side by side and share its wind rows through L2.  Taken when the
// geometry is constant along i and the fall speed is one value per grain.
// ---------------------------------------------------------------------------
constexpr int ACT_WARPS = 2;
// doubles per warp: two buffers of (q, v) chunks and two of staged geometry
constexpr int ACT_WARP_D = 2 * 2 * ACH * 32 + 2 * 2 * ACH;
static_assert((ACT_WARP_D * 8) % 128 == 0, "warp regions stay 128-byte aligned");

template <int DIR, int LIM>
__global__ void __launch_bounds__(32 * ACT_WARPS) k_advect_colt(
    const __grid_constant__ CUtensorMap tq, const __grid_constant__ CUtensorMap tv, Layout L, Box box,
    int nocycle, double eps, const double *__restrict__ cin, double *__restrict__ cout,
    const double *__restrict__ vel, const double *__restrict__ vghost, Geo4 vf, Geo3 sig, Geo3 dtvt,
    const int32_t *__restrict__ aloft, DevScalars *sc, double *__restrict__ out1, double *__restrict__ out2) {
  static_assert(DIR == 1 || DIR == 2, "lanes along i: y and z sweeps only");
  extern __shared__ __align__(128) unsigned char act_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint64_t *bar = reinterpret_cast<uint64_t *>(act_smem) + 2 * wid;
  double *wsm = reinterpret_cast<double *>(act_smem + 128) + (long)wid * ACT_WARP_D;
  // buffer b: q chunk at wsm + b*2*ACH*32, v chunk after it; geometry of
  // buffer b at wsm + 4*ACH*32 + b*2*ACH (sigma(c+2), then dt/kappa(c+1))
  const int nother = (DIR == 1) ? L.nz : L.ny;
  const int nti = (L.nx + 31) >> 5;
  const long t = (long)blockIdx.x * ACT_WARPS + wid;
  if (t >= (long)nti * nother * L.ns) return;  // whole warps only; no block barrier below
  const int g = (int)(t % L.ns);
  const long rr = t / L.ns;
  const int it = (int)(rr % nti);
  const int o = (int)(rr / nti) + 1;  // k (y sweep) or j (z sweep)
  const int a = (it << 5) + lane + 1;  // i
  const bool valid = a <= L.nx;
  const int n = (DIR == 1) ? L.ny : L.nz;
  const int rmin = (DIR == 1) ? box.jmin : box.kmin;
  const int rmax = (DIR == 1) ? box.jmax : box.kmax;
  const int ncells = rmax - rmin + 1;
  const int st = (DIR == 1) ? (int)L.P : (int)L.PY;
  const int ac = valid ? a : 1;
  const long base = (DIR == 1) ? L.cell(ac, 1, o) : L.cell(ac, o, 1);
  const bool lane_active = (DIR == 1) ? (a >= box.imin && a <= box.imax && o >= box.kmin && o <= box.kmax)
                                      : (a >= box.imin && a <= box.imax && o >= box.jmin && o <= box.jmax);
  const bool al = valid && lane_active && aloft[g] != 0;
  double *po = cout + (long)g * L.PG + base;
  if (!__any_sync(0xffffffffu, al)) {  // the reference leaves zeros
    if (valid)
      for (int c = 1; c <= n; c++) po[(c - 1) * st] = 0.0;
    return;
  }
  if (valid && !al)
    for (int c = 1; c <= n; c++) po[(c - 1) * st] = 0.0;
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncwarp();
  const double *pq = cin + (long)g * L.PG + base;
  const double *pv = vel + base;
  const double *pvg = vghost + base;
  const LineGeo gsig = line_of<DIR>(sig, ac, o);   // constant along i: the same line for every lane
  const LineGeo gdtv = line_of<DIR>(dtvt, ac, o);
  const double vf0 = (DIR == 2) ? vf.p[(long)g * vf.sg] : 0.0;  // one fall speed per grain
  const bool out_lo = rmin == 1;
  const bool out_hi = rmax == n;
  const int ctop = (DIR == 2) ? ncells + 1 : rmax + 1;  // update_cc(ncells+1) for z (:309-311)
  if (DIR == 2 && out_hi && ctop < rmin - 1 && lane == 0) raise_error(sc, A3G_ERR_UNSUPPORTED, 311);
  const long na = L.nx;
  const long oo = (long)g * na * nother + (long)(o - 1) * na + (ac - 1);
  auto fs_ok = [&](int I) { return I >= rmin - 1 && I <= rmax + 1; };
  auto fss_ok = [&](int I) { return I >= rmin && I <= rmax + 1; };
  auto qload = [&](int c) -> double {
    return (c >= rmin - 2 && c <= rmax + 2 && c >= 1 && c <= n) ? pq[(c - 1) * st] : 0.0;
  };
  auto vload = [&](int c) -> double {
    const int cl = c < 1 ? 1 : (c > n ? n : c);
    double v = ((DIR == 2 && (c < 1 || c > n)) ? pvg : pv)[(cl - 1) * st];
    if (DIR == 2) v = v + vf0;
    return v;
  };
  const int cs = out_lo ? 0 : 1;
  const int ce = out_hi ? n + 1 : n;
  // ---- interface cs and the window at cs (k_advect_col's prologue) ----------
  double q0 = qload(cs), q1 = qload(cs + 1);
  double d0 = q0 - qload(cs - 1), d1 = q1 - q0;
  double usA, usB, vB, dtv0 = gdtv.at(cs), fss0, fsr0;
  {
    const double vm2 = vload(cs - 2), vm1 = vload(cs - 1), v0 = vload(cs);
    vB = vload(cs + 1);
    const double usm1 = fs_ok(cs - 1) ? 0.5 * (vm2 + vm1) * gsig.at(cs - 1) : 0.0;
    usA = fs_ok(cs) ? 0.5 * (vm1 + v0) * gsig.at(cs) : 0.0;
    usB = fs_ok(cs + 1) ? 0.5 * (v0 + vB) * gsig.at(cs + 1) : 0.0;
    const double qm1 = qload(cs - 1);
    const double dm = qm1 - qload(cs - 2);
    const Iface f = make_iface(usm1, usA, usB, dtv0, fss_ok(cs), fs_ok(cs));
    fss0 = fss_select<LIM>(dm, d0, d1, f.up, f.cf, f.fss_ok, eps, nocycle);
    fsr0 = f.fs_ok ? (f.usp * d0) + q0 * f.divm : 0.0;
  }
  // ---- one step: interface c+1 and the update of cell c (k_advect_col's) ----
  auto step = [&](int c, auto checked, double q2, double vn, double s2, double dtv1) {
    constexpr bool CK = decltype(checked)::value;
    const int I = c + 1;
    const bool fsok2 = !CK || fs_ok(c + 2);
    const double usC = fsok2 ? 0.5 * (vB + vn) * s2 : 0.0;
    vB = vn;
    const Iface f = make_iface(usA, usB, usC, dtv1, !CK || fss_ok(I), !CK || fs_ok(I));
    usA = usB;
    usB = usC;
    const double d2 = q2 - q1;
    const double fss1 = fss_select<LIM>(d0, d1, d2, f.up, f.cf, f.fss_ok, eps, nocycle);
    double fsr1 = 0.0, fsl1 = 0.0;
    if (f.fs_ok) {
      fsr1 = f.usp * d1;
      fsl1 = f.usm * d1;
      fsr1 = fsr1 + q1 * f.divm;
      fsl1 = fsl1 + q0 * f.divp;
    }
    const double upd = cell_update(dtv0, fsl1, fsr0, fss1, fss0);
    if (al) {
      if (!CK || (c >= 1 && c <= n)) {
        const bool inbox = !CK || (c >= rmin && c <= rmax);
        po[(c - 1) * st] = inbox ? q0 + upd : 0.0;
      }
      if (CK && out_lo && c == 0) out1[oo] += upd;
      if (out_hi && c == ctop) out2[oo] += upd;
    }
    fss0 = fss1;
    fsr0 = fsr1;
    q0 = q1;
    q1 = q2;
    d0 = d1;
    d1 = d2;
    dtv0 = dtv1;
  };
  auto checked_step = [&](int c) {
    step(c, CkT{}, qload(c + 2), vload(c + 2), fs_ok(c + 2) ? gsig.at(c + 2) : 0.0, gdtv.at(c + 1));
  };
  // steps without range checks: c >= rmin, c+2 <= min(n, rmax+1)
  int fa = max(cs, rmin), fb = min(n - 2, rmax - 1);
  if (fb < fa) { fa = ce + 1; fb = ce; }
  int c = cs;
  for (; c < fa; c++) checked_step(c);
  if (fa <= fb) {
    // chunk m holds cells C0(m) .. C0(m)+ACH-1, C0(m) = fa+2+m*ACH: the cell
    // c+2 of the steps c = fa+m*ACH .. (clipped to fb)
    const int nchunk = (fb - fa) / ACH + 1;
    constexpr uint32_t bytes = 2u * ACH * 32u * 8u;
    auto issue = [&](int m) {
      const int bi = m & 1;
      double *qb = wsm + bi * 2 * ACH * 32;
      const int C0 = fa + 2 + m * ACH;
      if (lane == 0) {
        mbar_arrive_expect_tx(&bar[bi], bytes);
        if (DIR == 1) {
          tma_load_4d(qb, &tq, &bar[bi], it << 5, C0 - 1, o - 1, g);
          tma_load_4d(qb + ACH * 32, &tv, &bar[bi], it << 5, C0 - 1, o - 1, 0);
        } else {
          tma_load_4d(qb, &tq, &bar[bi], it << 5, o - 1, C0 - 1, g);
          tma_load_4d(qb + ACH * 32, &tv, &bar[bi], it << 5, o - 1, C0 - 1, 0);
        }
      }
      double *gb = wsm + 4 * ACH * 32 + bi * 2 * ACH;
      if (lane < ACH && C0 + lane <= fb + 2) {
        gb[lane] = gsig.at(C0 + lane);            // sigma(c+2)
        gb[ACH + lane] = gdtv.at(C0 + lane - 1);  // dt/kappa(c+1)
      }
    };
    uint32_t ph = 0u;
    issue(0);
    for (int m = 0; m < nchunk; m++) {
      const int bi = m & 1;
      if (m + 1 < nchunk) issue(m + 1);
      if (!mbar_wait(&bar[bi], (ph >> bi) & 1u)) {
        if (lane == 0) raise_error(sc, A3G_ERR_TIMEOUT, 3);
        return;
      }
      ph ^= 1u << bi;
      __syncwarp();
      const double *qb = wsm + bi * 2 * ACH * 32 + lane;
      const double *vb = qb + ACH * 32;
      const double *gb = wsm + 4 * ACH * 32 + bi * 2 * ACH;
      const int cend = min(fb, fa + m * ACH + ACH - 1);
      if (cend - c + 1 == ACH) {  // a whole chunk: straight-line steps
#pragma unroll
        for (int e = 0; e < ACH; e++, c++)
          step(c, FastT{}, qb[e * 32], (DIR == 2) ? vb[e * 32] + vf0 : vb[e * 32], gb[e], gb[ACH + e]);
      } else {
        for (int e = 0; c <= cend; c++, e++)
          step(c, FastT{}, qb[e * 32], (DIR == 2) ? vb[e * 32] + vf0 : vb[e * 32], gb[e], gb[ACH + e]);
      }
      __syncwarp();
    }
  }
  for (; c <= ce; c++) checked_step(c);
}

// Launches the TMA-fed column march; false when its conditions do not hold
// (the caller takes another variant).
template <int DIR, int LIM>
static bool launch_colt(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const Geo3 &sg = (DIR == 1) ? ctx->sny : ctx->snz;
  if (sg.si != 0 || ctx->dtv.si != 0) return false;  // geometry must not vary along i
  if (DIR == 2 && (ctx->vf.si != 0 || ctx->vf.sj != 0 || ctx->vf.sk != 0)) return false;
  CUtensorMap tq, tv;
  const double *vel = dir_vel(ctx, DIR);
  if (!tensor_map(ctx, ctx->c0, DIR == 1 ? TM_ADV_QY : TM_ADV_QZ, &tq) ||
      !tensor_map(ctx, vel, DIR == 1 ? TM_ADV_VY : TM_ADV_VZ, &tv))
    return false;
  const size_t smem = 128 + (size_t)ACT_WARPS * ACT_WARP_D * sizeof(double);
  static_assert(128 + ACT_WARPS * ACT_WARP_D * 8 <= 48 * 1024, "fits the default dynamic limit");
  const int nother = (DIR == 1) ? L.nz : L.ny;
  const long nw = (long)((L.nx + 31) / 32) * nother * L.ns;
  k_advect_colt<DIR, LIM><<<(unsigned)((nw + ACT_WARPS - 1) / ACT_WARPS), 32 * ACT_WARPS, smem, ctx->stream>>>(
      tq, tv, L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, ctx->c0, ctx->c1, vel, dir_vghost(ctx, DIR),
      ctx->vf, sg, ctx->dtv, ctx->aloft, ctx->sc, (DIR == 1) ? ctx->out_xz1 : ctx->out_xy1,
      (DIR == 1) ? ctx->out_xz2 : ctx->out_xy2);
  return true;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int DIR, int LIM, int GC, bool PER, bool TOPO = false>
static void launch_march_gc(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int na = (DIR == 0) ? L.ny : L.nx;
  const int nother = (DIR == 2) ? L.ny : L.nz;
  // segments of about 96 cells (whole lines when they are short)
  const int nseg = (n + 95) / 96;
  const int seg = (n + nseg - 1) / nseg;
  const int ngroups = (L.ns + GC - 1) / GC;
  dim3 grid(((na + 31) / 32) * ngroups, (nother + 3) / 4, (n + seg - 1) / seg);
  const long n2 = (long)(L.nx + 4) * (L.ny + 4);
  const double *deld = TOPO ? ctx->topo_buf + ((DIR == 0) ? 2 : 3) * n2 : nullptr;
  k_advect_march<DIR, LIM, GC, PER, TOPO><<<grid, dim3(32, 4), 0, ctx->stream>>>(
      L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, seg, ngroups, ctx->c0, ctx->c1,
      dir_vel(ctx, DIR), dir_vghost(ctx, DIR), deld, ctx->vf,
      (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz, ctx->dtv, ctx->aloft, ctx->sc,
      (DIR == 0) ? ctx->out_yz1 : (DIR == 1) ? ctx->out_xz1 : ctx->out_xy1,
      (DIR == 0) ? ctx->out_yz2 : (DIR == 1) ? ctx->out_xz2 : ctx->out_xy2);
}

template <int DIR, int LIM, int V, bool PER>
static void launch_block_v(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const int n = (DIR == 0) ? L.nx : (DIR == 1) ? L.ny : L.nz;
  const int nblk = (n + V - 1) / V;
  dim3 grid;
  if (DIR == 0) grid = dim3((nblk + 31) / 32, (L.ny + 3) / 4, L.nz * L.ns);
  else grid = dim3((L.nx + 31) / 32, (nblk * ((DIR == 1) ? L.nz : L.ny) + 3) / 4, L.ns);
  const Geo3 &sg = (DIR == 0) ? ctx->snx : (DIR == 1) ? ctx->sny : ctx->snz;
  const bool lc = along<DIR>(sg) == 0 && along<DIR>(ctx->dtv) == 0 && (DIR != 2 || ctx->vf.sk == 0);
#define A3G_BLK(LC_)                                                                                  \
  k_advect_block<DIR, LIM, V, PER, LC_><<<grid, dim3(32, 4), 0, ctx->stream>>>(                       \
      L, ctx->box, ctx->prm.nocycle, ctx->prm.eps_thresh, nblk, ctx->c0, ctx->c1,                     \
      dir_vel(ctx, DIR), dir_vghost(ctx, DIR), ctx->vf, sg, ctx->dtv, ctx->aloft, ctx->sc,            \
      (DIR == 0) ? ctx->out_yz1 : (DIR == 1) ? ctx->out_xz1 : ctx->out_xy1,                           \
      (DIR == 0) ? ctx->out_yz2 : (DIR == 1) ? ctx->out_xz2 : ctx->out_xy2)
  if (lc) A3G_BLK(true); else A3G_BLK(false);
#undef A3G_BLK
}

template <int DIR, int LIM>
static void launch_dir_lim(a3g_ctx *ctx) {
  const bool per = (DIR == 0) && ctx->grid.periodic;
  const int variant = ctx->tune_advect[DIR];
  if constexpr (DIR != 2) {
    // ZScaling_ID 2: the DelD*onD_cc terms live in the marching kernel only
    if (ctx->topo_on && ctx->prm.zscaling_id == 2) {
      const bool g2 = ctx->L.ns >= 2;
      if constexpr (DIR == 0) {
        if (per) {
          if (g2) launch_march_gc<DIR, LIM, 2, true, true>(ctx);
          else launch_march_gc<DIR, LIM, 1, true, true>(ctx);
          return;
        }
      }
      if (g2) launch_march_gc<DIR, LIM, 2, false, true>(ctx);
      else launch_march_gc<DIR, LIM, 1, false, true>(ctx);
      return;
    }
  }
  if constexpr (DIR == 0) {
    if (variant == 3) {
      launch_advect_xt<LIM>(ctx);
      return;
    }
    if (variant == 4 || variant == 5) {
      launch_advect_xw<LIM>(ctx, variant == 5);
      return;
    }
  }
  if constexpr (DIR != 0) {
    if (variant == 5) {
      launch_col<DIR, LIM>(ctx);
      return;
    }
    if (variant == 6) {
      if (!launch_colt<DIR, LIM>(ctx)) launch_block_v<DIR, LIM, 4, false>(ctx);
      return;
    }
  }
  if (variant == 1) {
    if (per) launch_block_v<DIR, LIM, 4, true>(ctx);
    else launch_block_v<DIR, LIM, 4, false>(ctx);
    return;
  }
  if (variant == 2) {
    if (per) launch_block_v<DIR, LIM, 8, true>(ctx);
    else launch_block_v<DIR, LIM, 8, false>(ctx);
    return;
  }
  if (ctx->L.ns >= 2) {
    if (per) launch_march_gc<DIR, LIM, 2, true>(ctx);
    else launch_march_gc<DIR, LIM, 2, false>(ctx);
  } else {
    if (per) launch_march_gc<DIR, LIM, 1, true>(ctx);
    else launch_march_gc<DIR, LIM, 1, false>(ctx);
  }
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

}  // namespace a3g
