// k_reduce.cu -- reductions and small per-step kernels.
//
//  * CFL maxima and the dt arithmetic of Adjust_DT (src/Adjust_dt.f90:136-332):
//    maxima are exact and order independent, so the result is bit-identical
//    to the CPU loop; they are combined with atomicMax on the IEEE bit
//    patterns (valid for non-negative doubles; NaNs are skipped as the
//    reference's `if (tmp.gt.max)` skips them).
//  * mass totals (src/Output_Vars.f90:1255-1459): per-grain sums of c*kappa
//    accumulated in double-double (TwoSum) and combined in a fixed order, so
//    the result is deterministic and within a few ulp of the exact sum.
//  * subgrid plane occupancy for get_minmax_index (src/Calc_Mesh.f90:432-542).
//  * met-step interpolation (src/MesoInterpolater.f90:207-223) and the vent
//    column source insertion (src/Ash3d.F90:428-431).
#include "a3g_internal.cuh"
#include "exact_div.cuh"

namespace a3g {

__device__ __forceinline__ void atomic_max_pos(double *addr, double v) {
  if (!(v == v)) return;  // NaN: ignored like the reference's comparisons
  atomicMax(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_pos(double *addr, double v) {
  if (!(v == v)) return;
  atomicMin(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmx(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmn(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One thread per interior cell (grid-stride).  vmax[0]: |vx| (projected) or
// max |vx|*minsig/kappa (lon/lat); vmax[1] the same for y; vmax[2] the
// vertical (|vz| + max_g |vf|)/dz_k.  src/Adjust_dt.f90:136-173.
__global__ void __launch_bounds__(256) k_cfl(Layout L, int latlon, const double *__restrict__ vx,
                                             const double *__restrict__ vy,
                                             const double *__restrict__ vz, Geo4 vf, Geo3 snx,
                                             Geo3 sny, Geo3 kap, const double *__restrict__ dz_vec,
                                             DevScalars *sc) {
  // block-strided rows (j,k), threads along i (a maximum does not depend on
  // the visiting order)
  const int nrow = L.ny * L.nz;
  const bool vf_const = vf.si == 0 && vf.sj == 0 && vf.sk == 0;  // per-grain settling speeds
  double vf0 = 0.0;
  if (vf_const)
    for (int g = 0; g < L.ns; g++) {
      const double a = fabs(vf.at(1, 1, 1, g));
      if (g == 0 || a > vf0) vf0 = a;
    }
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  for (int r = blockIdx.x; r < nrow; r += gridDim.x) {
    const int j = r % L.ny + 1, k = r / L.ny + 1;
    const double rdz = dz_vec[k + 1];
    const long rb = L.cell(1, j, k);
    for (int i = threadIdx.x + 1; i <= L.nx; i += blockDim.x) {
      const long c = rb + (i - 1);
      const double ax = fabs(vx[c]), ay = fabs(vy[c]);
      double t1, t2;
      if (latlon) {
        const double kp = kap.at(i, j, k);
        t1 = ax * fmn(snx.at(i, j, k), snx.at(i + 1, j, k)) / kp;
        t2 = ay * fmn(sny.at(i, j, k), sny.at(i, j + 1, k)) / kp;
      } else {
        t1 = ax;
        t2 = ay;
      }
      double vfm = vf0;
      if (!vf_const) {
        vfm = 0.0;
        for (int g = 0; g < L.ns; g++) {
          const double a = fabs(vf.at(i, j, k, g));
          if (g == 0 || a > vfm) vfm = a;
        }
      }
      const double t3 = (fabs(vz[c]) + vfm) / rdz;
      if (t1 > m0) m0 = t1;
      if (t2 > m1) m1 = t2;
      if (t3 > m2) m2 = t3;
    }
  }
  m0 = warp_max(m0);
  m1 = warp_max(m1);
  m2 = warp_max(m2);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&sc->vmax[0], m0);
    atomic_max_pos(&sc->vmax[1], m1);
    atomic_max_pos(&sc->vmax[2], m2);
  }
}

// Diffusion time limit, src/Adjust_dt.f90:191-235 (min over cells of
// sum_d (kappa/minsig_d)^2 / k_d, starting from DT_MAX).
__global__ void __launch_bounds__(256) k_diff_limit(Layout L, Geo3 snx, Geo3 sny, Geo3 snz,
                                                    Geo3 kap, Geo3 kx, Geo3 ky, Geo3 kz,
                                                    DevScalars *sc) {
  const long ncell = (long)L.nx * L.ny * L.nz;
  double m = 1.0e300;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % L.nx) + 1;
    const long r = t / L.nx;
    const int j = (int)(r % L.ny) + 1;
    const int k = (int)(r / L.ny) + 1;
    const double kp = kap.at(i, j, k);
    const double r1 = kp / fmn(snx.at(i, j, k), snx.at(i + 1, j, k));
    const double t1 = (r1 * r1) / kx.at(i, j, k);
    const double r2 = kp / fmn(sny.at(i, j, k), sny.at(i, j + 1, k));
    const double t2 = (r2 * r2) / ky.at(i, j, k);
    const double r3 = kp / fmn(snz.at(i, j, k), snz.at(i, j, k + 1));
    const double t3 = (r3 * r3) / kz.at(i, j, k);
    const double t4 = t1 + t2 + t3;
    if (t4 < m) m = t4;
  }
  m = warp_min(m);
  if ((threadIdx.x & 31) == 0) atomic_min_pos(&sc->time_diffuse, m);
}

// dt arithmetic, src/Adjust_dt.f90:176-179 and :288-332.
// meso (FAST_DT, Adjust_DT(mesostep=.true.)): bit 1 first copies
// dt_meso_next to dt_meso_last (the toggle of src/MesoInterpolater.f90:187),
// bit 0 stores the dt formed here as dt_meso_next (src/Adjust_dt.f90:335-337).
__global__ void k_dt_finalize(int latlon, int use_diffusion, int use_cn, int n_gs_aloft, double dx,
                              double dy, double cfl, double dt_min, double dt_max, double imp_dt_fac,
                              double eps_small, double time, double next_write_time,
                              double simtime, int diff_fresh, int meso, DevScalars *sc) {
  if (meso & 2) sc->dt_meso_last = sc->dt_meso_next;
  double vx_dx = sc->vmax[0], vy_dy = sc->vmax[1], vz_dz = sc->vmax[2];
  if (!latlon) {
    vx_dx = vx_dx / dx;
    vy_dy = vy_dy / dy;
  }
  if (n_gs_aloft == 0) vz_dz = 0.0;
  const double time_advect = 1.0 / fmx(fmx(vx_dx, vy_dy), vz_dz);
  double td;
  if (use_diffusion) {
    if (diff_fresh) {
      td = sc->time_diffuse;  // min(DT_MAX, min_cells tmp4)
      td = use_cn ? td * imp_dt_fac : td * 0.5;
      sc->time_diffuse = td;
      sc->have_diffuse = 1;
    } else {
      td = sc->time_diffuse;
    }
  } else {
    td = dt_max;
  }
  const double dt_tmp = fmn(time_advect, td);
  double dt;
  if (dt_tmp < dt_min) dt = dt_min;
  else if (dt_tmp > dt_max) dt = dt_max;
  else dt = fmn(1.0, cfl) * dt_tmp;
  const long long fac = (long long)(dt / dt_min);
  dt = dt_min * (double)fac;
  if ((next_write_time - time) > eps_small && (next_write_time - time) < dt) dt = next_write_time - time;
  if (time + dt > simtime) dt = simtime - time;
  sc->dt = dt;
  if (meso & 1) sc->dt_meso_next = dt;
}

// Adjust_DT(mesostep=.true.), the FAST_DT branch of src/Adjust_dt.f90:96-135:
// the maxima over the FP32 met step `vx,vy,vz` (m/s, [k][j][i] without
// padding), widened and scaled as the reference writes them:
//   projected: real(max|vx_sp|)*3.6 (divided by dx in k_dt_finalize);
//   lon/lat:   real(|vx_sp|)*3.6*minsig/kappa per cell;
//   vertical:  real(|vz_sp| + max_g|vf_sp|)*3.6/dz_k, the sum in FP32.
// real(.)*3.6 is monotone, so the projected maximum of the scaled cells is the
// scaled maximum.  vfm: max_g |vf_meso_next_step_sp| per cell, or null for
// the single value vfm0.
__global__ void __launch_bounds__(256) k_cfl_meso(Layout L, int latlon, const float *__restrict__ vx,
                                                  const float *__restrict__ vy, const float *__restrict__ vz,
                                                  const float *__restrict__ vfm, float vfm0, Geo3 snx, Geo3 sny,
                                                  Geo3 kap, const double *__restrict__ dz_vec, DevScalars *sc) {
  const int nrow = L.ny * L.nz;
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  for (int r = blockIdx.x; r < nrow; r += gridDim.x) {
    const int j = r % L.ny + 1, k = r / L.ny + 1;
    const double rdz = dz_vec[k + 1];
    const long rb = (long)r * L.nx;
    for (int i = threadIdx.x + 1; i <= L.nx; i += blockDim.x) {
      const long c = rb + (i - 1);
      const double ax = (double)fabsf(vx[c]) * 3.6, ay = (double)fabsf(vy[c]) * 3.6;
      double t1, t2;
      if (latlon) {
        const double kp = kap.at(i, j, k);
        t1 = ax * fmn(snx.at(i, j, k), snx.at(i + 1, j, k)) / kp;
        t2 = ay * fmn(sny.at(i, j, k), sny.at(i, j + 1, k)) / kp;
      } else {
        t1 = ax;
        t2 = ay;
      }
      const float s = __fadd_rn(fabsf(vz[c]), vfm ? vfm[c] : vfm0);
      const double t3 = (double)s * 3.6 / rdz;
      if (t1 > m0) m0 = t1;
      if (t2 > m1) m1 = t2;
      if (t3 > m2) m2 = t3;
    }
  }
  m0 = warp_max(m0);
  m1 = warp_max(m1);
  m2 = warp_max(m2);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&sc->vmax[0], m0);
    atomic_max_pos(&sc->vmax[1], m1);
    atomic_max_pos(&sc->vmax[2], m2);
  }
}

// The FAST_DT step dt of src/MesoInterpolater.f90:250-258: interpolated
// between the met steps' dt (no DT_MIN rounding), then clipped to the next
// write time and the end of the simulation.
__global__ void k_fast_dt(double frac, double eps_small, double time, double next_write_time, double simtime,
                          DevScalars *sc) {
  const double last = sc->dt_meso_last, next = sc->dt_meso_next;
  double dt = last + (next - last) * frac;
  if ((next_write_time - time) > eps_small && (next_write_time - time) < dt) dt = next_write_time - time;
  if (time + dt > simtime) dt = simtime - time;
  sc->dt = dt;
}

int launch_cfl_maxima_meso(a3g_ctx *ctx, int slot) {
  const long n = ctx->met_n;
  return launch_cfl_maxima_meso_ptr(ctx, ctx->met + (size_t)3 * n * (slot == 0 ? ctx->met_last : ctx->met_next));
}

// the maxima over a met step (vx, vy, vz of nx*ny*nz FP32 each) at m
int launch_cfl_maxima_meso_ptr(a3g_ctx *ctx, const float *m) {
  const Layout &L = ctx->L;
  A3G_CUDA(cudaMemsetAsync(ctx->sc->vmax, 0, sizeof(ctx->sc->vmax), ctx->stream));
  const long n = (long)L.nx * L.ny * L.nz;
  const long ncell = (long)L.nx * L.ny * L.nz;
  int blocks = (int)((ncell + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  tbegin(ctx, A3G_K_CFL);
  k_cfl_meso<<<blocks, 256, 0, ctx->stream>>>(L, ctx->grid.latlon, m, m + n, m + 2 * n, ctx->vfm_sp,
                                              ctx->vfm_sp_const, ctx->snx, ctx->sny, ctx->kappa, ctx->dz_vec,
                                              ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_fast_dt(a3g_ctx *ctx, double frac, double time, double next_write_time, double simtime) {
  tbegin(ctx, A3G_K_OTHER);
  k_fast_dt<<<1, 1, 0, ctx->stream>>>(frac, ctx->prm.eps_small, time, next_write_time, simtime, ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_cfl_maxima(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  A3G_CUDA(cudaMemsetAsync(ctx->sc->vmax, 0, sizeof(ctx->sc->vmax), ctx->stream));
  const long ncell = (long)L.nx * L.ny * L.nz;
  int blocks = (int)((ncell + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  tbegin(ctx, A3G_K_CFL);
  k_cfl<<<blocks, 256, 0, ctx->stream>>>(L, ctx->grid.latlon, ctx->vx, ctx->vy, ctx->vz, ctx->vf,
                                         ctx->snx, ctx->sny, ctx->kappa, ctx->dz_vec, ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// dt from maxima already in sc->vmax (local, or set from an all-reduce).
int launch_dt_from_maxima(a3g_ctx *ctx, int n_gs_aloft, double time, double next_write_time,
                          double simtime, int meso) {
  const Layout &L = ctx->L;
  const long ncell = (long)L.nx * L.ny * L.nz;
  int blocks = (int)((ncell + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  int fresh = 0;
  if (ctx->prm.use_diffusion && !ctx->h_sc->have_diffuse) {
    const double init = ctx->prm.dt_max;
    A3G_CUDA(cudaMemcpyAsync(&ctx->sc->time_diffuse, &init, sizeof(double), cudaMemcpyHostToDevice,
                             ctx->stream));
    tbegin(ctx, A3G_K_CFL);
    k_diff_limit<<<blocks, 256, 0, ctx->stream>>>(L, ctx->snx, ctx->sny, ctx->snz, ctx->kappa,
                                                  ctx->kx, ctx->ky, ctx->kz, ctx->sc);
    tend(ctx);
    A3G_LAUNCH_CHECK(ctx);
    fresh = 1;
    ctx->h_sc->have_diffuse = 1;
  }
  tbegin(ctx, A3G_K_OTHER);
  k_dt_finalize<<<1, 1, 0, ctx->stream>>>(
      ctx->grid.latlon, ctx->prm.use_diffusion, ctx->prm.use_cn, n_gs_aloft, ctx->grid.dx,
      ctx->grid.dy, ctx->prm.cfl, ctx->prm.dt_min, ctx->prm.dt_max, ctx->prm.imp_dt_fac,
      ctx->prm.eps_small, time, next_write_time, simtime, fresh, meso, ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_cfl(a3g_ctx *ctx, double time, double next_write_time, double simtime) {
  const Layout &L = ctx->L;
  A3G_CUDA(cudaMemsetAsync(ctx->sc->vmax, 0, sizeof(ctx->sc->vmax), ctx->stream));
  const long ncell = (long)L.nx * L.ny * L.nz;
  int blocks = (int)((ncell + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  tbegin(ctx, A3G_K_CFL);
  k_cfl<<<blocks, 256, 0, ctx->stream>>>(L, ctx->grid.latlon, ctx->vx, ctx->vy, ctx->vz, ctx->vf,
                                         ctx->snx, ctx->sny, ctx->kappa, ctx->dz_vec, ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  int fresh = 0;
  if (ctx->prm.use_diffusion && !ctx->h_sc->have_diffuse) {
    const double init = ctx->prm.dt_max;
    A3G_CUDA(cudaMemcpyAsync(&ctx->sc->time_diffuse, &init, sizeof(double), cudaMemcpyHostToDevice,
                             ctx->stream));
    tbegin(ctx, A3G_K_CFL);
    k_diff_limit<<<blocks, 256, 0, ctx->stream>>>(L, ctx->snx, ctx->sny, ctx->snz, ctx->kappa,
                                                  ctx->kx, ctx->ky, ctx->kz, ctx->sc);
    tend(ctx);
    A3G_LAUNCH_CHECK(ctx);
    fresh = 1;
    ctx->h_sc->have_diffuse = 1;  // host mirror; the device flag is set by finalize
  }
  tbegin(ctx, A3G_K_OTHER);
  k_dt_finalize<<<1, 1, 0, ctx->stream>>>(
      ctx->grid.latlon, ctx->prm.use_diffusion, ctx->prm.use_cn, ctx->n_gs_aloft, ctx->grid.dx,
      ctx->grid.dy, ctx->prm.cfl, ctx->prm.dt_min, ctx->prm.dt_max, ctx->prm.imp_dt_fac,
      ctx->prm.eps_small, time, next_write_time, simtime, fresh, 0, ctx->sc);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// mass totals
// ---------------------------------------------------------------------------
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD dd_add(DD a, double b) {  // TwoSum accumulate
  const double s = a.hi + b;
  const double bb = s - a.hi;
  const double err = (a.hi - (s - bb)) + (b - bb);
  DD r;
  r.hi = s;
  r.lo = a.lo + err;
  return r;
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD r = dd_add(a, b.hi);
  r.lo = r.lo + b.lo;
  return r;
}
__device__ __forceinline__ DD dd_shfl(DD v, int o) {
  DD r;
  r.hi = __shfl_xor_sync(0xffffffffu, v.hi, o);
  r.lo = __shfl_xor_sync(0xffffffffu, v.lo, o);
  return r;
}

// Jobs: 0 aloft (c*kappa over the interior), 1 deposit (xy1*kappa(:,:,0)),
// 2 yz1*kappa(0,:,:), 3 yz2*kappa(nx+1,:,:), 4 xz1*kappa(:,0,:),
// 5 xz2*kappa(:,ny+1,:), 6 xy2*kappa(:,:,nz+1).
constexpr int NJOBS = 7;
constexpr int TOT_BLOCKS = 296;

__global__ void __launch_bounds__(256) k_totals(Layout L, const double *__restrict__ c,
                                                Geo3 kap, const double *__restrict__ yz1,
                                                const double *__restrict__ yz2,
                                                const double *__restrict__ xz1,
                                                const double *__restrict__ xz2,
                                                const double *__restrict__ xy1,
                                                const double *__restrict__ xy2,
                                                double *__restrict__ part) {
  // job is the slowest grid index: the airborne-mass blocks of every grain
  // are resident together (more loads in flight) before the small face sums
  const int job = blockIdx.z, g = blockIdx.y;
  __shared__ double sh[2][8];
  DD acc = {0.0, 0.0};
  long n;
  switch (job) {
    case 0: n = (long)L.nx * L.ny * L.nz; break;
    case 1: case 6: n = (long)L.nx * L.ny; break;
    case 2: case 3: n = (long)L.ny * L.nz; break;
    default: n = (long)L.nx * L.nz; break;
  }
  if (job == 0) {
    // airborne mass: block b sums a contiguous run of the (j,k) rows, threads
    // along i.  A thread adds its few cells of a row in double (their loads
    // all in flight at once), times kappa once per row when kappa does not
    // vary along i, and carries the row terms in double-double: a relative
    // error of a few ulps per row term, far inside the 1e-13 the totals keep
    const double *cg = c + (long)g * L.PG;
    const int nrow = L.ny * L.nz;
    const int per = (nrow + (int)gridDim.x - 1) / (int)gridDim.x;
    const int r0 = (int)blockIdx.x * per, r1 = min(nrow, r0 + per);
    int j = r0 % L.ny + 1, k = r0 / L.ny + 1;
    const bool row_const = kap.si == 0;
    const int bd = (int)blockDim.x;
    for (int r = r0; r < r1; r++) {
      const double *row = cg + (long)r * L.P;
      double part = 0.0;
      for (int i0 = 0; i0 < L.nx; i0 += 4 * bd) {
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int i = i0 + (int)threadIdx.x + q * bd;
          v[q] = i < L.nx ? (row_const ? row[i] : row[i] * kap.at(i + 1, j, k)) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) part = part + v[q];
      }
      if (row_const) part = part * kap.at(1, j, k);
      acc = dd_add(acc, part);
      if (++j > L.ny) {
        j = 1;
        k++;
      }
    }
    n = 0;
  }
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    double v;
    if (job == 1 || job == 6) {
      const int i = (int)(t % L.nx) + 1, j = (int)(t / L.nx) + 1;
      const double *a = (job == 1) ? xy1 : xy2;
      v = a[(long)g * L.nx * L.ny + t] * kap.at(i, j, job == 1 ? 0 : L.nz + 1);
    } else if (job == 2 || job == 3) {
      const int j = (int)(t % L.ny) + 1, k = (int)(t / L.ny) + 1;
      const double *a = (job == 2) ? yz1 : yz2;
      v = a[(long)g * L.ny * L.nz + t] * kap.at(job == 2 ? 0 : L.nx + 1, j, k);
    } else {
      const int i = (int)(t % L.nx) + 1, k = (int)(t / L.nx) + 1;
      const double *a = (job == 4) ? xz1 : xz2;
      v = a[(long)g * L.nx * L.nz + t] * kap.at(i, job == 4 ? 0 : L.ny + 1, k);
    }
    acc = dd_add(acc, v);
  }
  for (int o = 16; o > 0; o >>= 1) acc = dd_add(acc, dd_shfl(acc, o));
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sh[0][w] = acc.hi; sh[1][w] = acc.lo; }
  __syncthreads();
  if (threadIdx.x == 0) {
    DD s = {0.0, 0.0};
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s = dd_add(s, DD{sh[0][q], sh[1][q]});
    const long o = (((long)g * NJOBS + job) * gridDim.x + blockIdx.x) * 2;
    part[o] = s.hi;
    part[o + 1] = s.lo;
  }
}

// one warp per (g, job): lanes take every 32nd block partial, then a fixed
// shuffle tree (the same order on every run)
__global__ void k_totals_final(int ns, int nblk, const double *__restrict__ part,
                               double *__restrict__ out) {
  const int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;  // (g, job)
  if (t >= ns * NJOBS) return;  // whole warps
  DD s = {0.0, 0.0};
  for (int b = lane; b < nblk; b += 32) {
    const long o = ((long)t * nblk + b) * 2;
    s = dd_add(s, DD{part[o], part[o + 1]});
  }
  for (int o = 16; o > 0; o >>= 1) s = dd_add(s, dd_shfl(s, o));
  if (lane == 0) out[t] = s.hi + s.lo;  // out[g*NJOBS + job]
}

// the partial sums of the totals, copied (asynchronously) to h_dst
// (ns*NJOBS doubles of pinned memory)
int launch_totals_partials(a3g_ctx *ctx, double *h_dst) {
  const Layout &L = ctx->L;
  const int ns = L.ns;
  dim3 grid(TOT_BLOCKS, ns, NJOBS);
  tbegin(ctx, A3G_K_TOTALS);
  k_totals<<<grid, 256, 0, ctx->stream>>>(L, ctx->c0, ctx->kappa, ctx->out_yz1, ctx->out_yz2,
                                          ctx->out_xz1, ctx->out_xz2, ctx->out_xy1, ctx->out_xy2,
                                          ctx->red_buf);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  double *fin = ctx->red_buf + (size_t)2 * TOT_BLOCKS * NJOBS * ns;
  tbegin(ctx, A3G_K_TOTALS);
  k_totals_final<<<(ns * NJOBS * 32 + 127) / 128, 128, 0, ctx->stream>>>(ns, TOT_BLOCKS, ctx->red_buf, fin);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  A3G_CUDA(cudaMemcpyAsync(h_dst, fin, sizeof(double) * ns * NJOBS, cudaMemcpyDeviceToHost, ctx->stream));
  return A3G_OK;
}

// volumes in the reference's order, src/Output_Vars.f90:1285-1290,1395-1401,1440-1456
void totals_volumes(a3g_ctx *ctx, const double *h_src, double *out4, double *mass_aloft) {
  const int ns = ctx->L.ns;
  const double rho = ctx->prm.magma_density, km3 = 1.0e9;
  double aloft = 0.0, depv = 0.0, outv = 0.0;
  for (int g = 0; g < ns; g++) {
    const double *r = h_src + (size_t)g * NJOBS;
    if (mass_aloft) mass_aloft[g] = r[0];
    aloft = aloft + r[0] / rho / km3;
  }
  for (int g = 0; g < ns; g++) depv = depv + h_src[(size_t)g * NJOBS + 1] / rho / km3;
  for (int g = 0; g < ns; g++) {
    const double *r = h_src + (size_t)g * NJOBS;
    outv = outv + (r[2] + r[3] + r[4] + r[5] + r[6]) / rho / km3;
  }
  out4[0] = aloft;
  out4[1] = depv;
  out4[2] = outv;
  out4[3] = aloft + depv + outv;
}

int launch_totals(a3g_ctx *ctx, double *out4, double *mass_aloft) {
  const Layout &L = ctx->L;
  const int ns = L.ns;
  dim3 grid(TOT_BLOCKS, ns, NJOBS);
  tbegin(ctx, A3G_K_TOTALS);
  k_totals<<<grid, 256, 0, ctx->stream>>>(L, ctx->c0, ctx->kappa, ctx->out_yz1, ctx->out_yz2,
                                          ctx->out_xz1, ctx->out_xz2, ctx->out_xy1, ctx->out_xy2,
                                          ctx->red_buf);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  double *fin = ctx->red_buf + (size_t)2 * TOT_BLOCKS * NJOBS * ns;
  tbegin(ctx, A3G_K_TOTALS);
  k_totals_final<<<(ns * NJOBS * 32 + 127) / 128, 128, 0, ctx->stream>>>(ns, TOT_BLOCKS, ctx->red_buf, fin);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  A3G_CUDA(cudaMemcpyAsync(ctx->h_tot, fin, sizeof(double) * ns * NJOBS, cudaMemcpyDeviceToHost,
                           ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  // volumes in the reference's order, src/Output_Vars.f90:1285-1290,1395-1401,1440-1456
  const double rho = ctx->prm.magma_density, km3 = 1.0e9;
  double aloft = 0.0, depv = 0.0, outv = 0.0;
  for (int g = 0; g < ns; g++) {
    const double *r = ctx->h_tot + (size_t)g * NJOBS;
    if (mass_aloft) mass_aloft[g] = r[0];
    aloft = aloft + r[0] / rho / km3;
  }
  for (int g = 0; g < ns; g++) depv = depv + ctx->h_tot[(size_t)g * NJOBS + 1] / rho / km3;
  for (int g = 0; g < ns; g++) {
    const double *r = ctx->h_tot + (size_t)g * NJOBS;
    outv = outv + (r[2] + r[3] + r[4] + r[5] + r[6]) / rho / km3;
  }
  out4[0] = aloft;
  out4[1] = depv;
  out4[2] = outv;
  out4[3] = aloft + depv + outv;
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// subgrid plane occupancy: flags[i] (i=1..nx), flags[nx+1+j], flags[nx+ny+2+k]
// set when some grain has c >= thresh in that plane.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_plane_flags(Layout L, const double *__restrict__ c,
                                                     double thresh, int32_t *__restrict__ flags) {
  const long ncell = (long)L.nx * L.ny * L.nz;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % L.nx) + 1;
    const long r = t / L.nx;
    const int j = (int)(r % L.ny) + 1;
    const int k = (int)(r / L.ny) + 1;
    const long cell = L.cell(i, j, k);
    bool hit = false;
    for (int g = 0; g < L.ns && !hit; g++) hit = c[(long)g * L.PG + cell] >= thresh;
    if (hit) {
      if (!flags[i]) flags[i] = 1;
      if (!flags[L.nx + 1 + j]) flags[L.nx + 1 + j] = 1;
      if (!flags[L.nx + L.ny + 2 + k]) flags[L.nx + L.ny + 2 + k] = 1;
    }
  }
}

int launch_plane_flags(a3g_ctx *ctx) {
  const Layout &L = ctx->L;
  const size_t nf = (size_t)L.nx + L.ny + L.nz + 3;
  A3G_CUDA(cudaMemsetAsync(ctx->plane_flags, 0, nf * sizeof(int32_t), ctx->stream));
  const long ncell = (long)L.nx * L.ny * L.nz;
  int blocks = (int)((ncell + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  tbegin(ctx, A3G_K_OTHER);
  k_plane_flags<<<blocks, 256, 0, ctx->stream>>>(L, ctx->c0, ctx->prm.cloudcon_grid_thresh,
                                                 ctx->plane_flags);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  A3G_CUDA(cudaMemcpyAsync(ctx->h_plane_flags, ctx->plane_flags, nf * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// winds and source
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_interp_winds(Layout L, const float *__restrict__ last,
                                                      const float *__restrict__ next, long n, double frac,
                                                      double *__restrict__ vx, double *__restrict__ vy,
                                                      double *__restrict__ vz) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % L.nx) + 1;
    const long r = t / L.nx;
    const int j = (int)(r % L.ny) + 1;
    const int k = (int)(r / L.ny) + 1;
    const long c = L.cell(i, j, k);
    const float dx = next[t] - last[t];
    const float dy = next[n + t] - last[n + t];
    const float dz = next[2 * n + t] - last[2 * n + t];
    vx[c] = ((double)last[t] + (double)dx * frac) * 3.6;
    vy[c] = ((double)last[n + t] + (double)dy * frac) * 3.6;
    vz[c] = ((double)last[2 * n + t] + (double)dz * frac) * 3.6;
  }
}

int launch_interp_winds(a3g_ctx *ctx, double frac) {
  const long n = ctx->met_n;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  tbegin(ctx, A3G_K_WINDS);
  k_interp_winds<<<blocks, 256, 0, ctx->stream>>>(ctx->L, ctx->met + (size_t)3 * n * ctx->met_last,
                                                  ctx->met + (size_t)3 * n * ctx->met_next, n, frac, ctx->vx,
                                                  ctx->vy, ctx->vz);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// Calc_Vmod_Topo (src/Topography.f90:2138-2166) on the interior, fused with
// the sum the z sweep needs: vzh = vz + vh, vh = f(k)*(vx*dhdx + vy*dhdy)
// with f = -1.0 (ZScaling_ID 1) or s_cc(k)/Ztop - 1.0 (2), precomputed on the
// host in those operations.  The ghost levels keep plain vz (vh is zero
// there in the reference: vx_pd and vy_pd are never written at ghost k).
__global__ void __launch_bounds__(256) k_vmod_topo(Layout L, const double *__restrict__ topo,
                                                   const double *__restrict__ vx,
                                                   const double *__restrict__ vy,
                                                   const double *__restrict__ vz,
                                                   double *__restrict__ vzh) {
  const long n = (long)L.nx * L.ny * L.nz;
  const long n2 = (long)(L.nx + 4) * (L.ny + 4);
  const double *dhdx = topo, *dhdy = topo + n2, *fac = topo + 4 * n2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % L.nx) + 1;
    const long r = t / L.nx;
    const int j = (int)(r % L.ny) + 1;
    const int k = (int)(r / L.ny) + 1;
    const long c = L.cell(i, j, k);
    const long m = (long)(i + 1) + (long)(L.nx + 4) * (j + 1);
    const double vh = fac[k - 1] * (vx[c] * dhdx[m] + vy[c] * dhdy[m]);
    vzh[c] = vz[c] + vh;
  }
}

int launch_vmod_topo(a3g_ctx *ctx) {
  const long n = (long)ctx->L.nx * ctx->L.ny * ctx->L.nz;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  tbegin(ctx, A3G_K_WINDS);
  k_vmod_topo<<<blocks, 256, 0, ctx->stream>>>(ctx->L, ctx->topo_buf, ctx->vx, ctx->vy, ctx->vz, ctx->vzh);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// umbrella_winds' radial winds added to the interpolated winds over the
// cloud's bounding box and the levels ibase..itop
// (src/MesoInterpolater.f90:237-241): vx += uvx, vy += uvy.
__global__ void __launch_bounds__(256) k_umbrella_winds(Layout L, int i0, int ni, int j0, int nj, int kb,
                                                        int nk, const double *__restrict__ uv,
                                                        double *__restrict__ vx, double *__restrict__ vy) {
  const long n = (long)ni * nj * nk;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int a = (int)(t % ni);
    const long r = t / ni;
    const int b = (int)(r % nj);
    const int k = kb + (int)(r / nj);
    const long c = L.cell(i0 + a, j0 + b, k);
    const long m = a + (long)ni * b;
    vx[c] = vx[c] + uv[m];
    vy[c] = vy[c] + uv[(long)ni * nj + m];
  }
}

int launch_umbrella_winds(a3g_ctx *ctx, int i0, int ni, int j0, int nj, const double *uv) {
  const int nk = ctx->umb_itop - ctx->umb_ibase + 1;
  const long n = (long)ni * nj * nk;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  tbegin(ctx, A3G_K_WINDS);
  k_umbrella_winds<<<blocks, 256, 0, ctx->stream>>>(ctx->L, i0, ni, j0, nj, ctx->umb_ibase, nk, uv, ctx->vx,
                                                    ctx->vy);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// Umbrella source insertion (src/Ash3d.F90:446-458): on ibase..itop the 3x3
// patch around the vent is first set to its volume-weighted average
// (AvgCon_Umbrella, src/Source_Umbrella.f90:539-560, i outer, j inner), then
// every patch cell of levels 1..nz gains dt*SourceNodeFlux_Umbrella.  One
// thread per (level, grain).
__global__ void k_source_umbrella(Layout L, int ivent, int jvent, int ibase, int itop,
                                  const double *__restrict__ sten, const double *__restrict__ flux, double dt,
                                  double *__restrict__ c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // (k-1) + nz*g
  if (t >= L.nz * L.ns) return;
  const int k = t % L.nz + 1, g = t / L.nz;
  double v[3][3];
  long a[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      a[i][j] = (long)g * L.PG + L.cell(ivent - 1 + i, jvent - 1 + j, k);
      v[i][j] = c[a[i][j]];
    }
  if (k >= ibase && k <= itop) {
    double avg = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) avg = avg + v[i][j] * sten[i + 3 * j + 9 * (k - 1)];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) v[i][j] = avg;
  }
  const long f0 = 9 * ((long)(k - 1) + (long)(L.nz + 1) * g);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) c[a[i][j]] = v[i][j] + dt * flux[f0 + i + 3 * j];
}

int launch_source_umbrella(a3g_ctx *ctx, double dt) {
  const int n = ctx->L.nz * ctx->L.ns;
  const double *sten = ctx->umb_buf;
  const double *flux = ctx->umb_buf + 9 * (size_t)ctx->L.nz;
  tbegin(ctx, A3G_K_OTHER);
  k_source_umbrella<<<(n + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ctx->umb_ivent, ctx->umb_jvent,
                                                              ctx->umb_ibase, ctx->umb_itop, sten, flux, dt,
                                                              ctx->c0);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// Scheduled source on the device: CheckEruptivePulses (src/Source.f90:613-685)
// and TephraSourceNodes (:708-783) with the step's dt from the device
// scalars, then the vent-column insertion of src/Ash3d.F90:428-431.  One
// block; thread 0 runs the pulse bookkeeping (ieruption/jeruption persist in
// state), the block inserts the (level, grain) fluxes.
constexpr int SRC_MAX_PULSES = 64;

__global__ void k_source_sched(Layout L, int ivent, int jvent, int np, const double *__restrict__ sched,
                               int32_t *__restrict__ state, const DevScalars *__restrict__ sc, Geo3 kap,
                               double time, double *__restrict__ c) {
  __shared__ double frac[SRC_MAX_PULSES + 1];
  __shared__ int ie_s, je_s, in_s;
  const double *t0 = sched, *t1 = sched + np, *mfr = sched + 2 * np, *col = sched + 3 * np;
  const double *bin = col + (size_t)np * (L.nz + 1);
  const double dt = sc->dt;
  if (threadIdx.x == 0) {
    const double tstart = time, tend = time + dt;
    const int ie = state[0];
    int je = state[1];
    int in = 0;
    for (int i = 1; i <= np; i++) frac[i] = 0.0;
    for (int i = ie; i <= np; i++) {
      bool pc = false;
      if (tstart >= t0[i - 1] && tstart < t1[i - 1]) {
        pc = true;
        je = i;
      } else if (tend > t0[i - 1] && tend <= t1[i - 1]) {
        je = i;  // :646-651: the loop exits before this pulse's fraction is formed
        break;
      } else if (tstart < t0[i - 1] && tend > t1[i - 1]) {
        pc = true;
        je = i;
      }
      if (pc) {
        in = 1;
        frac[i] = (fmin(tend, t1[i - 1]) - fmax(tstart, t0[i - 1])) / dt;
      }
    }
    ie_s = ie;
    je_s = je;
    in_s = in;
  }
  __syncthreads();
  const int ie = ie_s, je = je_s;
  if (in_s) {
    for (int t = threadIdx.x; t < L.nz * L.ns; t += blockDim.x) {
      const int k = t % L.nz + 1, g = t / L.nz;
      double tfr = 0.0;
      for (int i = ie; i <= je; i++)
        tfr = tfr + mfr[i - 1] * frac[i] * col[(ie - 1) + (size_t)np * (k - 1)];
      const double kv = kap.p[(long)(ivent + 1) * kap.si + (long)(jvent + 1) * kap.sj + (long)(k + 1) * kap.sk];
      const double flux = bin[g] * tfr / kv;
      const long a = (long)g * L.PG + L.cell(ivent, jvent, k);
      c[a] = c[a] + dt * flux;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    state[1] = je;
    if (in_s) state[0] = je;  // :776, only when TephraSourceNodes ran
  }
}

int launch_source_sched(a3g_ctx *ctx, double time) {
  tbegin(ctx, A3G_K_OTHER);
  k_source_sched<<<1, 256, 0, ctx->stream>>>(ctx->L, ctx->src_iv, ctx->src_jv, ctx->src_np, ctx->src_sched,
                                             ctx->src_state, ctx->sc, ctx->kappa, time, ctx->c0);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

__global__ void k_source(Layout L, int ivent, int jvent, const double *__restrict__ flux, double dt,
                         double *__restrict__ c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // (k-1) + nz*g
  if (t >= L.nz * L.ns) return;
  const int k = t % L.nz + 1, g = t / L.nz;
  const long a = (long)g * L.PG + L.cell(ivent, jvent, k);
  c[a] = c[a] + dt * flux[(long)(k - 1) + (long)(L.nz + 1) * g];
}

// the vent-column insertion with the step's dt read from the device scalars
__global__ void k_source_devdt(Layout L, int ivent, int jvent, const double *__restrict__ flux,
                               const DevScalars *__restrict__ sc, double *__restrict__ c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // (k-1) + nz*g
  if (t >= L.nz * L.ns) return;
  const int k = t % L.nz + 1, g = t / L.nz;
  const long a = (long)g * L.PG + L.cell(ivent, jvent, k);
  c[a] = c[a] + sc->dt * flux[(long)(k - 1) + (long)(L.nz + 1) * g];
}

int launch_source_devdt(a3g_ctx *ctx, int ivent, int jvent) {
  const int n = ctx->L.nz * ctx->L.ns;
  tbegin(ctx, A3G_K_OTHER);
  k_source_devdt<<<(n + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ivent, jvent, ctx->src_buf, ctx->sc, ctx->c0);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_source(a3g_ctx *ctx, int ivent, int jvent, double dt) {
  const int n = ctx->L.nz * ctx->L.ns;
  tbegin(ctx, A3G_K_OTHER);
  k_source<<<(n + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ivent, jvent, ctx->src_buf, dt, ctx->c0);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// observation operators for the adjoint (no counterpart in the reference's
// transport path; the column load is Gen_Output_Vars' CloudLoad)
// ---------------------------------------------------------------------------
// CloudLoad(i,j) = sum_k sum_g c(i,j,k,g) * dz(k) / 1e3 (tonnes/km^2), in the
// order of src/Output_Vars.f90:1061-1069, without the cloud mask.
__global__ void k_cloud_load(Layout L, const double *__restrict__ c, const double *__restrict__ dz_vec,
                             double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1;
  if (i > L.nx) return;
  double load = 0.0;
  for (int k = 1; k <= L.nz; k++) {
    double s = 0.0;
    for (int g = 0; g < L.ns; g++) s = s + c[(long)g * L.PG + L.cell(i, j, k)];
    load = load + s * dz_vec[k + 1] / 1.0e3;
  }
  out[(long)(j - 1) * L.nx + (i - 1)] = load;
}

// lam(i,j,k,g) += w(i,j) * dz(k) / 1e3: the transpose of the column load.
__global__ void k_adj_cloud_load(Layout L, const double *__restrict__ w, const double *__restrict__ dz_vec,
                                 double *__restrict__ lam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1;
  const int kg = blockIdx.z;
  if (i > L.nx) return;
  const int k = kg % L.nz + 1, g = kg / L.nz;
  const long a = (long)g * L.PG + L.cell(i, j, k);
  lam[a] = lam[a] + w[(long)(j - 1) * L.nx + (i - 1)] * dz_vec[k + 1] / 1.0e3;
}

// lam at the vent column, (nz+1) x ns with k fastest (row nz+1, the ghost
// that Set_BC(1) zeroes, is 0): the adjoint of the source insertion.
__global__ void k_vent_column(Layout L, int ivent, int jvent, const double *__restrict__ lam,
                              double *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (L.nz + 1) * L.ns) return;
  const int k = t % (L.nz + 1) + 1, g = t / (L.nz + 1);
  out[t] = (k <= L.nz) ? lam[(long)g * L.PG + L.cell(ivent, jvent, k)] : 0.0;
}

int launch_cloud_load(a3g_ctx *ctx, const double *c, double *out) {
  const Layout &L = ctx->L;
  tbegin(ctx, A3G_K_ADJOINT);
  k_cloud_load<<<dim3((L.nx + 127) / 128, L.ny), 128, 0, ctx->stream>>>(L, c, ctx->dz_vec, out);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_adj_cloud_load(a3g_ctx *ctx, const double *w, double *lam) {
  const Layout &L = ctx->L;
  tbegin(ctx, A3G_K_ADJOINT);
  k_adj_cloud_load<<<dim3((L.nx + 127) / 128, L.ny, L.nz * L.ns), 128, 0, ctx->stream>>>(L, w, ctx->dz_vec,
                                                                                        lam);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// grad(k, g) += dt * lam(ivent, jvent, k, g) / kappa(ivent, jvent, k) for
// k = 1..nz: the source-gradient gather of one reverse step, on the device
// (the same operations as the host's dt*col/kappa added to grad).
__global__ void k_vent_accumulate(Layout L, int ivent, int jvent, const double *__restrict__ lam, Geo3 kap,
                                  double dt, double *__restrict__ dst) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // (k-1) + nz*g
  if (t >= L.nz * L.ns) return;
  const int k = t % L.nz + 1, g = t / L.nz;
  const double kv = kap.p[(long)(ivent + 1) * kap.si + (long)(jvent + 1) * kap.sj + (long)(k + 1) * kap.sk];
  dst[t] = dst[t] + dt * lam[(long)g * L.PG + L.cell(ivent, jvent, k)] / kv;
}

int launch_vent_accumulate(a3g_ctx *ctx, int ivent, int jvent, double dt, double *dst) {
  const int n = ctx->L.nz * ctx->L.ns;
  tbegin(ctx, A3G_K_ADJOINT);
  k_vent_accumulate<<<(n + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ivent, jvent, ctx->lam0, ctx->kappa, dt,
                                                              dst);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_vent_column(a3g_ctx *ctx, int ivent, int jvent, const double *lam, double *out) {
  const int n = (ctx->L.nz + 1) * ctx->L.ns;
  k_vent_column<<<(n + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ivent, jvent, lam, out);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// output products of Gen_Output_Vars, one thread per column (i,j), in the
// reference's order: ConcentrationCalculator (src/Output_Vars.f90:1026-1123),
// AshThicknessCalculator (:855-895), the arrival-time marks (:1226-1236).
// ---------------------------------------------------------------------------
__global__ void k_output_vars(Layout L, Box box, const double *__restrict__ c, const double *__restrict__ dz_vec,
                              const double *__restrict__ zcc, const double *__restrict__ dep, double cloudcon,
                              double cloudload_th, double depo_th, double density, double time,
                              double *__restrict__ load, double *__restrict__ maxh, double *__restrict__ minh,
                              double *__restrict__ maxc, int32_t *__restrict__ mcl, double *__restrict__ dthick,
                              int32_t *__restrict__ mdep, double *__restrict__ carr, double *__restrict__ darr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1;
  if (i > L.nx) return;
  const long o = (long)(j - 1) * L.nx + (i - 1);
  const long plane = (long)L.nx * L.ny;
  // deposit thickness (mm) from DepositGranularity
  double sg = 0.0;
  for (int g = 0; g < L.ns; g++) sg = sg + dep[(long)g * plane + o];
  const double th = sg * dz_vec[2] / 1.0e6 / density * 1.0e3;
  const bool md = th > depo_th;
  dthick[o] = th;
  mdep[o] = md;
  double ld = 0.0, mh = 0.0, nh = 100.0, mx = 0.0;
  bool mc = false;
  if (L.ns > 0 && i >= box.imin && i <= box.imax && j >= box.jmin && j <= box.jmax) {
    auto tc = [&](int k) {
      double s = 0.0;
      for (int g = 0; g < L.ns; g++) s = s + c[(long)g * L.PG + L.cell(i, j, k)];
      return s;
    };
    for (int k = 1; k <= L.nz; k++) {
      const double t = tc(k);
      ld = ld + t * dz_vec[k + 1] / 1.0e3;
      if (t >= cloudcon) mh = zcc[k - 1] + 0.5 * dz_vec[k + 1];
      mx = (k == 1) ? t : fmx(mx, t);
    }
    for (int k = L.nz; k >= 1; k--)
      if (tc(k) <= cloudcon) nh = zcc[k - 1] - 0.5 * dz_vec[k + 1];
    mc = ld >= cloudload_th;
    if (mc) {
      if (nh < 0.0 && mh > 0.0) nh = 0.0;
      nh = fmn(mh, nh);
      mx = mx * 1.0e6 / 1.0e9;
    } else {
      ld = 0.0; mx = 0.0; mh = 0.0; nh = 0.0;
    }
  }
  load[o] = ld;
  maxh[o] = mh;
  minh[o] = nh;
  maxc[o] = mx;
  mcl[o] = mc;
  if (md && darr[o] < 0.0) darr[o] = time;
  if (mc && carr[o] < 0.0) carr[o] = time;
}

// Calc_vprofile (src/Output_Vars.f90:1308-1360): per profile point the
// column total (Fortran SUM order: k fastest, then the grains) against
// CLOUDCON_THRESH, and per level the sum over the grains in mg/m3.  One block
// per point; thread 0 forms the total.
__global__ void k_vprofiles(Layout L, const int32_t *__restrict__ pts, double thresh,
                            const double *__restrict__ c, double *__restrict__ out,
                            int32_t *__restrict__ written) {
  const int p = blockIdx.x;
  const int i = pts[2 * p], j = pts[2 * p + 1];
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int g = 0; g < L.ns; g++)
      for (int k = 1; k <= L.nz; k++) total = total + c[(long)g * L.PG + L.cell(i, j, k)];
    written[p] = !(total < thresh);
  }
  for (int k = 1 + threadIdx.x; k <= L.nz; k += blockDim.x) {
    double sum = 0.0;
    for (int g = 0; g < L.ns; g++) sum = sum + c[(long)g * L.PG + L.cell(i, j, k)];
    out[(long)(k - 1) + (long)L.nz * p] = sum * 1.0e6 / 1.0e9;  // KG_2_MG / KM3_2_M3
  }
}

int launch_vprofiles(a3g_ctx *ctx, int npts, const int32_t *pts, double *out, int32_t *written) {
  tbegin(ctx, A3G_K_OTHER);
  k_vprofiles<<<npts, 64, 0, ctx->stream>>>(ctx->L, pts, ctx->ov_cloudcon, ctx->c0, out, written);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_output_vars(a3g_ctx *ctx, double time, double *load, double *maxh, double *minh, double *maxc,
                       int32_t *mcl, double *dthick, int32_t *mdep, double *carr, double *darr) {
  const Layout &L = ctx->L;
  tbegin(ctx, A3G_K_OTHER);
  k_output_vars<<<dim3((L.nx + 127) / 128, L.ny), 128, 0, ctx->stream>>>(
      L, ctx->box, ctx->c0, ctx->dz_vec, ctx->ov_zcc, ctx->out_xy1, ctx->ov_cloudcon, ctx->ov_cloudload,
      ctx->ov_depo, ctx->ov_density, time, load, maxh, minh, maxc, mcl, dthick, mdep, carr, darr);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// NetCDF output arrays and restart (src/write_NETCDF.f90): FP32 (op = 4,
// src/Ash3d_VariableModules.f90:31) arrays with x fastest, the layout the
// writer passes to nf90_put_var.  One thread per cell of a row; blockIdx.y =
// j, blockIdx.z strides over the (k, g) planes.
// ---------------------------------------------------------------------------
// ashcon(i,j,k,g) = real(concen_pd(i,j,k,g,ts1), kind=op) (:3296-3298)
__global__ void k_pack_ashcon(Layout L, const double *__restrict__ c, float *__restrict__ ashcon) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= L.nx) return;
  for (int kg = blockIdx.z; kg < L.nz * L.ns; kg += gridDim.z) {
    const int k = kg % L.nz, g = kg / L.nz;
    ashcon[((long)kg * L.ny + j) * L.nx + i] = __double2float_rn(c[(long)g * L.PG + L.cell(i + 1, j + 1, k + 1)]);
  }
}

// depocon(i,j,g) = real(DepositGranularity*dz_vec_pd(0)/KM2_2_M2, kind=op),
// then 0 where depocon <= EPS_SMALL, the FP32 value compared in FP64
// (:3320-3330).  DepositGranularity is outflow_xy1 ([g][j][i]).
__global__ void k_pack_depocon(Layout L, const double *__restrict__ xy1, const double *__restrict__ dz_vec,
                               float *__restrict__ depocon) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= L.nx) return;
  for (int g = blockIdx.z; g < L.ns; g += gridDim.z) {
    const long a = ((long)g * L.ny + j) * L.nx + i;
    float d = __double2float_rn(xy1[a] * dz_vec[1] / 1.0e6);  // dz_vec[1] = dz_vec_pd(0)
    if ((double)d <= 1.0e-6) d = 0.0f;
    depocon[a] = d;
  }
}

// NC_RestartFile_LoadConcen (:3701-3707): concen_pd(i,j,k,g) = real(ashcon, ip)
__global__ void k_unpack_ashcon(Layout L, const float *__restrict__ ashcon, double *__restrict__ c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= L.nx) return;
  for (int kg = blockIdx.z; kg < L.nz * L.ns; kg += gridDim.z) {
    const int k = kg % L.nz, g = kg / L.nz;
    c[(long)g * L.PG + L.cell(i + 1, j + 1, k + 1)] = (double)ashcon[((long)kg * L.ny + j) * L.nx + i];
  }
}

// outflow_xy1_pd(i,j,g) = DepositGranularity(i,j,g) = real(depocon(i,j,g), ip)
__global__ void k_unpack_depocon(Layout L, const float *__restrict__ depocon, double *__restrict__ xy1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= L.nx) return;
  for (int g = blockIdx.z; g < L.ns; g += gridDim.z) {
    const long a = ((long)g * L.ny + j) * L.nx + i;
    xy1[a] = (double)depocon[a];
  }
}

static dim3 netcdf_grid(const Layout &L, int planes) {
  return dim3((L.nx + 255) / 256, L.ny, planes < 65535 ? planes : 65535);
}

int launch_netcdf_pack(a3g_ctx *ctx, float *ashcon, float *depocon) {
  const Layout &L = ctx->L;
  tbegin(ctx, A3G_K_OTHER);
  if (ashcon) k_pack_ashcon<<<netcdf_grid(L, L.nz * L.ns), 256, 0, ctx->stream>>>(L, ctx->c0, ashcon);
  if (depocon)
    k_pack_depocon<<<netcdf_grid(L, L.ns), 256, 0, ctx->stream>>>(L, ctx->out_xy1, ctx->dz_vec, depocon);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int launch_netcdf_unpack(a3g_ctx *ctx, const float *ashcon, const float *depocon) {
  const Layout &L = ctx->L;
  tbegin(ctx, A3G_K_OTHER);
  if (ashcon) k_unpack_ashcon<<<netcdf_grid(L, L.nz * L.ns), 256, 0, ctx->stream>>>(L, ashcon, ctx->c0);
  if (depocon) k_unpack_depocon<<<netcdf_grid(L, L.ns), 256, 0, ctx->stream>>>(L, depocon, ctx->out_xy1);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// self-test of exact_div.cuh against the IEEE division operator
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

__device__ double test_operand(uint64_t h) {
  const int kind = (int)(h & 15);
  const double sgn = (h & 16) ? -1.0 : 1.0;
  const uint64_t m = (h >> 12) & 0x000fffffffffffffULL;
  int e;
  if (kind < 8) e = (int)((h >> 5) & 63) - 32;          // moderate magnitudes
  else if (kind < 12) e = (int)((h >> 5) & 1023) - 512;  // wide range (fallbacks)
  else if (kind < 13) e = (int)((h >> 5) & 15) - 8;
  else if (kind < 14) e = -830 - (int)((h >> 5) & 255);  // tiny, down to subnormal (below)
  else e = (int)((h >> 5) & 7) - 4;
  double v = __longlong_as_double(
      (long long)(((uint64_t)(1023 + (kind == 13 ? e + 300 : e)) << 52) | (kind == 14 ? 0 : m)));
  if (kind == 13) v = v * 0x1p-300;  // exact while normal, rounded below 2^-1022
  if (kind == 15) v = (double)((h >> 20) & 255) - 128.0;  // small integers, zeros, exact ratios
  return sgn * v;
}

__global__ void k_selftest_div(uint64_t n, uint64_t seed, unsigned long long *bad) {
  unsigned long long local = 0;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const double a = test_operand(mix64(seed ^ (2 * t)));
    const double b = test_operand(mix64(seed ^ (2 * t + 1)));
    if (b == 0.0) continue;
    const double q1 = div_rn(a, b), q2 = a / b;
    const double y = 1.0 / b;
    const double q3 = div_rn_rcp(a, b, y);
    const bool same1 = __double_as_longlong(q1) == __double_as_longlong(q2) || (q1 != q1 && q2 != q2);
    const bool same3 = __double_as_longlong(q3) == __double_as_longlong(q2) || (q3 != q3 && q2 != q2);
    local += (same1 ? 0 : 1) + (same3 ? 0 : 1);
  }
  if (local) atomicAdd(bad, local);
}

}  // namespace a3g

extern "C" int a3g_selftest_div(int device, uint64_t n, uint64_t seed, uint64_t *mismatches) {
  if (!mismatches) { a3g::set_error("null mismatches"); return A3G_ERR_ARG; }
  A3G_CUDA(cudaSetDevice(device));
  unsigned long long *d = nullptr;
  A3G_CUDA(cudaMalloc((void **)&d, sizeof(*d)));
  cudaError_t e = cudaMemset(d, 0, sizeof(*d));
  if (e == cudaSuccess) {
    a3g::k_selftest_div<<<148 * 8, 256>>>(n, seed, d);
    e = cudaGetLastError();
  }
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return a3g::cuda_fail(e, "a3g_selftest_div");
  *mismatches = h;
  return A3G_OK;
}
