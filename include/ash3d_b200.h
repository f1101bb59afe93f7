/*
 * ash3d_b200.h -- C-ABI of the B200 (sm_100a) transport path for Ash3d.
 *
 * The Fortran host (Ash3d.F90's main loop) reaches the GPU through these
 * functions, bound with ISO_C_BINDING (the shim module
 * volcano-ash3d_b200/fortran/ash3d_b200_shim.f90 holds the interfaces).
 * Every function returns an int status (A3G_OK = 0); a nonzero status is
 * what the reference turns into "write(errlog) ... ; stop 1".
 *
 * Arrays cross this boundary in the reference's own Fortran layouts
 * (column-major, ghost cells included) so that the shim can pass c_loc() of
 * the module arrays directly (USEPOINTERS=T build, src/makefile:80):
 *   concen level   (-1:nx+2,-1:ny+2,-1:nz+2,1:ns)  one of ts0/ts1
 *   vx/vy/vz, kappa, sigma_n{x,y,z}  (-1:nx+2,-1:ny+2,-1:nz+2)
 *   vf             (-1:nx+2,-1:ny+2,-1:nz+2,1:ns)
 *   dz_vec         (-1:nz+2)
 *   kx/ky/kz       (0:nx+1,0:ny+1,0:nz+1)
 *   outflow_yz1/2  (-1:ny+2,-1:nz+2,1:ns); _xz1/2 (-1:nx+2,-1:nz+2,1:ns);
 *   outflow_xy1/2  (-1:nx+2,-1:ny+2,1:ns); DepositGranularity (nx,ny,ns)
 * All floating point is FP64 except the FP32 met steps.  The concentration
 * stays resident on the device between calls; only the calls that return a
 * host value (Adjust_DT, TimeStepTotals, the subgrid box, downloads)
 * synchronise the context's stream.
 */
#ifndef ASH3D_B200_H
#define ASH3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define A3G_ABI_VERSION 1

/* status codes */
#define A3G_OK              0
#define A3G_ERR_ARG         1   /* bad argument (sizes, pointers, codes) */
#define A3G_ERR_CUDA        2   /* a CUDA call failed */
#define A3G_ERR_NOMEM       3   /* device allocation failed */
#define A3G_ERR_BC_CODE     4   /* Set_BC code not 1 or 2 (src/Set_BC.f90:119-123) */
#define A3G_ERR_SUBGRID     5   /* kmax<kmin in get_minmax_index (src/Calc_Mesh.f90:522-527) */
#define A3G_ERR_PIVOT       6   /* a Crank-Nicolson line needed a row interchange or hit a zero pivot */
#define A3G_ERR_STATE       7   /* call out of order (e.g. no geometry bound yet) */
#define A3G_ERR_UNSUPPORTED 8   /* option outside the implemented variants */
#define A3G_ERR_NONFINITE   9   /* NaN/Inf detected in a device reduction */
#define A3G_ERR_TIMEOUT    10   /* a bounded device-side wait (TMA tile copy) ran out */

/* limiters: the LIM_* preprocessor choices of src/makefile:126 */
#define A3G_LIM_NONE     0
#define A3G_LIM_LAXWEN   1
#define A3G_LIM_BW       2
#define A3G_LIM_FROMM    3
#define A3G_LIM_MINMOD   4
#define A3G_LIM_SUPERBEE 5
#define A3G_LIM_MC       6

typedef struct a3g_ctx a3g_ctx;

/* Grid extents and flags: module mesh (src/Ash3d_VariableModules.f90:600-760). */
typedef struct a3g_grid_desc {
  int32_t nx, ny, nz, ns;   /* nxmax, nymax, nzmax, nsmax (ash grain bins) */
  int32_t periodic;         /* IsPeriodic */
  int32_t latlon;           /* IsLatLon */
  double dx, dy;            /* projected cell sizes (km); Adjust_DT uses them when !latlon */
} a3g_grid_desc;

/* Run-time forms of the reference's compile-time and control-file options
 * (src/makefile:91-206, src/ResetParams.f90:18-37). */
typedef struct a3g_params {
  int32_t limiter;          /* A3G_LIM_*; reference default build: SUPERBEE */
  int32_t use_cn;           /* 1: CRANKNIC (diffCN_*), 0: EXPLDIFF (diff_*) */
  int32_t use_diffusion;    /* useDiffusion */
  int32_t fast_subgrid;     /* FAST_SUBGRID */
  int32_t nocycle;          /* NOCYCLE */
  int32_t zscaling_id;      /* ZScaling_ID 0 (s = z), 1 (shifted), 2 (scaled, advect_sigma) */
  double cfl;               /* CFL (0.8) */
  double dt_min, dt_max;    /* DT_MIN, DT_MAX (hours) */
  double imp_fac;           /* Imp_fac (0.5) */
  double imp_dt_fac;        /* Imp_DT_fac (4.0) */
  double eps_thresh;        /* EPS_THRESH (1e-10) */
  double eps_small;         /* EPS_SMALL (1e-6) */
  double cloudcon_grid_thresh; /* CLOUDCON_GRID_THRESH (1e-7) */
  double magma_density;     /* MagmaDensity (2500) */
} a3g_params;

/* Fills *p with the reference defaults (superbee, CN, no subgrid). */
void a3g_default_params(a3g_params *p);
int  a3g_abi_version(void);
/* Message for the last failing call on this thread ("" if none). */
const char *a3g_last_error(void);

/* ---- lifetime: replaces the device-side half of alloc_arrays,
 *      src/Alloc_Arrays.f90:14-55 ---- */
int a3g_create(const a3g_grid_desc *grid, const a3g_params *params, int device, a3g_ctx **out);
int a3g_destroy(a3g_ctx *ctx);
/* Blocks until all work queued on the context is done. */
int a3g_sync(a3g_ctx *ctx);
/* Device bytes held by the context. */
int a3g_device_bytes(a3g_ctx *ctx, size_t *bytes);

/* ---- static inputs ---- */
/* Geometry from calc_mesh_params (src/Calc_Mesh.f90:23-220).  Arrays that do
 * not vary along i (or j) are stored once per (j,k) (or k) on the device. */
int a3g_set_geometry(a3g_ctx *ctx, const double *kappa_pd, const double *sigma_nx_pd,
                     const double *sigma_ny_pd, const double *sigma_nz_pd,
                     const double *dz_vec_pd);
/* kx/ky/kz from Allocate_Diff (src/Diffusion.F90:83-104), km^2/h. */
int a3g_set_diffusivity(a3g_ctx *ctx, const double *kx, const double *ky, const double *kz);
/* Fall velocities vf_pd (km/h, negative downward; src/Input_Data.f90:3669).
 * Stored once per (k,grain) when they do not vary in x and y. */
int a3g_set_fall_velocity(a3g_ctx *ctx, const double *vf_pd);
/* IsAloft(1:ns) (Prune_GS, src/Tephra.f90:782-812); n_gs_aloft is recounted. */
int a3g_set_aloft(a3g_ctx *ctx, const int32_t *is_aloft);

/* ---- winds (MesoInterpolater, src/MesoInterpolater.f90:201-263) ---- */
/* FP64 winds already interpolated on the host (vx_pd,vy_pd,vz_pd, km/h). */
int a3g_set_winds(a3g_ctx *ctx, const double *vx_pd, const double *vy_pd, const double *vz_pd);
/* FP32 met steps on the computational grid (nx,ny,nz; m/s), the pair that
 * brackets the current time.  Uploaded once per met step. */
int a3g_set_met_steps(a3g_ctx *ctx, const float *vx_last, const float *vy_last,
                      const float *vz_last, const float *vx_next, const float *vy_next,
                      const float *vz_next);
/* Read_NextMesoStep's toggle (src/MesoInterpolater.f90:168-199) without a
 * stall: a3g_prefetch_met_step copies the met step after next (FP32 nx*ny*nz,
 * m/s) into a spare slot on a copy stream (asynchronous for pinned host
 * memory); at the met-step boundary a3g_advance_met_step makes the old next
 * step the last one and the prefetched step the next one (the compute stream
 * waits for the copy).  a3g_met_prefetch_fence makes the compute stream wait
 * for a prefetch in flight.  Pinned host arrays given to a prefetch must stay
 * unchanged until then. */
int a3g_prefetch_met_step(a3g_ctx *ctx, const float *vx, const float *vy, const float *vz);
int a3g_advance_met_step(a3g_ctx *ctx);
int a3g_met_prefetch_fence(a3g_ctx *ctx);
/* Device form of src/MesoInterpolater.f90:207-223:
 * v = (dble(last) + dble(next-last)*frac)*3.6 */
int a3g_interp_winds(a3g_ctx *ctx, double interval_frac);

/* ---- lag-one host loop (no counterpart in the reference) ----
 * The reference's host reads dt back every step; these let a host queue a
 * whole step without waiting for the GPU, and read dt and the totals back
 * later, while the GPU works on the step's sweeps.
 * a3g_adjust_dt_async: Adjust_DT as a3g_adjust_dt, with dt left on the device
 * (the sweeps and the scheduled source read it there) and copied to a pinned
 * ring behind an event.  a3g_wait_dt: dt of the latest a3g_adjust_dt_async,
 * waiting only for that copy (and reporting a device error word).
 * a3g_timestep_totals_async / a3g_totals_get: TimeStepTotals with the
 * partial sums copied behind an event; a ticket stays valid for the next 4
 * calls. */
int a3g_adjust_dt_async(a3g_ctx *ctx, double time, double next_write_time, double simtime);
int a3g_wait_dt(a3g_ctx *ctx, double *dt);
int a3g_timestep_totals_async(a3g_ctx *ctx, int64_t *ticket);
int a3g_totals_get(a3g_ctx *ctx, int64_t ticket, double *out4, double *mass_aloft);
/* The eruption schedule for a3g_add_source_scheduled: per pulse the start and
 * end times (h) and MassFluxRate (kg/h), NormSourceColumn(npulses, nz+1)
 * (Fortran layout), Tephra_bin_mass(1:ns) (src/Source.f90:508-592,287-490). */
int a3g_set_source_pulses(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t npulses, const double *start_h,
                          const double *end_h, const double *mass_flux_rate, const double *norm_col,
                          const double *bin_mass);
/* CheckEruptivePulses + TephraSourceNodes + the vent-column insertion
 * (src/Source.f90:613-783, src/Ash3d.F90:416-431) on the device, with the dt
 * of the last Adjust_DT; ieruption/jeruption are kept on the device. */
int a3g_add_source_scheduled(a3g_ctx *ctx, double time);

/* The vent-column insertion of a3g_add_source_column with the dt that the
 * last Adjust_DT left on the device (for a host that reads dt late). */
int a3g_add_source_column_devdt(a3g_ctx *ctx, int32_t ivent, int32_t jvent, const double *flux);

/* ---- umbrella source (SourceType 'umbrella' / 'umbrella_air'; lon/lat grids) ---- */
/* Allocate_Source_Umbrella (src/Source_Umbrella.f90:85-153): the vent, the
 * umbrella levels ibase..itop and AvgStenc_Umbrella (3,3,nz).  Allocates the
 * per-step buffers once; the 3x3 patch must lie inside the grid. */
int a3g_set_umbrella(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t ibase, int32_t itop,
                     const double *avg_stencil);
/* Adds umbrella_winds' radial winds (km/h; uvx, uvy over the box i0..i1 x
 * j0..j1, i fastest) to vx, vy on levels ibase..itop, as MesoInterpolater
 * does while the eruption lasts (src/MesoInterpolater.f90:233-248).  Call it
 * after a3g_interp_winds / a3g_set_winds and before Adjust_DT; with terrain
 * bound, vh is formed again from the updated winds. */
int a3g_add_umbrella_winds(a3g_ctx *ctx, int32_t i0, int32_t i1, int32_t j0, int32_t j1,
                           const double *uvx, const double *uvy);
/* Umbrella source insertion (src/Ash3d.F90:435-458): on ibase..itop the 3x3
 * patch is set to its AvgCon_Umbrella average, then every patch cell gains
 * dt*SourceNodeFlux_Umbrella(3,3,nz+1,ns) (TephraSourceNodes_Umbrella,
 * src/Source_Umbrella.f90:409-448). */
int a3g_add_source_umbrella(a3g_ctx *ctx, const double *flux_umbrella, double dt);

/* ---- terrain (useTopo; src/Topography.f90) ---- */
/* Binds the topography terms of the step: dhdx_comp, dhdy_comp, DelDxonD_cc,
 * DelDyonD_cc (-1:nx+2,-1:ny+2, as Calc_FDGrad_Topo leaves them,
 * src/Topography.f90:2471-2536), s_cc_pd (-1:nz+2) and Ztop (km).  From
 * then on every a3g_set_winds / a3g_interp_winds also forms vh on the device
 * (Calc_Vmod_Topo, src/Topography.f90:2138-2166, which the reference calls
 * right after MesoInterpolater, src/Ash3d.F90:398), and the z sweep uses
 * vz+vh+vf (src/AdvectionVert_DCU.f90:172-174).  vh is zero on the ghost
 * levels, where the reference's vx_pd and vy_pd are never written.  With
 * ZScaling_ID 2 the x and y sweeps add the DelD*onD_cc terms
 * (src/AdvectionHorz_DCU.f90:163-166,251-257) and AdvectVert runs
 * advect_sigma (:341-564, the same line update as advect_z); the scaled
 * kappa_pd and sigma_n{x,y}_pd of calc_s_mesh (src/Calc_Mesh.f90:316-328)
 * come in through a3g_set_geometry.  ZScaling_ID 0 makes vh zero.  The
 * adjoint (a3g_adj_*) returns A3G_ERR_UNSUPPORTED once terrain is bound. */
int a3g_set_topo(a3g_ctx *ctx, const double *dhdx_comp, const double *dhdy_comp,
                 const double *deldx_on_d, const double *deldy_on_d, const double *s_cc_pd,
                 double ztop);

/* ---- concentration state ---- */
/* Uploads/downloads the interior of one level (ghosts of the download are
 * written as zero: the state of ts0 after the step prologue). */
int a3g_upload_concen(a3g_ctx *ctx, const double *concen_level);
int a3g_download_concen(a3g_ctx *ctx, double *concen_level);
/* Outflow accumulators and DepositGranularity (any pointer may be NULL). */
int a3g_upload_outflow(a3g_ctx *ctx, const double *yz1, const double *yz2, const double *xz1,
                       const double *xz2, const double *xy1, const double *xy2);
int a3g_download_outflow(a3g_ctx *ctx, double *yz1, double *yz2, double *xz1, double *xz2,
                         double *xy1, double *xy2, double *deposit);

/* ---- NetCDF output arrays and restart (src/write_NETCDF.f90) ---- */
/* The 3-D and 4-D arrays the NetCDF writer puts, formed on the device from
 * the current state (src/write_NETCDF.f90:3287-3300, 3307-3330):
 *   ashcon(1:nx,1:ny,1:nz,1:ns) = real(concen_pd(1:nx,1:ny,1:nz,1:ns,ts1), kind=op)
 *   depocon(1:nx,1:ny,1:ns)     = real(DepositGranularity*dz_vec_pd(0)/KM2_2_M2, kind=op),
 *                                 then 0 where depocon <= EPS_SMALL (1e-6; the FP32
 *                                 value compared in FP64, as Fortran promotes it)
 * op = 4 (src/Ash3d_VariableModules.f90:31): FP32, x fastest, nx*ny*nz*ns and
 * nx*ny*ns floats.  Either pointer may be NULL.  Each may be host or device
 * memory: device memory of the context's device (or managed memory) is
 * written by the kernel directly, anything else through one FP32 copy, half
 * the bytes of a3g_download_concen.  Synchronous. */
int a3g_output_ashcon(a3g_ctx *ctx, float *ashcon, float *depocon);
/* NC_RestartFile_LoadConcen (src/write_NETCDF.f90:3646-3716):
 * concen_pd(1:nx,1:ny,1:nz,:,ts1) = real(ashcon, ip), then concen(ts0) =
 * concen(ts1); outflow_xy1_pd(1:nx,1:ny,:) = DepositGranularity =
 * real(depocon, ip).  As in the reference, depocon is loaded as the file
 * holds it (kg/m^2, the writer's dz_vec_pd(0)/KM2_2_M2 scaling is not undone)
 * and the other outflow accumulators are left as they are.  Layouts, NULL and
 * pointer rules as a3g_output_ashcon.  Synchronous. */
int a3g_restart_load(a3g_ctx *ctx, const float *ashcon, const float *depocon);

/* ---- the per-step path (callers: src/Ash3d.F90:372-642) ---- */
/* Step prologue, src/Ash3d.F90:376-378 (ts0 <- ts1; ts1 <- 0). */
int a3g_step_prologue(a3g_ctx *ctx);
/* Sets dt (hours) for the next operators, as Adjust_DT/FAST_DT leave it in
 * time_data::dt (src/Ash3d_VariableModules.f90:1071-1072). */
int a3g_set_dt(a3g_ctx *ctx, double dt);
/* Source insertion, src/Ash3d.F90:428-431: concen(ivent,jvent,1:nz+1,:,ts0)
 * += dt*SourceNodeFlux; flux is (nz+1) x ns, k fastest (kg/km^3/h). */
int a3g_add_source_column(a3g_ctx *ctx, int32_t ivent, int32_t jvent, const double *flux,
                          double dt);
/* Set_BC(bc_code), src/Set_BC.f90:15-126.  Ghost cells are generated inside
 * the sweep kernels, so this validates the code and records it. */
int a3g_set_bc(a3g_ctx *ctx, int32_t bc_code);
/* AdvectHorz(itoggle), src/AdvectionHorz.f90:47-85 (with get_minmax_index,
 * src/Calc_Mesh.f90:432-542, when fast_subgrid; ivent/jvent/kvent used then). */
int a3g_advect_horz(a3g_ctx *ctx, int32_t itoggle, int32_t ivent, int32_t jvent, int32_t kvent);
/* advect_x / advect_y, src/AdvectionHorz_DCU.f90:68-305 / 322-556. */
int a3g_advect_x(a3g_ctx *ctx);
int a3g_advect_y(a3g_ctx *ctx);
/* AdvectVert -> advect_z, src/AdvectionVert_DCU.f90:64-323. */
int a3g_advect_vert(a3g_ctx *ctx);
/* DiffuseHorz(i), src/Diffusion.F90:151-216 (diff_x/y or diffCN_x/y). */
int a3g_diffuse_horz(a3g_ctx *ctx, int32_t itime);
/* DiffuseVert, src/Diffusion.F90:232-247 (diff_z or diffCN_z). */
int a3g_diffuse_vert(a3g_ctx *ctx);
/* Adjust_DT(mesostep=.false.), src/Adjust_dt.f90:19-339.  Computes dt on the
 * device from the current winds, then clips it to the next write time and
 * the simulation end exactly as :321-332; *dt_out receives it. */
int a3g_adjust_dt(a3g_ctx *ctx, double time, double next_write_time, double simtime,
                  double *dt_out);
/* The two halves of Adjust_DT for grain-sharded runs (grains split across
 * GPUs, each rank one context): a3g_cfl_maxima returns this context's three
 * CFL maxima {vx term, vy term, (|vz|+max|vf|)/dz term} (src/Adjust_dt.f90:
 * 136-173); after a MAX all-reduce of those over the ranks,
 * a3g_adjust_dt_from_maxima applies :176-332 to them, so every rank gets the
 * dt the reference computes over all grains. */
int a3g_cfl_maxima(a3g_ctx *ctx, double *vmax3);
int a3g_adjust_dt_from_maxima(a3g_ctx *ctx, const double *vmax3, int32_t n_gs_aloft_total,
                              double time, double next_write_time, double simtime,
                              double *dt_out);
/* The same two halves with the maxima kept on the device, for a sharded loop
 * that does not wait on the GPU (the same sources): a3g_cfl_maxima_device
 * queues the reduction on the context's stream into three doubles of the
 * context's device memory and returns their address (fixed for the
 * context's life); the caller all-reduces them (MAX) in place, ordered on
 * the context's stream (a3g_get_stream); a3g_adjust_dt_device_maxima_async
 * then forms dt from them on the device and queues its copy to the host,
 * which a3g_wait_dt returns, as a3g_adjust_dt_async does. */
int a3g_cfl_maxima_device(a3g_ctx *ctx, double **vmax3_dev);
int a3g_adjust_dt_device_maxima_async(a3g_ctx *ctx, int32_t n_gs_aloft_total, double time,
                                      double next_write_time, double simtime);
/* ---- FAST_DT: the time step of the reference's default build
 *      (FASTFPPFLAG = -DFAST_DT, src/makefile:91) ----
 * With FAST_DT the CFL maxima are taken only when a met step is loaded, on the
 * FP32 met step itself (Adjust_DT(mesostep=.true.), src/Adjust_dt.f90:96-135),
 * and every step's dt is interpolated between the dt of the last and of the
 * next met step (src/MesoInterpolater.f90:250-258).
 * a3g_set_fall_velocity_meso: vf_meso_next_step_sp (m/s, FP32), which
 * Read_NextMesoStep fills: per_grain=0, the whole (nx,ny,nz,ns) array in
 * Fortran order (fall models evaluated per cell); per_grain=1, ns values, the
 * real(Tephra_v_s(isize), sp) that Read_NextMesoStep puts in every cell when
 * the fall velocities come from the input file (src/MesoInterpolater.f90:
 * 567-574).  Only max_g |vf| per cell is kept.
 * a3g_cfl_maxima_meso: the three maxima of src/Adjust_dt.f90:96-135 over the
 * FP32 met step in device slot `slot` (0: last, 1: next, as a3g_set_met_steps
 * and a3g_advance_met_step leave them): real(max|vx|)*3.6 (projected; divided
 * by dx later) or real(|vx|)*3.6*minsig/kappa (lon/lat), and
 * real(|vz| + max_g|vf|)*3.6/dz_k with the sum in FP32.
 * a3g_adjust_dt_meso: Adjust_DT(mesostep=.true.) on that slot: dt formed from
 * those maxima as in :176-332 (snapped to DT_MIN, clipped to the next write
 * time and the end) becomes time_data::dt and dt_meso_next, both kept on the
 * device.  shift=1 first copies dt_meso_next to dt_meso_last, the toggle of
 * src/MesoInterpolater.f90:187.  dt_out may be NULL (nothing waits then).
 * The first met-step load of a run is a3g_adjust_dt_meso(slot 0, shift 0)
 * then (slot 1, shift 1) (src/MesoInterpolater.f90:142-150,187-195); every
 * later load, after a3g_advance_met_step, is (slot 1, shift 1).
 * a3g_adjust_dt_meso_from_maxima: the same from maxima all-reduced over the
 * ranks of a grain-sharded run (a3g_cfl_maxima_meso on each).
 * a3g_fast_dt_async: the step's dt = dt_meso_last + (dt_meso_next -
 * dt_meso_last)*interval_frac, clipped to the next write time and the end,
 * on the device (the sweeps read it there) and copied back behind an event
 * like a3g_adjust_dt_async; a3g_wait_dt returns it. */
int a3g_set_fall_velocity_meso(a3g_ctx *ctx, const float *vf_meso_sp, int32_t per_grain);
int a3g_cfl_maxima_meso(a3g_ctx *ctx, int32_t slot, double *vmax3);
int a3g_adjust_dt_meso(a3g_ctx *ctx, int32_t slot, int32_t shift, double time, double next_write_time,
                       double simtime, double *dt_out);
int a3g_adjust_dt_meso_from_maxima(a3g_ctx *ctx, const double *vmax3, int32_t n_gs_aloft_total, int32_t shift,
                                   double time, double next_write_time, double simtime, double *dt_out);
int a3g_fast_dt_async(a3g_ctx *ctx, double interval_frac, double time, double next_write_time, double simtime);
/* TimeStepTotals sums, src/TimeStepTotals.f90:57-66 with Calc_AshVol_Aloft/
 * Deposit/Outflow (src/Output_Vars.f90:1255-1459).  out4 = {aloft_vol,
 * dep_vol, outflow_vol, tot_vol} (km^3 DRE); mass_aloft (ns, kg) may be NULL.
 * Returns A3G_ERR_NONFINITE (the values still written) when a total is NaN or
 * infinite, which the reference would carry on with silently. */
int a3g_timestep_totals(a3g_ctx *ctx, double *out4, double *mass_aloft);
/* get_minmax_index, src/Calc_Mesh.f90:432-542: box = {imin,imax,jmin,jmax,kmin,kmax}. */
int a3g_get_minmax_index(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t kvent,
                         int32_t *box);
/* Sets the current box (solution::imin..kmax) explicitly. */
int a3g_set_subgrid(a3g_ctx *ctx, const int32_t *box);
int a3g_get_subgrid(a3g_ctx *ctx, int32_t *box);

/* One whole transport step in the order of src/Ash3d.F90:376-510 with the
 * dt already set: prologue, source column (flux may be NULL), Set_BC(1),
 * AdvectHorz(itime), AdvectVert, [Set_BC(2), DiffuseHorz(itime),
 * DiffuseVert].  Nothing is allocated inside. */
int a3g_step(a3g_ctx *ctx, int32_t itime, int32_t ivent, int32_t jvent, int32_t kvent,
             const double *flux);

/* Count of kernels this context has launched (diagnostics). */
int a3g_kernel_launches(a3g_ctx *ctx, uint64_t *count);

/* ---- measurement (no counterpart in the reference, which only reports
 *      cpu_time/system_clock totals, src/Ash3d.F90:727-759) ---- */
/* The cudaStream_t all of this context's work is queued on. */
int a3g_get_stream(a3g_ctx *ctx, void **stream);
/* Kernel classes reported by a3g_kernel_times. */
#define A3G_K_ADVECT_X   0
#define A3G_K_ADVECT_Y   1
#define A3G_K_ADVECT_Z   2
#define A3G_K_DIFF_X     3
#define A3G_K_DIFF_Y     4
#define A3G_K_DIFF_Z     5
#define A3G_K_CN_TABLE   6
#define A3G_K_CN_SOLVE_X 7
#define A3G_K_CN_SOLVE_Y 8
#define A3G_K_CN_SOLVE_Z 9
#define A3G_K_CFL        10
#define A3G_K_TOTALS     11
#define A3G_K_WINDS      12
#define A3G_K_OTHER      13
#define A3G_K_ADJOINT    14
#define A3G_K_COUNT      15
/* Starts (enable=1) or stops per-kernel CUDA-event timing; starting clears
 * the accumulators.  Timing brackets every launch with two events on the
 * context's stream. */
int a3g_kernel_timing(a3g_ctx *ctx, int32_t enable);
/* Sums per kernel class since timing was enabled (synchronises the stream):
 * ms[A3G_K_COUNT] total milliseconds, count[A3G_K_COUNT] launches. */
int a3g_kernel_times(a3g_ctx *ctx, double *ms, uint64_t *count);

/* ---- tuning (no counterpart in the reference) ---- */
/* Selects a kernel variant.  dir 0, 1, 2: the advection sweep along x, y, z,
 * variant 0 marching threads, 1 blocks of 4 cells, 2 blocks of 8 cells, and
 * for x only 3, warps marching 32 rows through shared-memory tiles, 4,
 * one warp per row walking it in 32-cell chunks with the lanes along i, and
 * 5, the same with the interior chunks staged one ahead by TMA tensor copies
 * (defaults: x 5, y 6, z 6).
 * dir 3: the Crank-Nicolson x solve, variant 0 warp-tiled, 1 one thread per
 * line, 2 warp-tiled with each tile loaded one chunk ahead by a TMA tensor
 * copy (default).  dir 4: the Crank-Nicolson y and z solves, variant 0 one
 * grain per thread, 1 two grains of a line per thread, 2 four, 3 tiles of
 * 32 lines staged in shared memory by TMA tensor copies (default; where the
 * coefficients vary along i, or nz > 256, variant 3 runs variant 1).
 * dir 1, 2 variant 5: the column march (one thread per line and grain, lanes
 * along i, each interface formed once); variant 6, the same march reading
 * the concentration and wind from chunks that TMA tensor copies stage in
 * shared memory (default for y and z; where the geometry varies along i or
 * the fall speed within a grain, variant 6 runs variant 1).  dir 5: the adjoint advection sweeps,
 * variant 0 four-cell blocks (default), 1 one cell per thread.  All variants
 * produce identical results; only their speed differs. */
int a3g_set_variant(a3g_ctx *ctx, int32_t dir, int32_t variant);
int a3g_get_variant(a3g_ctx *ctx, int32_t dir, int32_t *variant);

/* ---- output products (Gen_Output_Vars, src/Output_Vars.f90:1192-1240) ----
 * The 2-D products the reference writes at output and log steps, computed
 * on the device from the current state: ConcentrationCalculator (column
 * cloud load in t/km2 masked below CLOUDLOAD_THRESH, cloud top and bottom
 * heights from CLOUDCON_THRESH, peak concentration in mg/m3, the cloud mask;
 * :1026-1123), AshThicknessCalculator (deposit thickness in mm from
 * DepositGranularity and its mask; :855-895), CloudAreaCalculator (:1138-1177)
 * and the arrival-time marks (:1226-1236), which persist in the context.
 * z_cc: z_cc_pd(1:nz) (km).  Defaults: CLOUDCON_THRESH 1e-3 kg/km3,
 * CLOUDLOAD_THRESH 0.2 t/km2, DEPO_THRESH 0.01 mm, DepositDensity 1000 kg/m3. */
int a3g_set_output_params(a3g_ctx *ctx, const double *z_cc, double cloudcon_thresh,
                          double cloudload_thresh, double depo_thresh, double deposit_density);
/* Arrival times back to "not arrived" (-1). */
int a3g_output_reset(a3g_ctx *ctx);
/* All 2-D arrays (nx,ny), i fastest; any output may be NULL.  areas =
 * {CloudArea, DepositAreaCovered, CloudLoadArea(1:5)} (km2), summed in the
 * reference's loop order over the current subgrid box. */
int a3g_output_vars(a3g_ctx *ctx, double time, double *cloud_load, double *max_height,
                    double *min_height, double *max_conc, int32_t *mask_cloud, double *dep_thick,
                    int32_t *mask_dep, double *cloud_arrival, double *dep_arrival, double *areas);
/* Calc_vprofile (src/Output_Vars.f90:1308-1360): for each of npts points
 * (i_pts, j_pts, 1-based) whose column total of the current state is at
 * least CLOUDCON_THRESH (a3g_set_output_params), pr_ash(1:nz, point) = the
 * sum over the grains, in mg/m3, and written[point] = 1; the profiles of the
 * other points are left as they are and written[point] = 0.  The reference
 * reads the scratch level ts1, equal to the state after a step. */
int a3g_vprofiles(a3g_ctx *ctx, int32_t npts, const int32_t *i_pts, const int32_t *j_pts, double *pr_ash,
                  int32_t *written);

/* ---- discrete adjoint (no counterpart in the reference) ----
 * Reverse mode of the transport step for source inversion.  Every sweep is
 * piecewise linear in the concentration; with the limiter branches fixed by
 * the state the sweep was applied to it is a linear map J, and these calls
 * apply J^T to the adjoint field lam kept on the device.  They need the full
 * box (fast_subgrid off: the subgrid box depends on the state) and leave the
 * forward state and the outflow accumulators untouched.  dt and the winds
 * must be those of the forward step (a3g_set_dt / a3g_set_winds or
 * a3g_interp_winds). */
/* Allocates lam, the deposit adjoint and the step's stage buffer (3 levels
 * plus one face); lam starts at zero.  a3g_adj_step recomputes its second
 * intermediate state into the scratch level ts1. */
int a3g_adj_enable(a3g_ctx *ctx);
int a3g_adj_zero(a3g_ctx *ctx);
/* lam in the layout of concen_pd(:,:,:,:,ts0) (ghost values ignored on
 * upload, left untouched on download). */
int a3g_adj_set_lambda(a3g_ctx *ctx, const double *lam);
int a3g_adj_get_lambda(a3g_ctx *ctx, double *lam);
/* adjoint of DepositGranularity (nx,ny,ns), the bottom outflow of AdvectVert */
int a3g_adj_set_lambda_dep(a3g_ctx *ctx, const double *lam_dep);
int a3g_adj_get_lambda_dep(a3g_ctx *ctx, double *lam_dep);
/* One sweep's transpose, linearised at the current state (the sweep's
 * input): lam <- J^T lam.  a3g_adj_advect_vert also adds the deposit
 * adjoint's contribution.  a3g_adj_diffuse_horz(itime) reverses
 * DiffuseHorz(itime)'s order of x and y. */
int a3g_adj_advect_x(a3g_ctx *ctx);
int a3g_adj_advect_y(a3g_ctx *ctx);
int a3g_adj_advect_vert(a3g_ctx *ctx);
int a3g_adj_diffuse_horz(a3g_ctx *ctx, int32_t itime);
int a3g_adj_diffuse_vert(a3g_ctx *ctx);
/* The whole transport step itime (Set_BC(1), AdvectHorz(itime), AdvectVert,
 * Set_BC(2), DiffuseHorz(itime), DiffuseVert) in reverse, with the state
 * after the step's source insertion in the context.  The step's
 * intermediate states are recomputed on the device. */
int a3g_adj_step(a3g_ctx *ctx, int32_t itime);
/* lam at the vent column, (nz+1) x ns with k fastest (the layout of the
 * source flux): the adjoint of the source insertion before dt/kappa. */
int a3g_adj_vent_column(a3g_ctx *ctx, int32_t ivent, int32_t jvent, double *out);
/* The source gradient gathered on the device: a3g_adj_grad_reset zeroes
 * nbins x ns x nz bins; each reverse step a3g_adj_vent_accumulate adds
 * dt*lam(ivent,jvent,k,g)/kappa(ivent,jvent,k) (k = 1..nz) to bin `bin`, in
 * the order of the calls; a3g_adj_grad_get copies the bins back (bin-major,
 * then grain, k fastest). */
int a3g_adj_grad_reset(a3g_ctx *ctx, int32_t nbins);
int a3g_adj_vent_accumulate(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t bin, double dt);
int a3g_adj_grad_get(a3g_ctx *ctx, double *out);
/* Unmasked column load (CloudLoad of src/Output_Vars.f90:1061-1069,
 * tonnes/km^2) of the current state, (nx,ny); and lam += H^T w for a
 * weight w (nx,ny), H that column load. */
int a3g_cloud_load(a3g_ctx *ctx, double *out);
int a3g_adj_add_cloud_load(a3g_ctx *ctx, const double *w);
/* Device-resident copies of the concentration (checkpoints of the forward
 * run for the reverse sweep). */
int a3g_snapshot_alloc(a3g_ctx *ctx, int32_t nslots);
int a3g_snapshot_save(a3g_ctx *ctx, int32_t slot);
int a3g_snapshot_load(a3g_ctx *ctx, int32_t slot);

/* ---- source inversion over a whole run: forward/adjoint pair (no counterpart
 *      in the reference, which runs forward only) ----
 * The control p is the erupted mass rate (kg/h) per model level, hourly bin
 * and grain bin, Fortran order (nz, nbins, ns), inserted at the vent column
 * as src/Ash3d.F90:428-431 inserts SourceNodeFlux: concen(ivent,jvent,k,g)
 * += dt*p(k,bin,g)/kappa(ivent,jvent,k), bin = the hour the step starts in.
 * Observations: the unmasked column load (CloudLoad, src/Output_Vars.f90:
 * 1061-1069, tonnes/km^2) at the end of every hour, (nx,ny) per hour, and the
 * deposit thickness (AshThicknessCalculator, src/Output_Vars.f90:880-884, mm,
 * unmasked) accumulated after hour dep_from, (nx,ny).  Misfit:
 *   J = 1/2 sum_{hours h >= load_from} |load_h - y_h|^2 + 1/2 |dep - y_dep|^2
 * (either term as `misfit` selects).  The run starts from a clean atmosphere
 * at time 0; dt is clipped to the next hour so that observations fall on step
 * ends; FAST_SUBGRID must be off and no terrain or umbrella source bound. */
#define A3G_MISFIT_LOAD    1
#define A3G_MISFIT_DEPOSIT 2
typedef struct a3g_inv_desc {
  int32_t ivent, jvent;      /* vent column (1-based) */
  int32_t nbins;             /* hourly source bins of the control */
  int32_t misfit;            /* A3G_MISFIT_LOAD | A3G_MISFIT_DEPOSIT */
  int32_t fast_dt;           /* 1: FAST_DT (met-step dt interpolated), 0: Adjust_DT every step */
  int32_t load_from;         /* first observed hour of the column loads (0-based) */
  int32_t dep_from;          /* the deposit misfit counts the deposit laid down after this hour */
  int32_t adj_from;          /* the reverse run covers the steps from this hour on (0: the whole run);
                              * the gradient then holds the bins of those steps, and lam
                              * (a3g_adj_get_lambda) is the misfit's adjoint at that hour */
  double sim_hours;          /* run length, whole hours */
  double snapshot_bytes;     /* device memory for checkpoints; <= 0: the free memory less 2 GiB */
  int32_t met_cache;         /* 0: every met step of the run on the device when they take at most a
                              * quarter of the free memory; 1: never (the three met slots of the
                              * context, each step uploaded from the provider when a run reaches it) */
} a3g_inv_desc;
/* Met-step provider: sets three pointers to the FP32 met step of `hour`
 * (vx, vy, vz; nx*ny*nz, m/s, i fastest) in host memory, valid until the next
 * call; returns 0, nonzero on failure. */
typedef int (*a3g_met_provider)(void *user, int32_t hour, const float **vx, const float **vy, const float **vz);
/* Binds the problem: observations (obs_load: nhours*nx*ny, hour-major;
 * obs_dep: nx*ny; either may be NULL when its misfit term is off), the met
 * steps (all copied to the device when they take at most a quarter of the
 * free memory, else fetched per hour), and the dt of every step, formed here
 * from the winds alone.  Allocates the adjoint buffers. */
int a3g_inv_setup(a3g_ctx *ctx, const a3g_inv_desc *desc, a3g_met_provider met, void *user,
                  const double *obs_load, const double *obs_dep);
/* The forward run for control p: every step in the reference's order, the
 * observations, J (J_out may be NULL) and the step count.  Keeps the
 * checkpoints the reversal starts from: binomial placement under the budget
 * (with room for every state, every state). */
int a3g_forward_checkpointed(a3g_ctx *ctx, const double *p, double *J_out, int32_t *nsteps);
/* The reverse run after a3g_forward_checkpointed: grad (nz, nbins, ns) =
 * J_obs^T w, the vector-Jacobian product with weights w_load (nhours*nx*ny)
 * and w_dep (nx*ny) on every observation (both given); NULL weights take the
 * residuals of the misfit's terms, so that grad = dJ/dp.  Steps between checkpoints are recomputed
 * on the device; the forward run's checkpoints are spent. */
int a3g_adjoint(a3g_ctx *ctx, const double *w_load, const double *w_dep, double *grad);
/* The tangent-linear run: the observations' perturbation for a control
 * perturbation dp at control p (limiter branches of the run at p). */
int a3g_tangent_linear(a3g_ctx *ctx, const double *p, const double *dp, double *dloads, double *ddep);
/* The last run's observations (loads: nhours*nx*ny, dep: nx*ny; either may
 * be NULL) and stats = {steps, checkpoint slots, forward steps the last
 * reversal recomputed, steps in the reversal window} (four entries). */
int a3g_inv_observations(a3g_ctx *ctx, double *loads, double *dep, int64_t *stats);
/* Forward steps the binomial reversal of nsteps steps repeats with nslots
 * free checkpoint slots, and its first split (host arithmetic only). */
int a3g_checkpoint_cost(int32_t nsteps, int32_t nslots, int64_t *recomputed, int32_t *first_split);

/* ---- allocation-free entry point (no counterpart in the reference) ---- */
/* Per-grain airborne mass, sum(c*kappa) over the interior cells, for callers
 * that cannot allocate device memory at the time of the call: hosts that
 * reserve all GPU memory at start-up and forbid allocation afterwards, or
 * hosts that hand the library buffers from their own memory manager.  It
 * calls no allocation routine: its partial sums live in a fixed device array
 * of the library (64 grains x 296 blocks x 2 doubles, about 296 KiB per
 * device, held until the process exits).  It launches two kernels, so call
 * it from ordinary host code, not from a stream callback or host function.
 *   conc:  device array [ns][nz][ny][row_pitch] (i fastest, interior cells)
 *   kappa: device array [nz][ny][nx] (interior cell volumes)
 *   mass_out: device array [ns] (written)
 *   stream: a cudaStream_t, or NULL for the default stream; the call is
 *           asynchronous on it.
 * ns above 64 is rejected with A3G_ERR_ARG.  The launches run with `device`
 * current; the caller's current device is restored before the call returns.
 * The first call on a device looks up the array's device address with that
 * device current and caches it for the life of the process: make that first
 * call before any stream capture, and do not call again on a device after a
 * cudaDeviceReset of it (the cached address would be stale).  All calls
 * share the array and it keeps the last call's contents (nothing in it needs
 * to start at zero); calls whose kernels overlap on the same device race on
 * it. */
int a3g_mass_aloft_noalloc(int device, const double *conc, const double *kappa, int32_t nx,
                           int32_t ny, int32_t nz, int32_t ns, int64_t row_pitch,
                           double *mass_out, void *stream);

/* ---- diagnostics (no counterpart in the reference) ---- */
/* Checks the library's division against the IEEE division operator on n
 * seeded operand pairs (mixed magnitudes, signs, powers of two, zeros) on
 * the given device; *mismatches receives the number of differing quotients
 * (0 is expected: the sweeps rely on bit-identical quotients). */
int a3g_selftest_div(int device, uint64_t n, uint64_t seed, uint64_t *mismatches);

#ifdef __cplusplus
}
#endif

#endif
