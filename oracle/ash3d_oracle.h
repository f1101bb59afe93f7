/*
 * ash3d_oracle.h -- CPU restatement of Ash3d's per-time-step transport path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA library
 * (volcano-ash3d_b200/csrc) and the timed CPU baseline; it is never linked
 * into, called by, or used as a fallback for the product path.  Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline legs of bench.py load it.
 *
 * It keeps the reference's data layout exactly: Fortran column-major arrays
 * with two ghost cells on each side (concen_pd(-1:nx+2,-1:ny+2,-1:nz+2,1:ns,
 * ts0:ts1), src/Ash3d_VariableModules.f90:923-946), the ts0/ts1 working and
 * scratch levels, the zero-then-copy-back of every sweep and the operator
 * order of src/Ash3d.F90:372-510.  OpenMP appears exactly where the reference
 * has it: the row loops of the three advection sweeps.
 *
 * Parity pinning: the Fortran reference cannot be compiled in this image (no
 * Fortran compiler, no MetReader/HoursSince/projection libraries).  The
 * restatement is pinned against the reference binary's own regression
 * outputs instead: tests/test_ref_goldens.py reruns the reference's
 * tests/test_02 (advection + explicit diffusion, Suzuki source) to 2e-4 of
 * its L2 check (tolerance 0.1) and tests/test_01 (a rotating 1-D wind
 * sounding) to 0.04-0.09 (tolerance 0.01; the sounding's interpolation onto
 * the grid belongs to MetReader, outside the reference tree).  The
 * tridiagonal solver (a restatement of LAPACK dgtsv, the third-party routine
 * on this path) is pinned against SciPy's LAPACK dgtsv in
 * tests/test_oracle_dgtsv.py.  CN diffusion, lon/lat grids, settling and the
 * non-superbee limiters follow the reference source but no reference output
 * covers them.
 */
#ifndef ASH3D_ORACLE_H
#define ASH3D_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Limiter ids: the LIM_* preprocessor choices of src/makefile:126. */
enum { ORC_LIM_NONE = 0, ORC_LIM_LAXWEN = 1, ORC_LIM_BW = 2, ORC_LIM_FROMM = 3,
       ORC_LIM_MINMOD = 4, ORC_LIM_SUPERBEE = 5, ORC_LIM_MC = 6 };

/*
 * All arrays are owned by the caller and laid out exactly as the Fortran
 * module arrays (column-major, ghost extents included):
 *   concen   (-1:nx+2,-1:ny+2,-1:nz+2,1:ns,0:1)
 *   vx,vy,vz,vh,kappa,sig_nx,sig_ny,sig_nz (-1:nx+2,-1:ny+2,-1:nz+2)
 *   vf       (-1:nx+2,-1:ny+2,-1:nz+2,1:ns)
 *   dz_vec   (-1:nz+2)
 *   kx,ky,kz (0:nx+1,0:ny+1,0:nz+1)
 *   outflow_yz1/2 (-1:ny+2,-1:nz+2,1:ns)
 *   outflow_xz1/2 (-1:nx+2,-1:nz+2,1:ns)
 *   outflow_xy1/2 (-1:nx+2,-1:ny+2,1:ns)
 *   deposit  DepositGranularity(1:nx,1:ny,1:ns)
 *   is_aloft IsAloft(1:ns) (0/1)
 *   mass_aloft (1:ns)
 */
typedef struct orc_state {
  int32_t nx, ny, nz, ns;
  int32_t periodic, latlon;
  int32_t limiter, use_cn, use_diffusion, fast_subgrid, nocycle;
  int32_t imin, imax, jmin, jmax, kmin, kmax;
  int32_t have_dt_diffus, n_gs_aloft;
  int32_t nthreads, pad0;
  double dx, dy;
  double cfl, dt_min, dt_max, imp_fac, imp_dt_fac, eps_thresh;
  double eps_small, cloudcon_grid_thresh, magma_density;
  double dt;            /* time_data::dt (hours) */
  double time_diffuse;  /* Adjust_DT's saved diffusion limit */
  double *concen;
  double *vx, *vy, *vz, *vh, *vf;
  double *kappa, *sig_nx, *sig_ny, *sig_nz, *dz_vec;
  double *kx, *ky, *kz;
  double *outflow_yz1, *outflow_yz2, *outflow_xz1, *outflow_xz2;
  double *outflow_xy1, *outflow_xy2;
  double *deposit;
  int32_t *is_aloft;
  double *mass_aloft;
  /* Terrain (src/Topography.f90): ZScaling_ID, useTopo, Ztop (km) and, when
   * use_topo, dhdx_comp, dhdy_comp, DelDxonD_cc, DelDyonD_cc (-1:nx+2,
   * -1:ny+2) and s_cc_pd (-1:nz+2). */
  int32_t zscaling_id, use_topo;
  double ztop;
  double *dhdx, *dhdy, *deldx, *deldy, *s_cc;
} orc_state;

/* Set_BC(bc_code), src/Set_BC.f90:15-126.  Returns 1 for an unknown code. */
int  orc_set_bc(orc_state *s, int code);
/* advect_x / advect_y, src/AdvectionHorz_DCU.f90:68-305 / 322-556 (with
 * the DelD*onD_cc topography terms of :163-166,251-257 when ZScaling_ID 2). */
void orc_advect_x(orc_state *s);
void orc_advect_y(orc_state *s);
/* advect_z, src/AdvectionVert_DCU.f90:100-323. */
void orc_advect_z(orc_state *s);
/* AdvectHorz(itoggle), src/AdvectionHorz.f90:47-85 (get_minmax_index when
 * fast_subgrid, else the full box).  Returns nonzero on kmax<kmin. */
int  orc_advect_horz(orc_state *s, int itoggle, int ivent, int jvent, int kvent);
/* AdvectVert, src/AdvectionVert_DCU.f90:64-82.  ZScaling_ID 2 selects
 * advect_sigma (:341-564), whose body is advect_z's line for line. */
void orc_advect_vert(orc_state *s);
/* Calc_Vmod_Topo, src/Topography.f90:2138-2166: vh over the whole ghosted
 * array from the current vx, vy (ZScaling_ID 1: -(vx*dhdx + vy*dhdy);
 * 2: (s_cc/Ztop - 1)*(vx*dhdx + vy*dhdy); 0: 0). */
void orc_calc_vmod_topo(orc_state *s);
/* diff_x/diff_y/diff_z, src/Diffusion.F90:266-650. */
void orc_diff_x(orc_state *s);
void orc_diff_y(orc_state *s);
void orc_diff_z(orc_state *s);
/* diffCN_x/diffCN_y/diffCN_z, src/Diffusion.F90:671-1428. */
void orc_diffcn_x(orc_state *s);
void orc_diffcn_y(orc_state *s);
void orc_diffcn_z(orc_state *s);
/* DiffuseHorz(i) / DiffuseVert, src/Diffusion.F90:151-247. */
void orc_diffuse_horz(orc_state *s, int itime);
void orc_diffuse_vert(orc_state *s);
/* Adjust_DT(.false.), src/Adjust_dt.f90:19-339 (per-step path).  Writes dt
 * (hours) to s->dt and *dt_out. */
void orc_adjust_dt(orc_state *s, double time, double next_write_time,
                   double simtime, double *dt_out);
/* The two halves of orc_adjust_dt (grain-sharded runs reduce the maxima
 * across ranks in between): maxima {vx, vy, vz+vf terms}; projected grids
 * return max|vx|, max|vy| undivided. */
void orc_cfl_maxima(orc_state *s, double out3[3]);
/* Adjust_DT(mesostep=.true.) maxima on an FP32 met step (FAST_DT,
 * src/Adjust_dt.f90:96-135), and the FAST_DT step dt
 * (src/MesoInterpolater.f90:250-258). */
void orc_cfl_maxima_meso(orc_state *s, const float *vx_sp, const float *vy_sp, const float *vz_sp,
                         const float *vf_sp, int per_grain, double out3[3]);
double orc_fast_dt(orc_state *s, double dt_meso_last, double dt_meso_next, double interval_frac,
                   double time, double next_write_time, double simtime);
void orc_dt_from_maxima(orc_state *s, const double v3[3], int n_gs_aloft, double time,
                        double next_write_time, double simtime, double *dt_out);
/* Calc_AshVol_{Aloft,Deposit,Outflow} + TimeStepTotals sums,
 * src/TimeStepTotals.f90:57-66, src/Output_Vars.f90:1255-1459.
 * out = {aloft_vol, dep_vol, outflow_vol, tot_vol}; fills s->mass_aloft. */
void orc_timestep_totals(orc_state *s, double out[4]);
/* get_minmax_index, src/Calc_Mesh.f90:432-542.  Returns 1 on kmax<kmin. */
int  orc_get_minmax_index(orc_state *s, int ivent, int jvent, int kvent);
/* Step prologue, src/Ash3d.F90:376-378: ts0 <- ts1, ts1 <- 0. */
void orc_step_prologue(orc_state *s);
/* Source insertion, src/Ash3d.F90:428-431: concen(ivent,jvent,1:nz+1,g,ts0)
 * += dt*flux(k,g); flux is (nz+1) x ns with k fastest. */
void orc_add_source(orc_state *s, int ivent, int jvent, const double *flux,
                    double dt);
/* MesoInterpolater wind interpolation, src/MesoInterpolater.f90:207-223:
 * v = (dble(last) + dble(next-last)*frac)*3.6 on the interior; inputs are
 * nx*ny*nz FP32 met steps (i fastest). */
void orc_interp_winds(orc_state *s, const float *vx_last, const float *vx_next,
                      const float *vy_last, const float *vy_next,
                      const float *vz_last, const float *vz_next, double frac);
/* Umbrella source: umbrella_winds' box (i0..i1 x j0..j1, i fastest) added to
 * vx, vy on levels ibase..itop (src/MesoInterpolater.f90:237-241), and the
 * 3x3 insertion of src/Ash3d.F90:446-458 (AvgCon_Umbrella smoothing on
 * ibase..itop with stencil(3,3,nz), then concen += dt*flux(3,3,nz+1,ns) on
 * levels 1..nz+1). */
void orc_add_umbrella_winds(orc_state *s, int ibase, int itop, int i0, int i1, int j0, int j1,
                            const double *uvx, const double *uvy);
void orc_add_source_umbrella(orc_state *s, int ivent, int jvent, int ibase, int itop,
                             const double *stencil, const double *flux, double dt);
/* Prune_GS, src/Tephra.f90:782-812. */
void orc_prune_gs(orc_state *s, double airborne_thresh);
/* Restatement of LAPACK dgtsv for one right-hand side (reference LAPACK's
 * published algorithm: Gaussian elimination with partial pivoting of a
 * tridiagonal matrix, then back substitution).  Returns LAPACK's INFO. */
int  orc_dgtsv(int n, double *dl, double *d, double *du, double *b);
/* Discrete adjoint (no counterpart in the reference).  Each routine applies
 * the transpose of one sweep's Jacobian, with the limiter branches fixed by
 * the forward state in concen(:,:,:,:,ts0), to lam (one level, shaped like
 * concen(:,:,:,:,ts0)) in place.  Full box only.  lam_dep: adjoint of
 * DepositGranularity (nx,ny,ns) or NULL. */
void orc_lim_coef(int lim, double dq, double dqu, double eps, double *a, double *b);
void orc_adj_advect_x(orc_state *s, double *lam);
void orc_adj_advect_y(orc_state *s, double *lam);
void orc_adj_advect_z(orc_state *s, double *lam, const double *lam_dep);
void orc_adj_diffuse_horz(orc_state *s, double *lam, int itime);
void orc_adj_diffuse_vert(orc_state *s, double *lam);
/* Output products of Gen_Output_Vars (src/Output_Vars.f90:1192-1240):
 * cloud load (masked), cloud top/bottom, maximum concentration (mg/m3), cloud
 * and deposit masks, deposit thickness (mm), the arrival-time marks (arrays
 * start at -1 and keep the first time a mask holds) and areas = {CloudArea,
 * DepositAreaCovered, CloudLoadArea(1:5)}.  2-D arrays (nx,ny), i fastest;
 * z_cc = z_cc_pd(1:nz). */
void orc_output_vars(orc_state *s, const double *z_cc, double cloudcon_thresh,
                     double cloudload_thresh, double depo_thresh, double deposit_density,
                     double time, double *cloud_load, double *max_height, double *min_height,
                     double *max_conc, int32_t *mask_cloud, double *dep_thick, int32_t *mask_dep,
                     double *cloud_arrival, double *dep_arrival, double *areas);
/* Calc_vprofile (src/Output_Vars.f90:1308-1360) on concen(:,:,:,:,ts1):
 * out (nz x npts, k fastest) is filled for the points whose column total is
 * at least thresh (written = 1), left as it is for the others. */
void orc_vprofiles(orc_state *s, int npts, const int32_t *i_pts, const int32_t *j_pts, double thresh,
                   double *out, int32_t *written);
/* OpenMP thread count for the advection rows (<=0: runtime default). */
void orc_set_threads(int n);
int  orc_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
