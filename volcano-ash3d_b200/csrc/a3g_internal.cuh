// a3g_internal.cuh -- device data layout, context and shared helpers of the
// B200 transport library.
//
// Device layout (chosen for the sweeps, not copied from the host):
//   * concentration: interior cells only, [grain][k][j][i] with the x-row
//     padded to a pitch P (a multiple of 8 doubles, 64-byte aligned rows).
//     Ghost cells are never stored: every sweep generates the ghost values
//     Set_BC would have written (zero / edge copy / periodic wrap) when it
//     loads a row, which is exact because no ghost value survives from one
//     operator to the next in the reference (each operator re-runs Set_BC or
//     its own Neumann fill first).
//   * two levels c0/c1 ping-pong; a sweep reads c0 and writes every interior
//     cell of c1 (zeros outside the active box and for grains not aloft,
//     which is the zero-then-copy-back of the reference), then they swap.
//   * winds vx/vy/vz: interior only, same pitch.
//   * geometry and diffusivity: stored with ghosts but compressed by
//     broadcast strides (a stride of 0 means "does not vary along that
//     index"), so a projected grid keeps one value per k and a lon/lat grid
//     one per (j,k).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <string>
#include <vector>

#include "../../include/ash3d_b200.h"

namespace a3g {

// Geometry/diffusivity array with broadcast strides.  Element at Fortran
// indices (i,j,k) is p[(i-o)*si + (j-o)*sj + (k-o)*sk], o = lower bound
// (-1 for the ghosted mesh arrays, 0 for kx/ky/kz).
struct Geo3 {
  const double *p;
  long si, sj, sk;
  int o;
  __host__ __device__ __forceinline__ double at(int i, int j, int k) const {
    return p[(long)(i - o) * si + (long)(j - o) * sj + (long)(k - o) * sk];
  }
};

// vf_pd with broadcast strides; grain index 0-based.
struct Geo4 {
  const double *p;
  long si, sj, sk, sg;
  __host__ __device__ __forceinline__ double at(int i, int j, int k, int g) const {
    return p[(long)(i + 1) * si + (long)(j + 1) * sj + (long)(k + 1) * sk + (long)g * sg];
  }
};

// Interior layout of the concentration / wind arrays on the device.
struct Layout {
  int nx, ny, nz, ns;
  long P, PY, PG;  // row pitch, plane stride, grain stride (elements)
  __host__ __device__ __forceinline__ long cell(int i, int j, int k) const {  // 1-based
    return (long)(k - 1) * PY + (long)(j - 1) * P + (long)(i - 1);
  }
  __host__ __device__ __forceinline__ long at(int i, int j, int k, int g) const {
    return (long)g * PG + cell(i, j, k);
  }
};

struct Box {
  int imin, imax, jmin, jmax, kmin, kmax;
};

// A TMA tensor map over one concentration level or one wind array (cached
// per device pointer and tile shape; see tensor_map()).  Tile kinds:
//   TM_COLUMN      level, 32 i x 1 j x nz k (the CN z solve's column tile)
//   TM_YCHUNK_IN   level, 32 i x (YT_CH + 2) j (a CN y chunk and its neighbours)
//   TM_YCHUNK_OUT  level, 32 i x YT_CH j (the CN y chunk it stores)
//   TM_ADV_QY/QZ   level, 32 i x ACH j / ACH k (an advection chunk)
//   TM_ADV_VY/VZ   wind array, the same chunks
//   TM_ADV_QX1/QX2 level, 32 i x 1 j x 1 k x 1 / 2 grains (an x chunk)
//   TM_ADV_VX      wind array, 32 i (an x chunk)
//   TM_XROWS       level as a 2-D array of rows (i, row = (grain, k, j)),
//                  36 i x 32 rows (a CN x tile with its neighbour cells)
enum TmapKind {
  TM_COLUMN = 0,
  TM_YCHUNK_IN = 1,
  TM_YCHUNK_OUT = 2,
  TM_ADV_QY = 3,
  TM_ADV_QZ = 4,
  TM_ADV_VY = 5,
  TM_ADV_VZ = 6,
  TM_ADV_QX1 = 7,
  TM_ADV_QX2 = 8,
  TM_ADV_VX = 9,
  TM_XROWS = 10
};
constexpr int YT_CH = 16;            // cells per CN y chunk
constexpr int YT_ROWS = YT_CH + 2;   // with the cell before and the cell after
constexpr int ACH = 8;               // cells per advection chunk
constexpr int XT2_COLS = 36;         // cells per CN x tile row as loaded (even start, 16-byte rule)
struct TmapEntry {
  const void *p;
  int kind;
  CUtensorMap map;
};

// Per-step device scalars (read by kernels so that a step can be replayed).
struct DevScalars {
  double dt;              // time_data::dt
  double vmax[4];         // CFL maxima as bit patterns (atomicMax on uint64)
  double time_diffuse;    // cached diffusion limit
  double dt_meso_last;    // FAST_DT: dt of the last met step (time_data::dt_meso_last)
  double dt_meso_next;    // FAST_DT: dt of the next met step (time_data::dt_meso_next)
  int32_t have_diffuse;   // time_diffuse valid
  int32_t err;            // device error word (A3G_ERR_*), first error wins
  int32_t err_info;       // where it happened
  int32_t flags_pad;
};

}  // namespace a3g

struct a3g_inv;  // source inversion state (a3g_inverse.cu)

struct a3g_ctx {
  a3g_grid_desc grid;
  a3g_params prm;
  int device;
  cudaStream_t stream;
  a3g::Layout L;

  double *c0, *c1;          // concentration levels (state = c0)
  double *vx, *vy, *vz;     // winds (km/h)
  float *met;               // 3 met slots of 3 FP32 arrays (vx, vy, vz): last, next, spare
  long met_n;               // nx*ny*nz
  int met_last, met_next, met_spare;  // slot indices
  bool met_prefetched;      // the spare slot holds a prefetched step
  cudaStream_t copy_stream; // met-step prefetches
  cudaEvent_t met_copy_ev;  // end of the last prefetch copy
  cudaEvent_t met_free_ev;  // the spare slot's last reader is done
  double *geo_ptrs[8];      // compressed kappa,snx,sny,snz,kx,ky,kz,vf
  a3g::Geo3 kappa, snx, sny, snz, kx, ky, kz;
  a3g::Geo3 dtv;            // dt/kappa of the current step (kappa's layout)
  double *dtv_buf;
  size_t kappa_len;
  bool dtv_valid;
  uint64_t dt_stamp, dtv_stamp;  // dt_stamp changes whenever dt may have changed
  a3g::Geo4 vf;
  // FAST_DT: max over grains of |vf_meso_next_step_sp| (m/s, FP32), one value
  // when it is the same in every cell, else per cell (nx*ny*nz, i fastest)
  float vfm_sp_const;
  float *vfm_sp;
  bool have_vf_meso;
  double *dz_vec;           // (-1:nz+2) on device
  std::vector<double> h_dz; // host copy
  // outflow accumulators, interior only: yz (ns,nz,ny), xz (ns,nz,nx), xy (ns,ny,nx)
  double *out_yz1, *out_yz2, *out_xz1, *out_xz2, *out_xy1, *out_xy2;
  int32_t *aloft;           // IsAloft on device
  std::vector<int32_t> h_aloft;
  int n_gs_aloft;
  a3g::DevScalars *sc;      // device scalars
  a3g::DevScalars *h_sc;    // pinned host mirror
  double *red_buf;          // reduction partials
  size_t red_len;
  int32_t *plane_flags;     // subgrid plane occupancy (nx+ny+nz+3)
  int32_t *h_plane_flags;   // pinned
  double *src_buf;          // device source column (nz+1)*ns
  double *h_src;            // pinned staging
  cudaEvent_t src_event;    // guards reuse of h_src
  double *h_tot;            // pinned totals staging
  // CN factor tables, one region per direction (cn_tab[d] inside cn_buf),
  // reused while dt, the box, the geometry and the diffusivity stay the same:
  // cn_state = {dt of each table (3), skip flags (3)} on the device
  double *cn_buf;
  size_t cn_len;
  double *cn_tab[3];
  bool cn_valid[3];
  a3g::Box cn_box[3];
  double *cn_state;

  a3g::Box box;
  int last_bc;
  bool have_geometry, have_diffusivity, have_vf, have_winds;
  bool ts1_zeroed;          // the last sweep left ts1 zero without copy-back
  double host_dt;
  uint64_t launches;
  size_t bytes;
  // kernel variant per advection direction (0 march, 1 block V=4, 2 block V=8)
  int tune_advect[3];
  int tune_cn_x;            // CN x solve: 0 warp-tiled, 1 one thread per line
  int tune_cn_yz;           // CN y/z solves: 0 one grain per thread, 1 two grains per thread
  bool adj_gather;          // adjoint advection: cell-per-thread gather (true) or 4-cell blocks (false)
  // discrete adjoint (a3g_adj_*)
  double *lam0, *lam1;      // lam and its scratch level
  double *lam_dep;          // adjoint of DepositGranularity (ns,ny,nx)
  double *stage1;           // recomputed state inside a step (ts1 holds the second)
  double *adj_face;         // sink for outflow updates of recomputed sweeps
  double *obs_buf;          // (nx*ny) or ((nz+1)*ns), whichever is larger
  std::vector<double *> snaps;
  // output products (a3g_output_vars): 9 (nx*ny) planes, z_cc, parameters
  double *ov_buf;
  double *ov_zcc;
  double ov_cloudcon, ov_cloudload, ov_depo, ov_density;
  std::vector<double> h_area;  // sigma_nz_pd(1:nx,1:ny,1)
  // lag-one host loop: pinned rings of the device scalars (a3g_adjust_dt_async
  // / a3g_wait_dt) and of the totals partials (a3g_timestep_totals_async /
  // a3g_totals_get), each slot guarded by an event
  a3g::DevScalars *h_sc_ring;
  cudaEvent_t sc_ev[4];
  uint64_t dt_seq;
  double *h_tot_ring;
  cudaEvent_t tot_ev[4];
  uint64_t tot_seq;
  // scheduled source (a3g_set_source_pulses): start, end, rate, NormSourceColumn,
  // bin mass on the device; ieruption/jeruption live on the device
  double *src_sched;
  int32_t *src_state;
  int src_np, src_iv, src_jv;
  // device-accumulated source gradient (a3g_adj_grad_reset): nbins x ns x nz
  double *adj_grad;
  int adj_grad_bins;
  // vertical profiles (a3g_vprofiles): points and results, grown on demand
  double *vp_buf;
  size_t vp_cap;
  // NetCDF output / restart staging for host pointers (FP32), grown on demand
  float *nc_buf;
  size_t nc_cap;
  // terrain (a3g_set_topo): dhdx, dhdy, DelDxonD, DelDyonD ((nx+4)*(ny+4) each,
  // ghosted, i fastest) and the per-level factor of vh (nz); vzh = vz + vh on
  // the interior, the vertical wind of the z sweep
  bool topo_on;
  double *topo_buf;
  double *vzh;
  // umbrella source (a3g_set_umbrella): stencil (9*nz), patch flux
  // (9*(nz+1)*ns) and winds box (2*nx*ny) on the device, pinned staging
  bool umb_on;
  int umb_ivent, umb_jvent, umb_ibase, umb_itop;
  double *umb_buf;
  double *h_umb;
  cudaEvent_t umb_event;
  // source inversion (a3g_inv_setup)
  a3g_inv *inv;
  // TMA tensor maps over the levels and winds the tiled kernels read and
  // write, and per tiled CN kernel its set-up state: 0 until its first
  // launch, then the persistent grid size (z: [0], y: [1]) or 1 once its
  // shared-memory attributes are set (x: [2])
  std::vector<a3g::TmapEntry> tmaps;
  int tma_grid[4];
  // optional per-kernel timing (a3g_kernel_timing)
  bool timing;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_kind;   // kind of each recorded (start, stop) pair
  size_t ev_used;             // events consumed from the pool
};

namespace a3g {

// error plumbing (thread-local message)
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define A3G_CUDA(call)                                 \
  do {                                                 \
    cudaError_t e__ = (call);                          \
    if (e__ != cudaSuccess) return a3g::cuda_fail(e__, #call); \
  } while (0)

#define A3G_LAUNCH_CHECK(ctx)                                        \
  do {                                                               \
    (ctx)->launches++;                                               \
    cudaError_t e__ = cudaGetLastError();                            \
    if (e__ != cudaSuccess) return a3g::cuda_fail(e__, "kernel launch"); \
  } while (0)

// launchers (kernels live in k_*.cu)
int launch_advect_x(a3g_ctx *ctx);
int launch_advect_y(a3g_ctx *ctx);
int launch_advect_z(a3g_ctx *ctx);
int launch_diff_x(a3g_ctx *ctx);
int launch_diff_y(a3g_ctx *ctx);
int launch_diff_z(a3g_ctx *ctx);
int launch_diffcn_x(a3g_ctx *ctx);
int launch_diffcn_y(a3g_ctx *ctx);
int launch_diffcn_z(a3g_ctx *ctx);
int launch_cfl(a3g_ctx *ctx, double time, double next_write_time, double simtime);
int launch_cfl_maxima(a3g_ctx *ctx);
int launch_dt_from_maxima(a3g_ctx *ctx, int n_gs_aloft, double time, double next_write_time,
                          double simtime, int meso = 0);
int launch_cfl_maxima_meso(a3g_ctx *ctx, int slot);
int launch_cfl_maxima_meso_ptr(a3g_ctx *ctx, const float *met_step);
void inv_free(a3g_ctx *ctx);
int launch_fast_dt(a3g_ctx *ctx, double frac, double time, double next_write_time, double simtime);
int launch_totals(a3g_ctx *ctx, double *out4, double *mass_aloft);
int launch_plane_flags(a3g_ctx *ctx);
int launch_interp_winds(a3g_ctx *ctx, double frac);
int launch_vmod_topo(a3g_ctx *ctx);
int launch_totals_partials(a3g_ctx *ctx, double *h_dst);
void totals_volumes(a3g_ctx *ctx, const double *h_src, double *out4, double *mass_aloft);
int launch_source_sched(a3g_ctx *ctx, double time);
int launch_vprofiles(a3g_ctx *ctx, int npts, const int32_t *pts, double *out, int32_t *written);
int launch_netcdf_pack(a3g_ctx *ctx, float *ashcon, float *depocon);
int launch_netcdf_unpack(a3g_ctx *ctx, const float *ashcon, const float *depocon);
int launch_umbrella_winds(a3g_ctx *ctx, int i0, int ni, int j0, int nj, const double *uv);
int launch_source_umbrella(a3g_ctx *ctx, double dt);
int launch_source(a3g_ctx *ctx, int ivent, int jvent, double dt);
int launch_source_devdt(a3g_ctx *ctx, int ivent, int jvent);
int launch_vent_accumulate(a3g_ctx *ctx, int ivent, int jvent, double dt, double *dst);
int launch_zero_state(a3g_ctx *ctx);
int check_device_error(a3g_ctx *ctx);
int launch_adj_advect(a3g_ctx *ctx, int dir, const double *cq, const double *lin, double *lout,
                      const double *lam_lo);
int launch_adj_diffuse(a3g_ctx *ctx, int dir, const double *lin, double *lout);
int launch_tl_advect(a3g_ctx *ctx, int dir, const double *cq, const double *din, double *dout, double *dep);
int launch_cloud_load(a3g_ctx *ctx, const double *c, double *out);
int launch_adj_cloud_load(a3g_ctx *ctx, const double *w, double *lam);
int launch_vent_column(a3g_ctx *ctx, int ivent, int jvent, const double *lam, double *out);
int launch_output_vars(a3g_ctx *ctx, double time, double *load, double *maxh, double *minh, double *maxc,
                       int32_t *mcl, double *dthick, int32_t *mdep, double *carr, double *darr);
int refresh_dtv(a3g_ctx *ctx);
// The tensor map of kind `kind` over the level at p (encoded on first use,
// then cached), copied to *out; false when the driver cannot encode it (the
// caller falls back).
bool tensor_map(a3g_ctx *ctx, const double *p, int kind, CUtensorMap *out);
// per-kernel timing brackets (no-ops unless a3g_kernel_timing(ctx,1))
void tbegin(a3g_ctx *ctx, int kind);
void tend(a3g_ctx *ctx);

inline void swap_levels(a3g_ctx *ctx) {
  double *t = ctx->c0;
  ctx->c0 = ctx->c1;
  ctx->c1 = t;
}

// Fortran MAX/MIN for reals (no NaNs reach these in the transport path).
__device__ __forceinline__ double fmx(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double fmn(double a, double b) { return a < b ? a : b; }

__device__ __forceinline__ void raise_error(DevScalars *sc, int code, int info) {
  if (atomicCAS(&sc->err, 0, code) == 0) sc->err_info = info;
}

}  // namespace a3g
