// a3g_api.cu -- the C-ABI (include/ash3d_b200.h): context lifetime, data
// movement between the Fortran-layout host arrays and the device layout,
// and the per-step entry points that mirror the reference subroutines.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "a3g_internal.cuh"

namespace a3g {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
int cuda_fail(cudaError_t e, const char *what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return A3G_ERR_CUDA;
}
size_t cn_table_doubles(const a3g_ctx *ctx, int dir);

static int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

static bool same_bits(double a, double b) { return std::memcmp(&a, &b, sizeof(double)) == 0; }

// Compresses a column-major array with extents n0 x n1 x n2 (x ng blocks) to
// the indices it actually varies along.  Returns the strides of the
// compressed copy (0 where the array is constant along that index).
static void compress(const double *src, long n0, long n1, long n2, long ng, std::vector<double> &out,
                     long &si, long &sj, long &sk, long &sg) {
  bool vi = false, vj = false, vk = false;
  for (long g = 0; g < ng; g++)
    for (long c = 0; c < n2; c++)
      for (long b = 0; b < n1; b++) {
        const double *row = src + n0 * (b + n1 * (c + n2 * g));
        const double *row0 = src + n0 * (0 + n1 * (c + n2 * g));
        const double *row00 = src + n0 * (b + n1 * (0 + n2 * g));
        for (long a = 0; a < n0; a++) {
          if (!vi && !same_bits(row[a], row[0])) vi = true;
          if (!vj && !same_bits(row[a], row0[a])) vj = true;
          if (!vk && !same_bits(row[a], row00[a])) vk = true;
        }
      }
  const long m0 = vi ? n0 : 1, m1 = vj ? n1 : 1, m2 = vk ? n2 : 1;
  out.assign((size_t)(m0 * m1 * m2 * ng), 0.0);
  for (long g = 0; g < ng; g++)
    for (long c = 0; c < m2; c++)
      for (long b = 0; b < m1; b++)
        for (long a = 0; a < m0; a++)
          out[(size_t)(a + m0 * (b + m1 * (c + m2 * g)))] = src[a + n0 * (b + n1 * (c + n2 * g))];
  si = vi ? 1 : 0;
  sj = vj ? m0 : 0;
  sk = vk ? m0 * m1 : 0;
  sg = m0 * m1 * m2;
}

static int upload_vec(a3g_ctx *ctx, const std::vector<double> &v, double **dptr) {
  if (*dptr) { cudaFree(*dptr); ctx->bytes -= 0; *dptr = nullptr; }
  A3G_CUDA(cudaMalloc(dptr, v.size() * sizeof(double)));
  ctx->bytes += v.size() * sizeof(double);
  A3G_CUDA(cudaMemcpy(*dptr, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
  return A3G_OK;
}

// host ghosted level <-> device interior level (one 3-D copy per grain)
static int copy_level(a3g_ctx *ctx, double *host, double *dev, bool to_device, long nxg, long nyg,
                      long nzg, long ghost, int nx, int ny, int nz, int ng, long dpitch, long dslab,
                      long dgrain) {
  for (int g = 0; g < ng; g++) {
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    cudaPitchedPtr hp = make_cudaPitchedPtr(host + (size_t)g * nxg * nyg * nzg, nxg * sizeof(double),
                                            nxg * sizeof(double), nyg);
    cudaPitchedPtr dp = make_cudaPitchedPtr(dev + (size_t)g * dgrain, dpitch * sizeof(double),
                                            nx * sizeof(double), dslab / dpitch);
    cudaPos hpos = make_cudaPos(ghost * sizeof(double), ghost, ghost);
    cudaPos dpos = make_cudaPos(0, 0, 0);
    if (to_device) { p.srcPtr = hp; p.srcPos = hpos; p.dstPtr = dp; p.dstPos = dpos; p.kind = cudaMemcpyHostToDevice; }
    else { p.srcPtr = dp; p.srcPos = dpos; p.dstPtr = hp; p.dstPos = hpos; p.kind = cudaMemcpyDeviceToHost; }
    p.extent = make_cudaExtent(nx * sizeof(double), ny, nz);
    A3G_CUDA(cudaMemcpy3DAsync(&p, ctx->stream));
  }
  return A3G_OK;
}

int check_device_error(a3g_ctx *ctx) {
  if (ctx->h_sc->err != 0) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "device error %d (info %d)", ctx->h_sc->err, ctx->h_sc->err_info);
    set_error(buf);
    return ctx->h_sc->err;
  }
  return A3G_OK;
}

static int sync_scalars(a3g_ctx *ctx) {
  A3G_CUDA(cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);
}

void tbegin(a3g_ctx *ctx, int kind) {
  if (!ctx->timing) return;
  while (ctx->ev_pool.size() < ctx->ev_used + 2) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) { ctx->timing = false; return; }
    ctx->ev_pool.push_back(e);
  }
  cudaEventRecord(ctx->ev_pool[ctx->ev_used], ctx->stream);
  ctx->ev_kind.push_back(kind);
}

void tend(a3g_ctx *ctx) {
  if (!ctx->timing || ctx->ev_kind.size() * 2 != ctx->ev_used + 2) return;
  cudaEventRecord(ctx->ev_pool[ctx->ev_used + 1], ctx->stream);
  ctx->ev_used += 2;
}

static void full_box(a3g_ctx *ctx) {
  ctx->box = Box{1, ctx->grid.nx, 1, ctx->grid.ny, 1, ctx->grid.nz};
}

}  // namespace a3g

using namespace a3g;

#define CTX_CHECK(ctx)                                                   \
  do {                                                                   \
    if (!(ctx)) return fail(A3G_ERR_ARG, "null context");                \
    cudaError_t e__ = cudaSetDevice((ctx)->device);                      \
    if (e__ != cudaSuccess) return cuda_fail(e__, "cudaSetDevice");      \
  } while (0)

extern "C" {

void a3g_default_params(a3g_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->limiter = A3G_LIM_SUPERBEE;
  p->use_cn = 1;
  p->use_diffusion = 1;
  p->fast_subgrid = 0;
  p->nocycle = 0;
  p->zscaling_id = 0;
  p->cfl = 0.8;
  p->dt_min = 1.0e-5;
  p->dt_max = 1.0;
  p->imp_fac = 0.5;
  p->imp_dt_fac = 4.0;
  p->eps_thresh = 1.0e-10;
  p->eps_small = 1.0e-6;
  p->cloudcon_grid_thresh = 1.0e-7;
  p->magma_density = 2500.0;
}

int a3g_abi_version(void) { return A3G_ABI_VERSION; }
const char *a3g_last_error(void) { return g_err.c_str(); }

int a3g_create(const a3g_grid_desc *grid, const a3g_params *params, int device, a3g_ctx **out) {
  if (!grid || !params || !out) return fail(A3G_ERR_ARG, "null argument");
  *out = nullptr;
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->ns < 1)
    return fail(A3G_ERR_ARG, "grid extents must be >= 1");
  if (grid->periodic && grid->nx < 2) return fail(A3G_ERR_ARG, "periodic grid needs nx >= 2");
  if (params->zscaling_id < 0 || params->zscaling_id > 2)
    return fail(A3G_ERR_ARG, "ZScaling_ID must be 0, 1 or 2");
  if (params->limiter < A3G_LIM_NONE || params->limiter > A3G_LIM_MC)
    return fail(A3G_ERR_ARG, "unknown limiter");
  if (!(params->dt_min > 0.0) || !(params->dt_max >= params->dt_min))
    return fail(A3G_ERR_ARG, "need 0 < DT_MIN <= DT_MAX");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
    return fail(A3G_ERR_CUDA, "no CUDA device (the library has no CPU path)");
  if (device < 0 || device >= ndev) return fail(A3G_ERR_ARG, "bad device ordinal");
  A3G_CUDA(cudaSetDevice(device));
  a3g_ctx *ctx = new (std::nothrow) a3g_ctx();
  if (!ctx) return fail(A3G_ERR_NOMEM, "host allocation failed");
  ctx->grid = *grid;
  ctx->prm = *params;
  ctx->device = device;
  Layout &L = ctx->L;
  L.nx = grid->nx; L.ny = grid->ny; L.nz = grid->nz; L.ns = grid->ns;
  L.P = ((long)grid->nx + 7) / 8 * 8;  // the x sweep stores 8 cells per thread
  L.PY = L.P * grid->ny;
  L.PG = L.PY * grid->nz;
  full_box(ctx);
  ctx->h_aloft.assign(grid->ns, 1);
  ctx->n_gs_aloft = grid->ns;
  ctx->last_bc = 0;
  // fastest measured advection variants on B200 (x: warp-row chunks with
  // the interior chunks fed by TMA, C2 1.27 ms against 1.38 without and 2.16
  // for marching rows; y, z: the column march fed by TMA chunks, C2 y 1.43 ->
  // 1.24 ms and z 1.64 -> 1.28 ms against 4-cell blocks, which remain where
  // the march's conditions do not hold); a3g_set_variant overrides them
  ctx->tune_advect[0] = 5;
  ctx->tune_advect[1] = 6;
  ctx->tune_advect[2] = 6;
  // CN x solve: warp tiles loaded one chunk ahead by TMA (C2 1.35 -> 1.16 ms
  // against the synchronous tile loads of variant 0)
  ctx->tune_cn_x = 2;
  ctx->ov_cloudcon = 1.0e-3;   // CLOUDCON_THRESH, src/Output_Vars.f90:119
  ctx->ov_cloudload = 2.0e-1;  // CLOUDLOAD_THRESH, :114
  ctx->ov_depo = 1.0e-2;       // DEPO_THRESH, :113
  ctx->ov_density = 1000.0;    // DepositDensity, src/Tephra.f90:55
  // CN y and z solves through TMA tiles (C2 on B200: y 1.55 -> 1.25 ms, z
  // 1.23 -> 0.66 ms against two grains per thread)
  ctx->tune_cn_yz = 3;
  auto dmalloc = [&](void **p, size_t n) -> cudaError_t {
    cudaError_t e = cudaMalloc(p, n);
    if (e == cudaSuccess) { ctx->bytes += n; cudaMemsetAsync(*p, 0, n, ctx->stream); }
    return e;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  const size_t lev = (size_t)L.PG * L.ns * sizeof(double);
  const size_t w3 = (size_t)L.PG * sizeof(double);
  const int ns = L.ns;
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->c0, lev);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->c1, lev);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->vx, w3);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->vy, w3);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->vz, w3);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->out_yz1, sizeof(double) * ns * L.ny * L.nz);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->out_yz2, sizeof(double) * ns * L.ny * L.nz);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->out_xz1, sizeof(double) * ns * L.nx * L.nz);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->out_xz2, sizeof(double) * ns * L.nx * L.nz);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->out_xy1, sizeof(double) * ns * L.nx * L.ny);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->out_xy2, sizeof(double) * ns * L.nx * L.ny);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->aloft, sizeof(int32_t) * ns);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->sc, sizeof(DevScalars));
  ctx->red_len = (size_t)2 * 296 * 7 * ns + 7 * ns;
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->red_buf, sizeof(double) * ctx->red_len);
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->plane_flags, sizeof(int32_t) * (L.nx + L.ny + L.nz + 3));
  if (e == cudaSuccess) e = dmalloc((void **)&ctx->src_buf, sizeof(double) * (L.nz + 1) * ns);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_sc, sizeof(DevScalars));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_plane_flags, sizeof(int32_t) * (L.nx + L.ny + L.nz + 3));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_src, sizeof(double) * (L.nz + 1) * ns);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_tot, sizeof(double) * 7 * ns);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->src_event, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->met_copy_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->met_free_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_sc_ring, 4 * sizeof(DevScalars));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_tot_ring, sizeof(double) * 4 * 7 * ns);
  for (int q = 0; q < 4 && e == cudaSuccess; q++) {
    e = cudaEventCreateWithFlags(&ctx->sc_ev[q], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->tot_ev[q], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) {
    std::memset(ctx->h_sc, 0, sizeof(DevScalars));
    std::vector<int32_t> ones(ns, 1);
    e = cudaMemcpyAsync(ctx->aloft, ones.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    int rc = (e == cudaErrorMemoryAllocation) ? fail(A3G_ERR_NOMEM, "device allocation failed")
                                              : cuda_fail(e, "a3g_create");
    a3g_destroy(ctx);
    return rc;
  }
  ctx->ts1_zeroed = false;
  *out = ctx;
  return A3G_OK;
}

int a3g_destroy(a3g_ctx *ctx) {
  if (!ctx) return A3G_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  inv_free(ctx);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  double *dptrs[] = {ctx->c0, ctx->c1, ctx->vx, ctx->vy, ctx->vz, ctx->out_yz1, ctx->out_yz2,
                     ctx->out_xz1, ctx->out_xz2, ctx->out_xy1, ctx->out_xy2, ctx->red_buf,
                     ctx->src_buf, ctx->cn_buf, ctx->dz_vec, ctx->dtv_buf};
  for (double *p : dptrs) if (p) cudaFree(p);
  for (double *p : ctx->geo_ptrs) if (p) cudaFree(p);
  if (ctx->met) cudaFree(ctx->met);
  if (ctx->aloft) cudaFree(ctx->aloft);
  if (ctx->sc) cudaFree(ctx->sc);
  if (ctx->plane_flags) cudaFree(ctx->plane_flags);
  if (ctx->h_sc) cudaFreeHost(ctx->h_sc);
  if (ctx->h_plane_flags) cudaFreeHost(ctx->h_plane_flags);
  if (ctx->h_src) cudaFreeHost(ctx->h_src);
  if (ctx->h_tot) cudaFreeHost(ctx->h_tot);
  if (ctx->src_event) cudaEventDestroy(ctx->src_event);
  if (ctx->umb_event) cudaEventDestroy(ctx->umb_event);
  for (int q = 0; q < 4; q++) {
    if (ctx->sc_ev[q]) cudaEventDestroy(ctx->sc_ev[q]);
    if (ctx->tot_ev[q]) cudaEventDestroy(ctx->tot_ev[q]);
  }
  if (ctx->h_sc_ring) cudaFreeHost(ctx->h_sc_ring);
  if (ctx->h_tot_ring) cudaFreeHost(ctx->h_tot_ring);
  if (ctx->src_sched) cudaFree(ctx->src_sched);
  if (ctx->src_state) cudaFree(ctx->src_state);
  if (ctx->h_umb) cudaFreeHost(ctx->h_umb);
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  double *aptrs[] = {ctx->lam0, ctx->lam1, ctx->lam_dep, ctx->stage1, ctx->adj_face,
                     ctx->obs_buf, ctx->ov_buf, ctx->ov_zcc, ctx->topo_buf, ctx->vzh, ctx->umb_buf,
                     ctx->vp_buf, ctx->adj_grad, ctx->cn_state};
  for (double *p : aptrs) if (p) cudaFree(p);
  if (ctx->nc_buf) cudaFree(ctx->nc_buf);
  if (ctx->vfm_sp) cudaFree(ctx->vfm_sp);
  for (double *p : ctx->snaps) if (p) cudaFree(p);
  if (ctx->met_copy_ev) cudaEventDestroy(ctx->met_copy_ev);
  if (ctx->met_free_ev) cudaEventDestroy(ctx->met_free_ev);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return A3G_OK;
}

int a3g_sync(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  return sync_scalars(ctx);
}

int a3g_device_bytes(a3g_ctx *ctx, size_t *bytes) {
  if (!ctx || !bytes) return fail(A3G_ERR_ARG, "null argument");
  *bytes = ctx->bytes;
  return A3G_OK;
}

static int set_geo3(a3g_ctx *ctx, const double *src, long n0, long n1, long n2, int lower, Geo3 *g,
                    int slot) {
  std::vector<double> v;
  long si, sj, sk, sg;
  compress(src, n0, n1, n2, 1, v, si, sj, sk, sg);
  double *d = ctx->geo_ptrs[slot];
  ctx->geo_ptrs[slot] = nullptr;
  if (d) cudaFree(d);
  int rc = upload_vec(ctx, v, &ctx->geo_ptrs[slot]);
  if (rc) return rc;
  g->p = ctx->geo_ptrs[slot];
  g->si = si; g->sj = sj; g->sk = sk; g->o = lower;
  return A3G_OK;
}

static int ensure_cn_buf(a3g_ctx *ctx) {
  for (int d = 0; d < 3; d++) ctx->cn_valid[d] = false;  // geometry or diffusivity changed
  if (!ctx->have_geometry || !ctx->have_diffusivity) return A3G_OK;
  size_t len[3], need = 0;
  for (int d = 0; d < 3; d++) {
    len[d] = (cn_table_doubles(ctx, d) + 31) / 32 * 32;  // 256-byte aligned regions
    need += len[d];
  }
  if (!ctx->cn_state) {
    if (cudaMalloc((void **)&ctx->cn_state, 6 * sizeof(double)) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "CN table state allocation failed");
    A3G_CUDA(cudaMemsetAsync(ctx->cn_state, 0, 6 * sizeof(double), ctx->stream));
  }
  if (need > ctx->cn_len) {
    if (ctx->cn_buf) { cudaFree(ctx->cn_buf); ctx->bytes -= ctx->cn_len * sizeof(double); ctx->cn_buf = nullptr; }
    cudaError_t e = cudaMalloc((void **)&ctx->cn_buf, need * sizeof(double));
    if (e != cudaSuccess) { ctx->cn_len = 0; return fail(A3G_ERR_NOMEM, "CN table allocation failed"); }
    ctx->cn_len = need;
    ctx->bytes += need * sizeof(double);
  }
  size_t off = 0;
  for (int d = 0; d < 3; d++) {
    ctx->cn_tab[d] = ctx->cn_buf + off;
    off += len[d];
  }
  return A3G_OK;
}

int a3g_set_geometry(a3g_ctx *ctx, const double *kappa_pd, const double *sigma_nx_pd,
                     const double *sigma_ny_pd, const double *sigma_nz_pd, const double *dz_vec_pd) {
  CTX_CHECK(ctx);
  if (!kappa_pd || !sigma_nx_pd || !sigma_ny_pd || !sigma_nz_pd || !dz_vec_pd)
    return fail(A3G_ERR_ARG, "null geometry array");
  const long n0 = ctx->grid.nx + 4, n1 = ctx->grid.ny + 4, n2 = ctx->grid.nz + 4;
  int rc;
  if ((rc = set_geo3(ctx, kappa_pd, n0, n1, n2, -1, &ctx->kappa, 0))) return rc;
  {  // dt/kappa buffer with kappa's compressed layout
    const long m0 = ctx->kappa.si ? n0 : 1;
    const long m1 = ctx->kappa.sj ? n1 : 1;
    const long m2 = ctx->kappa.sk ? n2 : 1;
    ctx->kappa_len = (size_t)(m0 * m1 * m2);
    if (ctx->dtv_buf) { cudaFree(ctx->dtv_buf); ctx->dtv_buf = nullptr; }
    A3G_CUDA(cudaMalloc((void **)&ctx->dtv_buf, ctx->kappa_len * sizeof(double)));
    ctx->bytes += ctx->kappa_len * sizeof(double);
    ctx->dtv = ctx->kappa;
    ctx->dtv.p = ctx->dtv_buf;
    ctx->dtv_valid = false;
  }
  if ((rc = set_geo3(ctx, sigma_nx_pd, n0, n1, n2, -1, &ctx->snx, 1))) return rc;
  if ((rc = set_geo3(ctx, sigma_ny_pd, n0, n1, n2, -1, &ctx->sny, 2))) return rc;
  if ((rc = set_geo3(ctx, sigma_nz_pd, n0, n1, n2, -1, &ctx->snz, 3))) return rc;
  ctx->h_dz.assign(dz_vec_pd, dz_vec_pd + n2);
  // sigma_nz_pd(1:nx,1:ny,1): the cell areas the output products sum
  ctx->h_area.resize((size_t)ctx->grid.nx * ctx->grid.ny);
  for (int j = 1; j <= ctx->grid.ny; j++)
    for (int i = 1; i <= ctx->grid.nx; i++)
      ctx->h_area[(size_t)(i - 1) + (size_t)ctx->grid.nx * (j - 1)] =
          sigma_nz_pd[(size_t)(i + 1) + (size_t)n0 * ((size_t)(j + 1) + (size_t)n1 * 2)];
  if (ctx->dz_vec) { cudaFree(ctx->dz_vec); ctx->dz_vec = nullptr; }
  if ((rc = upload_vec(ctx, ctx->h_dz, &ctx->dz_vec))) return rc;
  ctx->have_geometry = true;
  return ensure_cn_buf(ctx);
}

int a3g_set_diffusivity(a3g_ctx *ctx, const double *kx, const double *ky, const double *kz) {
  CTX_CHECK(ctx);
  if (!kx || !ky || !kz) return fail(A3G_ERR_ARG, "null diffusivity array");
  const long n0 = ctx->grid.nx + 2, n1 = ctx->grid.ny + 2, n2 = ctx->grid.nz + 2;
  int rc;
  if ((rc = set_geo3(ctx, kx, n0, n1, n2, 0, &ctx->kx, 4))) return rc;
  if ((rc = set_geo3(ctx, ky, n0, n1, n2, 0, &ctx->ky, 5))) return rc;
  if ((rc = set_geo3(ctx, kz, n0, n1, n2, 0, &ctx->kz, 6))) return rc;
  ctx->have_diffusivity = true;
  ctx->h_sc->have_diffuse = 0;  // Adjust_DT recomputes its diffusion limit
  A3G_CUDA(cudaMemsetAsync(&ctx->sc->have_diffuse, 0, sizeof(int32_t), ctx->stream));
  return ensure_cn_buf(ctx);
}

int a3g_set_fall_velocity(a3g_ctx *ctx, const double *vf_pd) {
  CTX_CHECK(ctx);
  if (!vf_pd) return fail(A3G_ERR_ARG, "null vf_pd");
  const long n0 = ctx->grid.nx + 4, n1 = ctx->grid.ny + 4, n2 = ctx->grid.nz + 4;
  std::vector<double> v;
  long si, sj, sk, sg;
  compress(vf_pd, n0, n1, n2, ctx->grid.ns, v, si, sj, sk, sg);
  double *d = ctx->geo_ptrs[7];
  ctx->geo_ptrs[7] = nullptr;
  if (d) cudaFree(d);
  int rc = upload_vec(ctx, v, &ctx->geo_ptrs[7]);
  if (rc) return rc;
  ctx->vf = Geo4{ctx->geo_ptrs[7], si, sj, sk, sg};
  ctx->have_vf = true;
  return A3G_OK;
}

int a3g_set_aloft(a3g_ctx *ctx, const int32_t *is_aloft) {
  CTX_CHECK(ctx);
  if (!is_aloft) return fail(A3G_ERR_ARG, "null IsAloft");
  int n = 0;
  for (int g = 0; g < ctx->grid.ns; g++) {
    ctx->h_aloft[g] = is_aloft[g] ? 1 : 0;
    n += ctx->h_aloft[g];
  }
  ctx->n_gs_aloft = n;
  A3G_CUDA(cudaMemcpyAsync(ctx->aloft, ctx->h_aloft.data(), sizeof(int32_t) * ctx->grid.ns,
                           cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

int a3g_set_winds(a3g_ctx *ctx, const double *vx_pd, const double *vy_pd, const double *vz_pd) {
  CTX_CHECK(ctx);
  if (!vx_pd || !vy_pd || !vz_pd) return fail(A3G_ERR_ARG, "null wind array");
  const Layout &L = ctx->L;
  const double *src[3] = {vx_pd, vy_pd, vz_pd};
  double *dst[3] = {ctx->vx, ctx->vy, ctx->vz};
  for (int c = 0; c < 3; c++) {
    int rc = copy_level(ctx, const_cast<double *>(src[c]), dst[c], true, L.nx + 4, L.ny + 4, L.nz + 4, 2,
                        L.nx, L.ny, L.nz, 1, L.P, L.PY, L.PG);
    if (rc) return rc;
  }
  if (ctx->topo_on) {
    int rc = launch_vmod_topo(ctx);
    if (rc) return rc;
  }
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_winds = true;
  return A3G_OK;
}

static int ensure_met(a3g_ctx *ctx) {
  if (ctx->met) return A3G_OK;
  const long n = (long)ctx->grid.nx * ctx->grid.ny * ctx->grid.nz;
  if (cudaMalloc((void **)&ctx->met, sizeof(float) * 9 * n) != cudaSuccess)
    return fail(A3G_ERR_NOMEM, "met-step allocation failed");
  ctx->bytes += sizeof(float) * 9 * n;
  ctx->met_n = n;
  ctx->met_last = 0;
  ctx->met_next = 1;
  ctx->met_spare = 2;
  ctx->met_prefetched = false;
  return A3G_OK;
}

int a3g_set_met_steps(a3g_ctx *ctx, const float *vx_last, const float *vy_last, const float *vz_last,
                      const float *vx_next, const float *vy_next, const float *vz_next) {
  CTX_CHECK(ctx);
  const float *src[6] = {vx_last, vy_last, vz_last, vx_next, vy_next, vz_next};
  for (int c = 0; c < 6; c++)
    if (!src[c]) return fail(A3G_ERR_ARG, "null met-step array");
  int rc = ensure_met(ctx);
  if (rc) return rc;
  const long n = ctx->met_n;
  for (int c = 0; c < 6; c++) {
    float *dst = ctx->met + (size_t)3 * n * (c < 3 ? ctx->met_last : ctx->met_next) + (size_t)(c % 3) * n;
    A3G_CUDA(cudaMemcpyAsync(dst, src[c], sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  return A3G_OK;
}

// Read_NextMesoStep's toggle (src/MesoInterpolater.f90:168-199): the next met
// step is copied into the spare slot on the copy stream, ahead of need;
// a3g_advance_met_step makes it the next step and the old next the last one.
int a3g_prefetch_met_step(a3g_ctx *ctx, const float *vx, const float *vy, const float *vz) {
  CTX_CHECK(ctx);
  if (!vx || !vy || !vz) return fail(A3G_ERR_ARG, "null met-step array");
  int rc = ensure_met(ctx);
  if (rc) return rc;
  const long n = ctx->met_n;
  // the spare slot was last read by work queued before the latest advance
  A3G_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->met_free_ev, 0));
  const float *src[3] = {vx, vy, vz};
  for (int c = 0; c < 3; c++)
    A3G_CUDA(cudaMemcpyAsync(ctx->met + (size_t)3 * n * ctx->met_spare + (size_t)c * n, src[c],
                             sizeof(float) * n, cudaMemcpyHostToDevice, ctx->copy_stream));
  A3G_CUDA(cudaEventRecord(ctx->met_copy_ev, ctx->copy_stream));
  ctx->met_prefetched = true;
  return A3G_OK;
}

int a3g_advance_met_step(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  if (!ctx->met || !ctx->met_prefetched) return fail(A3G_ERR_STATE, "no met step prefetched");
  A3G_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->met_copy_ev, 0));
  A3G_CUDA(cudaEventRecord(ctx->met_free_ev, ctx->stream));  // the old last slot's readers end here
  const int old_last = ctx->met_last;
  ctx->met_last = ctx->met_next;
  ctx->met_next = ctx->met_spare;
  ctx->met_spare = old_last;
  ctx->met_prefetched = false;
  return A3G_OK;
}

int a3g_met_prefetch_fence(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  A3G_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->met_copy_ev, 0));
  return A3G_OK;
}

int a3g_interp_winds(a3g_ctx *ctx, double interval_frac) {
  CTX_CHECK(ctx);
  if (!ctx->met) return fail(A3G_ERR_STATE, "a3g_set_met_steps has not been called");
  int rc = launch_interp_winds(ctx, interval_frac);
  if (!rc && ctx->topo_on) rc = launch_vmod_topo(ctx);  // Calc_Vmod_Topo, src/Ash3d.F90:398
  if (!rc) ctx->have_winds = true;
  return rc;
}

int a3g_set_topo(a3g_ctx *ctx, const double *dhdx_comp, const double *dhdy_comp, const double *deldx_on_d,
                 const double *deldy_on_d, const double *s_cc_pd, double ztop) {
  CTX_CHECK(ctx);
  const int z = ctx->prm.zscaling_id;
  const long nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  const long n2 = (nx + 4) * (ny + 4);
  if (!dhdx_comp || !dhdy_comp) return fail(A3G_ERR_ARG, "null topography gradient");
  if (z == 2 && (!deldx_on_d || !deldy_on_d || !s_cc_pd)) return fail(A3G_ERR_ARG, "ZScaling_ID 2 needs DelD*onD_cc and s_cc_pd");
  if (z == 2 && !(ztop > 0.0)) return fail(A3G_ERR_ARG, "Ztop must be positive");
  // per-level factor of vh (src/Topography.f90:2151-2163), in the
  // reference's operations: -1.0 for ZScaling_ID 1, s_cc/Ztop - 1.0 for 2
  std::vector<double> h(4 * n2 + nz, 0.0);
  std::memcpy(h.data(), dhdx_comp, sizeof(double) * n2);
  std::memcpy(h.data() + n2, dhdy_comp, sizeof(double) * n2);
  if (deldx_on_d) std::memcpy(h.data() + 2 * n2, deldx_on_d, sizeof(double) * n2);
  if (deldy_on_d) std::memcpy(h.data() + 3 * n2, deldy_on_d, sizeof(double) * n2);
  for (long k = 1; k <= nz; k++)
    h[4 * n2 + k - 1] = (z == 1) ? -1.0 : (z == 2) ? (s_cc_pd[k + 1] / ztop - 1.0) : 0.0;
  if (!ctx->topo_buf) {
    if (cudaMalloc((void **)&ctx->topo_buf, sizeof(double) * h.size()) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "topography allocation failed");
    ctx->bytes += sizeof(double) * h.size();
  }
  if (!ctx->vzh) {
    const size_t w3 = (size_t)ctx->L.PG * sizeof(double);
    if (cudaMalloc((void **)&ctx->vzh, w3) != cudaSuccess) return fail(A3G_ERR_NOMEM, "vz+vh allocation failed");
    ctx->bytes += w3;
    A3G_CUDA(cudaMemsetAsync(ctx->vzh, 0, w3, ctx->stream));
  }
  A3G_CUDA(cudaMemcpyAsync(ctx->topo_buf, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
  ctx->topo_on = true;
  if (ctx->have_winds) {
    int rc = launch_vmod_topo(ctx);
    if (rc) return rc;
  }
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

int a3g_upload_concen(a3g_ctx *ctx, const double *concen_level) {
  CTX_CHECK(ctx);
  if (!concen_level) return fail(A3G_ERR_ARG, "null concen");
  const Layout &L = ctx->L;
  int rc = copy_level(ctx, const_cast<double *>(concen_level), ctx->c0, true, L.nx + 4, L.ny + 4,
                      L.nz + 4, 2, L.nx, L.ny, L.nz, L.ns, L.P, L.PY, L.PG);
  if (rc) return rc;
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->ts1_zeroed = false;
  return A3G_OK;
}

int a3g_download_concen(a3g_ctx *ctx, double *concen_level) {
  CTX_CHECK(ctx);
  if (!concen_level) return fail(A3G_ERR_ARG, "null concen");
  const Layout &L = ctx->L;
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memset(concen_level, 0, sizeof(double) * (size_t)(L.nx + 4) * (L.ny + 4) * (L.nz + 4) * L.ns);
  int rc = copy_level(ctx, concen_level, ctx->c0, false, L.nx + 4, L.ny + 4, L.nz + 4, 2, L.nx, L.ny,
                      L.nz, L.ns, L.P, L.PY, L.PG);
  if (rc) return rc;
  return sync_scalars(ctx);
}

// outflow arrays: host (-1:a+2,-1:b+2,1:ns) <-> device [g][b][a] interior
static int copy_outflow(a3g_ctx *ctx, double *host, double *dev, int na, int nb, bool to_device) {
  if (!host) return A3G_OK;
  cudaMemcpy3DParms p;
  std::memset(&p, 0, sizeof(p));
  cudaPitchedPtr hp = make_cudaPitchedPtr(host, (na + 4) * sizeof(double), (na + 4) * sizeof(double), nb + 4);
  cudaPitchedPtr dp = make_cudaPitchedPtr(dev, na * sizeof(double), na * sizeof(double), nb);
  cudaPos hpos = make_cudaPos(2 * sizeof(double), 2, 0);
  if (to_device) { p.srcPtr = hp; p.srcPos = hpos; p.dstPtr = dp; p.kind = cudaMemcpyHostToDevice; }
  else { p.srcPtr = dp; p.dstPtr = hp; p.dstPos = hpos; p.kind = cudaMemcpyDeviceToHost; }
  p.extent = make_cudaExtent(na * sizeof(double), nb, ctx->grid.ns);
  A3G_CUDA(cudaMemcpy3DAsync(&p, ctx->stream));
  return A3G_OK;
}

int a3g_upload_outflow(a3g_ctx *ctx, const double *yz1, const double *yz2, const double *xz1,
                       const double *xz2, const double *xy1, const double *xy2) {
  CTX_CHECK(ctx);
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  int rc = 0;
  if (!rc) rc = copy_outflow(ctx, const_cast<double *>(yz1), ctx->out_yz1, ny, nz, true);
  if (!rc) rc = copy_outflow(ctx, const_cast<double *>(yz2), ctx->out_yz2, ny, nz, true);
  if (!rc) rc = copy_outflow(ctx, const_cast<double *>(xz1), ctx->out_xz1, nx, nz, true);
  if (!rc) rc = copy_outflow(ctx, const_cast<double *>(xz2), ctx->out_xz2, nx, nz, true);
  if (!rc) rc = copy_outflow(ctx, const_cast<double *>(xy1), ctx->out_xy1, nx, ny, true);
  if (!rc) rc = copy_outflow(ctx, const_cast<double *>(xy2), ctx->out_xy2, nx, ny, true);
  if (rc) return rc;
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

int a3g_download_outflow(a3g_ctx *ctx, double *yz1, double *yz2, double *xz1, double *xz2,
                         double *xy1, double *xy2, double *deposit) {
  CTX_CHECK(ctx);
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  int rc = 0;
  if (!rc) rc = copy_outflow(ctx, yz1, ctx->out_yz1, ny, nz, false);
  if (!rc) rc = copy_outflow(ctx, yz2, ctx->out_yz2, ny, nz, false);
  if (!rc) rc = copy_outflow(ctx, xz1, ctx->out_xz1, nx, nz, false);
  if (!rc) rc = copy_outflow(ctx, xz2, ctx->out_xz2, nx, nz, false);
  if (!rc) rc = copy_outflow(ctx, xy1, ctx->out_xy1, nx, ny, false);
  if (!rc) rc = copy_outflow(ctx, xy2, ctx->out_xy2, nx, ny, false);
  if (rc) return rc;
  if (deposit)  // DepositGranularity = outflow_xy1(1:nx,1:ny,:), src/AdvectionVert_DCU.f90:321
    A3G_CUDA(cudaMemcpyAsync(deposit, ctx->out_xy1, sizeof(double) * nx * ny * ctx->grid.ns,
                             cudaMemcpyDeviceToHost, ctx->stream));
  return sync_scalars(ctx);
}

// ---- NetCDF output arrays and restart ---------------------------------------
// A caller's pointer that the kernels can address: device memory of this
// context's device, or managed memory.  Anything else goes through staging.
static bool device_addressable(a3g_ctx *ctx, const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice && a.device == ctx->device) || a.type == cudaMemoryTypeManaged;
}

static int ensure_nc_buf(a3g_ctx *ctx, size_t n) {
  if (n <= ctx->nc_cap) return A3G_OK;
  if (ctx->nc_buf) cudaFree(ctx->nc_buf);
  ctx->nc_buf = nullptr;
  ctx->nc_cap = 0;
  if (cudaMalloc((void **)&ctx->nc_buf, n * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return fail(A3G_ERR_NOMEM, "NetCDF staging buffer allocation failed");
  }
  ctx->nc_cap = n;
  return A3G_OK;
}

// Device addresses of ashcon and depocon for the kernels: the caller's own
// when addressable, else slices of the staging buffer.
static int nc_targets(a3g_ctx *ctx, const float *ashcon, const float *depocon, float **da, float **dd) {
  const Layout &L = ctx->L;
  const size_t na = (size_t)L.nx * L.ny * L.nz * L.ns, nd = (size_t)L.nx * L.ny * L.ns;
  const bool a_dev = ashcon && device_addressable(ctx, ashcon);
  const bool d_dev = depocon && device_addressable(ctx, depocon);
  const size_t sa = (ashcon && !a_dev) ? na : 0, sd = (depocon && !d_dev) ? nd : 0;
  int rc = ensure_nc_buf(ctx, sa + sd);
  if (rc) return rc;
  *da = !ashcon ? nullptr : a_dev ? const_cast<float *>(ashcon) : ctx->nc_buf;
  *dd = !depocon ? nullptr : d_dev ? const_cast<float *>(depocon) : ctx->nc_buf + sa;
  return A3G_OK;
}

int a3g_output_ashcon(a3g_ctx *ctx, float *ashcon, float *depocon) {
  CTX_CHECK(ctx);
  const Layout &L = ctx->L;
  const size_t na = (size_t)L.nx * L.ny * L.nz * L.ns, nd = (size_t)L.nx * L.ny * L.ns;
  float *da, *dd;
  int rc = nc_targets(ctx, ashcon, depocon, &da, &dd);
  if (rc) return rc;
  rc = launch_netcdf_pack(ctx, da, dd);
  if (rc) return rc;
  if (ashcon && da != ashcon)
    A3G_CUDA(cudaMemcpyAsync(ashcon, da, na * sizeof(float), cudaMemcpyDefault, ctx->stream));
  if (depocon && dd != depocon)
    A3G_CUDA(cudaMemcpyAsync(depocon, dd, nd * sizeof(float), cudaMemcpyDefault, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);
}

int a3g_restart_load(a3g_ctx *ctx, const float *ashcon, const float *depocon) {
  CTX_CHECK(ctx);
  const Layout &L = ctx->L;
  const size_t na = (size_t)L.nx * L.ny * L.nz * L.ns, nd = (size_t)L.nx * L.ny * L.ns;
  float *da, *dd;
  int rc = nc_targets(ctx, ashcon, depocon, &da, &dd);
  if (rc) return rc;
  if (ashcon && da != ashcon)
    A3G_CUDA(cudaMemcpyAsync(da, ashcon, na * sizeof(float), cudaMemcpyDefault, ctx->stream));
  if (depocon && dd != depocon)
    A3G_CUDA(cudaMemcpyAsync(dd, depocon, nd * sizeof(float), cudaMemcpyDefault, ctx->stream));
  rc = launch_netcdf_unpack(ctx, da, dd);
  if (rc) return rc;
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ashcon) ctx->ts1_zeroed = false;
  return check_device_error(ctx);
}

int a3g_step_prologue(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  // ts0 <- ts1: the state is unchanged unless the last sweep left ts1 zero.
  if (ctx->ts1_zeroed)
    A3G_CUDA(cudaMemsetAsync(ctx->c0, 0, sizeof(double) * ctx->L.PG * ctx->L.ns, ctx->stream));
  ctx->ts1_zeroed = true;  // ts1 <- 0; the next sweep that copies back clears this
  return A3G_OK;
}

int a3g_set_dt(a3g_ctx *ctx, double dt) {
  CTX_CHECK(ctx);
  ctx->host_dt = dt;
  ctx->dt_stamp++;
  A3G_CUDA(cudaMemcpyAsync(&ctx->sc->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  return A3G_OK;
}

int a3g_add_source_column(a3g_ctx *ctx, int32_t ivent, int32_t jvent, const double *flux, double dt) {
  CTX_CHECK(ctx);
  if (!flux) return fail(A3G_ERR_ARG, "null flux");
  if (ivent < 1 || ivent > ctx->grid.nx || jvent < 1 || jvent > ctx->grid.ny)
    return fail(A3G_ERR_ARG, "vent outside the grid");
  A3G_CUDA(cudaEventSynchronize(ctx->src_event));  // previous staging copy done
  const size_t n = (size_t)(ctx->grid.nz + 1) * ctx->grid.ns;
  std::memcpy(ctx->h_src, flux, n * sizeof(double));
  A3G_CUDA(cudaMemcpyAsync(ctx->src_buf, ctx->h_src, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->src_event, ctx->stream));
  return launch_source(ctx, ivent, jvent, dt);
}

// ---- umbrella source (src/Source_Umbrella.f90) ----------------------------
static size_t umb_flux_len(const a3g_ctx *ctx) { return (size_t)9 * (ctx->grid.nz + 1) * ctx->grid.ns; }
static size_t umb_wind_len(const a3g_ctx *ctx) { return (size_t)2 * ctx->grid.nx * ctx->grid.ny; }

int a3g_set_umbrella(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t ibase, int32_t itop,
                     const double *avg_stencil) {
  CTX_CHECK(ctx);
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  if (!avg_stencil) return fail(A3G_ERR_ARG, "null averaging stencil");
  if (ivent < 2 || ivent > nx - 1 || jvent < 2 || jvent > ny - 1)
    return fail(A3G_ERR_ARG, "the umbrella's 3x3 patch must lie inside the grid");
  if (ibase < 1 || itop < ibase || itop > nz) return fail(A3G_ERR_ARG, "need 1 <= ibase <= itop <= nz");
  const size_t nsten = (size_t)9 * nz;
  const size_t total = nsten + umb_flux_len(ctx) + umb_wind_len(ctx);
  if (!ctx->umb_buf) {
    if (cudaMalloc((void **)&ctx->umb_buf, total * sizeof(double)) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "umbrella buffer allocation failed");
    ctx->bytes += total * sizeof(double);
    A3G_CUDA(cudaMallocHost((void **)&ctx->h_umb, (umb_flux_len(ctx) + umb_wind_len(ctx)) * sizeof(double)));
    A3G_CUDA(cudaEventCreateWithFlags(&ctx->umb_event, cudaEventDisableTiming));
    A3G_CUDA(cudaEventRecord(ctx->umb_event, ctx->stream));
  }
  A3G_CUDA(cudaMemcpyAsync(ctx->umb_buf, avg_stencil, nsten * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->umb_ivent = ivent;
  ctx->umb_jvent = jvent;
  ctx->umb_ibase = ibase;
  ctx->umb_itop = itop;
  ctx->umb_on = true;
  return A3G_OK;
}

int a3g_add_umbrella_winds(a3g_ctx *ctx, int32_t i0, int32_t i1, int32_t j0, int32_t j1, const double *uvx,
                           const double *uvy) {
  CTX_CHECK(ctx);
  if (!ctx->umb_on) return fail(A3G_ERR_STATE, "a3g_set_umbrella has not been called");
  if (!uvx || !uvy) return fail(A3G_ERR_ARG, "null umbrella winds");
  if (i0 < 1 || i1 < i0 || i1 > ctx->grid.nx || j0 < 1 || j1 < j0 || j1 > ctx->grid.ny)
    return fail(A3G_ERR_ARG, "umbrella wind box outside the grid");
  const size_t m = (size_t)(i1 - i0 + 1) * (j1 - j0 + 1);
  A3G_CUDA(cudaEventSynchronize(ctx->umb_event));  // previous staging copy done
  double *h = ctx->h_umb + umb_flux_len(ctx);
  std::memcpy(h, uvx, m * sizeof(double));
  std::memcpy(h + m, uvy, m * sizeof(double));
  double *d = ctx->umb_buf + (size_t)9 * ctx->grid.nz + umb_flux_len(ctx);
  A3G_CUDA(cudaMemcpyAsync(d, h, 2 * m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->umb_event, ctx->stream));
  int rc = launch_umbrella_winds(ctx, i0, i1 - i0 + 1, j0, j1 - j0 + 1, d);
  // vh is formed from the winds with the umbrella's added (Calc_Vmod_Topo
  // runs after MesoInterpolater, src/Ash3d.F90:396-398)
  if (!rc && ctx->topo_on) rc = launch_vmod_topo(ctx);
  return rc;
}

int a3g_add_source_umbrella(a3g_ctx *ctx, const double *flux_umbrella, double dt) {
  CTX_CHECK(ctx);
  if (!ctx->umb_on) return fail(A3G_ERR_STATE, "a3g_set_umbrella has not been called");
  if (!flux_umbrella) return fail(A3G_ERR_ARG, "null umbrella flux");
  A3G_CUDA(cudaEventSynchronize(ctx->umb_event));
  std::memcpy(ctx->h_umb, flux_umbrella, umb_flux_len(ctx) * sizeof(double));
  A3G_CUDA(cudaMemcpyAsync(ctx->umb_buf + (size_t)9 * ctx->grid.nz, ctx->h_umb,
                           umb_flux_len(ctx) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->umb_event, ctx->stream));
  return launch_source_umbrella(ctx, dt);
}

int a3g_add_source_column_devdt(a3g_ctx *ctx, int32_t ivent, int32_t jvent, const double *flux) {
  CTX_CHECK(ctx);
  if (!flux) return fail(A3G_ERR_ARG, "null flux");
  if (ivent < 1 || ivent > ctx->grid.nx || jvent < 1 || jvent > ctx->grid.ny)
    return fail(A3G_ERR_ARG, "vent outside the grid");
  A3G_CUDA(cudaEventSynchronize(ctx->src_event));  // previous staging copy done
  const size_t n = (size_t)(ctx->grid.nz + 1) * ctx->grid.ns;
  std::memcpy(ctx->h_src, flux, n * sizeof(double));
  A3G_CUDA(cudaMemcpyAsync(ctx->src_buf, ctx->h_src, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->src_event, ctx->stream));
  return launch_source_devdt(ctx, ivent, jvent);
}

int a3g_set_bc(a3g_ctx *ctx, int32_t bc_code) {
  CTX_CHECK(ctx);
  if (bc_code != 1 && bc_code != 2) return fail(A3G_ERR_BC_CODE, "ERROR BC code not recognized");
  ctx->last_bc = bc_code;
  return A3G_OK;
}

static int ready(a3g_ctx *ctx) {
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  if (!ctx->have_vf) return fail(A3G_ERR_STATE, "fall velocities not set");
  if (!ctx->have_winds) return fail(A3G_ERR_STATE, "winds not set");
  return A3G_OK;
}

int a3g_advect_x(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = ready(ctx);
  if (rc) return rc;
  rc = launch_advect_x(ctx);
  if (!rc) ctx->ts1_zeroed = false;
  return rc;
}

int a3g_advect_y(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = ready(ctx);
  if (rc) return rc;
  rc = launch_advect_y(ctx);
  if (!rc) ctx->ts1_zeroed = false;
  return rc;
}

int a3g_get_minmax_index(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t kvent, int32_t *box) {
  CTX_CHECK(ctx);
  int rc = launch_plane_flags(ctx);
  if (rc) return rc;
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  const int32_t *fi = ctx->h_plane_flags, *fj = fi + nx + 1, *fk = fj + ny + 1;
  Box b;
  // "maxval(plane) < CLOUDCON_GRID_THRESH" <=> no cell of the plane reaches it
  b.imin = 1; b.imax = nx;
  for (int i = 2; i <= ivent - 1; i++) { if (!fi[i]) b.imin = i; else break; }
  for (int i = nx; i >= b.imin + 2; i--) { if (!fi[i]) b.imax = i; else break; }
  if (ctx->grid.periodic && (b.imin == 1 || b.imax == nx)) { b.imin = 1; b.imax = nx; }
  b.jmin = 1; b.jmax = ny;
  for (int j = 2; j <= jvent - 1; j++) { if (!fj[j]) b.jmin = j; else break; }
  for (int j = ny; j >= b.jmin + 2; j--) { if (!fj[j]) b.jmax = j; else break; }
  b.kmin = 1; b.kmax = nz;
  for (int k = 2; k <= kvent - 1; k++) { if (!fk[k]) b.kmin = k; else break; }
  for (int k = nz; k >= b.kmin + 2; k--) { if (!fk[k]) b.kmax = k; else break; }
  if (b.kmax < b.kmin) return fail(A3G_ERR_SUBGRID, "ERROR: kmax<kmin in get_minmax_index");
  if (b.imax - b.imin < 2) { b.imax = (b.imax + 1 < nx) ? b.imax + 1 : nx; b.imin = b.imax - 2; }
  if (b.jmax - b.jmin < 2) { b.jmax = (b.jmax + 1 < ny) ? b.jmax + 1 : ny; b.jmin = b.jmax - 2; }
  if (b.kmax - b.kmin < 2) { b.kmax = (b.kmax + 1 < nz) ? b.kmax + 1 : nz; b.kmin = b.kmax - 2; }
  ctx->box = b;
  if (box) { box[0] = b.imin; box[1] = b.imax; box[2] = b.jmin; box[3] = b.jmax; box[4] = b.kmin; box[5] = b.kmax; }
  return A3G_OK;
}

int a3g_set_subgrid(a3g_ctx *ctx, const int32_t *box) {
  CTX_CHECK(ctx);
  if (!box) return fail(A3G_ERR_ARG, "null box");
  Box b{box[0], box[1], box[2], box[3], box[4], box[5]};
  if (b.imin < 1 || b.imax > ctx->grid.nx || b.jmin < 1 || b.jmax > ctx->grid.ny || b.kmin < 1 ||
      b.kmax > ctx->grid.nz || b.imin > b.imax || b.jmin > b.jmax || b.kmin > b.kmax)
    return fail(A3G_ERR_ARG, "box outside the grid or empty");
  ctx->box = b;
  return A3G_OK;
}

int a3g_get_subgrid(a3g_ctx *ctx, int32_t *box) {
  if (!ctx || !box) return fail(A3G_ERR_ARG, "null argument");
  const Box &b = ctx->box;
  box[0] = b.imin; box[1] = b.imax; box[2] = b.jmin; box[3] = b.jmax; box[4] = b.kmin; box[5] = b.kmax;
  return A3G_OK;
}

int a3g_advect_horz(a3g_ctx *ctx, int32_t itoggle, int32_t ivent, int32_t jvent, int32_t kvent) {
  CTX_CHECK(ctx);
  int rc = ready(ctx);
  if (rc) return rc;
  if (ctx->prm.fast_subgrid) {
    if ((rc = a3g_get_minmax_index(ctx, ivent, jvent, kvent, nullptr))) return rc;
  } else {
    full_box(ctx);
  }
  if (itoggle % 2 == 0) {
    if ((rc = launch_advect_y(ctx))) return rc;
    if ((rc = launch_advect_x(ctx))) return rc;
  } else {
    if ((rc = launch_advect_x(ctx))) return rc;
    if ((rc = launch_advect_y(ctx))) return rc;
  }
  ctx->ts1_zeroed = false;
  return A3G_OK;
}

int a3g_advect_vert(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = ready(ctx);
  if (rc) return rc;
  rc = launch_advect_z(ctx);
  if (!rc) ctx->ts1_zeroed = false;
  return rc;
}

int a3g_diffuse_horz(a3g_ctx *ctx, int32_t itime) {
  CTX_CHECK(ctx);
  if (!ctx->have_geometry || !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "geometry/diffusivity not set");
  Box &b = ctx->box;
  if (ctx->prm.fast_subgrid) {  // src/Diffusion.F90:168-176
    b.imin = b.imin - 1 > 1 ? b.imin - 1 : 1;
    b.imax = b.imax + 1 < ctx->grid.nx ? b.imax + 1 : ctx->grid.nx;
    b.jmin = b.jmin - 1 > 1 ? b.jmin - 1 : 1;
    b.jmax = b.jmax + 1 < ctx->grid.ny ? b.jmax + 1 : ctx->grid.ny;
    b.kmin = b.kmin - 1 > 1 ? b.kmin - 1 : 1;
    b.kmax = b.kmax + 1 < ctx->grid.nz ? b.kmax + 1 : ctx->grid.nz;
  } else {
    full_box(ctx);
  }
  int rc;
  if (ctx->prm.use_cn) {
    if (itime % 2 == 0) {
      if ((rc = launch_diffcn_x(ctx))) return rc;
      if ((rc = launch_diffcn_y(ctx))) return rc;
    } else {
      if ((rc = launch_diffcn_y(ctx))) return rc;
      if ((rc = launch_diffcn_x(ctx))) return rc;
    }
  } else {
    if (itime % 2 == 0) {
      if ((rc = launch_diff_x(ctx))) return rc;
      if ((rc = launch_diff_y(ctx))) return rc;
    } else {
      if ((rc = launch_diff_y(ctx))) return rc;
      if ((rc = launch_diff_x(ctx))) return rc;
    }
    ctx->ts1_zeroed = false;
  }
  return A3G_OK;
}

int a3g_diffuse_vert(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  if (!ctx->have_geometry || !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "geometry/diffusivity not set");
  int rc;
  if (ctx->prm.use_cn) {
    rc = launch_diffcn_z(ctx);
  } else {
    rc = launch_diff_z(ctx);
    if (!rc) ctx->ts1_zeroed = false;
  }
  return rc;
}

int a3g_adjust_dt(a3g_ctx *ctx, double time, double next_write_time, double simtime, double *dt_out) {
  CTX_CHECK(ctx);
  if (!ctx->have_geometry || !ctx->have_vf || !ctx->have_winds)
    return fail(A3G_ERR_STATE, "geometry, fall velocities and winds must be set");
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  int rc = launch_cfl(ctx, time, next_write_time, simtime);
  if (rc) return rc;
  ctx->dt_stamp++;
  if ((rc = sync_scalars(ctx))) return rc;
  ctx->host_dt = ctx->h_sc->dt;
  if (dt_out) *dt_out = ctx->h_sc->dt;
  return A3G_OK;
}

// ---- lag-one host loop ------------------------------------------------------
int a3g_adjust_dt_async(a3g_ctx *ctx, double time, double next_write_time, double simtime) {
  CTX_CHECK(ctx);
  if (!ctx->have_geometry || !ctx->have_vf || !ctx->have_winds)
    return fail(A3G_ERR_STATE, "geometry, fall velocities and winds must be set");
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  int rc = launch_cfl(ctx, time, next_write_time, simtime);
  if (rc) return rc;
  ctx->dt_stamp++;
  const int slot = (int)(ctx->dt_seq % 4);
  A3G_CUDA(cudaMemcpyAsync(ctx->h_sc_ring + slot, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost,
                           ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->sc_ev[slot], ctx->stream));
  ctx->dt_seq++;
  return A3G_OK;
}

int a3g_wait_dt(a3g_ctx *ctx, double *dt_out) {
  CTX_CHECK(ctx);
  if (!dt_out) return fail(A3G_ERR_ARG, "null dt");
  if (ctx->dt_seq == 0) return fail(A3G_ERR_STATE, "a3g_adjust_dt_async has not been called");
  const int slot = (int)((ctx->dt_seq - 1) % 4);
  A3G_CUDA(cudaEventSynchronize(ctx->sc_ev[slot]));
  *ctx->h_sc = ctx->h_sc_ring[slot];
  ctx->host_dt = ctx->h_sc->dt;
  *dt_out = ctx->h_sc->dt;
  return check_device_error(ctx);
}

int a3g_timestep_totals_async(a3g_ctx *ctx, int64_t *ticket) {
  CTX_CHECK(ctx);
  if (!ticket) return fail(A3G_ERR_ARG, "null ticket");
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  const int slot = (int)(ctx->tot_seq % 4);
  // the slot's previous copy must have been consumed: at most 4 in flight
  A3G_CUDA(cudaEventSynchronize(ctx->tot_ev[slot]));
  int rc = launch_totals_partials(ctx, ctx->h_tot_ring + (size_t)slot * 7 * ctx->grid.ns);
  if (rc) return rc;
  A3G_CUDA(cudaEventRecord(ctx->tot_ev[slot], ctx->stream));
  *ticket = (int64_t)ctx->tot_seq++;
  return A3G_OK;
}

int a3g_totals_get(a3g_ctx *ctx, int64_t ticket, double *out4, double *mass_aloft) {
  CTX_CHECK(ctx);
  if (!out4) return fail(A3G_ERR_ARG, "null out4");
  if (ticket < 0 || (uint64_t)ticket >= ctx->tot_seq || (uint64_t)ticket + 4 < ctx->tot_seq)
    return fail(A3G_ERR_ARG, "totals ticket unknown or overwritten (at most 4 in flight)");
  const int slot = (int)(ticket % 4);
  A3G_CUDA(cudaEventSynchronize(ctx->tot_ev[slot]));
  totals_volumes(ctx, ctx->h_tot_ring + (size_t)slot * 7 * ctx->grid.ns, out4, mass_aloft);
  for (int q = 0; q < 4; q++)
    if (!std::isfinite(out4[q])) return fail(A3G_ERR_NONFINITE, "non-finite mass total (NaN/Inf in the state)");
  return A3G_OK;
}

int a3g_set_source_pulses(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t npulses, const double *start_h,
                          const double *end_h, const double *mass_flux_rate, const double *norm_col,
                          const double *bin_mass) {
  CTX_CHECK(ctx);
  const int nz = ctx->grid.nz, ns = ctx->grid.ns;
  if (npulses < 1 || npulses > 64) return fail(A3G_ERR_ARG, "need 1 <= npulses <= 64");
  if (!start_h || !end_h || !mass_flux_rate || !norm_col || !bin_mass) return fail(A3G_ERR_ARG, "null source array");
  if (ivent < 1 || ivent > ctx->grid.nx || jvent < 1 || jvent > ctx->grid.ny)
    return fail(A3G_ERR_ARG, "vent outside the grid");
  const size_t n = (size_t)3 * npulses + (size_t)npulses * (nz + 1) + ns;
  std::vector<double> h(n);
  std::memcpy(h.data(), start_h, sizeof(double) * npulses);
  std::memcpy(h.data() + npulses, end_h, sizeof(double) * npulses);
  std::memcpy(h.data() + 2 * npulses, mass_flux_rate, sizeof(double) * npulses);
  std::memcpy(h.data() + 3 * npulses, norm_col, sizeof(double) * npulses * (nz + 1));
  std::memcpy(h.data() + 3 * npulses + (size_t)npulses * (nz + 1), bin_mass, sizeof(double) * ns);
  if (ctx->src_sched) cudaFree(ctx->src_sched);
  ctx->src_sched = nullptr;
  if (cudaMalloc((void **)&ctx->src_sched, n * sizeof(double)) != cudaSuccess)
    return fail(A3G_ERR_NOMEM, "source schedule allocation failed");
  if (!ctx->src_state && cudaMalloc((void **)&ctx->src_state, 2 * sizeof(int32_t)) != cudaSuccess)
    return fail(A3G_ERR_NOMEM, "source state allocation failed");
  const int32_t st[2] = {1, 1};  // ieruption = jeruption = 1, src/Source.f90:173-174
  A3G_CUDA(cudaMemcpyAsync(ctx->src_sched, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaMemcpyAsync(ctx->src_state, st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->src_np = npulses;
  ctx->src_iv = ivent;
  ctx->src_jv = jvent;
  return A3G_OK;
}

int a3g_add_source_scheduled(a3g_ctx *ctx, double time) {
  CTX_CHECK(ctx);
  if (!ctx->src_sched) return fail(A3G_ERR_STATE, "a3g_set_source_pulses has not been called");
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  return launch_source_sched(ctx, time);
}

int a3g_cfl_maxima(a3g_ctx *ctx, double *vmax3) {
  CTX_CHECK(ctx);
  if (!vmax3) return fail(A3G_ERR_ARG, "null vmax3");
  if (!ctx->have_geometry || !ctx->have_vf || !ctx->have_winds)
    return fail(A3G_ERR_STATE, "geometry, fall velocities and winds must be set");
  int rc = launch_cfl_maxima(ctx);
  if (rc) return rc;
  if ((rc = sync_scalars(ctx))) return rc;
  for (int q = 0; q < 3; q++) vmax3[q] = ctx->h_sc->vmax[q];
  return A3G_OK;
}

int a3g_adjust_dt_from_maxima(a3g_ctx *ctx, const double *vmax3, int32_t n_gs_aloft_total,
                              double time, double next_write_time, double simtime, double *dt_out) {
  CTX_CHECK(ctx);
  if (!vmax3) return fail(A3G_ERR_ARG, "null vmax3");
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  double v[4] = {vmax3[0], vmax3[1], vmax3[2], 0.0};
  A3G_CUDA(cudaMemcpyAsync(ctx->sc->vmax, v, sizeof(v), cudaMemcpyHostToDevice, ctx->stream));
  int rc = launch_dt_from_maxima(ctx, n_gs_aloft_total, time, next_write_time, simtime);
  if (rc) return rc;
  ctx->dt_stamp++;
  if ((rc = sync_scalars(ctx))) return rc;
  ctx->host_dt = ctx->h_sc->dt;
  if (dt_out) *dt_out = ctx->h_sc->dt;
  return A3G_OK;
}

int a3g_cfl_maxima_device(a3g_ctx *ctx, double **vmax3_dev) {
  CTX_CHECK(ctx);
  if (!vmax3_dev) return fail(A3G_ERR_ARG, "null output");
  if (!ctx->have_geometry || !ctx->have_vf || !ctx->have_winds)
    return fail(A3G_ERR_STATE, "geometry, fall velocities and winds must be set");
  int rc = launch_cfl_maxima(ctx);
  if (rc) return rc;
  *vmax3_dev = ctx->sc->vmax;
  return A3G_OK;
}

int a3g_adjust_dt_device_maxima_async(a3g_ctx *ctx, int32_t n_gs_aloft_total, double time,
                                      double next_write_time, double simtime) {
  CTX_CHECK(ctx);
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  int rc = launch_dt_from_maxima(ctx, n_gs_aloft_total, time, next_write_time, simtime);
  if (rc) return rc;
  ctx->dt_stamp++;
  const int slot = (int)(ctx->dt_seq % 4);
  A3G_CUDA(cudaMemcpyAsync(ctx->h_sc_ring + slot, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost,
                           ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->sc_ev[slot], ctx->stream));
  ctx->dt_seq++;
  return A3G_OK;
}

// ---- FAST_DT (src/makefile:91; src/Adjust_dt.f90:96-135, src/MesoInterpolater.f90:
// 142-150, 187-195, 250-258) ------------------------------------------------
int a3g_set_fall_velocity_meso(a3g_ctx *ctx, const float *vf_meso_sp, int32_t per_grain) {
  CTX_CHECK(ctx);
  if (!vf_meso_sp) return fail(A3G_ERR_ARG, "null vf_meso_next_step_sp");
  const int ns = ctx->grid.ns;
  if (ctx->vfm_sp) cudaFree(ctx->vfm_sp);
  ctx->vfm_sp = nullptr;
  ctx->have_vf_meso = false;
  if (per_grain) {
    // real(Tephra_v_s(isize), sp) in every cell (src/MesoInterpolater.f90:567-574)
    float v = 0.0f;
    for (int g = 0; g < ns; g++) {
      const float a = std::fabs(vf_meso_sp[g]);
      if (g == 0 || a > v) v = a;
    }
    ctx->vfm_sp_const = v;
    ctx->have_vf_meso = true;
    return A3G_OK;
  }
  const long n = (long)ctx->grid.nx * ctx->grid.ny * ctx->grid.nz;
  // maxval(abs(vf_meso_next_step_sp(i,j,k,1:nsmax))) per cell
  std::vector<float> m((size_t)n);
  bool uniform = true;
  for (long c = 0; c < n; c++) {
    float v = 0.0f;
    for (int g = 0; g < ns; g++) {
      const float a = std::fabs(vf_meso_sp[(size_t)g * n + c]);
      if (g == 0 || a > v) v = a;
    }
    m[(size_t)c] = v;
    if (std::memcmp(&m[(size_t)c], &m[0], sizeof(float)) != 0) uniform = false;
  }
  ctx->vfm_sp_const = m[0];
  if (!uniform) {
    if (cudaMalloc((void **)&ctx->vfm_sp, sizeof(float) * n) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "fall-velocity maxima allocation failed");
    A3G_CUDA(cudaMemcpyAsync(ctx->vfm_sp, m.data(), sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
    A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  ctx->have_vf_meso = true;
  return A3G_OK;
}

static int meso_ready(a3g_ctx *ctx, int slot) {
  if (slot != 0 && slot != 1) return fail(A3G_ERR_ARG, "met slot must be 0 (last) or 1 (next)");
  if (!ctx->met) return fail(A3G_ERR_STATE, "a3g_set_met_steps has not been called");
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  if (!ctx->have_vf_meso) return fail(A3G_ERR_STATE, "a3g_set_fall_velocity_meso has not been called");
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  return A3G_OK;
}

int a3g_cfl_maxima_meso(a3g_ctx *ctx, int32_t slot, double *vmax3) {
  CTX_CHECK(ctx);
  if (!vmax3) return fail(A3G_ERR_ARG, "null vmax3");
  int rc = meso_ready(ctx, slot);
  if (rc) return rc;
  if ((rc = launch_cfl_maxima_meso(ctx, slot))) return rc;
  if ((rc = sync_scalars(ctx))) return rc;
  for (int q = 0; q < 3; q++) vmax3[q] = ctx->h_sc->vmax[q];
  return A3G_OK;
}

int a3g_adjust_dt_meso(a3g_ctx *ctx, int32_t slot, int32_t shift, double time, double next_write_time,
                       double simtime, double *dt_out) {
  CTX_CHECK(ctx);
  int rc = meso_ready(ctx, slot);
  if (rc) return rc;
  if ((rc = launch_cfl_maxima_meso(ctx, slot))) return rc;
  if ((rc = launch_dt_from_maxima(ctx, ctx->n_gs_aloft, time, next_write_time, simtime, shift ? 3 : 1)))
    return rc;
  ctx->dt_stamp++;
  if (!dt_out) return A3G_OK;
  if ((rc = sync_scalars(ctx))) return rc;
  ctx->host_dt = ctx->h_sc->dt;
  *dt_out = ctx->h_sc->dt;
  return A3G_OK;
}

int a3g_adjust_dt_meso_from_maxima(a3g_ctx *ctx, const double *vmax3, int32_t n_gs_aloft_total, int32_t shift,
                                   double time, double next_write_time, double simtime, double *dt_out) {
  CTX_CHECK(ctx);
  if (!vmax3) return fail(A3G_ERR_ARG, "null vmax3");
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  double v[4] = {vmax3[0], vmax3[1], vmax3[2], 0.0};
  A3G_CUDA(cudaMemcpyAsync(ctx->sc->vmax, v, sizeof(v), cudaMemcpyHostToDevice, ctx->stream));
  int rc = launch_dt_from_maxima(ctx, n_gs_aloft_total, time, next_write_time, simtime, shift ? 3 : 1);
  if (rc) return rc;
  ctx->dt_stamp++;
  if ((rc = sync_scalars(ctx))) return rc;
  ctx->host_dt = ctx->h_sc->dt;
  if (dt_out) *dt_out = ctx->h_sc->dt;
  return A3G_OK;
}

int a3g_fast_dt_async(a3g_ctx *ctx, double interval_frac, double time, double next_write_time, double simtime) {
  CTX_CHECK(ctx);
  int rc = launch_fast_dt(ctx, interval_frac, time, next_write_time, simtime);
  if (rc) return rc;
  ctx->dt_stamp++;
  const int slot = (int)(ctx->dt_seq % 4);
  A3G_CUDA(cudaMemcpyAsync(ctx->h_sc_ring + slot, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost,
                           ctx->stream));
  A3G_CUDA(cudaEventRecord(ctx->sc_ev[slot], ctx->stream));
  ctx->dt_seq++;
  return A3G_OK;
}

int a3g_timestep_totals(a3g_ctx *ctx, double *out4, double *mass_aloft) {
  CTX_CHECK(ctx);
  if (!out4) return fail(A3G_ERR_ARG, "null out4");
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  int rc = launch_totals(ctx, out4, mass_aloft);
  if (rc) return rc;
  if ((rc = sync_scalars(ctx))) return rc;
  // The reference carries a NaN on silently (its mass-conservation stop
  // test compares false); the totals are still written, but the caller is told.
  for (int q = 0; q < 4; q++)
    if (!std::isfinite(out4[q])) return fail(A3G_ERR_NONFINITE, "non-finite mass total (NaN/Inf in the state)");
  return A3G_OK;
}

int a3g_step(a3g_ctx *ctx, int32_t itime, int32_t ivent, int32_t jvent, int32_t kvent, const double *flux) {
  CTX_CHECK(ctx);
  int rc;
  if ((rc = a3g_step_prologue(ctx))) return rc;
  if (flux && (rc = a3g_add_source_column(ctx, ivent, jvent, flux, ctx->host_dt))) return rc;
  if ((rc = a3g_set_bc(ctx, 1))) return rc;
  if ((rc = a3g_advect_horz(ctx, itime, ivent, jvent, kvent))) return rc;
  if ((rc = a3g_advect_vert(ctx))) return rc;
  if (ctx->prm.use_diffusion) {
    if ((rc = a3g_set_bc(ctx, 2))) return rc;
    if ((rc = a3g_diffuse_horz(ctx, itime))) return rc;
    if ((rc = a3g_diffuse_vert(ctx))) return rc;
  }
  return A3G_OK;
}

int a3g_get_stream(a3g_ctx *ctx, void **stream) {
  if (!ctx || !stream) return fail(A3G_ERR_ARG, "null argument");
  *stream = (void *)ctx->stream;
  return A3G_OK;
}

int a3g_kernel_timing(a3g_ctx *ctx, int32_t enable) {
  CTX_CHECK(ctx);
  ctx->timing = enable != 0;
  ctx->ev_kind.clear();
  ctx->ev_used = 0;
  return A3G_OK;
}

int a3g_kernel_times(a3g_ctx *ctx, double *ms, uint64_t *count) {
  CTX_CHECK(ctx);
  if (!ms || !count) return fail(A3G_ERR_ARG, "null argument");
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < A3G_K_COUNT; k++) { ms[k] = 0.0; count[k] = 0; }
  const size_t pairs = ctx->ev_used / 2;
  for (size_t p = 0; p < pairs && p < ctx->ev_kind.size(); p++) {
    float t = 0.0f;
    A3G_CUDA(cudaEventElapsedTime(&t, ctx->ev_pool[2 * p], ctx->ev_pool[2 * p + 1]));
    const int k = ctx->ev_kind[p];
    ms[k] += t;
    count[k] += 1;
  }
  return A3G_OK;
}

int a3g_set_variant(a3g_ctx *ctx, int32_t dir, int32_t variant) {
  if (!ctx) return fail(A3G_ERR_ARG, "null context");
  const bool col = (dir == 1 || dir == 2) && (variant == 5 || variant == 6);  // the column marches (y, z)
  if (dir < 0 || dir > 5 || variant < 0 ||
      (!col && variant > (dir == 0 ? 5 : dir == 3 ? 2 : dir == 4 ? 3 : dir == 5 ? 1 : 2)))
    return fail(A3G_ERR_ARG, "bad direction or variant");
  if (dir == 3) ctx->tune_cn_x = variant;
  else if (dir == 4) ctx->tune_cn_yz = variant;
  else if (dir == 5) ctx->adj_gather = variant == 1;
  else ctx->tune_advect[dir] = variant;
  return A3G_OK;
}

int a3g_get_variant(a3g_ctx *ctx, int32_t dir, int32_t *variant) {
  if (!ctx || !variant || dir < 0 || dir > 5) return fail(A3G_ERR_ARG, "bad argument");
  *variant = (dir == 3)   ? ctx->tune_cn_x
             : (dir == 4) ? ctx->tune_cn_yz
             : (dir == 5) ? (ctx->adj_gather ? 1 : 0)
                          : ctx->tune_advect[dir];
  return A3G_OK;
}

int a3g_kernel_launches(a3g_ctx *ctx, uint64_t *count) {
  if (!ctx || !count) return fail(A3G_ERR_ARG, "null argument");
  *count = ctx->launches;
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// discrete adjoint
// ---------------------------------------------------------------------------
static size_t level_bytes(const a3g_ctx *ctx) { return sizeof(double) * ctx->L.PG * ctx->L.ns; }

static int adj_ready(a3g_ctx *ctx) {
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  if (ctx->prm.fast_subgrid) return fail(A3G_ERR_UNSUPPORTED, "the adjoint needs fast_subgrid off");
  if (ctx->topo_on) return fail(A3G_ERR_UNSUPPORTED, "the adjoint does not cover the terrain terms");
  int rc = ready(ctx);
  if (rc) return rc;
  full_box(ctx);
  return A3G_OK;
}

static void swap_lam(a3g_ctx *ctx) {
  double *t = ctx->lam0;
  ctx->lam0 = ctx->lam1;
  ctx->lam1 = t;
}

int a3g_adj_enable(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  if (ctx->lam0) return a3g_adj_zero(ctx);
  const size_t lev = level_bytes(ctx);
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz, ns = ctx->grid.ns;
  const size_t face = sizeof(double) * (size_t)ns *
                      (size_t)std::max(std::max((long)ny * nz, (long)nx * nz), (long)nx * ny);
  const size_t obs = sizeof(double) * std::max((size_t)nx * ny, (size_t)(nz + 1) * ns);
  double **bufs[] = {&ctx->lam0, &ctx->lam1, &ctx->stage1};
  for (double **b : bufs) {
    if (cudaMalloc((void **)b, lev) != cudaSuccess) return fail(A3G_ERR_NOMEM, "adjoint level allocation failed");
    ctx->bytes += lev;
  }
  if (cudaMalloc((void **)&ctx->lam_dep, sizeof(double) * (size_t)nx * ny * ns) != cudaSuccess ||
      cudaMalloc((void **)&ctx->adj_face, face) != cudaSuccess ||
      cudaMalloc((void **)&ctx->obs_buf, obs) != cudaSuccess)
    return fail(A3G_ERR_NOMEM, "adjoint buffer allocation failed");
  ctx->bytes += sizeof(double) * (size_t)nx * ny * ns + face + obs;
  return a3g_adj_zero(ctx);
}

int a3g_adj_zero(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  A3G_CUDA(cudaMemsetAsync(ctx->lam0, 0, level_bytes(ctx), ctx->stream));
  A3G_CUDA(cudaMemsetAsync(ctx->lam1, 0, level_bytes(ctx), ctx->stream));
  A3G_CUDA(cudaMemsetAsync(ctx->lam_dep, 0,
                           sizeof(double) * (size_t)ctx->grid.nx * ctx->grid.ny * ctx->grid.ns, ctx->stream));
  return A3G_OK;
}

int a3g_adj_set_lambda(a3g_ctx *ctx, const double *lam) {
  CTX_CHECK(ctx);
  if (!lam) return fail(A3G_ERR_ARG, "null lam");
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  A3G_CUDA(cudaMemsetAsync(ctx->lam0, 0, level_bytes(ctx), ctx->stream));
  int rc = copy_level(ctx, const_cast<double *>(lam), ctx->lam0, true, nx + 4, ny + 4, nz + 4, 2, nx, ny, nz,
                      ctx->grid.ns, ctx->L.P, ctx->L.PY, ctx->L.PG);
  if (rc) return rc;
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

int a3g_adj_get_lambda(a3g_ctx *ctx, double *lam) {
  CTX_CHECK(ctx);
  if (!lam) return fail(A3G_ERR_ARG, "null lam");
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz;
  int rc = copy_level(ctx, lam, ctx->lam0, false, nx + 4, ny + 4, nz + 4, 2, nx, ny, nz, ctx->grid.ns,
                      ctx->L.P, ctx->L.PY, ctx->L.PG);
  if (rc) return rc;
  return sync_scalars(ctx);
}

int a3g_adj_set_lambda_dep(a3g_ctx *ctx, const double *lam_dep) {
  CTX_CHECK(ctx);
  if (!lam_dep) return fail(A3G_ERR_ARG, "null lam_dep");
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  A3G_CUDA(cudaMemcpyAsync(ctx->lam_dep, lam_dep, sizeof(double) * (size_t)ctx->grid.nx * ctx->grid.ny * ctx->grid.ns,
                           cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

int a3g_adj_get_lambda_dep(a3g_ctx *ctx, double *lam_dep) {
  CTX_CHECK(ctx);
  if (!lam_dep) return fail(A3G_ERR_ARG, "null lam_dep");
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  A3G_CUDA(cudaMemcpyAsync(lam_dep, ctx->lam_dep, sizeof(double) * (size_t)ctx->grid.nx * ctx->grid.ny * ctx->grid.ns,
                           cudaMemcpyDeviceToHost, ctx->stream));
  return sync_scalars(ctx);
}

static int adj_advect_dir(a3g_ctx *ctx, int dir, const double *state) {
  int rc = launch_adj_advect(ctx, dir, state, ctx->lam0, ctx->lam1, dir == 2 ? ctx->lam_dep : nullptr);
  if (rc) return rc;
  swap_lam(ctx);
  return A3G_OK;
}

static int adj_diffuse_dir(a3g_ctx *ctx, int dir) {
  int rc = launch_adj_diffuse(ctx, dir, ctx->lam0, ctx->lam1);
  if (rc) return rc;
  swap_lam(ctx);
  return A3G_OK;
}

int a3g_adj_advect_x(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = adj_ready(ctx);
  return rc ? rc : adj_advect_dir(ctx, 0, ctx->c0);
}

int a3g_adj_advect_y(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = adj_ready(ctx);
  return rc ? rc : adj_advect_dir(ctx, 1, ctx->c0);
}

int a3g_adj_advect_vert(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = adj_ready(ctx);
  return rc ? rc : adj_advect_dir(ctx, 2, ctx->c0);
}

int a3g_adj_diffuse_horz(a3g_ctx *ctx, int32_t itime) {
  CTX_CHECK(ctx);
  int rc = adj_ready(ctx);
  if (rc) return rc;
  if (!ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  // DiffuseHorz: even x then y, odd y then x (src/Diffusion.F90:186-214)
  const int first = (itime % 2 == 0) ? 0 : 1;
  if ((rc = adj_diffuse_dir(ctx, 1 - first))) return rc;
  return adj_diffuse_dir(ctx, first);
}

int a3g_adj_diffuse_vert(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  int rc = adj_ready(ctx);
  if (rc) return rc;
  if (!ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  return adj_diffuse_dir(ctx, 2);
}

int a3g_adj_step(a3g_ctx *ctx, int32_t itime) {
  CTX_CHECK(ctx);
  int rc = adj_ready(ctx);
  if (rc) return rc;
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return fail(A3G_ERR_STATE, "diffusivity not set");
  // Recompute the states entering the second horizontal sweep and the
  // vertical sweep, keeping the forward state and accumulators intact: the
  // recomputed sweeps write into the stage buffer and the scratch level ts1
  // (which every sweep overwrites whole) and add their outflow updates to a
  // scratch face.
  double *keep_c0 = ctx->c0, *keep_c1 = ctx->c1;
  double *outs[6] = {ctx->out_yz1, ctx->out_yz2, ctx->out_xz1, ctx->out_xz2, ctx->out_xy1, ctx->out_xy2};
  ctx->out_yz1 = ctx->out_yz2 = ctx->out_xz1 = ctx->out_xz2 = ctx->out_xy1 = ctx->out_xy2 = ctx->adj_face;
  const int first = (itime % 2 == 0) ? 1 : 0;  // AdvectHorz: even y then x, odd x then y
  ctx->c1 = ctx->stage1;
  rc = (first == 0) ? launch_advect_x(ctx) : launch_advect_y(ctx);  // c0 := stage1 (state b)
  if (!rc) {
    ctx->c1 = keep_c1;
    rc = (first == 0) ? launch_advect_y(ctx) : launch_advect_x(ctx);  // c0 := ts1 (state c)
  }
  ctx->out_yz1 = outs[0]; ctx->out_yz2 = outs[1]; ctx->out_xz1 = outs[2];
  ctx->out_xz2 = outs[3]; ctx->out_xy1 = outs[4]; ctx->out_xy2 = outs[5];
  ctx->c0 = keep_c0;
  ctx->c1 = keep_c1;
  if (rc) return rc;
  if (ctx->prm.use_diffusion) {
    if ((rc = adj_diffuse_dir(ctx, 2))) return rc;  // DiffuseVert^T
    const int dfirst = (itime % 2 == 0) ? 0 : 1;     // DiffuseHorz: even x then y
    if ((rc = adj_diffuse_dir(ctx, 1 - dfirst))) return rc;
    if ((rc = adj_diffuse_dir(ctx, dfirst))) return rc;
  }
  if ((rc = adj_advect_dir(ctx, 2, ctx->c1))) return rc;             // AdvectVert^T at state c
  if ((rc = adj_advect_dir(ctx, 1 - first, ctx->stage1))) return rc; // second horizontal sweep at b
  return adj_advect_dir(ctx, first, ctx->c0);                        // first horizontal sweep at a
}

int a3g_adj_grad_reset(a3g_ctx *ctx, int32_t nbins) {
  CTX_CHECK(ctx);
  if (nbins < 1) return fail(A3G_ERR_ARG, "need nbins >= 1");
  const size_t n = (size_t)nbins * ctx->grid.nz * ctx->grid.ns;
  if (nbins != ctx->adj_grad_bins) {
    if (ctx->adj_grad) cudaFree(ctx->adj_grad);
    ctx->adj_grad = nullptr;
    if (cudaMalloc((void **)&ctx->adj_grad, n * sizeof(double)) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "gradient buffer allocation failed");
    ctx->adj_grad_bins = nbins;
  }
  A3G_CUDA(cudaMemsetAsync(ctx->adj_grad, 0, n * sizeof(double), ctx->stream));
  return A3G_OK;
}

int a3g_adj_vent_accumulate(a3g_ctx *ctx, int32_t ivent, int32_t jvent, int32_t bin, double dt) {
  CTX_CHECK(ctx);
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  if (!ctx->adj_grad) return fail(A3G_ERR_STATE, "a3g_adj_grad_reset has not been called");
  if (bin < 0 || bin >= ctx->adj_grad_bins) return fail(A3G_ERR_ARG, "gradient bin out of range");
  if (ivent < 1 || ivent > ctx->grid.nx || jvent < 1 || jvent > ctx->grid.ny)
    return fail(A3G_ERR_ARG, "vent outside the grid");
  return launch_vent_accumulate(ctx, ivent, jvent, dt,
                                ctx->adj_grad + (size_t)bin * ctx->grid.nz * ctx->grid.ns);
}

int a3g_adj_grad_get(a3g_ctx *ctx, double *out) {
  CTX_CHECK(ctx);
  if (!out) return fail(A3G_ERR_ARG, "null out");
  if (!ctx->adj_grad) return fail(A3G_ERR_STATE, "a3g_adj_grad_reset has not been called");
  const size_t n = (size_t)ctx->adj_grad_bins * ctx->grid.nz * ctx->grid.ns;
  A3G_CUDA(cudaMemcpyAsync(out, ctx->adj_grad, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return sync_scalars(ctx);
}

int a3g_adj_vent_column(a3g_ctx *ctx, int32_t ivent, int32_t jvent, double *out) {
  CTX_CHECK(ctx);
  if (!out) return fail(A3G_ERR_ARG, "null out");
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  if (ivent < 1 || ivent > ctx->grid.nx || jvent < 1 || jvent > ctx->grid.ny)
    return fail(A3G_ERR_ARG, "vent outside the grid");
  int rc = launch_vent_column(ctx, ivent, jvent, ctx->lam0, ctx->obs_buf);
  if (rc) return rc;
  A3G_CUDA(cudaMemcpyAsync(out, ctx->obs_buf, sizeof(double) * (size_t)(ctx->grid.nz + 1) * ctx->grid.ns,
                           cudaMemcpyDeviceToHost, ctx->stream));
  return sync_scalars(ctx);
}

int a3g_cloud_load(a3g_ctx *ctx, double *out) {
  CTX_CHECK(ctx);
  if (!out) return fail(A3G_ERR_ARG, "null out");
  if (!ctx->obs_buf) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  int rc = launch_cloud_load(ctx, ctx->c0, ctx->obs_buf);
  if (rc) return rc;
  A3G_CUDA(cudaMemcpyAsync(out, ctx->obs_buf, sizeof(double) * (size_t)ctx->grid.nx * ctx->grid.ny,
                           cudaMemcpyDeviceToHost, ctx->stream));
  return sync_scalars(ctx);
}

int a3g_adj_add_cloud_load(a3g_ctx *ctx, const double *w) {
  CTX_CHECK(ctx);
  if (!w) return fail(A3G_ERR_ARG, "null w");
  if (!ctx->lam0) return fail(A3G_ERR_STATE, "a3g_adj_enable has not been called");
  A3G_CUDA(cudaMemcpyAsync(ctx->obs_buf, w, sizeof(double) * (size_t)ctx->grid.nx * ctx->grid.ny,
                           cudaMemcpyHostToDevice, ctx->stream));
  int rc = launch_adj_cloud_load(ctx, ctx->obs_buf, ctx->lam0);
  if (rc) return rc;
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));  // w may be reused by the caller
  return A3G_OK;
}

int a3g_snapshot_alloc(a3g_ctx *ctx, int32_t nslots) {
  CTX_CHECK(ctx);
  if (nslots < 0) return fail(A3G_ERR_ARG, "negative slot count");
  while ((int)ctx->snaps.size() < nslots) {
    double *p = nullptr;
    if (cudaMalloc((void **)&p, level_bytes(ctx)) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "snapshot allocation failed");
    ctx->bytes += level_bytes(ctx);
    ctx->snaps.push_back(p);
  }
  return A3G_OK;
}

int a3g_snapshot_save(a3g_ctx *ctx, int32_t slot) {
  CTX_CHECK(ctx);
  if (slot < 0 || slot >= (int)ctx->snaps.size()) return fail(A3G_ERR_ARG, "snapshot slot out of range");
  A3G_CUDA(cudaMemcpyAsync(ctx->snaps[slot], ctx->c0, level_bytes(ctx), cudaMemcpyDeviceToDevice, ctx->stream));
  return A3G_OK;
}

int a3g_snapshot_load(a3g_ctx *ctx, int32_t slot) {
  CTX_CHECK(ctx);
  if (slot < 0 || slot >= (int)ctx->snaps.size()) return fail(A3G_ERR_ARG, "snapshot slot out of range");
  A3G_CUDA(cudaMemcpyAsync(ctx->c0, ctx->snaps[slot], level_bytes(ctx), cudaMemcpyDeviceToDevice, ctx->stream));
  ctx->ts1_zeroed = false;  // a restored state survives the next prologue
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// output products (Gen_Output_Vars)
// ---------------------------------------------------------------------------
int a3g_set_output_params(a3g_ctx *ctx, const double *z_cc, double cloudcon_thresh, double cloudload_thresh,
                          double depo_thresh, double deposit_density) {
  CTX_CHECK(ctx);
  if (!z_cc) return fail(A3G_ERR_ARG, "null z_cc");
  if (!(deposit_density > 0.0)) return fail(A3G_ERR_ARG, "deposit density must be positive");
  if (!ctx->ov_zcc) {
    A3G_CUDA(cudaMalloc((void **)&ctx->ov_zcc, sizeof(double) * ctx->grid.nz));
    ctx->bytes += sizeof(double) * ctx->grid.nz;
  }
  A3G_CUDA(cudaMemcpyAsync(ctx->ov_zcc, z_cc, sizeof(double) * ctx->grid.nz, cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->ov_cloudcon = cloudcon_thresh;
  ctx->ov_cloudload = cloudload_thresh;
  ctx->ov_depo = depo_thresh;
  ctx->ov_density = deposit_density;
  return A3G_OK;
}

static int ensure_ov(a3g_ctx *ctx) {
  if (ctx->ov_buf) return A3G_OK;
  const size_t n = (size_t)ctx->grid.nx * ctx->grid.ny;
  // 5 double planes, 2 int planes (as doubles' room), 2 arrival planes
  const size_t bytes = sizeof(double) * n * 9;
  if (cudaMalloc((void **)&ctx->ov_buf, bytes) != cudaSuccess) return fail(A3G_ERR_NOMEM, "output buffers");
  ctx->bytes += bytes;
  return a3g_output_reset(ctx);
}

int a3g_output_reset(a3g_ctx *ctx) {
  CTX_CHECK(ctx);
  if (!ctx->ov_buf) return ensure_ov(ctx);
  const size_t n = (size_t)ctx->grid.nx * ctx->grid.ny;
  std::vector<double> neg(2 * n, -1.0);
  A3G_CUDA(cudaMemcpyAsync(ctx->ov_buf + 7 * n, neg.data(), sizeof(double) * 2 * n, cudaMemcpyHostToDevice,
                           ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  return A3G_OK;
}

int a3g_vprofiles(a3g_ctx *ctx, int32_t npts, const int32_t *i_pts, const int32_t *j_pts, double *pr_ash,
                  int32_t *written) {
  CTX_CHECK(ctx);
  if (npts < 0 || (npts > 0 && (!i_pts || !j_pts || !pr_ash || !written)))
    return fail(A3G_ERR_ARG, "bad profile point arrays");
  if (npts == 0) return A3G_OK;
  const int nz = ctx->grid.nz;
  for (int p = 0; p < npts; p++)
    if (i_pts[p] < 1 || i_pts[p] > ctx->grid.nx || j_pts[p] < 1 || j_pts[p] > ctx->grid.ny)
      return fail(A3G_ERR_ARG, "profile point outside the grid");
  // doubles: results (nz*npts), then points and flags as int32 pairs
  const size_t need = (size_t)nz * npts + (size_t)npts * 2;
  if (need > ctx->vp_cap) {
    if (ctx->vp_buf) cudaFree(ctx->vp_buf);
    ctx->vp_buf = nullptr;
    if (cudaMalloc((void **)&ctx->vp_buf, need * sizeof(double)) != cudaSuccess)
      return fail(A3G_ERR_NOMEM, "profile buffer allocation failed");
    ctx->vp_cap = need;
  }
  double *out = ctx->vp_buf;
  int32_t *pts = reinterpret_cast<int32_t *>(ctx->vp_buf + (size_t)nz * npts);
  int32_t *flags = pts + 2 * (size_t)npts;
  std::vector<int32_t> hp(2 * (size_t)npts);
  for (int p = 0; p < npts; p++) { hp[2 * p] = i_pts[p]; hp[2 * p + 1] = j_pts[p]; }
  A3G_CUDA(cudaMemcpyAsync(pts, hp.data(), hp.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  int rc = launch_vprofiles(ctx, npts, pts, out, flags);
  if (rc) return rc;
  std::vector<double> ho((size_t)nz * npts);
  A3G_CUDA(cudaMemcpyAsync(ho.data(), out, ho.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  A3G_CUDA(cudaMemcpyAsync(written, flags, npts * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  A3G_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int p = 0; p < npts; p++)  // points below the threshold keep their previous profile
    if (written[p]) std::memcpy(pr_ash + (size_t)nz * p, ho.data() + (size_t)nz * p, nz * sizeof(double));
  return check_device_error(ctx);
}

int a3g_output_vars(a3g_ctx *ctx, double time, double *cloud_load, double *max_height, double *min_height,
                    double *max_conc, int32_t *mask_cloud, double *dep_thick, int32_t *mask_dep,
                    double *cloud_arrival, double *dep_arrival, double *areas) {
  CTX_CHECK(ctx);
  if (!ctx->have_geometry) return fail(A3G_ERR_STATE, "geometry not set");
  if (!ctx->ov_zcc) return fail(A3G_ERR_STATE, "a3g_set_output_params has not been called");
  int rc = ensure_ov(ctx);
  if (rc) return rc;
  const int nx = ctx->grid.nx, ny = ctx->grid.ny;
  const size_t n = (size_t)nx * ny;
  double *b = ctx->ov_buf;
  int32_t *mc = reinterpret_cast<int32_t *>(b + 5 * n);
  int32_t *md = mc + n;
  if ((rc = launch_output_vars(ctx, time, b, b + n, b + 2 * n, b + 3 * n, mc, b + 4 * n, md, b + 7 * n,
                               b + 8 * n)))
    return rc;
  // the host needs the loads and masks for the areas (sequential sums, reference order)
  std::vector<double> h_load(n), h_dep(n);
  std::vector<int32_t> h_mc(n), h_md(n);
  A3G_CUDA(cudaMemcpyAsync(h_load.data(), b, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  A3G_CUDA(cudaMemcpyAsync(h_mc.data(), mc, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  A3G_CUDA(cudaMemcpyAsync(h_md.data(), md, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  double *outs[] = {max_height, min_height, max_conc, dep_thick};
  for (int q = 0; q < 4; q++)
    if (outs[q])
      A3G_CUDA(cudaMemcpyAsync(outs[q], b + (q + 1) * n, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  if (cloud_arrival)
    A3G_CUDA(cudaMemcpyAsync(cloud_arrival, b + 7 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  if (dep_arrival)
    A3G_CUDA(cudaMemcpyAsync(dep_arrival, b + 8 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  if ((rc = sync_scalars(ctx))) return rc;
  if (cloud_load) std::memcpy(cloud_load, h_load.data(), sizeof(double) * n);
  if (mask_cloud) std::memcpy(mask_cloud, h_mc.data(), sizeof(int32_t) * n);
  if (mask_dep) std::memcpy(mask_dep, h_md.data(), sizeof(int32_t) * n);
  if (areas) {
    // DepositAreaCovered (:881-889), CloudArea (:1101), CloudLoadArea (:1157-1170)
    const Box &bx = ctx->box;
    auto o = [&](int i, int j) { return (size_t)(i - 1) + (size_t)nx * (j - 1); };
    double dep_area = 0.0, cloud_area = 0.0, la[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    static const double load_val[5] = {0.24, 1.0, 2.0, 4.0, 6.0};
    for (int i = 1; i <= nx; i++)
      for (int j = 1; j <= ny; j++)
        if (h_md[o(i, j)]) dep_area = dep_area + ctx->h_area[o(i, j)];
    for (int i = bx.imin; i <= bx.imax; i++)
      for (int j = bx.jmin; j <= bx.jmax; j++)
        if (h_mc[o(i, j)]) cloud_area = cloud_area + ctx->h_area[o(i, j)];
    for (int i = bx.imin; i <= bx.imax; i++)
      for (int j = bx.jmin; j <= bx.jmax; j++)
        for (int k = 0; k < 5; k++)
          if (h_load[o(i, j)] > load_val[k]) la[k] = la[k] + ctx->h_area[o(i, j)];
    areas[0] = cloud_area;
    areas[1] = dep_area;
    for (int k = 0; k < 5; k++) areas[2 + k] = la[k];
  }
  return A3G_OK;
}

}  // extern "C"
