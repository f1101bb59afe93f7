// a3g_inverse.cu -- source inversion through a whole run: the forward run
// with checkpoints under a device-memory budget, the discrete adjoint that
// reverses it, and the tangent-linear run.  No counterpart in the reference
// (Ash3d runs forward only).
//
// The control p(k, bin, g) (Fortran order (nz, nbins, ns), kg/h) is the
// erupted mass rate per model level, hourly bin and grain bin, inserted at
// the vent column as src/Ash3d.F90:428-431 inserts SourceNodeFlux:
// concen(ivent,jvent,k,g) += dt * p(k,bin,g) / kappa(ivent,jvent,k), bin =
// the hour the step starts in.  The observations are the unmasked column
// loads (CloudLoad, src/Output_Vars.f90:1061-1069) at the end of every hour
// and the deposit thickness (AshThicknessCalculator, :880-884) accumulated
// after a given hour; the misfit is
//   J = 1/2 sum_{h >= load_from} |L c(h) - y_h|^2 + 1/2 |T(D_end - D_from) - y_dep|^2.
//
// Run structure (the loop of src/Ash3d.F90:372-510 restricted to the
// transport): dt depends only on the winds, so a first pass forms the dt of
// every step (Adjust_DT every step, or FAST_DT's met-step dt interpolated;
// dt clipped to the next hour so that the observations fall on step ends)
// and the runs replay it.  Checkpoints are the state at the start of a step;
// their placement is binomial: reversing n steps with s free slots stores
// the state at the split k that minimises k + C(n-k, s-1) + C(k, s), the
// forward steps the reversal repeats (C(1, s) = 0, C(n, 0) = n(n-1)/2).  The
// first forward run stores the checkpoints of the recursion's rightmost
// path, so with a budget of n-1 slots nothing is recomputed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>
#include <vector>

#include "a3g_internal.cuh"

namespace a3g {

struct InvStep {
  int itime;    // 1-based step number (the toggles of AdvectHorz/DiffuseHorz)
  int hour;     // met interval (MR_iMetStep_Now)
  int bin;      // source bin: the hour the step starts in
  int ob;       // hour index (0-based) whose end this step reaches, or -1
  double time;  // time at the start of the step
  double dt;
  double frac;  // Interval_Frac
};

}  // namespace a3g

struct a3g_inv {
  a3g_inv_desc d;
  a3g_met_provider met;
  void *user;
  int nhours;
  std::vector<a3g::InvStep> steps;
  // device buffers
  double *dts;        // dt of every step
  double *p, *dp;     // control and its perturbation (nz, nbins, ns)
  double *grad;       // gradient (nz, nbins, ns)
  double *obs_load;   // y (nhours, ny, nx), i fastest
  double *obs_dep;    // y_dep (ny, nx)
  double *mod_load;   // L c at the hour ends
  double *mod_dep;    // T(D_end - D_from)
  double *dep_from;   // T(D_from)
  double *w_load;     // weights of the adjoint (residuals or the caller's)
  double *w_dep;
  double *tl0, *tl1, *tl_dep;  // tangent-linear state and deposit
  float *met_cache;   // every met step of the run on the device (or null)
  int met_cache_n;
  int slot_hour[3];   // met step each of the context's three met slots holds (-1: none)
  std::vector<double *> slots;
  size_t max_slots;
  double J;
  bool have_forward;
  long recomputed;    // forward steps repeated by the last reversal
  bool w_all;         // the adjoint's weights are the caller's: every observation counts
  double *outs_keep[6];
};

namespace a3g {

int cuda_fail(cudaError_t e, const char *what);
void set_error(const std::string &msg);

static int ifail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// c(ivent,jvent,k,g) += dt * p(k,bin,g) / kappa(ivent,jvent,k)
__global__ void k_inv_source(Layout L, int ivent, int jvent, const double *__restrict__ p, int bin, int nbins,
                             Geo3 kap, const double *__restrict__ dts, int n, double *__restrict__ c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // (k-1) + nz*g
  if (t >= L.nz * L.ns) return;
  const int k = t % L.nz + 1, g = t / L.nz;
  const double kv = kap.p[(long)(ivent + 1) * kap.si + (long)(jvent + 1) * kap.sj + (long)(k + 1) * kap.sk];
  const double flux = p[(long)(k - 1) + (long)L.nz * (bin + (long)nbins * g)] / kv;
  const long a = (long)g * L.PG + L.cell(ivent, jvent, k);
  c[a] = c[a] + dts[n] * flux;
}

// grad(k,bin,g) += dt * lam(ivent,jvent,k,g) / kappa(ivent,jvent,k)
__global__ void k_inv_grad(Layout L, int ivent, int jvent, const double *__restrict__ lam, Geo3 kap,
                           const double *__restrict__ dts, int n, int bin, int nbins, double *__restrict__ grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.nz * L.ns) return;
  const int k = t % L.nz + 1, g = t / L.nz;
  const double kv = kap.p[(long)(ivent + 1) * kap.si + (long)(jvent + 1) * kap.sj + (long)(k + 1) * kap.sk];
  const long o = (long)(k - 1) + (long)L.nz * (bin + (long)nbins * g);
  grad[o] = grad[o] + dts[n] * lam[(long)g * L.PG + L.cell(ivent, jvent, k)] / kv;
}

__global__ void k_set_dt(DevScalars *sc, const double *__restrict__ dts, int n) { sc->dt = dts[n]; }

// DepositThickness(i,j) = sum_g dep(i,j,g) * dz_vec(1) / KM2_2_M2 / DepositDensity * M_2_MM
// (src/Output_Vars.f90:880-884), unmasked; dep in the device's [g][j][i] order
__global__ void k_dep_thickness(int nx, int ny, int ns, const double *__restrict__ dep,
                                const double *__restrict__ dz_vec, double density, const double *__restrict__ sub,
                                double *__restrict__ out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nx * ny) return;
  double s = 0.0;
  for (int g = 0; g < ns; g++) s = s + dep[(long)g * nx * ny + t];
  double v = s * dz_vec[2] / 1.0e6 / density * 1.0e3;
  if (sub) v = v - sub[t];
  out[t] = v;
}

// lam_dep(g,j,i) = w(i,j) * dz_vec(1) / KM2_2_M2 / DepositDensity * M_2_MM (the transpose)
__global__ void k_adj_dep(int nx, int ny, int ns, const double *__restrict__ w, const double *__restrict__ dz_vec,
                          double density, double *__restrict__ lam_dep) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nx * ny * ns) return;
  lam_dep[t] = w[t % ((long)nx * ny)] * dz_vec[2] / 1.0e6 / density * 1.0e3;
}

// r = model - obs (the residual, the adjoint's weight)
__global__ void k_resid(long n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ r) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < n) r[t] = a[t] - b[t];
}

__global__ void k_interp_from(Layout L, const float *__restrict__ last, const float *__restrict__ next, long n,
                              double frac, double *__restrict__ vx, double *__restrict__ vy, double *__restrict__ vz) {
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

}  // namespace a3g

using namespace a3g;

// ---------------------------------------------------------------------------
// binomial checkpoint schedule
// ---------------------------------------------------------------------------
namespace {

struct Schedule {
  int S = 0;          // free slots (besides the state the reversal starts from)
  int N = 0;
  bool all = false;   // S >= N-1: every state fits, nothing is recomputed
  std::vector<long> cost;  // (n, s) -> forward steps repeated
  std::vector<int> split;  // (n, s) -> best first-segment length
  long &C(int n, int s) { return cost[(size_t)n * (S + 1) + s]; }
  int &K(int n, int s) { return split[(size_t)n * (S + 1) + s]; }
  void build(int n_max, int s_max) {
    N = n_max;
    S = std::max(s_max, 0);
    all = S >= N - 1;
    if (all) return;
    // the table costs about N^2*S/2 operations: fewer slots beyond that
    while (S > 1 && (double)N * N * S / 2.0 > 4.0e8) S--;
    cost.assign((size_t)(N + 1) * (S + 1), 0);
    split.assign((size_t)(N + 1) * (S + 1), 1);
    for (int n = 1; n <= N; n++) {
      C(n, 0) = (long)n * (n - 1) / 2;
      for (int s = 1; s <= S; s++) {
        if (n == 1) { C(n, s) = 0; continue; }
        if (s >= n - 1) { C(n, s) = n - 1; K(n, s) = 1; continue; }
        long best = -1;
        int bk = 1;
        for (int k = 1; k < n; k++) {
          const long c = k + C(n - k, s - 1) + C(k, s);
          if (best < 0 || c < best) { best = c; bk = k; }
        }
        C(n, s) = best;
        K(n, s) = bk;
      }
    }
  }
  int split_of(int n, int s) {
    if (s <= 0 || n <= 1 || all || s >= n - 1) return 1;
    return K(n, std::min(s, S));
  }
  long cost_of(int n, int s) {
    if (n <= 1) return 0;
    if (all || s >= n - 1) return n - 1;
    if (s <= 0) return (long)n * (n - 1) / 2;
    return C(n, std::min(s, S));
  }
};

}  // namespace

extern "C" int a3g_checkpoint_cost(int32_t nsteps, int32_t nslots, int64_t *recomputed, int32_t *first_split) {
  if (nsteps < 1 || nslots < 0 || !recomputed) {
    set_error("a3g_checkpoint_cost: need nsteps >= 1, nslots >= 0 and an output");
    return A3G_ERR_ARG;
  }
  Schedule sc;
  sc.build(nsteps, nslots);
  *recomputed = sc.cost_of(nsteps, nslots);
  if (first_split) *first_split = sc.split_of(nsteps, nslots);
  return A3G_OK;
}

// ---------------------------------------------------------------------------
// run pieces
// ---------------------------------------------------------------------------
namespace {

int met_hour(double time, int hour) {  // driver.met_hour (src/MesoInterpolater.f90:122-145)
  if (hour < 0) return (int)std::floor(time);
  return (time > hour + 1) ? hour + 1 : hour;
}

size_t level_bytes(const a3g_ctx *ctx) { return sizeof(double) * ctx->L.PG * ctx->L.ns; }

int dev_alloc(a3g_ctx *ctx, double **p, size_t n) {
  if (*p) return A3G_OK;
  if (cudaMalloc((void **)p, n * sizeof(double)) != cudaSuccess) return ifail(A3G_ERR_NOMEM, "inversion buffer allocation failed");
  ctx->bytes += n * sizeof(double);
  return cudaMemsetAsync(*p, 0, n * sizeof(double), ctx->stream) == cudaSuccess ? A3G_OK
                                                                             : ifail(A3G_ERR_CUDA, "memset");
}

// the met step `hour` from the provider into met slot `slot`
int upload_met(a3g_ctx *ctx, a3g_inv *v, int hour, int slot) {
  const float *a[3];
  if (v->met(v->user, hour, &a[0], &a[1], &a[2])) return ifail(A3G_ERR_ARG, "the met-step provider failed");
  const long n = ctx->met_n;
  for (int q = 0; q < 3; q++) {
    if (!a[q]) return ifail(A3G_ERR_ARG, "the met-step provider returned a null array");
    // a copy from pageable memory returns once the source has been staged,
    // so the provider may reuse its buffers after this call
    A3G_CUDA(cudaMemcpyAsync(ctx->met + (size_t)3 * n * slot + (size_t)q * n, a[q], sizeof(float) * n,
                             cudaMemcpyHostToDevice, ctx->stream));
  }
  v->slot_hour[slot] = hour;
  return A3G_OK;
}

// the met pair (hour, hour+1): its place in the cache, or the context's met
// slots, which keep the steps they hold: a run that moves on by one hour
// (forward) or back by one hour (the reversal) uploads one step, not two
int load_pair(a3g_ctx *ctx, a3g_inv *v, int hour, const float **last, const float **next) {
  const long n = ctx->met_n ? ctx->met_n : (long)ctx->grid.nx * ctx->grid.ny * ctx->grid.nz;
  if (v->met_cache && hour + 1 < v->met_cache_n) {
    *last = v->met_cache + (size_t)3 * n * hour;
    *next = v->met_cache + (size_t)3 * n * (hour + 1);
    return A3G_OK;
  }
  int rc;
  if (!ctx->met) {  // the slots do not exist yet: a3g_set_met_steps allocates them
    const float *a[3], *b[3];
    if (v->met(v->user, hour, &a[0], &a[1], &a[2]) || v->met(v->user, hour + 1, &b[0], &b[1], &b[2]))
      return ifail(A3G_ERR_ARG, "the met-step provider failed");
    if ((rc = a3g_set_met_steps(ctx, a[0], a[1], a[2], b[0], b[1], b[2]))) return rc;
    v->slot_hour[ctx->met_last] = hour;
    v->slot_hour[ctx->met_next] = hour + 1;
    v->slot_hour[ctx->met_spare] = -1;
  } else {
    const int want[2] = {hour, hour + 1};
    int at[2] = {-1, -1};
    for (int q = 0; q < 2; q++)
      for (int s = 0; s < 3; s++)
        if (v->slot_hour[s] == want[q]) at[q] = s;
    for (int q = 0; q < 2; q++) {
      if (at[q] >= 0) continue;
      int s = 0;  // a slot that holds neither step of the pair
      while (s < 3 && (s == at[1 - q] || v->slot_hour[s] == want[0] || v->slot_hour[s] == want[1])) s++;
      if (s == 3) return ifail(A3G_ERR_STATE, "no free met slot");  // cannot happen: one step is missing
      if ((rc = upload_met(ctx, v, want[q], s))) return rc;
      at[q] = s;
    }
    ctx->met_last = at[0];
    ctx->met_next = at[1];
    ctx->met_spare = 3 - at[0] - at[1];
  }
  *last = ctx->met + (size_t)3 * n * ctx->met_last;
  *next = ctx->met + (size_t)3 * n * ctx->met_next;
  return A3G_OK;
}

// The inversion's runs use the context's three met slots as their own: a
// prefetch still pending is waited for and dropped, and what the slots hold
// is forgotten, since other calls may have written them since the last run.
int claim_met_slots(a3g_ctx *ctx, a3g_inv *v) {
  for (int s = 0; s < 3; s++) v->slot_hour[s] = -1;
  if (ctx->met && ctx->met_prefetched) {
    A3G_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->met_copy_ev, 0));
    ctx->met_prefetched = false;
  }
  return A3G_OK;
}

int winds(a3g_ctx *ctx, a3g_inv *v, int hour, double frac) {
  const float *last, *next;
  int rc = load_pair(ctx, v, hour, &last, &next);
  if (rc) return rc;
  const Layout &L = ctx->L;
  const long n = (long)L.nx * L.ny * L.nz;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  tbegin(ctx, A3G_K_WINDS);
  k_interp_from<<<blocks, 256, 0, ctx->stream>>>(L, last, next, n, frac, ctx->vx, ctx->vy, ctx->vz);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  ctx->have_winds = true;
  return A3G_OK;
}

int set_step_dt(a3g_ctx *ctx, a3g_inv *v, int n) {
  k_set_dt<<<1, 1, 0, ctx->stream>>>(ctx->sc, v->dts, n);
  A3G_LAUNCH_CHECK(ctx);
  ctx->host_dt = v->steps[n].dt;
  ctx->dt_stamp++;
  return A3G_OK;
}

int add_source(a3g_ctx *ctx, a3g_inv *v, const double *p, int n, double *c) {
  const InvStep &s = v->steps[n];
  if (s.bin < 0 || s.bin >= v->d.nbins) return A3G_OK;
  const int m = ctx->L.nz * ctx->L.ns;
  tbegin(ctx, A3G_K_OTHER);
  k_inv_source<<<(m + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, v->d.ivent, v->d.jvent, p, s.bin, v->d.nbins,
                                                         ctx->kappa, v->dts, n, c);
  tend(ctx);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

// the sweeps of step n on ctx->c0 (Set_BC(1), AdvectHorz, AdvectVert,
// Set_BC(2), DiffuseHorz, DiffuseVert)
int sweeps(a3g_ctx *ctx, int itime) {
  int rc;
  const int iv = 1, jv = 1;
  if ((rc = a3g_set_bc(ctx, 1))) return rc;
  if ((rc = a3g_advect_horz(ctx, itime, iv, jv, 1))) return rc;
  if ((rc = a3g_advect_vert(ctx))) return rc;
  if (ctx->prm.use_diffusion) {
    if ((rc = a3g_set_bc(ctx, 2))) return rc;
    if ((rc = a3g_diffuse_horz(ctx, itime))) return rc;
    if ((rc = a3g_diffuse_vert(ctx))) return rc;
  }
  return A3G_OK;
}

void redirect_outflows(a3g_ctx *ctx, a3g_inv *v, bool on) {
  double **o[6] = {&ctx->out_yz1, &ctx->out_yz2, &ctx->out_xz1, &ctx->out_xz2, &ctx->out_xy1, &ctx->out_xy2};
  for (int q = 0; q < 6; q++) {
    if (on) {
      v->outs_keep[q] = *o[q];
      *o[q] = ctx->adj_face;
    } else {
      *o[q] = v->outs_keep[q];
    }
  }
}

// one forward step n from the state in c0 (the state at the step's start)
int advance(a3g_ctx *ctx, a3g_inv *v, int n) {
  const InvStep &s = v->steps[n];
  int rc;
  if ((rc = a3g_step_prologue(ctx))) return rc;
  if ((rc = winds(ctx, v, s.hour, s.frac))) return rc;
  if ((rc = set_step_dt(ctx, v, n))) return rc;
  if ((rc = add_source(ctx, v, v->p, n, ctx->c0))) return rc;
  return sweeps(ctx, s.itime);
}

int save_state(a3g_ctx *ctx, a3g_inv *v, int slot) {
  while ((int)v->slots.size() <= slot) {
    double *p = nullptr;
    if (cudaMalloc((void **)&p, level_bytes(ctx)) != cudaSuccess)
      return ifail(A3G_ERR_NOMEM, "checkpoint allocation failed (lower snapshot_bytes)");
    ctx->bytes += level_bytes(ctx);
    v->slots.push_back(p);
  }
  if (cudaMemcpyAsync(v->slots[slot], ctx->c0, level_bytes(ctx), cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
    return ifail(A3G_ERR_CUDA, "checkpoint copy failed");
  return A3G_OK;
}

int restore_state(a3g_ctx *ctx, a3g_inv *v, int slot) {
  if (cudaMemcpyAsync(ctx->c0, v->slots[slot], level_bytes(ctx), cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
    return ifail(A3G_ERR_CUDA, "checkpoint copy failed");
  ctx->ts1_zeroed = false;  // a restored state survives the next prologue
  return A3G_OK;
}

int thickness(a3g_ctx *ctx, const double *sub, double *out) {
  const long n = (long)ctx->grid.nx * ctx->grid.ny;
  k_dep_thickness<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(ctx->grid.nx, ctx->grid.ny, ctx->grid.ns,
                                                                         ctx->out_xy1, ctx->dz_vec, ctx->ov_density,
                                                                         sub, out);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int thickness_of(a3g_ctx *ctx, const double *dep, const double *sub, double *out) {
  const long n = (long)ctx->grid.nx * ctx->grid.ny;
  k_dep_thickness<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(ctx->grid.nx, ctx->grid.ny, ctx->grid.ns,
                                                                         dep, ctx->dz_vec, ctx->ov_density, sub, out);
  A3G_LAUNCH_CHECK(ctx);
  return A3G_OK;
}

int sync_check(a3g_ctx *ctx) {
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "inversion run");
  return check_device_error(ctx);
}

bool obs_used(const a3g_inv *v, int ob) {
  if (ob < 0 || ob >= v->nhours) return false;
  return v->w_all || ((v->d.misfit & A3G_MISFIT_LOAD) && ob >= v->d.load_from);
}

// the first step of the reversal window (the first step starting at or after adj_from)
int first_reversed(const a3g_inv *v) {
  int n = 0;
  while (n < (int)v->steps.size() && v->steps[n].time + 1.0e-9 < (double)v->d.adj_from) n++;
  return n;
}

bool dep_used(const a3g_inv *v) { return v->w_all || (v->d.misfit & A3G_MISFIT_DEPOSIT) != 0; }

// the step ends inside the deposit window (after hour dep_from)
bool in_dep_window(const a3g_inv *v, int n) { return v->steps[n].time + 1.0e-12 >= (double)v->d.dep_from; }

int inv_ready(a3g_ctx *ctx) {
  if (!ctx->inv) return ifail(A3G_ERR_STATE, "a3g_inv_setup has not been called");
  if (ctx->prm.fast_subgrid) return ifail(A3G_ERR_UNSUPPORTED, "the inversion needs fast_subgrid off");
  if (ctx->topo_on) return ifail(A3G_ERR_UNSUPPORTED, "the inversion does not cover the terrain terms");
  if (ctx->umb_on) return ifail(A3G_ERR_UNSUPPORTED, "the inversion covers the vent-column source only");
  return claim_met_slots(ctx, ctx->inv);
}

}  // namespace

void a3g::inv_free(a3g_ctx *ctx) {
  a3g_inv *v = ctx->inv;
  if (!v) return;
  double *bufs[] = {v->dts, v->p, v->dp, v->grad, v->obs_load, v->obs_dep, v->mod_load, v->mod_dep,
                    v->dep_from, v->w_load, v->w_dep, v->tl0, v->tl1, v->tl_dep};
  for (double *b : bufs) if (b) cudaFree(b);
  if (v->met_cache) cudaFree(v->met_cache);
  for (double *s : v->slots) if (s) cudaFree(s);
  delete v;
  ctx->inv = nullptr;
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" int a3g_inv_setup(a3g_ctx *ctx, const a3g_inv_desc *d, a3g_met_provider met, void *user,
                             const double *obs_load, const double *obs_dep) {
  if (!ctx || !d || !met) return ifail(A3G_ERR_ARG, "a3g_inv_setup: null argument");
  const int nx = ctx->grid.nx, ny = ctx->grid.ny, nz = ctx->grid.nz, ns = ctx->grid.ns;
  if (d->ivent < 1 || d->ivent > nx || d->jvent < 1 || d->jvent > ny) return ifail(A3G_ERR_ARG, "vent outside the grid");
  if (d->nbins < 1) return ifail(A3G_ERR_ARG, "need nbins >= 1");
  if (!(d->sim_hours >= 1.0) || d->sim_hours != std::floor(d->sim_hours))
    return ifail(A3G_ERR_ARG, "sim_hours must be a whole number of hours >= 1");
  if ((d->misfit & ~3) || !d->misfit) return ifail(A3G_ERR_ARG, "misfit must be A3G_MISFIT_LOAD and/or A3G_MISFIT_DEPOSIT");
  if (d->met_cache != 0 && d->met_cache != 1) return ifail(A3G_ERR_ARG, "met_cache must be 0 or 1");
  if ((d->misfit & A3G_MISFIT_LOAD) && !obs_load) return ifail(A3G_ERR_ARG, "column-load misfit without observations");
  if ((d->misfit & A3G_MISFIT_DEPOSIT) && !obs_dep) return ifail(A3G_ERR_ARG, "deposit misfit without an observation");
  if (d->dep_from < 0 || d->dep_from >= (int)d->sim_hours || d->load_from < 0 || d->adj_from < 0 ||
      d->adj_from >= (int)d->sim_hours)
    return ifail(A3G_ERR_ARG, "observation or reversal windows outside the run");
  int rc;
  if (ctx->prm.fast_subgrid) return ifail(A3G_ERR_UNSUPPORTED, "the inversion needs fast_subgrid off");
  if (ctx->topo_on) return ifail(A3G_ERR_UNSUPPORTED, "the inversion does not cover the terrain terms");
  if (!ctx->have_geometry || !ctx->have_vf) return ifail(A3G_ERR_STATE, "geometry and fall velocities must be set");
  if (ctx->prm.use_diffusion && !ctx->have_diffusivity) return ifail(A3G_ERR_STATE, "diffusivity not set");
  if (d->fast_dt && !ctx->have_vf_meso) return ifail(A3G_ERR_STATE, "FAST_DT needs a3g_set_fall_velocity_meso");
  inv_free(ctx);
  a3g_inv *v = new a3g_inv();
  ctx->inv = v;
  v->d = *d;
  v->met = met;
  v->user = user;
  v->nhours = (int)d->sim_hours;
  if ((rc = claim_met_slots(ctx, v))) return rc;
  if ((rc = a3g_adj_enable(ctx))) return rc;
  ctx->box = Box{1, nx, 1, ny, 1, nz};
  const size_t ctl = (size_t)nz * d->nbins * ns, plane = (size_t)nx * ny;
  if ((rc = dev_alloc(ctx, &v->p, ctl)) || (rc = dev_alloc(ctx, &v->dp, ctl)) || (rc = dev_alloc(ctx, &v->grad, ctl)) ||
      (rc = dev_alloc(ctx, &v->obs_load, plane * v->nhours)) || (rc = dev_alloc(ctx, &v->obs_dep, plane)) ||
      (rc = dev_alloc(ctx, &v->mod_load, plane * v->nhours)) || (rc = dev_alloc(ctx, &v->mod_dep, plane)) ||
      (rc = dev_alloc(ctx, &v->dep_from, plane)) || (rc = dev_alloc(ctx, &v->w_load, plane * v->nhours)) ||
      (rc = dev_alloc(ctx, &v->w_dep, plane)))
    return rc;
  if (obs_load)
    A3G_CUDA(cudaMemcpyAsync(v->obs_load, obs_load, sizeof(double) * plane * v->nhours, cudaMemcpyHostToDevice, ctx->stream));
  if (obs_dep) A3G_CUDA(cudaMemcpyAsync(v->obs_dep, obs_dep, sizeof(double) * plane, cudaMemcpyHostToDevice, ctx->stream));
  // every met step of the run on the device when they take at most a quarter
  // of the free memory
  {
    const long n3 = (long)nx * ny * nz;
    const int nmet = v->nhours + 2;
    const size_t need = sizeof(float) * 3 * (size_t)n3 * nmet;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if (d->met_cache == 0 && need <= fr / 4 && cudaMalloc((void **)&v->met_cache, need) == cudaSuccess) {
      ctx->bytes += need;
      v->met_cache_n = nmet;
      for (int h = 0; h < nmet; h++) {
        const float *a[3];
        if (met(user, h, &a[0], &a[1], &a[2])) return ifail(A3G_ERR_ARG, "the met-step provider failed");
        for (int q = 0; q < 3; q++)
          A3G_CUDA(cudaMemcpyAsync(v->met_cache + (size_t)3 * n3 * h + (size_t)q * n3, a[q], sizeof(float) * n3,
                                   cudaMemcpyHostToDevice, ctx->stream));
        A3G_CUDA(cudaStreamSynchronize(ctx->stream));  // the provider may reuse its buffers
      }
    }
  }
  // ---- the dt of every step (winds only) ----
  const double T = d->sim_hours;
  double time = 0.0;
  int hour = -1, itime = 0;
  while (time < T - 1.0e-12) {
    InvStep s;
    s.itime = ++itime;
    const int h = met_hour(time, hour);
    const bool load = h != hour;
    s.hour = h;
    s.frac = time - h;
    s.time = time;
    s.bin = (int)std::floor(time + 1.0e-12);
    const double nwt = std::floor(time + 1.0e-12) + 1.0;  // the next hour: observations on step ends
    if ((rc = winds(ctx, v, h, s.frac))) return rc;
    double dt = 0.0;
    if (d->fast_dt) {
      if (load) {
        // Adjust_DT(mesostep=.true.) at the met-step load (src/MesoInterpolater.f90:142-150,
        // 187-195): the first load takes the last step then the next one
        const float *last, *next;
        if ((rc = load_pair(ctx, v, h, &last, &next))) return rc;
        if (hour < 0) {
          if ((rc = launch_cfl_maxima_meso_ptr(ctx, last))) return rc;
          if ((rc = launch_dt_from_maxima(ctx, ctx->n_gs_aloft, time, nwt, T, 1))) return rc;
        }
        if ((rc = launch_cfl_maxima_meso_ptr(ctx, next))) return rc;
        if ((rc = launch_dt_from_maxima(ctx, ctx->n_gs_aloft, time, nwt, T, 3))) return rc;
      }
      if ((rc = a3g_fast_dt_async(ctx, s.frac, time, nwt, T))) return rc;
      if ((rc = a3g_wait_dt(ctx, &dt))) return rc;
    } else {
      if ((rc = a3g_adjust_dt(ctx, time, nwt, T, &dt))) return rc;
    }
    hour = h;
    s.dt = dt;
    time = time + dt;
    s.ob = -1;
    if (std::fabs(time - std::round(time)) < 1.0e-9 && std::round(time) >= 1.0) s.ob = (int)std::lround(time) - 1;
    v->steps.push_back(s);
    if (itime > 10000000) return ifail(A3G_ERR_STATE, "the run does not end (dt too small)");
  }
  if ((rc = dev_alloc(ctx, &v->dts, v->steps.size()))) return rc;
  std::vector<double> h_dt(v->steps.size());
  for (size_t q = 0; q < v->steps.size(); q++) h_dt[q] = v->steps[q].dt;
  A3G_CUDA(cudaMemcpyAsync(v->dts, h_dt.data(), sizeof(double) * h_dt.size(), cudaMemcpyHostToDevice, ctx->stream));
  // ---- checkpoint budget ----
  size_t fr = 0, tot = 0;
  A3G_CUDA(cudaMemGetInfo(&fr, &tot));
  double budget = d->snapshot_bytes;
  if (!(budget > 0.0)) budget = (double)fr - 2.0 * 1073741824.0;  // leave 2 GiB
  const double lb = (double)level_bytes(ctx);
  long slots = (long)std::floor(budget / lb);
  if (slots < 1) return ifail(A3G_ERR_NOMEM, "the snapshot budget holds no checkpoint");
  v->max_slots = (size_t)std::min<long>(slots, (long)v->steps.size() - first_reversed(v));
  return sync_check(ctx);
}

namespace {

// the forward run: zero state, every step, the observations; stores the
// states of `keep` (step indices, ascending) in slots 0, 1, ...
int forward_run(a3g_ctx *ctx, a3g_inv *v, const std::vector<int> &keep) {
  const Layout &L = ctx->L;
  int rc;
  A3G_CUDA(cudaMemsetAsync(ctx->c0, 0, level_bytes(ctx), ctx->stream));
  A3G_CUDA(cudaMemsetAsync(ctx->c1, 0, level_bytes(ctx), ctx->stream));
  double *outs[6] = {ctx->out_yz1, ctx->out_yz2, ctx->out_xz1, ctx->out_xz2, ctx->out_xy1, ctx->out_xy2};
  const size_t osz[6] = {(size_t)L.ns * L.ny * L.nz, (size_t)L.ns * L.ny * L.nz, (size_t)L.ns * L.nx * L.nz,
                         (size_t)L.ns * L.nx * L.nz, (size_t)L.ns * L.nx * L.ny, (size_t)L.ns * L.nx * L.ny};
  for (int q = 0; q < 6; q++) A3G_CUDA(cudaMemsetAsync(outs[q], 0, osz[q] * sizeof(double), ctx->stream));
  ctx->ts1_zeroed = false;
  const size_t plane = (size_t)ctx->grid.nx * ctx->grid.ny;
  A3G_CUDA(cudaMemsetAsync(v->dep_from, 0, plane * sizeof(double), ctx->stream));
  size_t kp = 0;
  for (int n = 0; n < (int)v->steps.size(); n++) {
    if (v->d.dep_from > 0 && std::fabs(v->steps[n].time - v->d.dep_from) < 1.0e-9)
      if ((rc = thickness(ctx, nullptr, v->dep_from))) return rc;  // T(D_from)
    if (kp < keep.size() && keep[kp] == n) {  // the state at the step's start
      if ((rc = save_state(ctx, v, (int)kp))) return rc;
      kp++;
    }
    if ((rc = advance(ctx, v, n))) return rc;
    const int ob = v->steps[n].ob;
    if (ob >= 0 && ob < v->nhours) {
      if ((rc = launch_cloud_load(ctx, ctx->c0, v->mod_load + plane * ob))) return rc;
    }
  }
  if ((rc = thickness(ctx, v->d.dep_from > 0 ? v->dep_from : nullptr, v->mod_dep))) return rc;
  return A3G_OK;
}

double host_misfit(a3g_ctx *ctx, a3g_inv *v, int *rc) {
  const size_t plane = (size_t)ctx->grid.nx * ctx->grid.ny;
  std::vector<double> m(plane * v->nhours), y(plane * v->nhours);
  double J = 0.0;
  *rc = A3G_OK;
  if (v->d.misfit & A3G_MISFIT_LOAD) {
    if (cudaMemcpy(m.data(), v->mod_load, sizeof(double) * m.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(y.data(), v->obs_load, sizeof(double) * y.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      *rc = ifail(A3G_ERR_CUDA, "misfit copy failed");
      return 0.0;
    }
    for (int ob = v->d.load_from; ob < v->nhours; ob++)
      for (size_t t = 0; t < plane; t++) {
        const double r = m[plane * ob + t] - y[plane * ob + t];
        J += 0.5 * (r * r);
      }
  }
  if (v->d.misfit & A3G_MISFIT_DEPOSIT) {
    if (cudaMemcpy(m.data(), v->mod_dep, sizeof(double) * plane, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(y.data(), v->obs_dep, sizeof(double) * plane, cudaMemcpyDeviceToHost) != cudaSuccess) {
      *rc = ifail(A3G_ERR_CUDA, "misfit copy failed");
      return 0.0;
    }
    for (size_t t = 0; t < plane; t++) {
      const double r = m[t] - y[t];
      J += 0.5 * (r * r);
    }
  }
  return J;
}

// the checkpoints the first forward run stores: the rightmost path of the
// reversal's recursion over [0, N) with S free slots
std::vector<int> spine(Schedule &sc, int N, int S) {
  std::vector<int> keep{0};
  int a = 0, s = S;
  while (N - a > 1 && s > 0) {
    const int m = a + sc.split_of(N - a, s);
    keep.push_back(m);
    a = m;
    s--;
  }
  return keep;
}

struct Reverser {
  a3g_ctx *ctx;
  a3g_inv *v;
  Schedule sc;
  std::vector<int> slot_step;  // step whose state each slot holds (-1: free)
  bool dep_on = false;
  long recomputed = 0;

  int slot_of(int step) {
    for (size_t q = 0; q < slot_step.size(); q++)
      if (slot_step[q] == step) return (int)q;
    return -1;
  }
  int free_slot() {
    for (size_t q = 0; q < slot_step.size(); q++)
      if (slot_step[q] < 0) return (int)q;
    slot_step.push_back(-1);
    return (int)slot_step.size() - 1;
  }
  // state of step a (in a slot) advanced to step t, into c0; outflows to scratch
  int state_at(int a, int t) {
    int rc;
    if ((rc = restore_state(ctx, v, slot_of(a)))) return rc;
    redirect_outflows(ctx, v, true);
    for (int n = a; n < t && !rc; n++) {
      rc = advance(ctx, v, n);
      recomputed++;
    }
    redirect_outflows(ctx, v, false);
    return rc;
  }
  // the reverse of step n with its start state in c0
  int reverse_step(int n) {
    const InvStep &s = v->steps[n];
    const size_t plane = (size_t)ctx->grid.nx * ctx->grid.ny;
    int rc;
    if ((rc = winds(ctx, v, s.hour, s.frac))) return rc;
    if ((rc = set_step_dt(ctx, v, n))) return rc;
    if ((rc = add_source(ctx, v, v->p, n, ctx->c0))) return rc;  // the post-source state adj_step expects
    if (obs_used(v, s.ob) && (rc = launch_adj_cloud_load(ctx, v->w_load + plane * s.ob, ctx->lam0))) return rc;
    if (dep_used(v)) {
      const bool on = in_dep_window(v, n);
      if (on != dep_on) {
        const long m = (long)plane * ctx->grid.ns;
        if (on)
          k_adj_dep<<<(unsigned)((m + 255) / 256), 256, 0, ctx->stream>>>(ctx->grid.nx, ctx->grid.ny, ctx->grid.ns,
                                                                          v->w_dep, ctx->dz_vec, ctx->ov_density,
                                                                          ctx->lam_dep);
        else
          A3G_CUDA(cudaMemsetAsync(ctx->lam_dep, 0, sizeof(double) * m, ctx->stream));
        A3G_LAUNCH_CHECK(ctx);
        dep_on = on;
      }
    }
    if ((rc = a3g_adj_step(ctx, s.itime))) return rc;
    if (s.bin >= 0 && s.bin < v->d.nbins) {
      const int m = ctx->L.nz * ctx->L.ns;
      k_inv_grad<<<(m + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, v->d.ivent, v->d.jvent, ctx->lam0, ctx->kappa,
                                                           v->dts, n, s.bin, v->d.nbins, v->grad);
      A3G_LAUNCH_CHECK(ctx);
    }
    return A3G_OK;
  }
  // reverses steps a..b-1; the state of step a is in a slot; s free slots
  int reverse(int a, int b, int s) {
    int rc;
    if (b - a == 1) {
      if ((rc = state_at(a, a))) return rc;
      return reverse_step(a);
    }
    if (s <= 0) {
      for (int t = b - 1; t >= a; t--) {
        if ((rc = state_at(a, t))) return rc;
        if ((rc = reverse_step(t))) return rc;
      }
      return A3G_OK;
    }
    const int m = a + sc.split_of(b - a, s);
    const bool had = slot_of(m) >= 0;  // stored by the first forward run
    if (!had) {
      if ((rc = state_at(a, m))) return rc;  // the state at m's start
      const int q = free_slot();
      if ((rc = save_state(ctx, v, q))) return rc;
      slot_step[q] = m;
    }
    if ((rc = reverse(m, b, s - 1))) return rc;
    slot_step[slot_of(m)] = -1;
    return reverse(a, m, s);
  }
};

}  // namespace

extern "C" int a3g_forward_checkpointed(a3g_ctx *ctx, const double *p, double *J_out, int32_t *nsteps) {
  if (!ctx || !p) return ifail(A3G_ERR_ARG, "a3g_forward_checkpointed: null argument");
  int rc = inv_ready(ctx);
  if (rc) return rc;
  a3g_inv *v = ctx->inv;
  const size_t ctl = (size_t)ctx->grid.nz * v->d.nbins * ctx->grid.ns;
  A3G_CUDA(cudaMemcpyAsync(v->p, p, sizeof(double) * ctl, cudaMemcpyHostToDevice, ctx->stream));
  ctx->box = Box{1, ctx->grid.nx, 1, ctx->grid.ny, 1, ctx->grid.nz};
  const int N = (int)v->steps.size(), n0 = first_reversed(v);
  Schedule sc;
  sc.build(N - n0, (int)v->max_slots - 1);
  std::vector<int> keep = spine(sc, N - n0, (int)v->max_slots - 1);
  for (int &k : keep) k += n0;
  if ((rc = forward_run(ctx, v, keep))) return rc;
  if ((rc = sync_check(ctx))) return rc;
  v->J = host_misfit(ctx, v, &rc);
  if (rc) return rc;
  v->have_forward = true;
  if (J_out) *J_out = v->J;
  if (nsteps) *nsteps = N;
  return A3G_OK;
}

extern "C" int a3g_adjoint(a3g_ctx *ctx, const double *w_load, const double *w_dep, double *grad) {
  if (!ctx || !grad) return ifail(A3G_ERR_ARG, "a3g_adjoint: null argument");
  int rc = inv_ready(ctx);
  if (rc) return rc;
  a3g_inv *v = ctx->inv;
  if (!v->have_forward) return ifail(A3G_ERR_STATE, "a3g_forward_checkpointed has not run");
  const size_t plane = (size_t)ctx->grid.nx * ctx->grid.ny;
  const long nl = (long)plane * v->nhours;
  // the adjoint's weights: the caller's (every observation), or the residuals
  // of the misfit's terms
  if ((w_load == nullptr) != (w_dep == nullptr))
    return ifail(A3G_ERR_ARG, "a3g_adjoint: give both weights or neither");
  v->w_all = w_load != nullptr;
  if (w_load)
    A3G_CUDA(cudaMemcpyAsync(v->w_load, w_load, sizeof(double) * nl, cudaMemcpyHostToDevice, ctx->stream));
  else
    k_resid<<<(unsigned)((nl + 255) / 256), 256, 0, ctx->stream>>>(nl, v->mod_load, v->obs_load, v->w_load);
  if (w_dep)
    A3G_CUDA(cudaMemcpyAsync(v->w_dep, w_dep, sizeof(double) * plane, cudaMemcpyHostToDevice, ctx->stream));
  else
    k_resid<<<(unsigned)((plane + 255) / 256), 256, 0, ctx->stream>>>((long)plane, v->mod_dep, v->obs_dep, v->w_dep);
  A3G_LAUNCH_CHECK(ctx);
  if ((rc = a3g_adj_zero(ctx))) return rc;
  const size_t ctl = (size_t)ctx->grid.nz * v->d.nbins * ctx->grid.ns;
  A3G_CUDA(cudaMemsetAsync(v->grad, 0, sizeof(double) * ctl, ctx->stream));
  ctx->box = Box{1, ctx->grid.nx, 1, ctx->grid.ny, 1, ctx->grid.nz};
  const int N = (int)v->steps.size(), n0 = first_reversed(v);
  Reverser R;
  R.ctx = ctx;
  R.v = v;
  R.sc.build(N - n0, (int)v->max_slots - 1);
  std::vector<int> keep = spine(R.sc, N - n0, (int)v->max_slots - 1);
  for (int &k : keep) k += n0;
  R.slot_step.assign(keep.begin(), keep.end());
  rc = R.reverse(n0, N, (int)v->max_slots - 1);
  if (rc) return rc;
  v->recomputed = R.recomputed;
  A3G_CUDA(cudaMemcpyAsync(grad, v->grad, sizeof(double) * ctl, cudaMemcpyDeviceToHost, ctx->stream));
  // the forward state is the first step's start now; mark the run as spent
  v->have_forward = false;
  return sync_check(ctx);
}

extern "C" int a3g_inv_observations(a3g_ctx *ctx, double *loads, double *dep, int64_t *stats) {
  if (!ctx) return ifail(A3G_ERR_ARG, "null context");
  if (!ctx->inv) return ifail(A3G_ERR_STATE, "a3g_inv_setup has not been called");
  a3g_inv *v = ctx->inv;
  const size_t plane = (size_t)ctx->grid.nx * ctx->grid.ny;
  if (loads)
    A3G_CUDA(cudaMemcpyAsync(loads, v->mod_load, sizeof(double) * plane * v->nhours, cudaMemcpyDeviceToHost, ctx->stream));
  if (dep) A3G_CUDA(cudaMemcpyAsync(dep, v->mod_dep, sizeof(double) * plane, cudaMemcpyDeviceToHost, ctx->stream));
  if (stats) {
    stats[0] = (int64_t)v->steps.size();
    stats[1] = (int64_t)v->max_slots;
    stats[2] = (int64_t)v->recomputed;
    stats[3] = (int64_t)v->steps.size() - first_reversed(v);
  }
  return sync_check(ctx);
}

extern "C" int a3g_tangent_linear(a3g_ctx *ctx, const double *p, const double *dp, double *dloads, double *ddep) {
  if (!ctx || !p || !dp) return ifail(A3G_ERR_ARG, "a3g_tangent_linear: null argument");
  int rc = inv_ready(ctx);
  if (rc) return rc;
  a3g_inv *v = ctx->inv;
  const Layout &L = ctx->L;
  const size_t lev = level_bytes(ctx);
  const size_t plane = (size_t)ctx->grid.nx * ctx->grid.ny;
  const size_t ctl = (size_t)ctx->grid.nz * v->d.nbins * ctx->grid.ns;
  if ((rc = dev_alloc(ctx, &v->tl0, lev / sizeof(double))) || (rc = dev_alloc(ctx, &v->tl1, lev / sizeof(double))) ||
      (rc = dev_alloc(ctx, &v->tl_dep, plane * ctx->grid.ns)))
    return rc;
  A3G_CUDA(cudaMemcpyAsync(v->p, p, sizeof(double) * ctl, cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaMemcpyAsync(v->dp, dp, sizeof(double) * ctl, cudaMemcpyHostToDevice, ctx->stream));
  A3G_CUDA(cudaMemsetAsync(ctx->c0, 0, lev, ctx->stream));
  A3G_CUDA(cudaMemsetAsync(ctx->c1, 0, lev, ctx->stream));
  A3G_CUDA(cudaMemsetAsync(v->tl0, 0, lev, ctx->stream));
  A3G_CUDA(cudaMemsetAsync(v->tl1, 0, lev, ctx->stream));
  A3G_CUDA(cudaMemsetAsync(v->tl_dep, 0, sizeof(double) * plane * ctx->grid.ns, ctx->stream));
  A3G_CUDA(cudaMemsetAsync(v->mod_load, 0, sizeof(double) * plane * v->nhours, ctx->stream));  // d(L c)
  A3G_CUDA(cudaMemsetAsync(v->dep_from, 0, sizeof(double) * plane, ctx->stream));
  ctx->ts1_zeroed = false;
  ctx->box = Box{1, ctx->grid.nx, 1, ctx->grid.ny, 1, ctx->grid.nz};
  v->have_forward = false;  // the buffers now hold perturbations
  redirect_outflows(ctx, v, true);  // the state's own outflows are not needed
  // the perturbation's sweeps: advection by the tangent-linear kernels
  // (branches from the state entering each sweep), diffusion by the forward
  // kernels themselves (linear)
  auto tl_swap = [&]() { std::swap(v->tl0, v->tl1); };
  auto diffuse_tl = [&](auto fn) -> int {
    double *c0 = ctx->c0, *c1 = ctx->c1;
    ctx->c0 = v->tl0;
    ctx->c1 = v->tl1;
    int r = fn();
    v->tl0 = ctx->c0;
    v->tl1 = ctx->c1;
    ctx->c0 = c0;
    ctx->c1 = c1;
    return r;
  };
  for (int n = 0; n < (int)v->steps.size() && !rc; n++) {
    const InvStep &s = v->steps[n];
    if (v->d.dep_from > 0 && std::fabs(s.time - v->d.dep_from) < 1.0e-9)
      if ((rc = thickness_of(ctx, v->tl_dep, nullptr, v->dep_from))) break;
    if ((rc = a3g_step_prologue(ctx))) break;
    if ((rc = winds(ctx, v, s.hour, s.frac))) break;
    if ((rc = set_step_dt(ctx, v, n))) break;
    if ((rc = add_source(ctx, v, v->p, n, ctx->c0))) break;
    if ((rc = add_source(ctx, v, v->dp, n, v->tl0))) break;
    const int first = (s.itime % 2 == 0) ? 1 : 0;  // AdvectHorz: even y then x
    for (int q = 0; q < 2 && !rc; q++) {
      const int dir = (q == 0) ? first : 1 - first;
      if ((rc = launch_tl_advect(ctx, dir, ctx->c0, v->tl0, v->tl1, nullptr))) break;
      tl_swap();
      rc = (dir == 0) ? launch_advect_x(ctx) : launch_advect_y(ctx);
    }
    if (rc) break;
    if ((rc = launch_tl_advect(ctx, 2, ctx->c0, v->tl0, v->tl1, v->tl_dep))) break;
    tl_swap();
    if ((rc = launch_advect_z(ctx))) break;
    ctx->ts1_zeroed = false;
    if (ctx->prm.use_diffusion) {
      if ((rc = a3g_diffuse_horz(ctx, s.itime))) break;
      if ((rc = diffuse_tl([&]() { return a3g_diffuse_horz(ctx, s.itime); }))) break;
      if ((rc = a3g_diffuse_vert(ctx))) break;
      if ((rc = diffuse_tl([&]() { return a3g_diffuse_vert(ctx); }))) break;
    }
    if (s.ob >= 0 && s.ob < v->nhours && (rc = launch_cloud_load(ctx, v->tl0, v->mod_load + plane * s.ob))) break;
  }
  redirect_outflows(ctx, v, false);
  if (rc) return rc;
  if ((rc = thickness_of(ctx, v->tl_dep, v->d.dep_from > 0 ? v->dep_from : nullptr, v->mod_dep))) return rc;
  if (dloads)
    A3G_CUDA(cudaMemcpyAsync(dloads, v->mod_load, sizeof(double) * plane * v->nhours, cudaMemcpyDeviceToHost, ctx->stream));
  if (ddep) A3G_CUDA(cudaMemcpyAsync(ddep, v->mod_dep, sizeof(double) * plane, cudaMemcpyDeviceToHost, ctx->stream));
  (void)L;
  return sync_check(ctx);
}
