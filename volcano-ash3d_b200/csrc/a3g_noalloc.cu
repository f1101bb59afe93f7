// a3g_noalloc.cu -- mass-aloft reduction that allocates no device memory.
//
// Some callers cannot allocate device memory when they need this sum: an
// operational forecast host that reserves all GPU memory at start-up and
// forbids allocation afterwards (so a long run cannot fail part-way with an
// out-of-memory error), or a host that hands the library device buffers from
// its own memory manager and keeps allocation to itself.
// a3g_mass_aloft_noalloc serves them: it computes the per-grain airborne
// mass sum(c*kappa) over the interior cells, with the same blocking and
// double-double accumulation as the context path (a3g_timestep_totals), but
// keeps its per-block partial sums in the file-scope device array below
// instead of a buffer obtained from cudaMalloc.  It launches kernels, so it
// is called from ordinary host code (CUDA forbids CUDA calls inside a stream
// callback or host function).
//
// Limits and sharing: the array holds A3G_NOALLOC_MAX_GRAINS grains x
// NOALLOC_BLOCKS blocks x 2 doubles (about 296 KiB) on every device that
// loads this library, for as long as the process lives.  Every block
// overwrites its own slot before the final pass reads it, so nothing in the
// array has to start at zero; the array keeps the last call's contents, and
// two calls whose kernels overlap on the same device race on it.
//
// The array's device address is looked up once per device and cached for the
// life of the process.  A cudaDeviceReset (or any other reset of the primary
// context) unloads the module and leaves that cached address stale, so a
// process that resets a device must not call this entry point on it again.
#include <mutex>

#include "a3g_internal.cuh"

#define A3G_NOALLOC_MAX_GRAINS 64
#define A3G_NOALLOC_MAX_DEVICES 64

namespace a3g {
namespace noalloc {

constexpr int NOALLOC_BLOCKS = 296;

// per-block partial sums: [grain][block][hi, lo]
static __device__ __align__(256) double g_partials[A3G_NOALLOC_MAX_GRAINS * NOALLOC_BLOCKS * 2];

struct DDn {
  double hi, lo;
};
__device__ __forceinline__ DDn add(DDn a, double b) {  // TwoSum accumulate
  const double s = a.hi + b;
  const double bb = s - a.hi;
  const double err = (a.hi - (s - bb)) + (b - bb);
  return DDn{s, a.lo + err};
}
__device__ __forceinline__ DDn add(DDn a, DDn b) {
  DDn r = add(a, b.hi);
  r.lo = r.lo + b.lo;
  return r;
}

__global__ void __launch_bounds__(256) k_mass_partial(const double *__restrict__ conc,
                                                      const double *__restrict__ kappa, int nx, int ny,
                                                      int nz, long pitch, double *__restrict__ part) {
  const int g = blockIdx.y;
  __shared__ double sh[2][8];
  const long n = (long)nx * ny * nz;
  const double *cg = conc + (long)g * pitch * ny * nz;
  DDn acc = {0.0, 0.0};
  const long nrow = n / nx;  // rows (j,k), r = (k-1)*ny + (j-1)
  for (long r = blockIdx.x; r < nrow; r += gridDim.x)
    for (int i = threadIdx.x; i < nx; i += blockDim.x) acc = add(acc, cg[r * pitch + i] * kappa[r * nx + i]);
  for (int o = 16; o > 0; o >>= 1) {
    DDn other;
    other.hi = __shfl_xor_sync(0xffffffffu, acc.hi, o);
    other.lo = __shfl_xor_sync(0xffffffffu, acc.lo, o);
    acc = add(acc, other);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[0][w] = acc.hi;
    sh[1][w] = acc.lo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    DDn s = {0.0, 0.0};
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s = add(s, DDn{sh[0][q], sh[1][q]});
    const long o = ((long)g * gridDim.x + blockIdx.x) * 2;
    part[o] = s.hi;
    part[o + 1] = s.lo;
  }
}

__global__ void k_mass_final(int ns, int nblk, const double *__restrict__ part, double *__restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ns) return;
  DDn s = {0.0, 0.0};
  for (int b = 0; b < nblk; b++) {
    const long o = ((long)g * nblk + b) * 2;
    s = add(s, DDn{part[o], part[o + 1]});
  }
  out[g] = s.hi + s.lo;
}

// Device address of g_partials, looked up once per device (with that device
// current) on the first call there.
static std::mutex g_mu;
static double *g_addr[A3G_NOALLOC_MAX_DEVICES];

static int scratch_for(int device, double **out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_partials)");
    g_addr[device] = static_cast<double *>(p);
  }
  *out = g_addr[device];
  return A3G_OK;
}

}  // namespace noalloc
}  // namespace a3g

extern "C" int a3g_mass_aloft_noalloc(int device, const double *conc, const double *kappa, int32_t nx,
                                      int32_t ny, int32_t nz, int32_t ns, int64_t row_pitch,
                                      double *mass_out, void *stream) {
  using namespace a3g::noalloc;
  if (!conc || !kappa || !mass_out) {
    a3g::set_error("a3g_mass_aloft_noalloc: null pointer");
    return A3G_ERR_ARG;
  }
  if (nx < 1 || ny < 1 || nz < 1 || ns < 1 || row_pitch < nx) {
    a3g::set_error("a3g_mass_aloft_noalloc: need nx, ny, nz, ns >= 1 and row_pitch >= nx");
    return A3G_ERR_ARG;
  }
  if (ns > A3G_NOALLOC_MAX_GRAINS) {
    a3g::set_error("a3g_mass_aloft_noalloc: ns exceeds the 64 grain bins its fixed scratch array holds");
    return A3G_ERR_ARG;
  }
  if (device < 0 || device >= A3G_NOALLOC_MAX_DEVICES) {
    a3g::set_error("a3g_mass_aloft_noalloc: device ordinal out of range");
    return A3G_ERR_ARG;
  }
  // the launches need `device` current; the caller's current device is put
  // back before returning, on every path
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) return a3g::cuda_fail(e, "cudaGetDevice");
  if (prev != device) {
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return a3g::cuda_fail(e, "cudaSetDevice");
  }
  int rc = A3G_OK;
  double *part = nullptr;
  rc = scratch_for(device, &part);
  if (rc == A3G_OK) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_mass_partial<<<dim3(NOALLOC_BLOCKS, ns), 256, 0, s>>>(conc, kappa, nx, ny, nz, (long)row_pitch, part);
    e = cudaGetLastError();
    if (e != cudaSuccess) rc = a3g::cuda_fail(e, "k_mass_partial launch");
  }
  if (rc == A3G_OK) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_mass_final<<<(ns + 63) / 64, 64, 0, s>>>(ns, NOALLOC_BLOCKS, part, mass_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) rc = a3g::cuda_fail(e, "k_mass_final launch");
  }
  if (prev != device) {
    e = cudaSetDevice(prev);
    if (e != cudaSuccess && rc == A3G_OK) rc = a3g::cuda_fail(e, "cudaSetDevice (restoring the caller's device)");
  }
  return rc;
}
