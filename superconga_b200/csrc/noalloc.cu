// Allocation-free variant of the vector-potential Poisson solve.
//
// Some callers cannot call cudaMalloc: for example a plugin that runs inside a
// framework which has already reserved the device memory for its own pool and
// hands the plugin only the buffers it owns, or a service that fixes its
// device-memory footprint at start-up and forbids allocation afterwards.  For
// them sc_poisson_noalloc solves A = -h^2 s sum_k (+/-) T_k (j - <j>) T_k with
// caller-owned inputs and output, and keeps its intermediates (the mean-free
// current and the two Toeplitz passes of one filter) in a fixed device array
// of this file instead of allocating.
//
// The array is a file-scope __device__ array of NOALLOC_SCRATCH_BYTES (24 MiB):
// every GPU that loads the library holds it until the process exits, and every
// call shares it.  The array keeps the last call's contents; each call
// overwrites everything it later reads, so nothing relies on them.  Calls whose
// work overlaps on the GPU (different streams, or different host threads on
// the same device) race on the array and must be ordered by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/scb200.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(24) << 20;
constexpr size_t NOALLOC_SCRATCH_DOUBLES = NOALLOC_SCRATCH_BYTES / sizeof(double);
constexpr int NA_REDUCE_BLOCKS = 64;
constexpr int NA_THREADS = 256;
constexpr int NA_PT = 32;

__device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Device address of g_noalloc_scratch, looked up once per device and CUDA
// context.  The context is part of the key because the array moves when the
// device's context is destroyed and created again (cudaDeviceReset, or the
// primary context released and retained): the module is then reloaded and the
// old address is no longer valid.
std::mutex g_mutex;
constexpr int MAX_DEVICES = 64;
struct ScratchSlot {
  CUcontext ctx = nullptr;
  double *addr = nullptr;
};
ScratchSlot g_scratch[MAX_DEVICES];

// Per-block sums of both current components (first half of `partial`: x,
// second half: y).
__global__ void __launch_bounds__(NA_THREADS) k_na_partial_sums(size_t nn, const double *__restrict__ j,
                                                                 double *partial) {
  __shared__ double sh[2][NA_THREADS];
  double sx = 0.0, sy = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
       i += (size_t)gridDim.x * blockDim.x) {
    sx += j[i];
    sy += j[nn + i];
  }
  sh[0][threadIdx.x] = sx;
  sh[1][threadIdx.x] = sy;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = sh[0][0];
    partial[gridDim.x + blockIdx.x] = sh[1][0];
  }
}

// s = j - <j>, with <j> = sum(j) / n_grain (ComputeVectorPotential.h:575-591).
__global__ void k_na_subtract_mean(size_t nn, int nblocks, double n_grain,
                                   const double *__restrict__ partial, const double *__restrict__ j,
                                   double *__restrict__ s) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= 2 * nn) return;
  const int d = (int)(i / nn);
  double sum = 0.0;
  for (int b = 0; b < nblocks; ++b) sum += partial[(size_t)d * nblocks + b];
  s[i] = j[i] - sum / n_grain;
}

// One Toeplitz correlation pass with one filter, written transposed
// (cvp_internal::crossCorrelate1DTranspose, ComputeVectorPotential.h:437-499).
__global__ void __launch_bounds__(NA_PT * 8) k_na_toeplitz(int n, const double *__restrict__ filt,
                                                           const double *__restrict__ src,
                                                           double *__restrict__ dst) {
  __shared__ double s_src[NA_PT][NA_PT + 1];
  __shared__ double s_f[2 * NA_PT];
  const int d = blockIdx.z;
  const int x0 = blockIdx.x * NA_PT, y0 = blockIdx.y * NA_PT;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const size_t nn = (size_t)n * n;
  const double *S = src + (size_t)d * nn;
  double acc[4] = {0, 0, 0, 0};
  for (int i0 = 0; i0 < n; i0 += NA_PT) {
    for (int r = ty; r < NA_PT; r += 8) {
      const int i = i0 + r, xx = x0 + tx;
      s_src[r][tx] = (i < n && xx < n) ? S[(size_t)i * n + xx] : 0.0;
    }
    const int t = ty * 32 + tx;
    if (t < 2 * NA_PT) {
      const int fi = i0 + n - 1 - y0 - (NA_PT - 1) + t;
      s_f[t] = (fi >= 0 && fi < 2 * n - 1) ? filt[fi] : 0.0;
    }
    __syncthreads();
    for (int r = 0; r < NA_PT; ++r) {
      const double sv = s_src[r][tx];
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] += s_f[r - (ty + 8 * u) + NA_PT - 1] * sv;
    }
    __syncthreads();
  }
  const int xx = x0 + tx;
  if (xx < n) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int yy = y0 + ty + 8 * u;
      if (yy < n) dst[(size_t)n * (d * n + xx) + yy] = acc[u];
    }
  }
}

// a = (first ? 0 : a) +/- t, in filter order (ComputeVectorPotential.h:713-722).
__global__ void k_na_accumulate(size_t n2, int first, int positive, const double *__restrict__ t,
                                double *a) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n2) return;
  const double v = first ? 0.0 : a[i];
  a[i] = positive ? v + t[i] : v - t[i];
}

__global__ void k_na_scale(size_t n2, double factor, double *a) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n2) a[i] *= factor;
}

// The CUDA context current on this thread, through the driver's
// cuCtxGetCurrent (reached via the runtime, so the library needs no link to
// libcuda).  nullptr when no context is current yet.
CUcontext current_context() {
  using GetCurrent = CUresult (*)(CUcontext *);
  static GetCurrent fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCurrent>(f);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Set-up of the current device: its address of g_noalloc_scratch.  The first
// call on a device (and the first after its context was re-created) makes the
// lookup with cudaGetSymbolAddress, which also loads this library's device code
// on that device; later calls in the same context reuse the address.
cudaError_t scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  ScratchSlot &slot = g_scratch[dev];
  const CUcontext ctx = current_context();
  if (!slot.addr || !ctx || slot.ctx != ctx) {
    double *ptr = nullptr;
    e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    slot.addr = ptr;
    slot.ctx = current_context();  // current now, if it was not before the lookup
  }
  *out = slot.addr;
  return cudaSuccess;
}

// Launches kernel on the stream and returns that launch's own status, so a
// failure is reported whatever error an earlier call of the caller left behind.
template <typename... KArgs, typename... Args>
cudaError_t launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = nullptr;
  cfg.numAttrs = 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

unsigned blocks_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

extern "C" int sc_poisson_noalloc(int n0, int n_filters, const double *d_filters,
                                  const int *positive, double factor, int n_grain,
                                  const double *d_j, double *d_a, void *stream) {
  if (n0 < 2 || n_filters < 1 || !d_filters || !positive || n_grain < 1 || !d_j || !d_a)
    return SC_ERR_ARG;
  const size_t nn = (size_t)n0 * n0;
  const size_t need = 2 * (size_t)NA_REDUCE_BLOCKS + 3 * 2 * nn;  // partials, s, t0, t1
  if (need > NOALLOC_SCRATCH_DOUBLES) return SC_ERR_SIZE;
  double *scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) return SC_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  double *partial = scratch;
  double *s = scratch + 2 * NA_REDUCE_BLOCKS;
  double *t0 = s + 2 * nn;
  double *t1 = t0 + 2 * nn;
  const size_t n2 = 2 * nn;
  const dim3 thr(NA_THREADS), elem(blocks_for(n2, NA_THREADS));
  cudaError_t e = launch(k_na_partial_sums, dim3(NA_REDUCE_BLOCKS), thr, st, nn, d_j, partial);
  if (e == cudaSuccess)
    e = launch(k_na_subtract_mean, elem, thr, st, nn, NA_REDUCE_BLOCKS, (double)n_grain, partial, d_j, s);
  const dim3 blk(NA_PT, 8), grid((n0 + NA_PT - 1) / NA_PT, (n0 + NA_PT - 1) / NA_PT, 2);
  for (int k = 0; k < n_filters && e == cudaSuccess; ++k) {
    const double *f = d_filters + (size_t)k * (2 * n0 - 1);
    e = launch(k_na_toeplitz, grid, blk, st, n0, f, s, t0);
    if (e == cudaSuccess) e = launch(k_na_toeplitz, grid, blk, st, n0, f, t0, t1);
    if (e == cudaSuccess) e = launch(k_na_accumulate, elem, thr, st, n2, k == 0 ? 1 : 0, positive[k] != 0 ? 1 : 0, t1, d_a);
  }
  if (e == cudaSuccess) e = launch(k_na_scale, elem, thr, st, n2, factor, d_a);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // the error is this call's own: report it and clear it
    return SC_ERR_CUDA;
  }
  return SC_OK;
}
