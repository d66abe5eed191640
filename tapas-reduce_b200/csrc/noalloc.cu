// FP64 direct sum for sampled targets that allocates no memory.
//
// Why it exists: tapas_b200_direct stages its target list and per-target sums
// in device buffers it allocates on every call.  Some callers cannot allow a
// device allocation where they check accuracy: a time-stepping loop that
// reserves all of its device memory up front (a cudaMalloc there can fail or
// push the solver out of memory), or code that shares the GPU with other
// streams (cudaMalloc / cudaFree synchronise the whole device and stall that
// work).  This entry point takes only caller-owned device buffers and keeps
// its partial sums in one fixed device array compiled into the library.
//
// Limits and sharing:
//  - at most kMaxTargets targets per call; more are rejected with
//    TAPAS_B200_ERR_CAPACITY and a message;
//  - the scratch array (kMaxTargets x kSplit x 4 doubles = 2 MiB) exists once
//    per GPU that loads the library and is held until the process exits;
//  - every call on a device uses the same array, and it keeps the last call's
//    contents.  Each call writes every slot it later reads, so nothing needs
//    clearing; calls that overlap on the GPU (different streams, or different
//    host threads without ordering) race on the array and must be serialised
//    by the caller;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make
//    that first call before any stream capture.
#include <mutex>

#include "common.cuh"

namespace tb {
namespace {

constexpr int kMaxTargets = 4096;
constexpr int kSplit = 16;       // blocks per target, each over 1/kSplit of the sources
constexpr int kNoallocThreads = 256;
constexpr int kMaxDevices = 64;

// The scratch: per (target, split) the 4 partial sums.
static __device__ __align__(256) double g_direct_scratch[(size_t)kMaxTargets * kSplit * 4];

double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

__global__ void __launch_bounds__(kNoallocThreads) direct_partial(
    const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z,
    const double *__restrict__ q, int64_t n, const int64_t *__restrict__ targets,
    double *__restrict__ scratch) {
  const int t = blockIdx.x, split = blockIdx.y;
  const int64_t i = targets[t];
  const bool ok = i >= 0 && i < n;
  double p = 0, ax = 0, ay = 0, az = 0;
  if (ok) {
    const double xi = x[i], yi = y[i], zi = z[i];
    for (int64_t j = (int64_t)split * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)kSplit * blockDim.x) {
      const double dx = xi - x[j], dy = yi - y[j], dz = zi - z[j];
      const double R2 = dx * dx + dy * dy + dz * dz;
      if (R2 != 0) {
        const double invR = 1.0 / sqrt(R2);
        const double qr = q[j] * invR;
        const double s3 = qr * invR * invR;
        p += qr;
        ax -= dx * s3;
        ay -= dy * s3;
        az -= dz * s3;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    p += __shfl_down_sync(0xffffffffu, p, o);
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
    az += __shfl_down_sync(0xffffffffu, az, o);
  }
  __shared__ double red[4][kNoallocThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = p; red[1][w] = ax; red[2][w] = ay; red[3][w] = az; }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int k = 0; k < kNoallocThreads / 32; k++) s += red[threadIdx.x][k];
    // A target index outside [0, n) yields NaN for that target.
    scratch[((size_t)t * kSplit + split) * 4 + threadIdx.x] = ok ? s : __longlong_as_double(-1);
  }
}

__global__ void direct_finish(const double *__restrict__ scratch, int64_t k,
                              double *__restrict__ out4) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < k * 4;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = idx / 4;
    const int c = (int)(idx % 4);
    double s = 0;
    for (int sp = 0; sp < kSplit; sp++) s += scratch[((size_t)t * kSplit + sp) * 4 + c];
    out4[idx] = s;
  }
}

}  // namespace
}  // namespace tb

using namespace tb;

extern "C" int tapas_b200_direct_noalloc(const double *x, const double *y, const double *z,
                                         const double *q, int64_t n, const int64_t *targets,
                                         int64_t k, double *out4, void *stream) {
  if (!x || !y || !z || !q || !targets || !out4 || n <= 0 || k <= 0) {
    set_error(nullptr, "direct_noalloc: need n > 0, k > 0 and non-null device pointers");
    return TAPAS_B200_ERR_ARG;
  }
  if (k > kMaxTargets) {
    set_error(nullptr,
              "direct_noalloc: %lld targets exceed the fixed scratch capacity of %d targets "
              "per call; split the target list",
              (long long)k, kMaxTargets);
    return TAPAS_B200_ERR_CAPACITY;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error(nullptr, "direct_noalloc: no usable current device (%s)", cudaGetErrorString(e));
    return TAPAS_B200_ERR_CUDA;
  }
  double *scratch;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
      // Host code cannot use g_direct_scratch's name as a device address:
      // look the address up once for this device (the current one).
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_direct_scratch);
      if (e != cudaSuccess || !p) {
        set_error(nullptr, "direct_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                  cudaGetErrorString(e));
        return TAPAS_B200_ERR_CUDA;
      }
      g_scratch_addr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // An error left by earlier asynchronous work would otherwise be read back
  // after the launch below and reported as this call's launch failure.
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(nullptr, "direct_noalloc: a CUDA error from earlier work was pending: %s",
              cudaGetErrorString(e));
    return TAPAS_B200_ERR_CUDA;
  }
  direct_partial<<<dim3((unsigned)k, kSplit), kNoallocThreads, 0, s>>>(x, y, z, q, n, targets,
                                                                       scratch);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    direct_finish<<<(unsigned)((k * 4 + 255) / 256), 256, 0, s>>>(scratch, k, out4);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(nullptr, "direct_noalloc: launch failed: %s", cudaGetErrorString(e));
    return TAPAS_B200_ERR_CUDA;
  }
  return TAPAS_B200_OK;
}
