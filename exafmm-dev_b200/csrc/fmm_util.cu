// Utilities behind the C ABI: FP64 direct summation on the GPU (Traversal::direct +
// normalize, include/traversal.h:304-337, accumulated in double), the FP32 FMA throughput
// probe used as the roofline denominator of the FP32-pipe kernels, and the count of this
// library's kernel launches.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <string>

#include "fmm_solver.cuh"

namespace fmmb200 {
std::atomic<long long> g_launches{0};
std::atomic<long long> g_device_allocs{0};
}
using namespace fmmb200;

namespace {

constexpr int kDirTile = 256;

__global__ void __launch_bounds__(kDirTile)
    k_direct(int nt, const double* __restrict__ xt, int ns, const double* __restrict__ xs,
             const double* __restrict__ qs, double eps2, double* __restrict__ out) {
  __shared__ double sh[kDirTile][4];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double x = 0, y = 0, z = 0;
  if (i < nt) {
    x = xt[3 * i];
    y = xt[3 * i + 1];
    z = xt[3 * i + 2];
  }
  double pot = 0, ax = 0, ay = 0, az = 0;
  for (int j0 = 0; j0 < ns; j0 += kDirTile) {
    const int j = j0 + threadIdx.x;
    __syncthreads();
    if (j < ns) {
      sh[threadIdx.x][0] = xs[3 * j];
      sh[threadIdx.x][1] = xs[3 * j + 1];
      sh[threadIdx.x][2] = xs[3 * j + 2];
      sh[threadIdx.x][3] = qs[j];
    }
    __syncthreads();
    const int cnt = min(kDirTile, ns - j0);
    for (int k = 0; k < cnt; k++) {
      const double dx = sh[k][0] - x, dy = sh[k][1] - y, dz = sh[k][2] - z;
      const double r2 = dx * dx + dy * dy + dz * dz + eps2;
      if (r2 != 0) {
        const double inv = 1.0 / sqrt(r2);
        const double qi = sh[k][3] * inv;
        const double inv3 = qi * inv * inv;
        pot += qi;
        ax += dx * inv3;
        ay += dy * inv3;
        az += dz * inv3;
      }
    }
  }
  if (i < nt) {
    out[4 * i] = pot;
    out[4 * i + 1] = ax;
    out[4 * i + 2] = ay;
    out[4 * i + 3] = az;
  }
}

// independent FMA chains: 8 per thread, ITER iterations, 2 flops each
template <int ITER>
__global__ void __launch_bounds__(256) k_fma_probe(float* out, float s) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-7f + k;
#pragma unroll 16
  for (int i = 0; i < ITER; i++)
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], s, 1e-7f);
  float t = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) t += a[k];
  if (t == 123.456f) out[0] = t;  // keeps the chains live
}

// ---- FP64 direct sum without allocation (fmm_b200_direct_noalloc) ---------------------
// The staging buffers of fmm_b200_direct (targets, sources, charges, output) live in one
// fixed array in device memory instead of per-call cudaMalloc/cudaFree.  Layout for a call
// (nt, ns), in doubles: targets [0, 3 nt), sources [3 nt, 3 nt + 3 ns), charges next (ns),
// output next (4 nt): 7 nt + 4 ns doubles, at most 7 * 32768 + 4 * 65536 = 491,520
// doubles (3.75 MiB) per device.  No part of it has to start at zero: a call copies in
// every input it reads and the kernel writes every output that is copied back.
constexpr int kNoAllocMaxTargets = FMM_DIRECT_NOALLOC_MAX_TARGETS;
constexpr int kNoAllocMaxSources = FMM_DIRECT_NOALLOC_MAX_SOURCES;
constexpr size_t kNoAllocDoubles =
    7 * (size_t)kNoAllocMaxTargets + 4 * (size_t)kNoAllocMaxSources;
static __device__ __align__(256) double g_direct_scratch[kNoAllocDoubles];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_base[kNoAllocMaxDevices] = {};
cudaStream_t g_noalloc_stream[kNoAllocMaxDevices] = {};

// Set-up of one device (which must be current), done once: the device address of the array
// (host code only sees a host-side stand-in under the array's name) and the call's own
// non-blocking stream (creating a stream allocates no device memory), so that the call
// neither waits for nor holds up the caller's other streams, the legacy default stream's
// implicit synchronisation included.
void noalloc_setup(int device, double** base, cudaStream_t* stream) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_base[device]) {
    void* p = nullptr;
    FMM_CUDA(cudaGetSymbolAddress(&p, g_direct_scratch));
    cudaStream_t st = nullptr;
    FMM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    g_noalloc_stream[device] = st;
    g_noalloc_base[device] = static_cast<double*>(p);
  }
  *base = g_noalloc_base[device];
  *stream = g_noalloc_stream[device];
}

}  // namespace

extern "C" {

long long fmm_b200_kernel_launches(void) { return g_launches.load(); }
long long fmm_b200_device_allocations(void) { return g_device_allocs.load(); }

int fmm_b200_direct_noalloc(int device, int nt, const double* xt, int ns, const double* xs,
                            const double* qs, double eps2, double* out) {
  fmmb200::set_call_error("");
  if (nt < 0 || ns < 0 || (nt > 0 && (!xt || !out)) || (ns > 0 && (!xs || !qs)) ||
      device < 0 || device >= kNoAllocMaxDevices) {
    fmmb200::set_call_error("fmm_b200_direct_noalloc: invalid argument");
    return FMM_ERR_INVALID;
  }
  if (nt > kNoAllocMaxTargets || ns > kNoAllocMaxSources) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "fmm_b200_direct_noalloc: %d targets / %d sources exceed the static scratch "
                  "limits of %d targets / %d sources (fmm_b200_direct has none)",
                  nt, ns, kNoAllocMaxTargets, kNoAllocMaxSources);
    fmmb200::set_call_error(msg);
    return FMM_ERR_INVALID;
  }
  if (nt == 0) return FMM_OK;
  try {
    FMM_CUDA(cudaSetDevice(device));
    double* base = nullptr;
    cudaStream_t st = nullptr;
    noalloc_setup(device, &base, &st);
    double *dxt = base, *dxs = base + 3 * (size_t)nt, *dqs = dxs + 3 * (size_t)ns,
           *dout = dqs + ns;
    FMM_CUDA(cudaMemcpyAsync(dxt, xt, 24 * (size_t)nt, cudaMemcpyHostToDevice, st));
    if (ns) {
      FMM_CUDA(cudaMemcpyAsync(dxs, xs, 24 * (size_t)ns, cudaMemcpyHostToDevice, st));
      FMM_CUDA(cudaMemcpyAsync(dqs, qs, 8 * (size_t)ns, cudaMemcpyHostToDevice, st));
    }
    k_direct<<<ceil_div(nt, kDirTile), kDirTile, 0, st>>>(nt, dxt, ns, dxs, dqs, eps2, dout);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaMemcpyAsync(out, dout, 32 * (size_t)nt, cudaMemcpyDeviceToHost, st));
    FMM_CUDA(cudaStreamSynchronize(st));
  } catch (const FmmError& e) {
    fmmb200::set_call_error(e.what());
    return e.code;
  }
  return FMM_OK;
}

int fmm_b200_direct(int device, int nt, const double* xt, int ns, const double* xs,
                    const double* qs, double eps2, double* out) {
  fmmb200::set_call_error("");
  if (nt < 0 || ns < 0 || (nt > 0 && (!xt || !out)) || (ns > 0 && (!xs || !qs))) {
    fmmb200::set_call_error("fmm_b200_direct: invalid argument");
    return FMM_ERR_INVALID;
  }
  if (nt == 0) return FMM_OK;
  try {
    FMM_CUDA(cudaSetDevice(device));
    DevArr<double> b;
    b.ensure(3 * (size_t)nt + 4 * (size_t)ns + 4 * (size_t)nt);
    double *dxt = b.p, *dxs = b.p + 3 * (size_t)nt, *dqs = dxs + 3 * (size_t)ns,
           *dout = dqs + ns;
    FMM_CUDA(cudaMemcpy(dxt, xt, 24 * (size_t)nt, cudaMemcpyHostToDevice));
    if (ns) {
      FMM_CUDA(cudaMemcpy(dxs, xs, 24 * (size_t)ns, cudaMemcpyHostToDevice));
      FMM_CUDA(cudaMemcpy(dqs, qs, 8 * (size_t)ns, cudaMemcpyHostToDevice));
    }
    k_direct<<<ceil_div(nt, kDirTile), kDirTile>>>(nt, dxt, ns, dxs, dqs, eps2, dout);
    FMM_LAUNCH_CHECK();
    FMM_CUDA(cudaMemcpy(out, dout, 32 * (size_t)nt, cudaMemcpyDeviceToHost));
    b.release();
  } catch (const FmmError& e) {
    fmmb200::set_call_error(e.what());
    return e.code;
  }
  return FMM_OK;
}

int fmm_b200_fp32_peak(int device, double* tflops) {
  if (!tflops) return FMM_ERR_INVALID;
  try {
    FMM_CUDA(cudaSetDevice(device));
    int sms = 0;
    FMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    DevArr<float> o;
    o.ensure(1);
    constexpr int ITER = 8192;
    const int blocks = sms * 8, threads = 256;
    k_fma_probe<ITER><<<blocks, threads>>>(o.p, 0.9999f);  // warm-up
    FMM_LAUNCH_CHECK();
    cudaEvent_t a, b;
    FMM_CUDA(cudaEventCreate(&a));
    FMM_CUDA(cudaEventCreate(&b));
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
      FMM_CUDA(cudaEventRecord(a));
      k_fma_probe<ITER><<<blocks, threads>>>(o.p, 0.9999f);
      FMM_LAUNCH_CHECK();
      FMM_CUDA(cudaEventRecord(b));
      FMM_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      FMM_CUDA(cudaEventElapsedTime(&ms, a, b));
      best = ms < best ? ms : best;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    o.release();
    const double flops = 2.0 * 8 * ITER * (double)blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
  } catch (const FmmError& e) {
    return e.code;
  }
  return FMM_OK;
}

}  // extern "C"
