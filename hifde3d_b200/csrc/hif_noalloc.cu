// Dense Schur elimination that allocates no device memory.
//
// hif_schur_device (hif_engine.cpp) takes its working copy of the block and its
// pivot-block inverses from cudaMallocAsync. Some callers cannot allocate device
// memory at all: a process whose framework allocator has already reserved the
// whole GPU, or a loop that must not touch the allocator between its own
// kernels. For them, hif_schur_device_noalloc computes the same result with all
// scratch in one file-scope device array of fixed size, reserved when the
// library is loaded on a device and kept until the process exits.
//
// Limits and sharing:
//   * blocks of at most kNoAllocMaxN DOFs (kNoAllocScratchBytes of scratch);
//   * every call on a device uses the same array; calls whose kernels overlap
//     on the GPU (different streams, or host threads sharing a device) race on
//     it and must be serialised by the caller;
//   * the first call on a device looks the array's address up once, with that
//     device current; that first call should come before any stream capture
//     begins on the device. The address is kept for the life of the process, so the
//     library must not be used on a device after cudaDeviceReset has torn its
//     context down;
//   * every call ends by copying the pivot status word to the host and
//     synchronising its stream: it returns after its kernels have finished;
//   * the kernels favour simplicity over speed (the panel kernels keep a 64-entry
//     row or column per thread and read the pivot-block inverse from global
//     memory); the results are those of hif_schur_device within rounding.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/hif_b200.h"
#include "hif_kernels.cuh"

namespace hif {
extern thread_local std::string g_last_error;
}

namespace {

constexpr int kNoAllocMaxN = 512;
constexpr int kNB = 64;  // pivot block of this variant
constexpr size_t kScratchDoubles = (size_t)kNoAllocMaxN * kNoAllocMaxN + kNB * kNB + 32;
constexpr size_t kNoAllocScratchBytes = kScratchDoubles * sizeof(double);
static_assert(kNoAllocScratchBytes < (2u << 20) + (64u << 10), "scratch stays about 2 MiB");

// Working block (n x n, ld n) | pivot-block inverse (64 x 64) | status word.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// W = B with the skeleton-skeleton block zeroed (so the elimination yields
// S = -A12 X there), and the status word cleared.
__global__ void k_na_load(const double* __restrict__ B, double* __restrict__ W, int n, int r,
                          int* __restrict__ status) {
  const long long nn = (long long)n * n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    W[e] = (i >= r && j >= r) ? 0.0 : B[e];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *status = 0;
}

// Gauss-Jordan inverse of the pivot block D = W[K, K] into Dinv.
__global__ void k_na_diag(double* __restrict__ W, int n, int r, int k0, double* __restrict__ Dinv,
                          int* __restrict__ status) {
  const int nb = min(kNB, r - k0);
  __shared__ double S[kNB * kNB];
  __shared__ double s_ip;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x)
    S[e] = W[(k0 + e % nb) + (long long)(k0 + e / nb) * n];
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    if (threadIdx.x == 0) {
      const double p = S[k + k * nb];
      if (!(fabs(p) > 1e-300) || !isfinite(p)) atomicOr(status, hif::kStatusTinyPivot);
      s_ip = 1.0 / p;
    }
    __syncthreads();
    const double ip = s_ip;
    for (int j = threadIdx.x; j < nb; j += blockDim.x)
      if (j != k) S[k + j * nb] *= ip;
    __syncthreads();
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
      const int i = e % nb, j = e / nb;
      if (i != k && j != k) S[e] = fma(-S[i + k * nb], S[k + j * nb], S[e]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
      if (i != k) S[i + k * nb] *= -ip;
    if (threadIdx.x == 0) S[k + k * nb] = ip;
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) Dinv[e] = S[e];
}

// Pivot rows: W[K, j] = Dinv W[K, j] for every column j outside K.
__global__ void k_na_rowpanel(double* __restrict__ W, int n, int r, int k0,
                              const double* __restrict__ Dinv) {
  const int nb = min(kNB, r - k0);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || (j >= k0 && j < k0 + nb)) return;
  double col[kNB];
  for (int t = 0; t < nb; ++t) col[t] = W[(k0 + t) + (long long)j * n];
  for (int i = 0; i < nb; ++i) {
    double acc = 0.0;
    for (int t = 0; t < nb; ++t) acc = fma(Dinv[i + t * nb], col[t], acc);
    W[(k0 + i) + (long long)j * n] = acc;
  }
}

// Rank-nb update of every entry outside the pivot rows / columns, except the
// skeleton rows' already-pivoted columns (never read again):
//   W[i, j] -= W[i, K] W[K, j].
__global__ void __launch_bounds__(256) k_na_update(double* __restrict__ W, int n, int r,
                                                   int k0) {
  const int nb = min(kNB, r - k0);
  const int k1 = k0 + nb;
  __shared__ double Cs[32][kNB + 1];  // W[i0.., K]
  __shared__ double Rs[kNB][33];      // W[K, j0..]
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int e = threadIdx.x; e < 32 * nb; e += blockDim.x) {
    const int a = e % 32, t = e / 32;
    Cs[a][t] = (i0 + a < n) ? W[(i0 + a) + (long long)(k0 + t) * n] : 0.0;
    Rs[t][a] = (j0 + a < n) ? W[(k0 + t) + (long long)(j0 + a) * n] : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int a = e % 32, b = e / 32;
    const int i = i0 + a, j = j0 + b;
    if (i >= n || j >= n) continue;
    if ((i >= k0 && i < k1) || (j >= k0 && j < k1)) continue;
    if (i >= r && j < k0) continue;
    double acc = W[i + (long long)j * n];
    for (int t = 0; t < nb; ++t) acc = fma(-Cs[a][t], Rs[t][b], acc);
    W[i + (long long)j * n] = acc;
  }
}

// Pivot columns of the redundant rows: W[i, K] = -W[i, K] Dinv; W[K, K] = Dinv.
__global__ void k_na_colpanel(double* __restrict__ W, int n, int r, int k0,
                              const double* __restrict__ Dinv) {
  const int nb = min(kNB, r - k0);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r) return;
  if (i >= k0 && i < k0 + nb) {
    for (int t = 0; t < nb; ++t) W[i + (long long)(k0 + t) * n] = Dinv[(i - k0) + t * nb];
    return;
  }
  double row[kNB];
  for (int t = 0; t < nb; ++t) row[t] = W[i + (long long)(k0 + t) * n];
  for (int c = 0; c < nb; ++c) {
    double acc = 0.0;
    for (int t = 0; t < nb; ++t) acc = fma(row[t], Dinv[t + c * nb], acc);
    W[i + (long long)(k0 + c) * n] = -acc;
  }
}

// Outputs: A22^{-1} = W[0:r, 0:r], X = W[0:r, r:n], S = W[r:n, r:n].
__global__ void k_na_store(const double* __restrict__ W, int n, int r, double* __restrict__ inv,
                           double* __restrict__ X, double* __restrict__ S) {
  const long long nn = (long long)n * n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (i < r && j < r) inv[i + (long long)j * r] = W[e];
    else if (i < r) X[i + (long long)(j - r) * r] = W[e];
    else if (j >= r) S[(i - r) + (long long)(j - r) * (n - r)] = W[e];
  }
}

int fail(int code, const char* msg) {
  hif::g_last_error = msg;
  return code;
}

}  // namespace

extern "C" int hif_schur_device_noalloc(const double* dB, int n, int r, double* dA22inv,
                                        double* dX, double* dS, void* stream) {
  // the same argument and device checks as hif_schur_device, in the same order
  if (!dB || n < 0 || r < 0 || r > n) return fail(HIF_ERR_ARG, "hif_schur_device_noalloc: bad block");
  if (n > kNoAllocMaxN)
    return fail(HIF_ERR_ARG, "hif_schur_device_noalloc: block larger than 512 DOFs "
                             "(the fixed scratch size); use hif_schur_device");
  if ((r > 0 && !dA22inv) || (r > 0 && r < n && !dX) || (r < n && !dS))
    return fail(HIF_ERR_ARG, "hif_schur_device_noalloc: missing output");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(HIF_ERR_NODEVICE, "no CUDA device");
  if (n == 0) return HIF_OK;  // an empty block: nothing to eliminate or write
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(HIF_ERR_NODEVICE, "hif_schur_device_noalloc: no current CUDA device");
  double* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) {
        return fail(HIF_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") +
                                   cudaGetErrorString(e)).c_str());
      }
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    base = g_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* W = base;
  double* Dinv = base + (size_t)kNoAllocMaxN * kNoAllocMaxN;
  int* status = reinterpret_cast<int*>(Dinv + kNB * kNB);

  const long long nn = (long long)n * n;
  const int gl = (int)std::min<long long>((nn + 255) / 256, 4096);
  k_na_load<<<gl, 256, 0, s>>>(dB, W, n, r, status);
  for (int k0 = 0; k0 < r; k0 += kNB) {
    k_na_diag<<<1, 256, 0, s>>>(W, n, r, k0, Dinv, status);
    k_na_rowpanel<<<(n + 127) / 128, 128, 0, s>>>(W, n, r, k0, Dinv);
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    k_na_update<<<grid, 256, 0, s>>>(W, n, r, k0);
    k_na_colpanel<<<(r + 127) / 128, 128, 0, s>>>(W, n, r, k0, Dinv);
  }
  k_na_store<<<gl, 256, 0, s>>>(W, n, r, dA22inv, dX, dS);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(HIF_ERR_CUDA, cudaGetErrorString(e));
  int hst = 0;
  e = cudaMemcpyAsync(&hst, status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(HIF_ERR_CUDA, cudaGetErrorString(e));
  if (hst & hif::kStatusTinyPivot) return fail(HIF_ERR_SINGULAR, "zero or non-finite pivot");
  return HIF_OK;
}
