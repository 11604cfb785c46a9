// Device kernels of the HIF factor / apply path (sm_100a, FP64).
//
// The reference performs these steps with LAPACK/BLAS on one CPU core
// (arbenson/HIFDE3D src/Factor.cpp, include/Schur.hpp, src/InterpDecomp.cpp).
// Here each level phase is a handful of batched launches over every cell or
// face of the level:
//   gather      dense blocks from the 7-point stencil plus the live Schur
//               complement blocks (replaces DenseSubmatrix over std::map and
//               UpdateMatrixAndDOFs, src/Factor.cpp:262-311);
//   sweep       in-place Gauss-Jordan elimination of the redundant DOFs of a
//               block [A22 A21; A12 A11]: yields A22^{-1}, X = A22^{-1} A21 and
//               A11 - A12 X in one pass (Schur.hpp:72-100);
//   dgemm       batched FP64 GEMM (rank-64 sweep updates, ID rotations);
//   id          column-pivoted Householder QR, rank test and interpolation
//               matrix (InterpDecomp.cpp:86-138);
//   gemv        gather / multiply / scatter sweeps of Apply (Factor.cpp:992-1081).
#include "hif_kernels.cuh"

#include <cfloat>
#include <climits>
#include <cmath>

namespace hif {

namespace {

__device__ __forceinline__ int find_desc(const int* __restrict__ off, int nd, int t) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; every thread gets the result. scratch: >= 32 doubles.
__device__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double t = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
  if (warp == 0) t = warp_sum(t);
  if (threadIdx.x == 0) scratch[32] = t;
  __syncthreads();
  double r = scratch[32];
  __syncthreads();
  return r;
}

}  // namespace

// ===========================================================================
// Gather / assembly
// ===========================================================================
constexpr int kGT = 32;  // gather tile edge

int gather_tiles(int m, int n) {
  return ((m + kGT - 1) / kGT) * ((n + kGT - 1) / kGT);
}

__device__ __forceinline__ void resolve_cover(const GatherTarget& g, int p,
                                              const int* __restrict__ dof_src,
                                              const int* __restrict__ src_owner,
                                              long long ncell3, CoverEntry* out) {
#pragma unroll
  for (int c = 0; c < kCover; ++c) {
    CoverEntry ce{-1, 0};
    if (p >= 0 && g.mode != 2) {
      const int s = dof_src[(2 * c) * ncell3 + p];
      if (s >= 0) {
        const bool ok = (g.mode == 0) ? (src_owner[s] == g.owner)
                                      : (s == g.allowA || s == g.allowB);
        if (ok) ce = CoverEntry{s, dof_src[(2 * c + 1) * ncell3 + p]};
      }
    }
    out[c] = ce;
  }
}

__global__ void __launch_bounds__(256) k_gather(const GatherTarget* __restrict__ tg,
                                                const int* __restrict__ tile_off, int ntg,
                                                const SourceDesc* __restrict__ src,
                                                const int* __restrict__ src_owner,
                                                const int* __restrict__ dof_src,
                                                const double* __restrict__ band,
                                                long long ncell3, int NC) {
  const int d = find_desc(tile_off, ntg, blockIdx.x);
  const GatherTarget g = tg[d];
  const int local = blockIdx.x - tile_off[d];
  const int tiles_m = (g.m + kGT - 1) / kGT;
  const int i0 = (local % tiles_m) * kGT, j0 = (local / tiles_m) * kGT;

  __shared__ int s_row[kGT], s_col[kGT];
  __shared__ CoverEntry s_rc[kGT][kCover], s_cc[kGT][kCover];
  for (int x = threadIdx.x; x < 2 * kGT; x += blockDim.x) {
    if (x < kGT) {
      const int i = i0 + x;
      const int p = (i < g.m) ? g.rows[i] : -1;
      s_row[x] = p;
      resolve_cover(g, p, dof_src, src_owner, ncell3, s_rc[x]);
    } else {
      const int y = x - kGT, j = j0 + y;
      const int q = (j < g.n) ? g.cols[j] : -1;
      s_col[y] = q;
      resolve_cover(g, q, dof_src, src_owner, ncell3, s_cc[y]);
    }
  }
  __syncthreads();
  const long long NC2 = (long long)NC * NC;
  for (int e = threadIdx.x; e < kGT * kGT; e += blockDim.x) {
    const int x = e % kGT, y = e / kGT;
    const int i = i0 + x, j = j0 + y;
    if (i >= g.m || j >= g.n) continue;
    const long long p = s_row[x], q = s_col[y];
    double v = 0.0;
    if (!(i >= g.a0_skip && j >= g.a0_skip)) {
      const long long dd = q - p;
      int b = -1;
      if (dd == 0) b = 0;
      else if (dd == -1) b = 1;
      else if (dd == 1) b = 2;
      else if (dd == -NC) b = 3;
      else if (dd == NC) b = 4;
      else if (dd == -NC2) b = 5;
      else if (dd == NC2) b = 6;
      if (b >= 0) v = band[b * ncell3 + p];
    }
#pragma unroll
    for (int a = 0; a < kCover; ++a) {
      const int sa = s_rc[x][a].src;
      if (sa < 0) continue;
#pragma unroll
      for (int c = 0; c < kCover; ++c) {
        if (s_cc[y][c].src == sa) {
          const SourceDesc sd = src[sa];
          v += sd.ptr[(long long)s_rc[x][a].pos + (long long)s_cc[y][c].pos * sd.ld];
        }
      }
    }
    g.out[i + (long long)j * g.ld] = v;
    if (g.a22_out != nullptr && i < g.r && j < g.r) g.a22_out[i + (long long)j * g.r] = v;
  }
}

void launch_gather(const GatherTarget* d_tg, const int* d_tile_off, int ntg, int total_tiles,
                   const SourceDesc* d_src, const int* d_src_owner, const int* d_dof_src,
                   const double* d_band, long long ncell3, int NC, cudaStream_t s) {
  if (total_tiles <= 0) return;
  k_gather<<<total_tiles, 256, 0, s>>>(d_tg, d_tile_off, ntg, d_src, d_src_owner, d_dof_src,
                                       d_band, ncell3, NC);
}

// ===========================================================================
// Batched FP64 GEMM: 64x64x16 tiles, 256 threads, 4x4 outputs per thread.
// Thread (tx, ty) owns rows tx + 16 a and columns ty + 16 b so that the
// epilogue stores are coalesced along the (column-major) rows.
// ===========================================================================
constexpr int kBM = 64, kBN = 64, kBK = 16;

int dgemm_tiles(int m, int n) {
  if (m <= 0 || n <= 0) return 0;
  return ((m + kBM - 1) / kBM) * ((n + kBN - 1) / kBN);
}

__global__ void __launch_bounds__(256) k_dgemm(const GemmDesc* __restrict__ descs,
                                               const int* __restrict__ tile_off, int nd) {
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const GemmDesc g = descs[di];
  const int local = blockIdx.x - tile_off[di];
  const int tiles_m = (g.m + kBM - 1) / kBM;
  const int m0 = (local % tiles_m) * kBM, n0 = (local / tiles_m) * kBN;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

  __shared__ double As[2][kBK][kBM + 1];
  __shared__ double Bs[2][kBK][kBN + 1];

  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

  double ra[4], rb[4];
  auto load_a = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      int mm, kk;
      if (g.transA == 0) { mm = e % kBM; kk = e / kBM; } else { mm = e / kBK; kk = e % kBK; }
      const int gm = m0 + mm, gk = k0 + kk;
      double v = 0.0;
      if (gm < g.m && gk < g.k)
        v = (g.transA == 0) ? g.A[gm + (long long)gk * g.lda] : g.A[gk + (long long)gm * g.lda];
      ra[q] = v;
    }
  };
  auto load_b = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      int nn, kk;
      if (g.transB == 0) { kk = e % kBK; nn = e / kBK; } else { nn = e % kBN; kk = e / kBN; }
      const int gn = n0 + nn, gk = k0 + kk;
      double v = 0.0;
      if (gn < g.n && gk < g.k)
        v = (g.transB == 0) ? g.B[gk + (long long)gn * g.ldb] : g.B[gn + (long long)gk * g.ldb];
      rb[q] = v;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      int mm, kk;
      if (g.transA == 0) { mm = e % kBM; kk = e / kBM; } else { mm = e / kBK; kk = e % kBK; }
      As[buf][kk][mm] = ra[q];
      int nn, kb;
      if (g.transB == 0) { kb = e % kBK; nn = e / kBK; } else { nn = e % kBN; kb = e / kBN; }
      Bs[buf][kb][nn] = rb[q];
    }
  };

  const int nk = (g.k + kBK - 1) / kBK;
  if (nk > 0) {
    load_a(0);
    load_b(0);
    store(0);
  }
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int buf = t & 1;
    if (t + 1 < nk) {
      load_a((t + 1) * kBK);
      load_b((t + 1) * kBK);
    }
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[buf][kk][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[buf][kk][ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    if (t + 1 < nk) store(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int gn = n0 + ty + 16 * b;
    if (gn >= g.n) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int gm = m0 + tx + 16 * a;
      if (gm >= g.m) continue;
      double* c = g.C + gm + (long long)gn * g.ldc;
      const double v = g.alpha * acc[a][b];
      *c = (g.beta == 0.0) ? v : fma(g.beta, *c, v);
    }
  }
}

void launch_dgemm(const GemmDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                  cudaStream_t s) {
  if (total_tiles <= 0) return;
  k_dgemm<<<total_tiles, 256, 0, s>>>(d_desc, d_tile_off, nd);
}

// ===========================================================================
// Gauss-Jordan sweep. For B = [A22 A21; A12 A11] (red first), eliminating
// pivots 0..r-1 in place gives [A22^{-1} X; * A11 - A12 X] with
// X = A22^{-1} A21: the three outputs of the reference's Schur().
// Entries of the bottom-left block whose column is already pivoted are never
// read again and are not updated.
// ===========================================================================
__global__ void __launch_bounds__(256) k_sweep_small(const SweepDesc* __restrict__ descs,
                                                     int* __restrict__ status) {
  const SweepDesc d = descs[blockIdx.x];
  const int n = d.n, r = d.r;
  extern __shared__ double S[];  // n x n, ld n
  const int nn = n * n;
  for (int e = threadIdx.x; e < nn; e += blockDim.x) S[e] = d.B[e];
  __syncthreads();
  __shared__ double s_ip;
  int bad = 0;
  for (int k = 0; k < r; ++k) {
    if (threadIdx.x == 0) {
      const double p = S[k + k * n];
      if (!(fabs(p) > 1e-300) || !isfinite(p)) bad = 1;
      s_ip = 1.0 / p;
    }
    __syncthreads();
    const double ip = s_ip;
    // new pivot row
    for (int j = threadIdx.x; j < n; j += blockDim.x)
      if (j != k) S[k + j * n] *= ip;
    __syncthreads();
    // rank-1 update of every entry outside row / column k
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int i = e % n, j = e / n;
      if (i == k || j == k) continue;
      if (i >= r && j < k) continue;
      S[e] = fma(-S[i + k * n], S[k + j * n], S[e]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < r; i += blockDim.x)
      if (i != k) S[i + k * n] *= -ip;
    if (threadIdx.x == 0) S[k + k * n] = ip;
    __syncthreads();
  }
  if (bad) atomicOr(status, kStatusTinyPivot);
  // compact outputs: A22^{-1} (r x r), X (r x s); T = A11 - A12 X stays in B
  const int s = n - r;
  for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
    const int i = e % r, j = e / r;
    d.a22inv[e] = S[i + j * n];
  }
  for (int e = threadIdx.x; e < r * s; e += blockDim.x) {
    const int i = e % r, j = e / r;
    d.X[e] = S[i + (r + j) * n];
  }
  for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
    const int i = e % s, j = e / s;
    d.B[(r + i) + (long long)(r + j) * n] = S[(r + i) + (r + j) * n];
  }
}

void launch_sweep_small(const SweepDesc* d_desc, int nd, int max_n, int* d_status,
                        cudaStream_t s) {
  if (nd <= 0) return;
  const size_t smem = (size_t)max_n * max_n * sizeof(double);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_sweep_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSmallSweepN * kSmallSweepN * (int)sizeof(double));
    attr_set = true;
  }
  k_sweep_small<<<nd, 256, smem, s>>>(d_desc, d_status);
}

// --- blocked sweep ---------------------------------------------------------
// Step for pivot block K = [k0, k1): D = B[K, K].
//   diag:     Dinv = D^{-1} (Gauss-Jordan in shared memory)
//   rowpanel: B[K, j] = Dinv B[K, j]           for j outside K
//   update:   B[i, j] -= B[i, K] B[K, j]       for i, j outside K (dgemm)
//   colpanel: B[i, K] = -B[i, K] Dinv           for red rows i outside K
//   setdiag:  B[K, K] = Dinv
__global__ void __launch_bounds__(256) k_sweep_diag(const SweepDesc* __restrict__ descs,
                                                    const int* __restrict__ active, int k0,
                                                    double* __restrict__ dinv,
                                                    int* __restrict__ status) {
  const int di = active[blockIdx.x];
  const SweepDesc d = descs[di];
  const int nb = min(kSweepNB, d.r - k0);
  __shared__ double S[kSweepNB * kSweepNB];
  __shared__ double s_ip;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    S[e] = d.B[(k0 + i) + (long long)(k0 + j) * d.n];
  }
  __syncthreads();
  int bad = 0;
  for (int k = 0; k < nb; ++k) {
    if (threadIdx.x == 0) {
      const double p = S[k + k * nb];
      if (!(fabs(p) > 1e-300) || !isfinite(p)) bad = 1;
      s_ip = 1.0 / p;
    }
    __syncthreads();
    const double ip = s_ip;
    for (int j = threadIdx.x; j < nb; j += blockDim.x)
      if (j != k) S[k + j * nb] *= ip;
    __syncthreads();
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
      const int i = e % nb, j = e / nb;
      if (i == k || j == k) continue;
      S[e] = fma(-S[i + k * nb], S[k + j * nb], S[e]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
      if (i != k) S[i + k * nb] *= -ip;
    if (threadIdx.x == 0) S[k + k * nb] = ip;
    __syncthreads();
  }
  if (bad) atomicOr(status, kStatusTinyPivot);
  double* out = dinv + (long long)di * kSweepNB * kSweepNB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) out[e] = S[e];
}

void launch_sweep_diag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                       double* d_dinv, int* d_status, cudaStream_t s) {
  if (nact <= 0) return;
  k_sweep_diag<<<nact, 256, 0, s>>>(d_desc, d_active, k0, d_dinv, d_status);
}

// Row panel: tile of up to 64 columns [lo, hi) of rows K.
__global__ void __launch_bounds__(256) k_sweep_rowpanel(const SweepDesc* __restrict__ descs,
                                                        const int4* __restrict__ tiles, int k0,
                                                        const double* __restrict__ dinv) {
  const int4 t = tiles[blockIdx.x];
  const SweepDesc d = descs[t.x];
  const int nb = min(kSweepNB, d.r - k0);
  const int w = t.z - t.y;
  extern __shared__ double panel_smem[];
  double* Ds = panel_smem;
  double* Ts = panel_smem + kSweepNB * kSweepNB;
  const double* Dg = dinv + (long long)t.x * kSweepNB * kSweepNB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) Ds[e] = Dg[e];
  for (int e = threadIdx.x; e < nb * w; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    Ts[e] = d.B[(k0 + i) + (long long)(t.y + j) * d.n];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * w; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    double acc = 0.0;
    for (int kk = 0; kk < nb; ++kk) acc = fma(Ds[i + kk * nb], Ts[kk + j * nb], acc);
    d.B[(k0 + i) + (long long)(t.y + j) * d.n] = acc;
  }
}

void launch_sweep_rowpanel(const SweepDesc* d_desc, const int* d_tile_map, int ntiles, int k0,
                           const double* d_dinv, cudaStream_t s) {
  if (ntiles <= 0) return;
  const int smem = 2 * kSweepNB * kSweepNB * (int)sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_sweep_rowpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = true;
  }
  k_sweep_rowpanel<<<ntiles, 256, smem, s>>>(d_desc, reinterpret_cast<const int4*>(d_tile_map),
                                             k0, d_dinv);
}

// Column panel: tile of up to 64 rows [lo, hi) of columns K: B = -B Dinv.
__global__ void __launch_bounds__(256) k_sweep_colpanel(const SweepDesc* __restrict__ descs,
                                                        const int4* __restrict__ tiles, int k0,
                                                        const double* __restrict__ dinv) {
  const int4 t = tiles[blockIdx.x];
  const SweepDesc d = descs[t.x];
  const int nb = min(kSweepNB, d.r - k0);
  const int h = t.z - t.y;
  extern __shared__ double panel_smem[];
  double* Ds = panel_smem;
  double* Ts = panel_smem + kSweepNB * kSweepNB;
  const double* Dg = dinv + (long long)t.x * kSweepNB * kSweepNB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) Ds[e] = Dg[e];
  for (int e = threadIdx.x; e < h * nb; e += blockDim.x) {
    const int i = e % h, j = e / h;
    Ts[e] = d.B[(t.y + i) + (long long)(k0 + j) * d.n];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < h * nb; e += blockDim.x) {
    const int i = e % h, j = e / h;
    double acc = 0.0;
    for (int kk = 0; kk < nb; ++kk) acc = fma(Ts[i + kk * h], Ds[kk + j * nb], acc);
    d.B[(t.y + i) + (long long)(k0 + j) * d.n] = -acc;
  }
}

void launch_sweep_colpanel(const SweepDesc* d_desc, const int* d_tile_map, int ntiles, int k0,
                           const double* d_dinv, cudaStream_t s) {
  if (ntiles <= 0) return;
  const int smem = 2 * kSweepNB * kSweepNB * (int)sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_sweep_colpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = true;
  }
  k_sweep_colpanel<<<ntiles, 256, smem, s>>>(d_desc, reinterpret_cast<const int4*>(d_tile_map),
                                             k0, d_dinv);
}

__global__ void k_sweep_setdiag(const SweepDesc* __restrict__ descs,
                                const int* __restrict__ active, int k0,
                                const double* __restrict__ dinv) {
  const int di = active[blockIdx.x];
  const SweepDesc d = descs[di];
  const int nb = min(kSweepNB, d.r - k0);
  const double* Dg = dinv + (long long)di * kSweepNB * kSweepNB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    d.B[(k0 + i) + (long long)(k0 + j) * d.n] = Dg[e];
  }
}

void launch_sweep_setdiag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                          const double* d_dinv, cudaStream_t s) {
  if (nact <= 0) return;
  k_sweep_setdiag<<<nact, 256, 0, s>>>(d_desc, d_active, k0, d_dinv);
}

// ===========================================================================
// Interpolative decomposition (one CTA per face).
//
// Column-pivoted Householder QR (Businger-Golub greedy pivoting on partial
// column norms, with the norm-downdating safeguard of Drmac and Bujanovic:
// recompute a norm when the downdated value lost more than half its digits),
// the reference's per-diagonal skeleton test |R_ii| > eps |R_00|
// (InterpDecomp.cpp:101-110) and W = R11^{-1} R12 restricted to the redundant
// columns, computed with the reference's construction of W_full and R_skel
// (InterpDecomp.cpp:115-137).
// ===========================================================================
__global__ void __launch_bounds__(512) k_id(const IdDesc* __restrict__ descs, double eps,
                                            int* __restrict__ status) {
  const IdDesc d = descs[blockIdx.x];
  const int m = d.m, n = d.n;
  double* M = d.M;
  extern __shared__ double sm[];
  double* vn1 = sm;
  double* vn2 = vn1 + n;
  double* scratch = vn2 + n;             // 64 doubles
  int* jp = reinterpret_cast<int*>(scratch + 64);
  int* flag = jp + n;                    // n
  int* pos = flag + n;                   // n (skeleton positions, then redundant)
  int* iscratch = pos + n;               // 32 (per-warp argmax indices)
  __shared__ int s_pvt;
  __shared__ int s_k;

  const int tid = threadIdx.x, nthr = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nthr >> 5;
  const double tol3z = sqrt(DBL_EPSILON * 0.5);

  for (int j = tid; j < n; j += nthr) jp[j] = j;
  for (int j = warp; j < n; j += nw) {
    double s = 0.0;
    for (int i = lane; i < m; i += 32) {
      const double v = M[i + (long long)j * m];
      s = fma(v, v, s);
    }
    s = warp_sum(s);
    if (lane == 0) { vn1[j] = sqrt(s); vn2[j] = vn1[j]; }
  }
  __syncthreads();

  const int steps = min(m, n);
  for (int i = 0; i < steps; ++i) {
    // ---- pivot choice
    if (d.order != nullptr) {
      if (tid == 0) s_pvt = i;
      __syncthreads();
      const int want = d.order[i];
      for (int j = i + tid; j < n; j += nthr)
        if (jp[j] == want) s_pvt = j;
      __syncthreads();
    } else {
      // first index of the maximum of vn1[i..n)
      double best = -1.0;
      int bi = INT_MAX;
      for (int j = i + tid; j < n; j += nthr) {
        const double v = vn1[j];
        if (v > best || (v == best && j < bi)) { best = v; bi = j; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      __syncthreads();
      if (lane == 0) { scratch[warp] = best; iscratch[warp] = bi; }
      __syncthreads();
      if (tid == 0) {
        double b = scratch[0];
        int bb = iscratch[0];
        for (int w = 1; w < nw; ++w)
          if (scratch[w] > b || (scratch[w] == b && iscratch[w] < bb)) {
            b = scratch[w];
            bb = iscratch[w];
          }
        s_pvt = (bb == INT_MAX) ? i : bb;
      }
      __syncthreads();
    }
    const int pvt = s_pvt;
    if (pvt != i) {
      for (int r = tid; r < m; r += nthr) {
        const double a = M[r + (long long)i * m];
        M[r + (long long)i * m] = M[r + (long long)pvt * m];
        M[r + (long long)pvt * m] = a;
      }
      if (tid == 0) {
        const int t = jp[pvt];
        jp[pvt] = jp[i];
        jp[i] = t;
        vn1[pvt] = vn1[i];
        vn2[pvt] = vn2[i];
      }
    }
    __syncthreads();
    // ---- Householder reflector for column i, rows i..m-1
    double xs = 0.0;
    for (int r = i + 1 + tid; r < m; r += nthr) {
      const double v = M[r + (long long)i * m];
      xs = fma(v, v, xs);
    }
    const double xnorm = sqrt(block_sum(xs, scratch));
    const double alpha = M[i + (long long)i * m];
    double tau = 0.0, beta = alpha;
    if (xnorm != 0.0) {
      beta = -copysign(hypot(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      const double scal = 1.0 / (alpha - beta);
      for (int r = i + 1 + tid; r < m; r += nthr) M[r + (long long)i * m] *= scal;
    }
    __syncthreads();
    if (tid == 0) {
      M[i + (long long)i * m] = beta;
      d.rdiag[i] = beta;
    }
    __syncthreads();
    // ---- apply H = I - tau [1; v][1; v]^T to columns i+1..n-1
    if (tau != 0.0) {
      for (int j = i + 1 + warp; j < n; j += nw) {
        double* cj = M + (long long)j * m;
        const double* ci = M + (long long)i * m;
        double w = (lane == 0) ? cj[i] : 0.0;
        for (int r = i + 1 + lane; r < m; r += 32) w = fma(ci[r], cj[r], w);
        w = warp_sum(w) * tau;
        if (lane == 0) cj[i] -= w;
        for (int r = i + 1 + lane; r < m; r += 32) cj[r] = fma(-w, ci[r], cj[r]);
      }
    }
    __syncthreads();
    // ---- partial norm downdate
    for (int j = i + 1 + tid; j < n; j += nthr) {
      flag[j] = 0;
      if (vn1[j] != 0.0) {
        double temp = fabs(M[i + (long long)j * m]) / vn1[j];
        temp = fmax(1.0 - temp * temp, 0.0);
        const double q = vn1[j] / vn2[j];
        const double temp2 = temp * q * q;
        if (temp2 <= tol3z) flag[j] = 1;
        else vn1[j] *= sqrt(temp);
      }
    }
    __syncthreads();
    for (int j = i + 1 + warp; j < n; j += nw) {
      if (!flag[j]) continue;
      double s = 0.0;
      for (int r = i + 1 + lane; r < m; r += 32) {
        const double v = M[r + (long long)j * m];
        s = fma(v, v, s);
      }
      s = warp_sum(s);
      if (lane == 0) {
        vn1[j] = (i + 1 < m) ? sqrt(s) : 0.0;
        vn2[j] = vn1[j];
      }
    }
    __syncthreads();
  }

  // ---- rank test
  const double r00 = fabs(M[0]);
  const double tol = r00 * eps;
  if (tid == 0) {
    int k = 0;
    for (int i = 0; i < n; ++i) {
      const int kp = fabs(M[i + (long long)i * m]) > tol;
      flag[i] = kp;
      if (kp) pos[k++] = i;
    }
    int rr = k;
    for (int i = 0; i < n; ++i)
      if (!flag[i]) pos[rr++] = i;
    s_k = k;
    *d.rank = k;
    if (r00 == 0.0) atomicOr(status, kStatusIdZero);
  }
  __syncthreads();
  const int k = s_k;
  for (int j = tid; j < n; j += nthr) {
    d.jpvt[j] = jp[j];
    d.keep[j] = flag[j];
  }
  // ---- W (k x (n-k)): back substitution with R_skel, one redundant column per thread
  //   W_full(a, c) = R(pos[a], c) if c >= a else 0;  R_skel = W_full(:, 0:k)
  const int nred = n - k;
  for (int b = tid; b < nred; b += nthr) {
    const int c = pos[k + b];
    double* x = d.W + (long long)b * k;
    for (int a = 0; a < k; ++a) x[a] = (c >= a) ? M[pos[a] + (long long)c * m] : 0.0;
    for (int a = k - 1; a >= 0; --a) {
      const double xa = x[a] / M[pos[a] + (long long)a * m];
      x[a] = xa;
      for (int t = 0; t < a; ++t) x[t] = fma(-M[pos[t] + (long long)a * m], xa, x[t]);
    }
  }
}

void launch_id(const IdDesc* d_desc, int nd, int max_n, double eps, int* d_status,
               cudaStream_t s) {
  if (nd <= 0) return;
  const size_t smem = (size_t)max_n * 2 * sizeof(double) + 64 * sizeof(double) +
                      (size_t)max_n * 3 * sizeof(int) + 32 * sizeof(int);
  static size_t attr = 0;
  if (smem > 48 * 1024 && smem > attr) {
    cudaFuncSetAttribute(k_id, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = smem;
  }
  k_id<<<nd, 512, smem, s>>>(d_desc, eps, d_status);
}

// ===========================================================================
// Batched sub-matrix copy (32 x 32 tiles)
// ===========================================================================
int copy_tiles(int m, int n) {
  if (m <= 0 || n <= 0) return 0;
  return ((m + 31) / 32) * ((n + 31) / 32);
}

__global__ void __launch_bounds__(256) k_copy(const CopyDesc* __restrict__ descs,
                                              const int* __restrict__ tile_off, int nd) {
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const CopyDesc c = descs[di];
  const int local = blockIdx.x - tile_off[di];
  const int tm = (c.m + 31) / 32;
  const int i0 = (local % tm) * 32, j0 = (local / tm) * 32;
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
    const int i = i0 + (e & 31), j = j0 + (e >> 5);
    if (i < c.m && j < c.n) c.dst[i + (long long)j * c.ldd] = c.src[i + (long long)j * c.lds];
  }
}

void launch_copy(const CopyDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                 cudaStream_t s) {
  if (total_tiles <= 0) return;
  k_copy<<<total_tiles, 256, 0, s>>>(d_desc, d_tile_off, nd);
}

__global__ void k_trsm_upper(const double* __restrict__ R, long long ldr, int k,
                             double* __restrict__ B, long long ldb, int nb) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nb) return;
  double* x = B + (long long)c * ldb;
  for (int a = k - 1; a >= 0; --a) {
    const double xa = x[a] / R[a + (long long)a * ldr];
    x[a] = xa;
    for (int t = 0; t < a; ++t) x[t] = fma(-R[t + (long long)a * ldr], xa, x[t]);
  }
}

void launch_trsm_upper(const double* R, long long ldr, int k, double* B, long long ldb, int nb,
                       cudaStream_t s) {
  if (nb <= 0 || k <= 0) return;
  k_trsm_upper<<<(nb + 127) / 128, 128, 0, s>>>(R, ldr, k, B, ldb, nb);
}

// ===========================================================================
// Apply: batched gather - GEMV - scatter over right-hand sides.
// trans = 0: 256 output rows per CTA, one row per thread (coalesced along M's
//            columns); trans = 1: 32 output columns per CTA, one warp per
//            column (coalesced down the column).
// ===========================================================================
constexpr int kRhsGroup = 4;
constexpr int kXChunk = 256;

int gemv_tiles(int m, int n, int trans) {
  if (m <= 0 || n <= 0) return 0;
  return trans == 0 ? (m + 255) / 256 : (n + 31) / 32;
}

__device__ __forceinline__ void gemv_emit(const GemvDesc& g, int i, int c, double y,
                                          double* u_out, long long ldu, long long contrib_ld) {
  if (g.mode == 1) g.contrib[i + (long long)c * contrib_ld] = y;
  else if (g.mode == 0) u_out[g.out_idx[i] + (long long)c * ldu] += g.alpha * y;
  else u_out[g.out_idx[i] + (long long)c * ldu] = g.alpha * y;
}

__global__ void __launch_bounds__(256) k_gemv(const GemvDesc* __restrict__ descs,
                                              const int* __restrict__ tile_off, int nd,
                                              const double* __restrict__ u_in,
                                              double* __restrict__ u_out, int nrhs,
                                              long long ldu, long long contrib_ld) {
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const GemvDesc g = descs[di];
  const int local = blockIdx.x - tile_off[di];
  __shared__ double xs[kXChunk][kRhsGroup];
  const int tid = threadIdx.x;
  if (g.trans == 0) {
    const int i = local * 256 + tid;
    for (int c0 = 0; c0 < nrhs; c0 += kRhsGroup) {
      const int nc = min(kRhsGroup, nrhs - c0);
      double acc[kRhsGroup] = {0.0, 0.0, 0.0, 0.0};
      for (int j0 = 0; j0 < g.n; j0 += kXChunk) {
        const int nj = min(kXChunk, g.n - j0);
        __syncthreads();
        for (int e = tid; e < nj * kRhsGroup; e += 256) {
          const int jj = e / kRhsGroup, cc = e % kRhsGroup;
          xs[jj][cc] = (cc < nc) ? u_in[g.in_idx[j0 + jj] + (long long)(c0 + cc) * ldu] : 0.0;
        }
        __syncthreads();
        if (i < g.m) {
          const double* col = g.M + i + (long long)j0 * g.ld;
          for (int jj = 0; jj < nj; ++jj) {
            const double mv = col[(long long)jj * g.ld];
#pragma unroll
            for (int cc = 0; cc < kRhsGroup; ++cc) acc[cc] = fma(mv, xs[jj][cc], acc[cc]);
          }
        }
      }
      if (i < g.m)
        for (int cc = 0; cc < nc; ++cc) gemv_emit(g, i, c0 + cc, acc[cc], u_out, ldu, contrib_ld);
    }
  } else {
    const int lane = tid & 31, warp = tid >> 5;
    for (int c0 = 0; c0 < nrhs; c0 += kRhsGroup) {
      const int nc = min(kRhsGroup, nrhs - c0);
      double acc[4][kRhsGroup];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < kRhsGroup; ++cc) acc[q][cc] = 0.0;
      for (int i0 = 0; i0 < g.m; i0 += kXChunk) {
        const int ni = min(kXChunk, g.m - i0);
        __syncthreads();
        for (int e = tid; e < ni * kRhsGroup; e += 256) {
          const int ii = e / kRhsGroup, cc = e % kRhsGroup;
          xs[ii][cc] = (cc < nc) ? u_in[g.in_idx[i0 + ii] + (long long)(c0 + cc) * ldu] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int j = local * 32 + warp * 4 + q;
          if (j >= g.n) continue;
          const double* col = g.M + (long long)j * g.ld + i0;
          for (int ii = lane; ii < ni; ii += 32) {
            const double mv = col[ii];
#pragma unroll
            for (int cc = 0; cc < kRhsGroup; ++cc) acc[q][cc] = fma(mv, xs[ii][cc], acc[q][cc]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = local * 32 + warp * 4 + q;
#pragma unroll
        for (int cc = 0; cc < kRhsGroup; ++cc) {
          const double y = warp_sum(acc[q][cc]);
          if (lane == 0 && j < g.n && cc < nc) gemv_emit(g, j, c0 + cc, y, u_out, ldu, contrib_ld);
        }
      }
    }
  }
}

void launch_gemv(const GemvDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                 const double* u_in, double* u_out, int nrhs, long long ldu,
                 long long contrib_ld, cudaStream_t s) {
  if (total_tiles <= 0) return;
  k_gemv<<<total_tiles, 256, 0, s>>>(d_desc, d_tile_off, nd, u_in, u_out, nrhs, ldu,
                                     contrib_ld);
}

__global__ void k_reduce_scatter(const int* __restrict__ dof, const int* __restrict__ off,
                                 const int* __restrict__ slot,
                                 const double* __restrict__ contrib, int ndof,
                                 long long contrib_ld, double alpha, double* __restrict__ u,
                                 int nrhs, long long ldu) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ndof * nrhs) return;
  const int d = (int)(t % ndof), c = (int)(t / ndof);
  double s = 0.0;
  for (int q = off[d]; q < off[d + 1]; ++q) s += contrib[slot[q] + (long long)c * contrib_ld];
  u[dof[d] + (long long)c * ldu] += alpha * s;
}

void launch_reduce_scatter(const int* d_dof, const int* d_off, const int* d_slot,
                           const double* d_contrib, int ndof, long long contrib_ld,
                           double alpha, double* u, int nrhs, long long ldu, cudaStream_t s) {
  const long long total = (long long)ndof * nrhs;
  if (total <= 0) return;
  k_reduce_scatter<<<(int)((total + 255) / 256), 256, 0, s>>>(d_dof, d_off, d_slot, d_contrib,
                                                             ndof, contrib_ld, alpha, u, nrhs,
                                                             ldu);
}

// ===========================================================================
// Operators: 7 bands over the NC^3 DOF grid, band b at band[b * NC^3 + p]:
// 0 diagonal, 1 (-i), 2 (+i), 3 (-j), 4 (+j), 5 (-k), 6 (+k). A band entry is
// zero where the neighbour is not a DOF (an index-0 plane or beyond N).
// ===========================================================================
__global__ void k_setup_node(const double* __restrict__ A, const double* __restrict__ V, int N,
                             double hh, double* __restrict__ band) {
  // SetupStencil, include/setup_stencil.hpp:34-69: entry (p, q) = -A(q)/h^2,
  // diagonal = sum of the six neighbours' A / h^2 + V(p). A, V are (NC+1)^3, i fastest.
  const int NC = N + 1, T = NC + 1;
  const long long n3 = (long long)NC * NC * NC;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n3) return;
  const int i = (int)(p % NC), j = (int)((p / NC) % NC), k = (int)(p / ((long long)NC * NC));
  if (i == 0 || j == 0 || k == 0) {
    for (int b = 0; b < 7; ++b) band[b * n3 + p] = 0.0;
    return;
  }
  auto a = [&](int x, int y, int z) { return A[x + (long long)T * y + (long long)T * T * z]; };
  double dg = 0.0;
  dg += (a(i - 1, j, k) + a(i + 1, j, k)) / hh;
  dg += (a(i, j - 1, k) + a(i, j + 1, k)) / hh;
  dg += (a(i, j, k - 1) + a(i, j, k + 1)) / hh;
  dg += V[i + (long long)T * j + (long long)T * T * k];
  band[p] = dg;
  band[1 * n3 + p] = (i - 1 >= 1) ? -a(i - 1, j, k) / hh : 0.0;
  band[2 * n3 + p] = (i + 1 <= N) ? -a(i + 1, j, k) / hh : 0.0;
  band[3 * n3 + p] = (j - 1 >= 1) ? -a(i, j - 1, k) / hh : 0.0;
  band[4 * n3 + p] = (j + 1 <= N) ? -a(i, j + 1, k) / hh : 0.0;
  band[5 * n3 + p] = (k - 1 >= 1) ? -a(i, j, k - 1) / hh : 0.0;
  band[6 * n3 + p] = (k + 1 <= N) ? -a(i, j, k + 1) / hh : 0.0;
}

void launch_setup_node(const double* d_A, const double* d_V, int N, double h, double* d_band,
                       cudaStream_t s) {
  const long long n3 = (long long)(N + 1) * (N + 1) * (N + 1);
  k_setup_node<<<(int)((n3 + 255) / 256), 256, 0, s>>>(d_A, d_V, N, h * h, d_band);
}

__global__ void k_setup_faces(const double* __restrict__ ax, const double* __restrict__ ay,
                              const double* __restrict__ az, const double* __restrict__ V,
                              int N, double hh, double* __restrict__ band) {
  // Flux form: face coefficients ax(i,j,k) between (i,j,k) and (i+1,j,k), etc.,
  // on (NC+1)^3 arrays, i fastest. Symmetric by construction.
  const int NC = N + 1, T = NC + 1;
  const long long n3 = (long long)NC * NC * NC;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n3) return;
  const int i = (int)(p % NC), j = (int)((p / NC) % NC), k = (int)(p / ((long long)NC * NC));
  if (i == 0 || j == 0 || k == 0) {
    for (int b = 0; b < 7; ++b) band[b * n3 + p] = 0.0;
    return;
  }
  auto at = [&](const double* F, int x, int y, int z) {
    return F[x + (long long)T * y + (long long)T * T * z];
  };
  const double xm = at(ax, i - 1, j, k), xp = at(ax, i, j, k);
  const double ym = at(ay, i, j - 1, k), yp = at(ay, i, j, k);
  const double zm = at(az, i, j, k - 1), zp = at(az, i, j, k);
  band[p] = (xm + xp + ym + yp + zm + zp) / hh + V[i + (long long)T * j + (long long)T * T * k];
  band[1 * n3 + p] = (i - 1 >= 1) ? -xm / hh : 0.0;
  band[2 * n3 + p] = (i + 1 <= N) ? -xp / hh : 0.0;
  band[3 * n3 + p] = (j - 1 >= 1) ? -ym / hh : 0.0;
  band[4 * n3 + p] = (j + 1 <= N) ? -yp / hh : 0.0;
  band[5 * n3 + p] = (k - 1 >= 1) ? -zm / hh : 0.0;
  band[6 * n3 + p] = (k + 1 <= N) ? -zp / hh : 0.0;
}

void launch_setup_faces(const double* d_ax, const double* d_ay, const double* d_az,
                        const double* d_V, int N, double h, double* d_band, cudaStream_t s) {
  const long long n3 = (long long)(N + 1) * (N + 1) * (N + 1);
  k_setup_faces<<<(int)((n3 + 255) / 256), 256, 0, s>>>(d_ax, d_ay, d_az, d_V, N, h * h,
                                                        d_band);
}

// y = A x (transpose = 0) or y = A^T x (transpose = 1, the reference's SpMV).
__global__ void k_stencil(const double* __restrict__ band, int NC, const double* __restrict__ x,
                          double* __restrict__ y, int nrhs, long long ldx, int transpose) {
  const long long n3 = (long long)NC * NC * NC;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n3 * nrhs) return;
  const long long p = t % n3;
  const int c = (int)(t / n3);
  const double* xc = x + c * ldx;
  const long long off[7] = {0, -1, 1, -(long long)NC, (long long)NC, -(long long)NC * NC,
                            (long long)NC * NC};
  const int rev[7] = {0, 2, 1, 4, 3, 6, 5};
  double s = 0.0;
  if (transpose == 0) {
    s = band[p] * xc[p];
#pragma unroll
    for (int b = 1; b < 7; ++b) {
      const double a = band[b * n3 + p];
      if (a != 0.0) s = fma(a, xc[p + off[b]], s);
    }
  } else {
    s = band[p] * xc[p];
#pragma unroll
    for (int b = 1; b < 7; ++b) {
      // (A^T)(p, q) = A(q, p) with q = p + off[b]: the band of q pointing back to p
      const long long q = p + off[b];
      if (q < 0 || q >= n3) continue;
      const double a = band[rev[b] * n3 + q];
      if (a != 0.0) s = fma(a, xc[q], s);
    }
  }
  y[p + c * ldx] = s;
}

void launch_stencil_apply(const double* d_band, int NC, const double* x, double* y, int nrhs,
                          long long ldx, int transpose, cudaStream_t s) {
  const long long total = (long long)NC * NC * NC * nrhs;
  k_stencil<<<(int)((total + 255) / 256), 256, 0, s>>>(d_band, NC, x, y, nrhs, ldx, transpose);
}

__global__ void k_zero_boundary(double* __restrict__ u, int NC, int nrhs, long long ldu) {
  const long long n3 = (long long)NC * NC * NC;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n3 * nrhs) return;
  const long long p = t % n3;
  const int c = (int)(t / n3);
  const int i = (int)(p % NC), j = (int)((p / NC) % NC), k = (int)(p / ((long long)NC * NC));
  if (i == 0 || j == 0 || k == 0) u[p + c * ldu] = 0.0;
}

void launch_zero_boundary(double* u, int NC, int nrhs, long long ldu, cudaStream_t s) {
  const long long total = (long long)NC * NC * NC * nrhs;
  k_zero_boundary<<<(int)((total + 255) / 256), 256, 0, s>>>(u, NC, nrhs, ldu);
}

__global__ void k_copy_vec(const double* __restrict__ x, double* __restrict__ y, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] = x[t];
}

void launch_copy_vec(const double* x, double* y, long long n, cudaStream_t s) {
  if (n <= 0) return;
  k_copy_vec<<<(int)((n + 255) / 256), 256, 0, s>>>(x, y, n);
}

// ---- deterministic dot products: fixed grid, fixed-order final sum --------
__global__ void __launch_bounds__(256) k_dot_partial(const double* __restrict__ x,
                                                     const double* __restrict__ y, long long n,
                                                     long long ld, double* __restrict__ part) {
  const int c = blockIdx.y;
  const double* xc = x + c * ld;
  const double* yc = y + c * ld;
  double s = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    s = fma(xc[t], yc[t], s);
  __shared__ double sc[40];
  s = block_sum(s, sc);
  if (threadIdx.x == 0) part[c * gridDim.x + blockIdx.x] = s;
}

__global__ void k_dot_final(const double* __restrict__ part, int nparts,
                            double* __restrict__ out) {
  const int c = blockIdx.x;
  __shared__ double sc[40];
  double s = 0.0;
  for (int t = threadIdx.x; t < nparts; t += blockDim.x) s += part[c * nparts + t];
  s = block_sum(s, sc);
  if (threadIdx.x == 0) out[c] = s;
}

void launch_dot(const double* x, const double* y, long long n, int nrhs, long long ld,
                double* d_partial, double* d_out, cudaStream_t s) {
  dim3 grid(kDotBlocks, nrhs);
  k_dot_partial<<<grid, 256, 0, s>>>(x, y, n, ld, d_partial);
  k_dot_final<<<nrhs, 256, 0, s>>>(d_partial, kDotBlocks, d_out);
}

__global__ void k_pcg_xr(double* __restrict__ x, double* __restrict__ r,
                         const double* __restrict__ p, const double* __restrict__ q,
                         const double* __restrict__ rz, const double* __restrict__ pq,
                         long long n, int nrhs, long long ld) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nrhs) return;
  const long long i = t % n;
  const int c = (int)(t / n);
  const double den = pq[c];
  const double a = (den != 0.0) ? rz[c] / den : 0.0;
  x[i + c * ld] = fma(a, p[i + c * ld], x[i + c * ld]);
  r[i + c * ld] = fma(-a, q[i + c * ld], r[i + c * ld]);
}

void launch_pcg_update_xr(double* x, double* r, const double* p, const double* q,
                          const double* rz, const double* pq, long long n, int nrhs,
                          long long ld, cudaStream_t s) {
  const long long total = n * nrhs;
  k_pcg_xr<<<(int)((total + 255) / 256), 256, 0, s>>>(x, r, p, q, rz, pq, n, nrhs, ld);
}

__global__ void k_pcg_p(double* __restrict__ p, const double* __restrict__ z,
                        const double* __restrict__ rz_new, const double* __restrict__ rz_old,
                        long long n, int nrhs, long long ld) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nrhs) return;
  const long long i = t % n;
  const int c = (int)(t / n);
  const double den = rz_old[c];
  const double b = (den != 0.0) ? rz_new[c] / den : 0.0;
  p[i + c * ld] = fma(b, p[i + c * ld], z[i + c * ld]);
}

void launch_pcg_update_p(double* p, const double* z, const double* rz_new,
                         const double* rz_old, long long n, int nrhs, long long ld,
                         cudaStream_t s) {
  const long long total = n * nrhs;
  k_pcg_p<<<(int)((total + 255) / 256), 256, 0, s>>>(p, z, rz_new, rz_old, n, nrhs, ld);
}

}  // namespace hif
