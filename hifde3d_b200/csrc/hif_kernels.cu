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

#include <cooperative_groups.h>

#include <cfloat>
#include <climits>
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

namespace hif {

namespace {

// Kernel attributes are per device (cudaFuncSetAttribute acts on the current
// device) and launchers run on several host threads at once (the serving
// loop's factor workers): every one-time setting goes through this table,
// keyed by (device, kernel), under one mutex.
std::mutex g_attr_mu;
std::map<std::pair<int, const void*>, size_t> g_attr_smem;

// Raises `fn`'s dynamic shared-memory limit on the current device to at least
// `bytes` (never lowers it).
// Multiprocessor count of the current device (cached per device).
int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_attr_mu);
  static std::map<int, int> sms;
  auto it = sms.find(dev);
  if (it != sms.end()) return it->second;
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (n <= 0) n = 1;
  sms[dev] = n;
  return n;
}

void ensure_smem(const void* fn, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_attr_mu);
  size_t& cur = g_attr_smem[{dev, fn}];
  if (bytes > cur) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cur = bytes;
  }
}

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
// Tiles of 32 rows x 64 columns: lane x of warp w assembles row x of columns
// w, w + 8, ..., w + 56, so a thread's row, its stencil row and its row covers
// (up to three sources, each turned into a pointer to the source's row) stay in
// registers, and a column's covers are warp-uniform shared-memory reads.
constexpr int kGTM = 32, kGTN = 64;

int gather_tiles(int m, int n) {
  return ((m + kGTM - 1) / kGTM) * ((n + kGTN - 1) / kGTN);
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

// Persistent over the tile list: CTA b assembles the contiguous tiles
// [b chunk, (b + 1) chunk), so the target of its first tile is found once by
// binary search and the rest by stepping through tile_off (a per-tile search
// costs ~log2(targets) dependent loads, more than a small tile's own work).
__global__ void __launch_bounds__(256) k_gather(const GatherTarget* __restrict__ tg,
                                                const int* __restrict__ tile_off, int ntg,
                                                int total_tiles,
                                                const SourceDesc* __restrict__ src,
                                                const int* __restrict__ src_owner,
                                                const int* __restrict__ dof_src,
                                                const double* __restrict__ band,
                                                long long ncell3, int NC) {
  const int chunk = (total_tiles + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * chunk, t1 = min(total_tiles, t0 + chunk);
  if (t0 >= t1) return;
  int d = find_desc(tile_off, ntg, t0);
  int dbeg = tile_off[d], dend = tile_off[d + 1];
  __shared__ int s_col[kGTN];
  __shared__ CoverEntry s_cc[kGTN][kCover];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int NC2 = NC * NC;
  for (int t = t0; t < t1; ++t) {
    while (t >= dend) {
      ++d;
      dbeg = dend;
      dend = tile_off[d + 1];
    }
    const GatherTarget g = tg[d];
    const int local = t - dbeg;
    const int tiles_m = (g.m + kGTM - 1) / kGTM;
    const int i0 = (local % tiles_m) * kGTM, j0 = (local / tiles_m) * kGTN;
    __syncthreads();  // the previous tile's readers of s_col / s_cc are done
    if (threadIdx.x < kGTN) {
      const int j = j0 + threadIdx.x;
      const int q = (j < g.n) ? g.cols[j] : -1;
      s_col[threadIdx.x] = q;
      resolve_cover(g, q, dof_src, src_owner, ncell3, s_cc[threadIdx.x]);
    }
    // this thread's row: DOF, stencil row and source rows (a source's entries
    // are addressed with 32-bit positions times its leading dimension)
    const int i = i0 + lane;
    const int p = (i < g.m) ? g.rows[i] : -1;
    CoverEntry rc[kCover];
    resolve_cover(g, p, dof_src, src_owner, ncell3, rc);
    const double* rp[kCover];
    int rs[kCover], rld[kCover];
#pragma unroll
    for (int a = 0; a < kCover; ++a) {
      rs[a] = rc[a].src;
      rp[a] = nullptr;
      rld[a] = 0;
      if (rc[a].src >= 0) {
        const SourceDesc sd = src[rc[a].src];
        rp[a] = sd.ptr + rc[a].pos;
        rld[a] = (int)sd.ld;
      }
    }
    __syncthreads();
    if (i < g.m) {
      const bool row_a0 = i < g.a0_skip;
      const bool row_a22 = g.a22_out != nullptr && i < g.r;
      const int ld = (int)g.ld;
      double* orow = g.out + i;
#pragma unroll 2
      for (int cc = warp; cc < kGTN; cc += 8) {
        const int j = j0 + cc;
        if (j >= g.n) break;
        double v = 0.0;
        if (row_a0 || j < g.a0_skip) {
          // stencil term: q - p in {0, -1, 1, -NC, NC, -NC^2, NC^2} -> bands 0..6
          const int dd = s_col[cc] - p, ad = abs(dd);
          if (ad == 0 || ad == 1 || ad == NC || ad == NC2) {
            const int b = (ad == 0 ? 0 : (ad == 1 ? 1 : (ad == NC ? 3 : 5))) + (dd > 0 ? 1 : 0);
            v = band[b * ncell3 + p];
          }
        }
        // sources holding both DOFs, in the column's cover order (a column cover
        // is warp-uniform, so an empty one is skipped by the whole warp)
#pragma unroll
        for (int c = 0; c < kCover; ++c) {
          const CoverEntry ce = s_cc[cc][c];
          if (ce.src < 0) continue;
#pragma unroll
          for (int a = 0; a < kCover; ++a)
            if (rs[a] == ce.src) v += rp[a][(long long)ce.pos * rld[a]];
        }
        orow[(long long)j * ld] = v;
        if (row_a22 && j < g.r) g.a22_out[i + (long long)j * g.r] = v;
      }
    }
  }
}

void launch_gather(const GatherTarget* d_tg, const int* d_tile_off, int ntg, int total_tiles,
                   const SourceDesc* d_src, const int* d_src_owner, const int* d_dof_src,
                   const double* d_band, long long ncell3, int NC, cudaStream_t s) {
  if (total_tiles <= 0) return;
  // 8 resident CTAs of 256 threads per SM, 148 SMs, several waves' worth of
  // chunks so that uneven tiles even out
  const int grid = std::min(total_tiles, 148 * 8 * 4);
  k_gather<<<grid, 256, 0, s>>>(d_tg, d_tile_off, ntg, total_tiles, d_src, d_src_owner,
                                d_dof_src, d_band, ncell3, NC);
}

// ===========================================================================
// Batched FP64 GEMM: 64x64x16 tiles, 256 threads, 4x4 outputs per thread.
// Thread (tx, ty) owns rows tx + 16 a and columns ty + 16 b so that the
// epilogue stores are coalesced along the (column-major) rows.
// ===========================================================================
constexpr int kBM = 64, kBN = 64, kBK = 16;

int dgemm_tiles(int m, int n, int tile) {
  if (m <= 0 || n <= 0) return 0;
  return ((m + tile - 1) / tile) * ((n + tile - 1) / tile);
}

__global__ void __launch_bounds__(256) k_dgemm(const GemmDesc* __restrict__ descs,
                                               const int* __restrict__ tile_off, int nd) {
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const GemmDesc g = descs[di];
  const int local = blockIdx.x - tile_off[di];
  const int tiles_m = (g.m + kBM - 1) / kBM;
  if (g.skip && *g.skip) return;
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

  const int kend = g.a_lower ? min(g.k, m0 + kBM) : g.k;
  const int kbeg = g.b_lower ? min(kend, n0) : 0;  // n0: a multiple of kBK
  const int nk = (kend - kbeg + kBK - 1) / kBK;
  if (nk > 0) {
    load_a(kbeg);
    load_b(kbeg);
    store(0);
  }
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int buf = t & 1;
    if (t + 1 < nk) {
      load_a(kbeg + (t + 1) * kBK);
      load_b(kbeg + (t + 1) * kBK);
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
  // with beta != 0 every C entry is loaded before the first store, so that the
  // 16 loads are in flight together
  double cv[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int gm = m0 + tx + 16 * a, gn = n0 + ty + 16 * b;
      cv[a][b] = (g.beta != 0.0 && gm < g.m && gn < g.n) ? g.C[gm + (long long)gn * g.ldc] : 0.0;
    }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int gn = n0 + ty + 16 * b;
    if (gn >= g.n) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int gm = m0 + tx + 16 * a;
      if (gm >= g.m) continue;
      const double v = g.alpha * acc[a][b];
      g.C[gm + (long long)gn * g.ldc] = (g.beta == 0.0) ? v : fma(g.beta, cv[a][b], v);
    }
  }
}

// ---------------------------------------------------------------------------
// 128 x 128 x 16 tiles, 256 threads, 8 x 8 outputs per thread, operands staged
// through a 3-stage cp.async pipeline (8-byte copies: sub-matrix views are
// only 8-byte aligned; out-of-range elements are zero-filled by the copy).
// ---------------------------------------------------------------------------
constexpr int kLBM = 128, kLBN = 128, kLBK = 16, kLStages = 3;
constexpr int kLAStride = kLBM + 2;  // doubles per k-row of the A stage
constexpr int kLBStride = kLBN + 2;
constexpr int kLSmem = kLStages * kLBK * (kLAStride + kLBStride) * (int)sizeof(double);
// with beta != 0 the C tile is prefetched into shared memory with the first stages
constexpr int kLSmemC = kLSmem + kLBM * kLBN * (int)sizeof(double);

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
  const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem),
               "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__global__ void __launch_bounds__(512, 1) k_dgemm128(const GemmDesc* __restrict__ descs,
                                                     const int* __restrict__ tile_off, int nd) {
  extern __shared__ double lsm[];
  double* As = lsm;                                  // [stage][k][kLAStride]
  double* Bs = lsm + kLStages * kLBK * kLAStride;    // [stage][k][kLBStride]
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const GemmDesc g = descs[di];
  const int local = blockIdx.x - tile_off[di];
  const int tiles_m = (g.m + kLBM - 1) / kLBM;
  if (g.lower && local % tiles_m < local / tiles_m) return;
  if (g.skip && *g.skip) return;
  const int m0 = (local % tiles_m) * kLBM, n0 = (local / tiles_m) * kLBN;
  const int tid = threadIdx.x;

  auto issue = [&](int stage, int k0) {
    double* as = As + stage * kLBK * kLAStride;
    double* bs = Bs + stage * kLBK * kLBStride;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 512 * q;
      int mm, kk;
      if (g.transA == 0) { mm = e % kLBM; kk = e / kLBM; } else { mm = e / kLBK; kk = e % kLBK; }
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < g.m && gk < g.k;
      const double* src = ok ? ((g.transA == 0) ? g.A + gm + (long long)gk * g.lda
                                                : g.A + gk + (long long)gm * g.lda)
                             : g.A;
      cp_async8(as + kk * kLAStride + mm, src, ok);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 512 * q;
      int nn, kk;
      if (g.transB == 0) { kk = e % kLBK; nn = e / kLBK; } else { nn = e % kLBN; kk = e / kLBN; }
      const int gn = n0 + nn, gk = k0 + kk;
      const bool ok = gn < g.n && gk < g.k;
      const double* src = ok ? ((g.transB == 0) ? g.B + gk + (long long)gn * g.ldb
                                                : g.B + gn + (long long)gk * g.ldb)
                             : g.B;
      cp_async8(bs + kk * kLBStride + nn, src, ok);
    }
  };

  // FP64 tensor cores: mma.sync m8n8k4 (DMMA). 16 warps as 4 (m) x 4 (n), warp
  // tile 32 x 32 = 4 x 4 MMA tiles (four warps per SM sub-partition keep the
  // DMMA pipe fed across the fixed issue spacing of one warp). Fragments (PTX
  // ISA, m8n8k4 .f64): with g = lane / 4, t = lane % 4, A holds (row g, k t),
  // B holds (k t, col g), C holds (row g, cols 2t and 2t + 1).
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
  const int gq = lane >> 2, tq = lane & 3;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

  double* Cs = lsm + kLStages * kLBK * (kLAStride + kLBStride);  // [col][row], 128 x 128
  const bool prefetch_c = g.beta != 0.0;
  if (prefetch_c) {
    for (int e = tid; e < kLBM * kLBN; e += 512) {
      const int i = e % kLBM, j = e / kLBM;
      const bool ok = (m0 + i) < g.m && (n0 + j) < g.n;
      cp_async8(Cs + e, ok ? g.C + (m0 + i) + (long long)(n0 + j) * g.ldc : g.C, ok);
    }
  }
  const int kend = g.a_lower ? min(g.k, m0 + kLBM) : g.k;
  const int kbeg = g.b_lower ? min(kend, n0) : 0;  // n0: a multiple of kLBK
  const int nk = (kend - kbeg + kLBK - 1) / kLBK;
#pragma unroll
  for (int st = 0; st < kLStages - 1; ++st) {
    if (st < nk) issue(st, kbeg + st * kLBK);
    cp_async_commit();  // the first group also carries the C tile
  }
  for (int t = 0; t < nk; ++t) {
    cp_async_wait<kLStages - 2>();
    __syncthreads();
    const int nt = t + kLStages - 1;
    if (nt < nk) issue(nt % kLStages, kbeg + nt * kLBK);
    cp_async_commit();
    const double* as = As + (t % kLStages) * kLBK * kLAStride;
    const double* bs = Bs + (t % kLStages) * kLBK * kLBStride;
#pragma unroll
    for (int k4 = 0; k4 < kLBK; k4 += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = as[(k4 + tq) * kLAStride + wm + a * 8 + gq];
#pragma unroll
      for (int b = 0; b < 4; ++b) bf[b] = bs[(k4 + tq) * kLBStride + wn + b * 8 + gq];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
          asm volatile(
              "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
              : "+d"(acc[a][b][0]), "+d"(acc[a][b][1])
              : "d"(af[a]), "d"(bf[b]));
    }
  }
  cp_async_wait<0>();
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int gm = m0 + wm + a * 8 + gq;
    if (gm >= g.m) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int cl = wn + b * 8 + tq * 2 + c;
        const int gn = n0 + cl;
        if (gn >= g.n) continue;
        double* cp = g.C + gm + (long long)gn * g.ldc;
        const double v = g.alpha * acc[a][b][c];
        *cp = prefetch_c ? fma(g.beta, Cs[cl * kLBM + wm + a * 8 + gq], v) : v;
      }
  }
}

void launch_dgemm(const GemmDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                  cudaStream_t s, int tile) {
  if (total_tiles <= 0) return;
  if (tile == 128) {
    ensure_smem((const void*)k_dgemm128, kLSmemC);
    k_dgemm128<<<total_tiles, 512, kLSmemC, s>>>(d_desc, d_tile_off, nd);
  } else {
    k_dgemm<<<total_tiles, 256, 0, s>>>(d_desc, d_tile_off, nd);
  }
}

__global__ void k_splitk_reduce(const SplitKDesc* __restrict__ descs) {
  const SplitKDesc d = descs[blockIdx.y];
  const long long mn = (long long)d.m * d.n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < mn;
       e += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int q = 0; q < d.S; ++q) acc += d.P[e + q * mn];
    const int i = (int)(e % d.m), j = (int)(e / d.m);
    double* c = d.C + i + (long long)j * d.ldc;
    *c = (d.beta == 0.0) ? d.alpha * acc : fma(d.beta, *c, d.alpha * acc);
  }
}

void launch_splitk_reduce(const SplitKDesc* d_desc, int nd, cudaStream_t s) {
  if (nd <= 0) return;
  dim3 grid(64, nd);
  k_splitk_reduce<<<grid, 256, 0, s>>>(d_desc);
}

// TF32 rounding of an FP32 value (round to nearest, ties away), as a 32-bit container.
__device__ __forceinline__ unsigned tf32_of(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

// ===========================================================================
// Split-TF32 GEMM on the 5th-generation tensor cores (tcgen05).
//
// 1. k_tc_convert splits every FP64 operand value into a TF32 pair
//    (hi = rn(x), lo = rn(x - hi)) and stores the pairs as tiles of 128 rows
//    x 32 values of k in the K-major canonical layout without swizzle that the
//    tensor cores read from shared memory: 8-row x 16-byte core matrices of
//    128 bytes, K-adjacent ones 128 bytes apart (LBO), 8-row groups 1024 bytes
//    apart (SBO); a tile is 16 KB of hi followed by 16 KB of lo.
// 2. k_gemm_tc computes one 128 x 128 tile of C per CTA with warp roles:
//    one thread of warp 0 brings the A and B tiles of each k step into a
//    3-stage ring with bulk asynchronous copies (cp.async.bulk, completion
//    counted in bytes on the stage's mbarrier); one thread of warp 1 issues,
//    per k-step of 8, the products lo*hi, hi*lo, hi*hi (M = N = 128, K = 8,
//    FP32 accumulation in tensor memory) and releases the stage with
//    tcgen05.commit; warps 4-7 read the accumulator (warp w: lanes
//    32 (w - 4) .. + 31) every 256 values of k and add it to an FP64
//    accumulator that also lives in tensor memory (two 32-bit columns per
//    value), so no FP32 sum runs over more than 256 terms and C is read and
//    written once (alpha acc + beta C). Two FP32 accumulators alternate, so
//    the products of the next chunk proceed while one is read; the CTA holds
//    all 512 tensor-memory columns (one CTA per SM by its shared memory).
// Every mbarrier wait is bounded (globaltimer, 2 s); a wait that runs out
// marks the CTA aborted (every role stops waiting), records kStatusTimeout and
// leaves the tile unwritten; the CTA still frees its tensor memory.
// ===========================================================================
constexpr int kTcM = 128, kTcN = 128, kTcK = 32, kTcStages = 3, kTcChunk = 256;
constexpr int kTcPart = kTcM * kTcK * 4;             // bytes of one operand part (hi or lo)
constexpr int kTcTile = 2 * kTcPart;                 // one converted operand tile (hi, lo)
constexpr int kTcStage = 2 * kTcTile;                // A tile, B tile
constexpr int kTcSmem = kTcStages * kTcStage + 256;  // + mbarriers, tensor memory address
constexpr unsigned long long kTcWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the completion of the mbarrier phase with the given parity;
// gives up at once when *abort is set, and sets it when the time runs out.
__device__ __forceinline__ bool mbar_wait(unsigned addr, unsigned parity,
                                          volatile int* abort = nullptr) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (abort && *abort) return false;
    if (global_ns() - t0 > kTcWaitNs) {
      if (abort) *abort = 1;
      return false;
    }
  }
}

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 1024 B,
// descriptor version 1 (sm_100).
__device__ __forceinline__ unsigned long long tc_desc(unsigned addr) {
  unsigned long long d = (unsigned long long)((addr >> 4) & 0x3FFF);
  d |= (unsigned long long)(128 >> 4) << 16;
  d |= (unsigned long long)(1024 >> 4) << 32;
  d |= 1ull << 46;
  return d;
}

// Instruction descriptor, kind::tf32: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr unsigned kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(kTcN >> 3) << 17) |
                              ((unsigned)(kTcM >> 4) << 24);

// Byte offset of element (row, k) of one 128 x 32 operand part.
__device__ __forceinline__ int tc_off(int row, int kc) {
  return (((row >> 3) * (kTcK / 4) + kc) << 7) + ((row & 7) << 4);
}

__global__ void __launch_bounds__(256) k_tc_convert(const TcOperand* __restrict__ ops,
                                                    const int* __restrict__ tile_off, int nops) {
  const int oi = find_desc(tile_off, nops, blockIdx.x);
  const TcOperand o = ops[oi];
  const int local = blockIdx.x - tile_off[oi];
  const int kt_n = (o.kdim + kTcK - 1) / kTcK;
  const int rt = local / kt_n, kt = local % kt_n;
  unsigned char* dst = o.out + (size_t)local * kTcTile;
  const int row = threadIdx.x & 127, half = threadIdx.x >> 7;
  const int gi = rt * kTcM + row;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kc = half + 2 * i;
    uint4 h, l;
    unsigned* ph = &h.x;
    unsigned* pl = &l.x;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gk = kt * kTcK + 4 * kc + e;
      const double x = (gi < o.rows && gk < o.kdim)
                           ? (o.trans ? o.X[gk + (long long)gi * o.ld] : o.X[gi + (long long)gk * o.ld])
                           : 0.0;
      const float f = (float)x;
      const unsigned fh = tf32_of(f);
      ph[e] = fh;
      pl[e] = tf32_of(f - __uint_as_float(fh));
    }
    const int off = tc_off(row, kc);
    *reinterpret_cast<uint4*>(dst + off) = h;
    *reinterpret_cast<uint4*>(dst + kTcPart + off) = l;
  }
}

void launch_tc_convert(const TcOperand* d_ops, const int* d_tile_off, int nops, int total_tiles,
                       cudaStream_t s) {
  if (total_tiles <= 0) return;
  k_tc_convert<<<total_tiles, 256, 0, s>>>(d_ops, d_tile_off, nops);
}

__global__ void __launch_bounds__(256, 1) k_gemm_tc(const TcGemm* __restrict__ descs,
                                                    const int* __restrict__ tile_off, int nd,
                                                    int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(tc_smem + kTcStages * kTcStage);
  unsigned long long* full = bars;                  // [kTcStages]
  unsigned long long* empty = bars + kTcStages;     // [kTcStages]
  unsigned long long* tfull = bars + 2 * kTcStages;  // [2]
  unsigned long long* tempty = tfull + 2;            // [2]
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(tempty + 2);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const TcGemm g = descs[di];
  const int local = blockIdx.x - tile_off[di];
  const int tiles_m = (g.m + kTcM - 1) / kTcM;
  const int mt = local % tiles_m, nt = local / tiles_m;
  if (g.lower && mt < nt) return;  // whole CTA, before any barrier or allocation
  const int m0 = mt * kTcM, n0 = nt * kTcN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kt_n = (g.k + kTcK - 1) / kTcK;
  constexpr int spc = kTcChunk / kTcK;  // k steps per chunk
  const int nchunk = (kt_n + spc - 1) / spc;

  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(4 * kTcN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int q = 0; q < kTcStages; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[q])) : "memory");
    }
    for (int q = 0; q < 2; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&tfull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&tempty[q])) : "memory");
    }
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // producer: bulk copies of the converted A and B tiles
    const unsigned char* a_src = g.A + (size_t)mt * kt_n * kTcTile;
    const unsigned char* b_src = g.B + (size_t)nt * kt_n * kTcTile;
    for (int kt = 0; kt < kt_n; ++kt) {
      const int s = kt % kTcStages;
      if (kt >= kTcStages &&
          !mbar_wait(smem_u32(&empty[s]), (unsigned)((kt / kTcStages - 1) & 1), abort))
        break;
      const unsigned fb = smem_u32(&full[s]);
      const unsigned dst = smem_u32(tc_smem + s * kTcStage);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                   "r"(kTcStage)
                   : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(dst),
          "l"(a_src + (size_t)kt * kTcTile), "r"(kTcTile), "r"(fb)
          : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(dst + kTcTile),
          "l"(b_src + (size_t)kt * kTcTile), "r"(kTcTile), "r"(fb)
          : "memory");
    }
  } else if (warp == 1 && lane == 0) {
    // tensor-core issue
    for (int kt = 0; kt < kt_n; ++kt) {
      const int s = kt % kTcStages, c = kt / spc, buf = c & 1;
      if (kt % spc == 0 && c >= 2 &&
          !mbar_wait(smem_u32(&tempty[buf]), (unsigned)((c / 2 - 1) & 1), abort))
        break;
      if (!mbar_wait(smem_u32(&full[s]), (unsigned)((kt / kTcStages) & 1), abort)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned base = smem_u32(tc_smem + s * kTcStage);
      const unsigned dacc = tmem + (unsigned)(buf * kTcN);
#pragma unroll
      for (int j = 0; j < kTcK / 8; ++j) {
        const unsigned long long dah = tc_desc(base + 0 * kTcPart + 256 * j);
        const unsigned long long dal = tc_desc(base + 1 * kTcPart + 256 * j);
        const unsigned long long dbh = tc_desc(base + 2 * kTcPart + 256 * j);
        const unsigned long long dbl = tc_desc(base + 3 * kTcPart + 256 * j);
        const unsigned long long da[3] = {dal, dah, dah}, db[3] = {dbh, dbl, dbh};
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const unsigned acc = (kt % spc > 0 || j > 0 || p > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred q;\n\t"
              "setp.ne.b32 q, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, q;\n\t}\n" ::"r"(dacc),
              "l"(da[p]), "l"(db[p]), "r"(kTcIdesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&empty[s]))
          : "memory");
      if (kt % spc == spc - 1 || kt == kt_n - 1)
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&tfull[buf]))
            : "memory");
    }
  } else if (warp >= 4) {
    // epilogue: every chunk's FP32 sums are added to an FP64 accumulator kept
    // in tensor memory (columns 2 kTcN + 2 j, + 1: low and high words of
    // column j's value); C is read and written once, after the last chunk
    const int q = warp - 4;
    const int gm = m0 + 32 * q + lane;
    const unsigned lanes = (unsigned)(32 * q) << 16;
    for (int c = 0; c < nchunk; ++c) {
      const int buf = c & 1;
      const bool last = c == nchunk - 1;
      if (!mbar_wait(smem_u32(&tfull[buf]), (unsigned)((c / 2) & 1), abort)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
      for (int cc = 0; cc < kTcN / 16; ++cc) {
        unsigned v[16], w[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tmem + lanes + (unsigned)(buf * kTcN + 16 * cc))
            : "memory");
        const unsigned a64 = tmem + lanes + (unsigned)(2 * kTcN + 32 * cc);
        if (c > 0) {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
              "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
              "[%32];"
              : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]),
                "=r"(w[6]), "=r"(w[7]), "=r"(w[8]), "=r"(w[9]), "=r"(w[10]), "=r"(w[11]),
                "=r"(w[12]), "=r"(w[13]), "=r"(w[14]), "=r"(w[15]), "=r"(w[16]), "=r"(w[17]),
                "=r"(w[18]), "=r"(w[19]), "=r"(w[20]), "=r"(w[21]), "=r"(w[22]), "=r"(w[23]),
                "=r"(w[24]), "=r"(w[25]), "=r"(w[26]), "=r"(w[27]), "=r"(w[28]), "=r"(w[29]),
                "=r"(w[30]), "=r"(w[31])
              : "r"(a64)
              : "memory");
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        double acc[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const double x = (double)__uint_as_float(v[e]);
          acc[e] = (c > 0) ? __hiloint2double((int)w[2 * e + 1], (int)w[2 * e]) + x : x;
        }
        if (!last) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            w[2 * e] = (unsigned)__double2loint(acc[e]);
            w[2 * e + 1] = (unsigned)__double2hiint(acc[e]);
          }
          asm volatile(
              "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
              "%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
              "%32};" ::"r"(a64),
              "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]),
              "r"(w[7]), "r"(w[8]), "r"(w[9]), "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]),
              "r"(w[14]), "r"(w[15]), "r"(w[16]), "r"(w[17]), "r"(w[18]), "r"(w[19]),
              "r"(w[20]), "r"(w[21]), "r"(w[22]), "r"(w[23]), "r"(w[24]), "r"(w[25]),
              "r"(w[26]), "r"(w[27]), "r"(w[28]), "r"(w[29]), "r"(w[30]), "r"(w[31])
              : "memory");
          asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        } else if (gm < g.m) {
          // the 16 C entries loaded before the first store (in flight together)
          double cv[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int gn = n0 + 16 * cc + e;
            cv[e] = (g.beta != 0.0 && gn < g.n) ? g.C[gm + (long long)gn * g.ldc] : 0.0;
          }
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int gn = n0 + 16 * cc + e;
            if (gn < g.n) {
              const double val = g.alpha * acc[e];
              g.C[gm + (long long)gn * g.ldc] = (g.beta == 0.0) ? val : fma(g.beta, cv[e], val);
            }
          }
        }
      }
      // this chunk's accumulator has been read: release it to the next chunk but one
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[buf]))
                     : "memory");
    }
    if (kt_n == 0 && gm < g.m) {
      for (int e = 0; e < kTcN; ++e) {
        const int gn = n0 + e;
        if (gn < g.n) {
          double* cp = g.C + gm + (long long)gn * g.ldc;
          *cp = (g.beta == 0.0) ? 0.0 : g.beta * *cp;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && *abort) atomicOr(status, kStatusTimeout);
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(4 * kTcN)
                 : "memory");
  }
}

void launch_gemm_tc(const TcGemm* d_desc, const int* d_tile_off, int nd, int total_tiles,
                    int* d_status, cudaStream_t s) {
  if (total_tiles <= 0) return;
  ensure_smem((const void*)k_gemm_tc, kTcSmem);
  k_gemm_tc<<<total_tiles, 256, kTcSmem, s>>>(d_desc, d_tile_off, nd, d_status);
}

// ===========================================================================
// FP64 products on the int8 tensor cores (Ozaki scheme).
//
// C = op(A) op(B) is computed from exact integer pieces of the operands.
// Every operand row (row i of op(A), column j of op(B)) is scaled by a power
// of two into (-1, 1) and cut into S signed 7-bit slices by truncation
// (v <- 128 v; q = trunc(v); v <- v - q, exact in FP64):
//   x_ik = 2^{e_i} sum_{s<S} q_s(i, k) 2^{-7(s+1)} + r_ik,  |r_ik| < 2^{e_i - 7S}.
// Then
//   C_ij = 2^{e_i + f_j - 14} sum_{d<S} 2^{-7d} P_d(i, j),  P_d = sum_{s+t=d} Q_s R_t^T,
// the slice pairs with s + t >= S being dropped (they weigh less than the
// representation error). |P_d| <= (d + 1) k 127^2 < 2^31 for k <= kOzMaxK, so
// each diagonal sum is exact in int32 and accumulates over the whole k range
// in its own tensor-memory accumulator (tcgen05.mma kind::i8, M = 128,
// N = BN, K = 32); the epilogue reads each once, sums them in FP64 (Horner in
// 2^-7) and scales by 2^{e_i + f_j - 14}. Integer accumulation makes the
// result independent of the order of the products. The error is of order
// k 2^{-7S} max_k |a_ik| max_k |b_kj| (an FP64 product's scales with
// u sum_k |a_ik| |b_kj|).
// A converted tile holds S slices of 128 rows x 64 bytes, each in the K-major
// canonical layout without swizzle: 8-row x 16-byte core matrices of 128 B,
// K-adjacent ones 128 B apart (LBO), 8-row groups 512 B apart (SBO), so rows
// 64..127 of a slice are its second 4 KB and a 64-row B tile is a contiguous
// half of each slice.
// Roles as in k_gemm_tc: one thread of warp 0 streams the A and B tiles of
// every 64-k step into a ring of stages (cp.async.bulk, completion counted in
// bytes on the stage's mbarrier); one thread of warp 1 issues the
// S (S + 1) / 2 slice products of each 32-k half and releases the stage with
// tcgen05.commit; warps 4-7 wait for the last products and write C. Waits are
// bounded as in k_gemm_tc.
// ===========================================================================
// Tile (128 rows x 64 k) of an operand into shared memory, read along the
// operand's contiguous dimension: for trans = 0 lanes run over rows, for
// trans = 1 over k, so that both layouts are read in whole cache lines. Each
// thread issues its 32 loads before the first store, so that they are in
// flight together. T[i * kOzTs + k]; entries past the operand are zero.
constexpr int kOzTs = kOzK + 1;
constexpr size_t kOzConvSmem = (size_t)128 * kOzTs * sizeof(double);
static_assert(128 * kOzK == 256 * 32, "tile loader: 256 threads x 32 elements");
__device__ __forceinline__ void oz_load_tile(const OzOperand& o, int rt, int kt, double* T) {
  const int r0 = rt * 128, k0 = kt * kOzK;
  double v[32];
  if (o.trans == 0) {
    // thread: row i = tid & 127, k = (tid >> 7) + 2 j
    const int i = threadIdx.x & 127, kb = threadIdx.x >> 7;
    const int gi = r0 + i;
    const double* src = o.X + gi;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int gk = k0 + kb + 2 * j;
      v[j] = (gi < o.rows && gk < o.kdim) ? __ldg(src + (long long)gk * o.ld) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) T[i * kOzTs + kb + 2 * j] = v[j];
  } else {
    // thread: k = tid & 63, row i = (tid >> 6) + 4 j
    const int k = threadIdx.x & (kOzK - 1), ib = threadIdx.x >> 6;
    const int gk = k0 + k;
    const double* src = o.X + gk;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int gi = r0 + ib + 4 * j;
      v[j] = (gi < o.rows && gk < o.kdim) ? __ldg(src + (long long)gi * o.ld) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) T[(ib + 4 * j) * kOzTs + k] = v[j];
  }
}

// Row exponents, read in place along the operand's contiguous dimension:
// trans = 0, two threads per row (lanes over consecutive rows), 32 k each;
// trans = 1, a warp per row (lanes over consecutive k), 16 rows per warp. The
// 32 loads of a thread are issued before the first maximum.
__global__ void __launch_bounds__(256) k_oz_exp(const OzOperand* __restrict__ ops,
                                                const int* __restrict__ tile_off, int nops) {
  const int oi = find_desc(tile_off, nops, blockIdx.x);
  const OzOperand o = ops[oi];
  const int local = blockIdx.x - tile_off[oi];
  const int kt_n = (o.kdim + kOzK - 1) / kOzK;
  const int rt = local / kt_n, kt = local % kt_n;
  const int k0 = kt * kOzK;
  double v[32];
  if (o.trans == 0) {
    const int row = threadIdx.x & 127, half = threadIdx.x >> 7;
    const int gi = rt * 128 + row;
    if (gi >= o.rows) return;
    const double* src = o.X + gi;
#pragma unroll
    for (int e = 0; e < 32; ++e) {
      const int gk = k0 + 32 * half + e;
      v[e] = gk < o.kdim ? __ldg(src + (long long)gk * o.ld) : 0.0;
    }
    double m = 0.0;
#pragma unroll
    for (int e = 0; e < 32; ++e) m = fmax(m, fabs(v[e]));
    if (m > 0.0) {
      int ex;
      frexp(m, &ex);  // m < 2^ex
      atomicMax(&o.rexp[gi], ex);
    }
  } else {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gk0 = k0 + lane, gk1 = k0 + 32 + lane;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int gi = rt * 128 + warp + 8 * j;
      const double* src = o.X + (long long)gi * o.ld;
      v[2 * j] = (gi < o.rows && gk0 < o.kdim) ? __ldg(src + gk0) : 0.0;
      v[2 * j + 1] = (gi < o.rows && gk1 < o.kdim) ? __ldg(src + gk1) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int gi = rt * 128 + warp + 8 * j;
      double m = fmax(fabs(v[2 * j]), fabs(v[2 * j + 1]));
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
      if (lane == 0 && gi < o.rows && m > 0.0) {
        int ex;
        frexp(m, &ex);
        atomicMax(&o.rexp[gi], ex);
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_oz_slice(const OzOperand* __restrict__ ops,
                                                  const int* __restrict__ tile_off, int nops,
                                                  int S) {
  extern __shared__ double oz_t[];
  const int oi = find_desc(tile_off, nops, blockIdx.x);
  const OzOperand o = ops[oi];
  const int local = blockIdx.x - tile_off[oi];
  const int kt_n = (o.kdim + kOzK - 1) / kOzK;
  const int rt = local / kt_n, kt = local % kt_n;
  oz_load_tile(o, rt, kt, oz_t);
  __syncthreads();
  const int row = threadIdx.x & 127, half = threadIdx.x >> 7;
  const int gi = rt * 128 + row;
  // rows without a nonzero keep the cleared exponent; their slices are zero
  const int ex = gi < o.rows ? max(o.rexp[gi], -4096) : 0;
  signed char* dst = o.out + (size_t)local * S * kOzPart;
#pragma unroll 1
  for (int c = 0; c < 2; ++c) {
    const int kc = 2 * half + c;  // 16-byte chunk of the row's 64 bytes
    unsigned w[kOzMaxS][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
      for (int s = 0; s < kOzMaxS; ++s) w[s][q] = 0u;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const double x = oz_t[row * kOzTs + 16 * kc + 4 * q + b];
        double v = ldexp(x, -ex);  // |v| < 1
#pragma unroll
        for (int s = 0; s < kOzMaxS; ++s) {
          if (s < S) {
            v *= 128.0;
            const double t = trunc(v);
            v -= t;
            w[s][q] |= ((unsigned)(int)t & 0xFFu) << (8 * b);
          }
        }
      }
    }
    const int off = ((row >> 3) * 4 + kc) * 128 + (row & 7) * 16;
#pragma unroll
    for (int s = 0; s < kOzMaxS; ++s)
      if (s < S)
        *reinterpret_cast<uint4*>(dst + (size_t)s * kOzPart + off) =
            make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
  }
}

void launch_oz_convert(const OzOperand* d_ops, const int* d_tile_off, int nops, int total_tiles,
                       int slices, int* d_rexp, long long n_rexp, cudaStream_t s) {
  if (total_tiles <= 0) return;
  // 0x80808080: below every exponent a double can have
  cudaMemsetAsync(d_rexp, 0x80, (size_t)n_rexp * sizeof(int), s);
  ensure_smem((const void*)k_oz_slice, kOzConvSmem);
  k_oz_exp<<<total_tiles, 256, 0, s>>>(d_ops, d_tile_off, nops);
  k_oz_slice<<<total_tiles, 256, kOzConvSmem, s>>>(d_ops, d_tile_off, nops, slices);
}

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 512 B.
__device__ __forceinline__ unsigned long long oz_desc(unsigned addr) {
  unsigned long long d = (unsigned long long)((addr >> 4) & 0x3FFF);
  d |= (unsigned long long)(128 >> 4) << 16;
  d |= (unsigned long long)(512 >> 4) << 32;
  d |= 1ull << 46;
  return d;
}

template <int S, int BN>
struct OzCfg {
  static constexpr int kA = S * kOzPart;   // A bytes of one stage
  static constexpr int kB = S * BN * kOzK;  // B bytes of one stage
  static constexpr int kStage = kA + kB;
  static constexpr int kStages = (200 * 1024) / kStage > 4 ? 4 : (200 * 1024) / kStage;
  static constexpr int kSmem = kStages * kStage + 256;
  static constexpr int kCols = S * BN <= 256 ? 256 : 512;  // tensor-memory columns
  // Instruction descriptor, kind::i8: D S32 (bits 4-5 = 2), A and B signed
  // 8-bit (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at 24.
  static constexpr unsigned kIdesc = (2u << 4) | (1u << 7) | (1u << 10) |
                                     ((unsigned)(BN >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
  static_assert(S * BN <= 512, "diagonal accumulators exceed tensor memory");
  static_assert(kStages >= 2, "stage ring");
};

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, int bytes, unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// One int8 slice product; U selects the A collector buffer's use: 0 read A
// from shared memory only, 1 read it and keep it (fill), 2 reuse the kept A,
// 3 reuse it for the last time.
template <int U>
__device__ __forceinline__ void oz_mma(unsigned d, unsigned long long da, unsigned long long db,
                                       unsigned idesc, unsigned acc) {
  if (U == 0)
    asm volatile(
        "{\n\t.reg .pred r;\n\tsetp.ne.b32 r, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, r;\n\t}\n" ::"r"(d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
  else if (U == 1)
    asm volatile(
        "{\n\t.reg .pred r;\n\tsetp.ne.b32 r, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::fill [%0], %1, %2, %3, r;\n\t}\n" ::"r"(
            d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
  else if (U == 2)
    asm volatile(
        "{\n\t.reg .pred r;\n\tsetp.ne.b32 r, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::use [%0], %1, %2, %3, r;\n\t}\n" ::"r"(d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred r;\n\tsetp.ne.b32 r, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::lastuse [%0], %1, %2, %3, r;\n\t}\n" ::"r"(
            d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

// Persistent: one CTA per SM walks the launch's tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ...; the tensor memory is allocated and the barriers
// set up once. The stage ring runs on across tiles. The accumulators of a tile
// are released (tempty) as soon as the epilogue warps have read them, so its
// C writes overlap the next tile's products.
template <int S, int BN>
__global__ void __launch_bounds__(256, 1) k_gemm_oz(const OzGemm* __restrict__ descs,
                                                    const int* __restrict__ tile_off, int nd,
                                                    int total_tiles, int* __restrict__ status) {
  using Cfg = OzCfg<S, BN>;
  constexpr int NS = Cfg::kStages;
  extern __shared__ __align__(1024) unsigned char oz_smem[];
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(oz_smem + NS * Cfg::kStage);
  unsigned long long* full = bars;        // [NS]
  unsigned long long* empty = bars + NS;  // [NS]
  unsigned long long* tfull = bars + 2 * NS;
  unsigned long long* tempty = tfull + 1;
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(tempty + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // tile decode shared by the roles
  // k tiles [kf, kt_cnt) of the launch's range run: with a lower-triangular A
  // none past the tile's last row, with a lower-triangular B none before its
  // first column
  auto tile = [&](int t, OzGemm& g, int& mt, int& nt, int& kf, int& kt_cnt) -> bool {
    const int di = find_desc(tile_off, nd, t);
    g = descs[di];
    const int local = t - tile_off[di];
    const int tiles_m = (g.m + 127) / 128;
    mt = local % tiles_m;
    nt = local / tiles_m;
    const int m0 = mt * 128, n0 = nt * BN;
    if (g.lower && n0 >= m0 + 128) return false;
    kt_cnt = g.a_lower ? min(g.kt_cnt, max(0, (m0 + 128 + kOzK - 1) / kOzK - g.kt0)) : g.kt_cnt;
    kf = g.b_lower ? min(kt_cnt, max(0, n0 / kOzK - g.kt0)) : 0;
    return true;
  };

  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(Cfg::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int q = 0; q < NS; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[q])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(tfull)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(tempty)) : "memory");
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // producer: per k tile, the S slices of the A tile, then those of the B tile
    int it = 0;
    for (int t = blockIdx.x; t < total_tiles && !*abort; t += gridDim.x) {
      OzGemm g;
      int mt, nt, kf, kt_cnt;
      if (!tile(t, g, mt, nt, kf, kt_cnt)) continue;
      const int n0 = nt * BN, bt = n0 / 128, bhalf = (n0 / 64) & 1;
      bool ok = true;
      for (int i = kf; i < kt_cnt; ++i, ++it) {
        const int kt = g.kt0 + i, s = it % NS;
        if (it >= NS && !mbar_wait(smem_u32(&empty[s]), (unsigned)((it / NS - 1) & 1), abort)) {
          ok = false;
          break;
        }
        const unsigned fb = smem_u32(&full[s]);
        const unsigned dst = smem_u32(oz_smem + s * Cfg::kStage);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                     "r"(Cfg::kStage)
                     : "memory");
        bulk_g2s(dst, g.A + ((size_t)mt * g.kt_total + kt) * S * kOzPart, Cfg::kA, fb);
        const signed char* b = g.B + ((size_t)bt * g.kt_total + kt) * S * kOzPart;
        if (BN == 128) {
          bulk_g2s(dst + Cfg::kA, b, Cfg::kB, fb);
        } else {
#pragma unroll
          for (int q = 0; q < S; ++q)
            bulk_g2s(dst + Cfg::kA + q * BN * kOzK, b + (size_t)q * kOzPart + bhalf * BN * kOzK,
                     BN * kOzK, fb);
        }
      }
      if (!ok) break;
    }
  } else if (warp == 1 && lane == 0) {
    // tensor-core issue: slice pair (p, q) adds into the accumulator of diagonal p + q
    int it = 0, a = 0;
    for (int t = blockIdx.x; t < total_tiles && !*abort; t += gridDim.x) {
      OzGemm g;
      int mt, nt, kf, kt_cnt;
      if (!tile(t, g, mt, nt, kf, kt_cnt) || kt_cnt <= kf) continue;
      // the previous tile's accumulators have been read
      if (a > 0 && !mbar_wait(smem_u32(tempty), (unsigned)((a - 1) & 1), abort)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      bool ok = true;
      for (int i = kf; i < kt_cnt; ++i, ++it) {
        const int s = it % NS;
        if (!mbar_wait(smem_u32(&full[s]), (unsigned)((it / NS) & 1), abort)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned base = smem_u32(oz_smem + s * Cfg::kStage);
#pragma unroll
        for (int j = 0; j < kOzK / 32; ++j) {
#pragma unroll
          for (int p = 0; p < S; ++p) {
            const unsigned long long da = oz_desc(base + p * kOzPart + 256 * j);
#pragma unroll
            for (int q = 0; p + q < S; ++q) {
              const unsigned long long db = oz_desc(base + Cfg::kA + q * BN * kOzK + 256 * j);
              const unsigned acc = (i > kf || j > 0 || p > 0) ? 1u : 0u;
              const unsigned d = tmem + (unsigned)((p + q) * BN);
              // A slice p is read from shared memory once per 32-k step and kept
              // in the collector buffer for its other slice pairs
              if (p == S - 1)
                oz_mma<0>(d, da, db, Cfg::kIdesc, acc);
              else if (q == 0)
                oz_mma<1>(d, da, db, Cfg::kIdesc, acc);
              else if (p + q < S - 1)
                oz_mma<2>(d, da, db, Cfg::kIdesc, acc);
              else
                oz_mma<3>(d, da, db, Cfg::kIdesc, acc);
            }
          }
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&empty[s]))
            : "memory");
      }
      if (!ok) break;
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(tfull))
          : "memory");
      ++a;
    }
  } else if (warp >= 4) {
    // epilogue: C = alpha 2^{e_i + f_j - 14} sum_d 2^{-7d} P_d + beta C, the
    // diagonals combined 64 columns at a time in registers
    const int q4 = warp - 4;
    const unsigned lanes = (unsigned)(32 * q4) << 16;
    int a = 0;
    for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
      OzGemm g;
      int mt, nt, kf, kt_cnt;
      if (!tile(t, g, mt, nt, kf, kt_cnt)) continue;
      kt_cnt -= kf;  // k tiles run
      const int gm = mt * 128 + 32 * q4 + lane, n0 = nt * BN;
      bool ok = true;
      if (kt_cnt > 0) {
        ok = mbar_wait(smem_u32(tfull), (unsigned)(a & 1), abort) && !*abort;
        if (ok) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      }
      if (!ok) break;
      const int ea = gm < g.m ? max(g.ea[gm], -4096) : 0;
#pragma unroll
      for (int half = 0; half < BN / 64; ++half) {
        double h[64];
#pragma unroll
        for (int e = 0; e < 64; ++e) h[e] = 0.0;
        if (kt_cnt > 0) {
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) {
#pragma unroll
            for (int d = S - 1; d >= 0; --d) {
              unsigned v[16];
              asm volatile(
                  "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,"
                  "%11,%12,%13,%14,%15}, [%16];"
                  : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                    "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                    "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                  : "r"(tmem + lanes + (unsigned)(d * BN + 64 * half + 16 * cc))
                  : "memory");
              asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
              for (int e = 0; e < 16; ++e)
                h[16 * cc + e] = fma(h[16 * cc + e], 0.0078125, (double)(int)v[e]);
            }
          }
          if (half == BN / 64 - 1) {
            // every accumulator of the tile is read: release them to the next tile
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
              asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(tempty))
                           : "memory");
          }
        }
        if (gm < g.m) {
          // 16 columns at a time: their C entries and column exponents are
          // loaded before any store, so the loads are in flight together (a
          // load after a store to C would wait for it: the compiler cannot rule
          // out aliasing)
          double* crow = g.C + gm;
#pragma unroll
          for (int e0 = 0; e0 < 64; e0 += 16) {
            double cv[16];
            int fe[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const int gn = n0 + 64 * half + e0 + e;
              const bool in = gn < g.n;
              fe[e] = in ? g.eb[gn] : 0;
              cv[e] = (in && g.beta != 0.0) ? crow[(long long)gn * g.ldc] : 0.0;
            }
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const int gn = n0 + 64 * half + e0 + e;
              if (gn < g.n) {
                const double val = g.alpha * ldexp(h[e0 + e], ea + max(fe[e], -4096) - 14);
                crow[(long long)gn * g.ldc] = (g.beta == 0.0) ? val : fma(g.beta, cv[e], val);
              }
            }
          }
        }
      }
      if (kt_cnt > 0) ++a;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && *abort) atomicOr(status, kStatusTimeout);
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(Cfg::kCols)
                 : "memory");
  }
}

int oz_tile_n(int slices) { return slices <= 4 ? 128 : 64; }

template <int S, int BN>
static void launch_gemm_oz_t(const OzGemm* d_desc, const int* d_tile_off, int nd, int total_tiles,
                             int* d_status, cudaStream_t s) {
  ensure_smem((const void*)k_gemm_oz<S, BN>, OzCfg<S, BN>::kSmem);
  const int grid = std::min(total_tiles, sm_count());
  k_gemm_oz<S, BN><<<grid, 256, OzCfg<S, BN>::kSmem, s>>>(d_desc, d_tile_off, nd, total_tiles,
                                                           d_status);
}

void launch_gemm_oz(const OzGemm* d_desc, const int* d_tile_off, int nd, int total_tiles,
                    int slices, int* d_status, cudaStream_t s) {
  if (total_tiles <= 0) return;
  switch (slices) {
    case 2: launch_gemm_oz_t<2, 128>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    case 3: launch_gemm_oz_t<3, 128>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    case 4: launch_gemm_oz_t<4, 128>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    case 5: launch_gemm_oz_t<5, 64>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    case 6: launch_gemm_oz_t<6, 64>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    case 7: launch_gemm_oz_t<7, 64>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    case 8: launch_gemm_oz_t<8, 64>(d_desc, d_tile_off, nd, total_tiles, d_status, s); break;
    default: break;
  }
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
  ensure_smem((const void*)k_sweep_small, kSmallSweepN * kSmallSweepN * sizeof(double));
  k_sweep_small<<<nd, 256, smem, s>>>(d_desc, d_status);
}

// --- blocked sweep ---------------------------------------------------------
// Step for pivot block K = [k0, k1) of A22: Dinv = B[K, K]^{-1} (k_sweep_diag);
// the row / column panels and the rank-128 update are batched GEMMs issued by
// the host; B[K, K] = Dinv (k_sweep_setdiag).
// Register-resident Gauss-Jordan inverse of the pivot block: thread (tx, ty)
// of a 16 x 32 grid holds the 4 x 8 sub-block rows 4 ty.., columns 8 tx.. in
// registers. At step k the owners of the old row k and column k publish them
// to shared memory (two buffers, alternating, so one barrier per step orders
// both the reads of step k and the writes of step k + 2); every thread then
// updates its 32 entries with the same operations as the in-place sweep:
// row k * (1 / p), column k * (-1 / p), the rest a - a_ik (a_kj / p).
__global__ void __launch_bounds__(512) k_sweep_diag(const SweepDesc* __restrict__ descs,
                                                    const int* __restrict__ active, int k0,
                                                    double* __restrict__ dinv,
                                                    int* __restrict__ status, int sym) {
  const int di = active[blockIdx.x];
  const SweepDesc d = descs[di];
  const int nb = min(kSweepNB, d.r - k0);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  __shared__ double rowk[2][kSweepNB], colk[2][kSweepNB];
  extern __shared__ double dg_sm[];  // kSweepNB x kSweepNB staging (coalesced load / store)
  // sym: the block is taken from its lower triangle (mirrored), so that the
  // inverse of a symmetric elimination stays consistent when the input carries
  // an asymmetric rounding error
  for (int e = threadIdx.x; e < kSweepNB * kSweepNB; e += blockDim.x) {
    const int i = e & (kSweepNB - 1), j = e / kSweepNB;
    const int ii = (sym && i < j) ? j : i, jj = (sym && i < j) ? i : j;
    dg_sm[e] = (i < nb && j < nb) ? d.B[(k0 + ii) + (long long)(k0 + jj) * d.n] : 0.0;
  }
  __syncthreads();
  double a[4][8];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) a[r][c] = dg_sm[(4 * ty + r) + (8 * tx + c) * kSweepNB];
  int bad = 0;
  for (int k = 0; k < nb; ++k) {
    const int buf = k & 1;
    if (ty == (k >> 2)) {
      const int kr = k & 3;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        double v = a[0][c];
#pragma unroll
        for (int r = 1; r < 4; ++r)
          if (r == kr) v = a[r][c];
        rowk[buf][8 * tx + c] = v;
      }
    }
    if (tx == (k >> 3)) {
      const int kc = k & 7;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double v = a[r][0];
#pragma unroll
        for (int c = 1; c < 8; ++c)
          if (c == kc) v = a[r][c];
        colk[buf][4 * ty + r] = v;
      }
    }
    __syncthreads();
    const double p = rowk[buf][k];
    if (threadIdx.x == 0 && (!(fabs(p) > 1e-300) || !isfinite(p))) bad = 1;
    const double ip = 1.0 / p;
    double rj[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) rj[c] = rowk[buf][8 * tx + c] * ip;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double cir = colk[buf][4 * ty + r];
#pragma unroll
      for (int c = 0; c < 8; ++c) a[r][c] = fma(-cir, rj[c], a[r][c]);
    }
    // row k, column k and the pivot replace what the general update wrote there
    if (ty == (k >> 2)) {
      const int kr = k & 3;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (r == kr) {
#pragma unroll
          for (int c = 0; c < 8; ++c) a[r][c] = rj[c];
        }
    }
    if (tx == (k >> 3)) {
      const int kc = k & 7;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c == kc) {
#pragma unroll
          for (int r = 0; r < 4; ++r)
            a[r][c] = (4 * ty + r == k) ? ip : colk[buf][4 * ty + r] * -ip;
        }
    }
  }
  if (bad) atomicOr(status, kStatusTinyPivot);
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) dg_sm[(4 * ty + r) + (8 * tx + c) * kSweepNB] = a[r][c];
  __syncthreads();
  double* out = dinv + (long long)di * kSweepNB * kSweepNB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    out[e] = dg_sm[i + j * kSweepNB];
  }
}

void launch_sweep_diag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                       double* d_dinv, int* d_status, cudaStream_t s, int sym) {
  if (nact <= 0) return;
  const int smem = kSweepNB * kSweepNB * (int)sizeof(double);
  ensure_smem((const void*)k_sweep_diag, smem);
  k_sweep_diag<<<nact, 512, smem, s>>>(d_desc, d_active, k0, d_dinv, d_status, sym);
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
// Cholesky elimination (symmetric positive definite interiors; the lower
// triangle of every block is the one read and written).
//   [A22 A12^T; A12 A11] = [L 0; Y^T I] [I 0; 0 S] [L^T Y; 0 I],
//   A22 = L L^T, Y = L^{-1} A12^T, S = A11 - Y^T Y.
// The factor keeps L (for F u), L^{-1} and Y (for F^{-1} u): in exact
// arithmetic X = L^{-T} Y and A22^{-1} = L^{-T} L^{-1}, the reference's
// Schur() outputs (include/Schur.hpp:72-100).
// ===========================================================================

// Small blocks whole in shared memory. Right-looking: for k < r, d = sqrt(S_kk),
// column k below the diagonal / d, then S_ij -= S_ik S_jk for k < j <= i; after
// r steps S[0:r, 0:r] = L, S[r:n, 0:r] = Y^T and S[r:n, r:n] = A11 - Y^T Y
// (lower). L^{-1} then replaces L in place by Gauss-Jordan on the lower
// triangle (entries above the diagonal stay zero under those steps).
__global__ void __launch_bounds__(256) k_chol_small(const SweepDesc* __restrict__ descs,
                                                    int* __restrict__ status) {
  const SweepDesc d = descs[blockIdx.x];
  const int n = d.n, r = d.r, s = n - r;
  extern __shared__ double S[];  // n x n, ld n; lower triangle used
  const int nn = n * n;
  for (int e = threadIdx.x; e < nn; e += blockDim.x) {
    const int i = e % n, j = e / n;
    S[e] = (i >= j) ? d.B[e] : 0.0;
  }
  __syncthreads();
  __shared__ double s_d;
  int bad = 0;
  for (int k = 0; k < r; ++k) {
    if (threadIdx.x == 0) {
      const double p = S[k + k * n];
      if (!(p > 1e-300) || !isfinite(p)) bad = 1;
      s_d = sqrt(fabs(p) > 1e-300 ? fabs(p) : 1.0);
    }
    __syncthreads();
    const double dk = s_d, idk = 1.0 / dk;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) S[i + k * n] *= idk;
    if (threadIdx.x == 0) S[k + k * n] = dk;
    __syncthreads();
    const int m = n - k - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int ii = e % m, jj = e / m;
      if (ii < jj) continue;
      const int i = k + 1 + ii, j = k + 1 + jj;
      S[i + j * n] = fma(-S[i + k * n], S[j + k * n], S[i + j * n]);
    }
    __syncthreads();
  }
  // outputs: L (zeros above), Y = (S[r:n, 0:r])^T, Schur complement (mirrored)
  for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
    const int i = e % r, j = e / r;
    d.L[e] = (i >= j) ? S[i + j * n] : 0.0;
  }
  for (int e = threadIdx.x; e < r * s; e += blockDim.x) {
    const int i = e % r, j = e / r;
    d.X[e] = S[(r + j) + i * n];
  }
  for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
    const int i = e % s, j = e / s;
    const int a = max(i, j), b = min(i, j);
    d.B[(r + i) + (long long)(r + j) * n] = S[(r + a) + (r + b) * n];
  }
  __syncthreads();
  // L^{-1} in place (lower triangle of S[0:r, 0:r])
  for (int k = 0; k < r; ++k) {
    const double ip = 1.0 / S[k + k * n];
    for (int j = threadIdx.x; j < k; j += blockDim.x) S[k + j * n] *= ip;
    __syncthreads();
    const int m = r - k - 1;
    for (int e = threadIdx.x; e < m * k; e += blockDim.x) {
      const int i = k + 1 + e % m, j = e / m;
      S[i + j * n] = fma(-S[i + k * n], S[k + j * n], S[i + j * n]);
    }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < r; i += blockDim.x) S[i + k * n] *= -ip;
    if (threadIdx.x == 0) S[k + k * n] = ip;
    __syncthreads();
  }
  if (bad) atomicOr(status, kStatusTinyPivot);
  for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
    const int i = e % r, j = e / r;
    d.a22inv[e] = (i >= j) ? S[i + j * n] : 0.0;
  }
}

void launch_chol_small(const SweepDesc* d_desc, int nd, int max_n, int* d_status,
                       cudaStream_t s) {
  if (nd <= 0) return;
  const size_t smem = (size_t)max_n * max_n * sizeof(double);
  ensure_smem((const void*)k_chol_small, kSmallSweepN * kSmallSweepN * sizeof(double));
  k_chol_small<<<nd, 256, smem, s>>>(d_desc, d_status);
}

// Pivot block of the blocked Cholesky: L_KK = chol(D) over B[K, K] (zeros
// above the diagonal) and L_KK^{-1} into dinv, with D (128 x 128, lower
// triangle read, padded with the identity past nb) in shared memory. This
// kernel is on the critical path of the top levels, where one or a few blocks
// remain, so it is built for latency: the only serial work is the pivot chain
// of each 32-wide panel.
//   for each panel p: warp 0 factors the 32 x 32 diagonal block with its rows
//   in registers (pivot and multipliers passed by shuffles; one reciprocal
//   square root per pivot, kept for the rest); the rows below are solved
//   against it by forward substitution, a thread per row; the trailing lower
//   triangle is updated with each thread holding a 16-strided micro-tile of
//   the outputs in registers (rows tx + 16a, columns ty + 16b), so that a
//   warp's loads are 16 consecutive doubles or broadcasts;
//   then the four 32 x 32 diagonal inverses, one warp each, and L^{-1} in
//   place, block row ib by block row: for every block column jb < ib at once,
//   Tb = L(ib, jb:ib) X(jb:ib, jb), then X(ib, jb) = -X_ib Tb.
constexpr int kCdP = 32;             // panel width
constexpr int kCdXs = kCdP + 1;      // padded stride of the diagonal inverses
constexpr int kCdThreads = 256;
constexpr size_t kCholDiagSmem =
    (size_t)(kSweepNB * kSweepNB + 4 * kCdP * kCdXs + 3 * kCdP * kCdXs + kSweepNB + 2 * kCdP) *
    sizeof(double);
static_assert(kSweepNB == 4 * kCdP && kCdThreads == 256, "16 x 16 thread grid over 32-row panels");

__global__ void __launch_bounds__(kCdThreads) k_chol_diag(const SweepDesc* __restrict__ descs,
                                                          const int* __restrict__ active, int k0,
                                                          double* __restrict__ dinv,
                                                          int* __restrict__ status) {
  const int di = active[blockIdx.x];
  const SweepDesc d = descs[di];
  const int nb = min(kSweepNB, d.r - k0);
  constexpr int T = kSweepNB;  // tile edge; column-major S[i + j T]
  extern __shared__ double cd_sm[];
  double* S = cd_sm;
  double* Xd = S + T * T;              // 4 diagonal inverses, [p][c][i] = X_pp(i, c)
  double* Tb = Xd + 4 * kCdP * kCdXs;  // 3 products of the inverse, [jb][c][k]
  double* rd = Tb + 3 * kCdP * kCdXs;  // 1 / L(i, i)
  double* colk = rd + T;               // 2 x 32: the current pivot column, double-buffered
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = tid & 15, ty = tid >> 4;
  // the lower triangle only (the only one read), in whole columns; 16 loads
  // of a thread in flight at once
  {
    const double* Bk = d.B + k0 + (long long)k0 * d.n;
#pragma unroll 1
    for (int base = 0; base < T * T; base += kCdThreads * 16) {
      double v[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int e = base + u * kCdThreads + tid, i = e % T, j = e / T;
        v[u] = (i < nb && j < nb) ? (i >= j ? Bk[i + (long long)j * d.n] : 0.0)
                                  : (i == j ? 1.0 : 0.0);
      }
#pragma unroll
      for (int u = 0; u < 16; ++u) S[base + u * kCdThreads + tid] = v[u];
    }
  }
  __syncthreads();
  int bad = 0;
  for (int p = 0; p < T / kCdP; ++p) {
    const int o = p * kCdP;
    if (warp == 0) {
      // Cholesky of the 32 x 32 diagonal block: lane = row, a[j] = D(lane, j)
      double a[kCdP];
#pragma unroll
      for (int j = 0; j < kCdP; ++j) a[j] = S[(o + lane) + (o + j) * T];
      double rmine = 1.0;  // 1 / L(lane, lane)
#pragma unroll
      for (int k = 0; k < kCdP; ++k) {
        const double pv = __shfl_sync(0xffffffffu, a[k], k);
        if (lane == 0 && o + k < nb && (!(pv > 1e-300) || !isfinite(pv))) bad = 1;
        const double q = fabs(pv) > 1e-300 ? fabs(pv) : 1.0;
        const double rk = rsqrt(q);
        if (lane > k) a[k] *= rk;
        if (lane == k) {
          a[k] = q * rk;
          rmine = rk;
        }
        // D(lane, j) -= L(lane, k) L(j, k), k < j <= lane; the column L(:, k) is
        // passed through shared memory (one store per lane, broadcast loads)
        // rather than by a pair of shuffles per entry; the buffer alternates
        // with k, so one warp barrier per pivot suffices
        double* ck = colk + (k & 1) * kCdP;
        ck[lane] = a[k];
        __syncwarp();
#pragma unroll
        for (int j = 1; j < kCdP; ++j) {
          if (j > k) {  // fixed trip count: a[] stays in registers
            const double ljk = ck[j];
            if (lane >= j) a[j] = fma(-a[k], ljk, a[j]);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kCdP; ++j) S[(o + lane) + (o + j) * T] = a[j];
      rd[o + lane] = rmine;
    }
    __syncthreads();
    const int r0 = o + kCdP, nrow = T - r0;
    if (nrow > 0) {
      // panel rows below, a thread per row: L(i, c) = (A(i, c) - sum_{k<c} L(i, k) L(c, k)) / L(c, c)
      if (tid < nrow) {
        const int i = r0 + tid;
        double l[kCdP];
#pragma unroll
        for (int c = 0; c < kCdP; ++c) l[c] = S[i + (o + c) * T];
#pragma unroll
        for (int c = 0; c < kCdP; ++c) {
          double acc = l[c];
#pragma unroll
          for (int k = 0; k < kCdP - 1; ++k)
            if (k < c) acc = fma(-l[k], S[(o + c) + (o + k) * T], acc);
          l[c] = acc * rd[o + c];
        }
#pragma unroll
        for (int c = 0; c < kCdP; ++c) S[i + (o + c) * T] = l[c];
      }
      __syncthreads();
      // trailing lower triangle: A(i, j) -= sum_k L(i, k) L(j, k)
      const int na = nrow / 16;  // 6, 4 or 2 row strides
      double t[6][6];
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = 0; b < 6; ++b)
          t[a][b] = (a < na && b < na) ? S[(r0 + tx + 16 * a) + (r0 + ty + 16 * b) * T] : 0.0;
#pragma unroll 2
      for (int k = 0; k < kCdP; ++k) {
        double li[6], lj[6];
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          li[a] = a < na ? S[(r0 + tx + 16 * a) + (o + k) * T] : 0.0;
          lj[a] = a < na ? S[(r0 + ty + 16 * a) + (o + k) * T] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
          for (int b = 0; b < 6; ++b)
            if (a < na && b < na) t[a][b] = fma(-li[a], lj[b], t[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = 0; b < 6; ++b)
          if (a < na && b < na && tx + 16 * a >= ty + 16 * b)
            S[(r0 + tx + 16 * a) + (r0 + ty + 16 * b) * T] = t[a][b];
      __syncthreads();
    }
  }
  if (bad) atomicOr(status, kStatusTinyPivot);
  // L over B[K, K]: warp per column
  for (int j = warp; j < nb; j += kCdThreads / 32)
    for (int i = lane; i < nb; i += 32)
      d.B[(k0 + i) + (long long)(k0 + j) * d.n] = (i >= j) ? S[i + j * T] : 0.0;
  // the diagonal inverses, warp p for block p, lane = column c:
  // X(c, c) = 1 / l_cc, X(i, c) = -(sum_{k=c}^{i-1} l_ik X(k, c)) / l_ii, zero above
  if (warp < T / kCdP) {
    const int o = warp * kCdP, c = lane;
    double x[kCdP];
#pragma unroll
    for (int i = 0; i < kCdP; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < kCdP - 1; ++k)
        if (k < i) acc = fma(S[(o + i) + (o + k) * T], x[k], acc);
      x[i] = i == c ? rd[o + i] : (i > c ? -acc * rd[o + i] : 0.0);
    }
    double* X = Xd + warp * kCdP * kCdXs;
#pragma unroll
    for (int i = 0; i < kCdP; ++i) X[c * kCdXs + i] = x[i];
  }
  __syncthreads();
  // L^{-1} in place: the diagonal blocks first (X_jj, zeros above)
  for (int e = tid; e < 4 * kCdP * kCdP; e += blockDim.x) {
    const int jb = e / (kCdP * kCdP), r = e % (kCdP * kCdP), i = r % kCdP, c = r / kCdP;
    S[(jb * kCdP + i) + (jb * kCdP + c) * T] = Xd[jb * kCdP * kCdXs + c * kCdXs + i];
  }
  __syncthreads();
  for (int ib = 1; ib < T / kCdP; ++ib) {
    const int oi = ib * kCdP;
    // Tb[jb](i, c) = sum_{k in [jb 32, oi)} L(oi + i, k) X(k, jb 32 + c)
    for (int jb = 0; jb < ib; ++jb) {
      const int oj = jb * kCdP;
      double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 4
      for (int k = oj; k < oi; ++k) {
        const double l0 = S[(oi + tx) + k * T], l1 = S[(oi + tx + 16) + k * T];
        const double x0 = S[k + (oj + ty) * T], x1 = S[k + (oj + ty + 16) * T];
        acc[0][0] = fma(l0, x0, acc[0][0]);
        acc[0][1] = fma(l0, x1, acc[0][1]);
        acc[1][0] = fma(l1, x0, acc[1][0]);
        acc[1][1] = fma(l1, x1, acc[1][1]);
      }
      double* Tj = Tb + jb * kCdP * kCdXs;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) Tj[(ty + 16 * b) * kCdXs + tx + 16 * a] = acc[a][b];
    }
    __syncthreads();
    // X(ib, jb) = -X_ib Tb[jb]
    const double* Xi = Xd + ib * kCdP * kCdXs;
    for (int jb = 0; jb < ib; ++jb) {
      const int oj = jb * kCdP;
      const double* Tj = Tb + jb * kCdP * kCdXs;
      double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 4
      for (int k = 0; k < kCdP; ++k) {
        const double x0 = Xi[k * kCdXs + tx], x1 = Xi[k * kCdXs + tx + 16];
        const double t0 = Tj[ty * kCdXs + k], t1 = Tj[(ty + 16) * kCdXs + k];
        acc[0][0] = fma(x0, t0, acc[0][0]);
        acc[0][1] = fma(x0, t1, acc[0][1]);
        acc[1][0] = fma(x1, t0, acc[1][0]);
        acc[1][1] = fma(x1, t1, acc[1][1]);
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) S[(oi + tx + 16 * a) + (oj + ty + 16 * b) * T] = -acc[a][b];
    }
    __syncthreads();
  }
  double* out = dinv + (long long)di * kSweepNB * kSweepNB;
  for (int j = warp; j < nb; j += kCdThreads / 32)
    for (int i = lane; i < nb; i += 32) out[i + j * nb] = (i >= j) ? S[i + j * T] : 0.0;
}

void launch_chol_diag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                      double* d_dinv, int* d_status, cudaStream_t s) {
  if (nact <= 0) return;
  ensure_smem((const void*)k_chol_diag, kCholDiagSmem);
  k_chol_diag<<<nact, kCdThreads, kCholDiagSmem, s>>>(d_desc, d_active, k0, d_dinv, d_status);
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
// stage_ld > 0: the face matrix is copied into shared memory (after the
// work arrays, at offset stage_off doubles) and the QR runs there; it is
// copied back at the end, so M ends overwritten as without staging.
__global__ void __launch_bounds__(512) k_id(const IdDesc* __restrict__ descs, double eps,
                                            int* __restrict__ status, int stage_off) {
  const IdDesc d = descs[blockIdx.x];
  const int m = d.m, n = d.n;
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
  double* M = d.M;
  if (stage_off > 0) {
    M = sm + stage_off;
    for (long long e = threadIdx.x; e < (long long)m * n; e += blockDim.x) M[e] = d.M[e];
    __syncthreads();
  }

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
  if (stage_off > 0)
    for (long long e = threadIdx.x; e < (long long)m * n; e += blockDim.x) d.M[e] = M[e];
}

// ---------------------------------------------------------------------------
// Grouped ID (see hif_kernels.cuh).
// ---------------------------------------------------------------------------
namespace {

// Barrier of the `group` CTAs of one face: arrival counter sync[0], generation
// sync[1]. Bounded spin; on timeout the status word records kStatusTimeout and
// *ok turns false (every CTA then skips to the end).
__device__ void group_barrier(int* sync, int group, int* status, bool* ok) {
  __syncthreads();
  if (group > 1 && threadIdx.x == 0) {
    volatile int* gen = sync + 1;
    const int g0 = *gen;
    __threadfence();
    if (atomicAdd(sync, 1) == group - 1) {
      atomicExch(sync, 0);
      __threadfence();
      atomicAdd(sync + 1, 1);
    } else {
      long long spins = 0;
      while (*gen == g0) {
        if (++spins > (1LL << 28)) {
          atomicOr(status, kStatusTimeout);
          *ok = false;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

}  // namespace

__global__ void __launch_bounds__(512) k_id_group(const IdGroupDesc* __restrict__ descs,
                                                  int group, double eps,
                                                  int* __restrict__ status) {
  const int face = blockIdx.x / group, me = blockIdx.x % group;
  const IdGroupDesc gd = descs[face];
  const IdDesc d = gd.id;
  const int m = d.m, n = d.n;
  double* M = d.M;
  double* vn1 = gd.norms;
  double* vn2 = gd.norms + n;
  int* jp = d.jpvt;
  extern __shared__ double gsm[];
  double* vsh = gsm;          // reflector rows i..m-1 (m doubles)
  __shared__ double scratch[64];
  __shared__ int iscr[32];
  __shared__ int s_pvt;
  __shared__ bool s_ok;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nthr >> 5;
  const double tol3z = sqrt(DBL_EPSILON * 0.5);
  if (tid == 0) s_ok = true;
  __syncthreads();

  // own columns: j = me, me + group, ...
  for (int j = me + warp * group; j < n; j += nw * group) {
    double sacc = 0.0;
    for (int r = lane; r < m; r += 32) {
      const double v = __ldcg(M + r + (long long)j * m);
      sacc = fma(v, v, sacc);
    }
    sacc = warp_sum(sacc);
    if (lane == 0) {
      __stcg(vn1 + j, sqrt(sacc));
      __stcg(vn2 + j, sqrt(sacc));
      __stcg(jp + j, j);
    }
  }
  group_barrier(gd.sync, group, status, &s_ok);

  const int steps = min(m, n);
  for (int i = 0; i < steps && s_ok; ++i) {
    // ---- candidates over own columns >= i
    double best = -1.0;
    int bi = INT_MAX;
    if (d.order != nullptr) {
      const int want = d.order[i];
      for (int j = i + ((me - i % group + group) % group) + tid * group; j < n; j += nthr * group)
        if (__ldcg(jp + j) == want) { best = 1.0; bi = j; }
    } else {
      for (int j = i + ((me - i % group + group) % group) + tid * group; j < n; j += nthr * group) {
        const double v = __ldcg(vn1 + j);
        if (v > best || (v == best && j < bi)) { best = v; bi = j; }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (lane == 0) { scratch[warp] = best; iscr[warp] = bi; }
    __syncthreads();
    if (tid == 0) {
      double b = scratch[0];
      int bb = iscr[0];
      for (int w = 1; w < nw; ++w)
        if (scratch[w] > b || (scratch[w] == b && iscr[w] < bb)) { b = scratch[w]; bb = iscr[w]; }
      __stcg(gd.cand + me, b);
      __stcg(gd.sync + 32 + me, bb);
    }
    group_barrier(gd.sync, group, status, &s_ok);
    if (!s_ok) break;
    if (tid == 0) {
      double b = -1.0;
      int bb = INT_MAX;
      for (int c = 0; c < group; ++c) {
        const double cb = __ldcg(gd.cand + c);
        const int ci = __ldcg(gd.sync + 32 + c);
        if (cb > b || (cb == b && ci < bb)) { b = cb; bb = ci; }
      }
      s_pvt = (bb == INT_MAX) ? i : bb;
    }
    __syncthreads();
    const int pvt = s_pvt;
    // ---- owner of column i: swap, reflector
    if (i % group == me) {
      if (pvt != i) {
        for (int r = tid; r < m; r += nthr) {
          const double a = __ldcg(M + r + (long long)i * m);
          const double b = __ldcg(M + r + (long long)pvt * m);
          __stcg(M + r + (long long)i * m, b);
          __stcg(M + r + (long long)pvt * m, a);
        }
        if (tid == 0) {
          const int t = __ldcg(jp + pvt);
          __stcg(jp + pvt, __ldcg(jp + i));
          __stcg(jp + i, t);
          __stcg(vn1 + pvt, __ldcg(vn1 + i));
          __stcg(vn2 + pvt, __ldcg(vn2 + i));
        }
      }
      __syncthreads();
      double xs = 0.0;
      for (int r = i + 1 + tid; r < m; r += nthr) {
        const double v = __ldcg(M + r + (long long)i * m);
        xs = fma(v, v, xs);
      }
      const double xnorm = sqrt(block_sum(xs, scratch));
      const double alpha = __ldcg(M + i + (long long)i * m);
      double tau = 0.0, beta = alpha;
      if (xnorm != 0.0) {
        beta = -copysign(hypot(alpha, xnorm), alpha);
        tau = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        for (int r = i + 1 + tid; r < m; r += nthr)
          __stcg(M + r + (long long)i * m, __ldcg(M + r + (long long)i * m) * scal);
      }
      __syncthreads();
      if (tid == 0) {
        __stcg(M + i + (long long)i * m, beta);
        d.rdiag[i] = beta;
        __stcg(gd.tau, tau);
      }
    }
    group_barrier(gd.sync, group, status, &s_ok);
    if (!s_ok) break;
    // ---- every CTA: cache the reflector, update its own columns > i
    const double tau = __ldcg(gd.tau);
    for (int r = i + 1 + tid; r < m; r += nthr) vsh[r - i - 1] = __ldcg(M + r + (long long)i * m);
    __syncthreads();
    const int len = m - i - 1;
    const int jfirst = i + 1 + ((me - (i + 1) % group + group) % group);
    if (tau != 0.0) {
      for (int j = jfirst + warp * group; j < n; j += nw * group) {
        double* cj = M + (long long)j * m;
        double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
        int r = lane;
        for (; r + 96 < len; r += 128) {
          w0 = fma(vsh[r], __ldcg(cj + i + 1 + r), w0);
          w1 = fma(vsh[r + 32], __ldcg(cj + i + 1 + r + 32), w1);
          w2 = fma(vsh[r + 64], __ldcg(cj + i + 1 + r + 64), w2);
          w3 = fma(vsh[r + 96], __ldcg(cj + i + 1 + r + 96), w3);
        }
        for (; r < len; r += 32) w0 = fma(vsh[r], __ldcg(cj + i + 1 + r), w0);
        double w = warp_sum((w0 + w1) + (w2 + w3));
        const double ci = __ldcg(cj + i);
        w = (w + ci) * tau;
        if (lane == 0) __stcg(cj + i, ci - w);
        for (r = lane; r < len; r += 32)
          __stcg(cj + i + 1 + r, fma(-w, vsh[r], __ldcg(cj + i + 1 + r)));
      }
    }
    __syncthreads();
    // ---- norm downdate of own columns (thread per column), recompute on cancellation
    for (int j = jfirst + tid * group; j < n; j += nthr * group) {
      const double v1 = __ldcg(vn1 + j);
      if (v1 != 0.0) {
        double temp = fabs(__ldcg(M + i + (long long)j * m)) / v1;
        temp = fmax(1.0 - temp * temp, 0.0);
        const double q = v1 / __ldcg(vn2 + j);
        if (temp * q * q <= tol3z) __stcg(vn2 + j, -1.0);  // flag: recompute
        else __stcg(vn1 + j, v1 * sqrt(temp));
      }
    }
    __syncthreads();
    for (int j = jfirst + warp * group; j < n; j += nw * group) {
      if (__ldcg(vn2 + j) != -1.0) continue;
      double sacc = 0.0;
      for (int r = i + 1 + lane; r < m; r += 32) {
        const double v = __ldcg(M + r + (long long)j * m);
        sacc = fma(v, v, sacc);
      }
      sacc = warp_sum(sacc);
      if (lane == 0) {
        const double nv = (i + 1 < m) ? sqrt(sacc) : 0.0;
        __stcg(vn1 + j, nv);
        __stcg(vn2 + j, nv);
      }
    }
    __syncthreads();
  }
  group_barrier(gd.sync, group, status, &s_ok);
  if (!s_ok) return;

  // ---- rank test (every CTA computes the same list) and W (red columns split over the group)
  int* flag = reinterpret_cast<int*>(vsh);
  int* pos = flag + n;
  __shared__ int s_k;
  const double r00 = fabs(__ldcg(M));
  const double tol = r00 * eps;
  if (tid == 0) {
    int k = 0;
    for (int i = 0; i < n; ++i) {
      const int kp = fabs(__ldcg(M + i + (long long)i * m)) > tol;
      flag[i] = kp;
      if (kp) pos[k++] = i;
    }
    int rr = k;
    for (int i = 0; i < n; ++i)
      if (!flag[i]) pos[rr++] = i;
    s_k = k;
    if (me == 0) {
      *d.rank = k;
      if (r00 == 0.0) atomicOr(status, kStatusIdZero);
    }
  }
  __syncthreads();
  const int k = s_k;
  if (me == 0)
    for (int j = tid; j < n; j += nthr) {
      d.jpvt[j] = __ldcg(jp + j);
      d.keep[j] = flag[j];
    }
  const int nred = n - k;
  for (int b = me * nthr + tid; b < nred; b += nthr * group) {
    const int c = pos[k + b];
    double* x = d.W + (long long)b * k;
    for (int a = 0; a < k; ++a) x[a] = (c >= a) ? __ldcg(M + pos[a] + (long long)c * m) : 0.0;
    for (int a = k - 1; a >= 0; --a) {
      const double xa = x[a] / __ldcg(M + pos[a] + (long long)a * m);
      x[a] = xa;
      for (int t = 0; t < a; ++t) x[t] = fma(-__ldcg(M + pos[t] + (long long)a * m), xa, x[t]);
    }
  }
}

cudaError_t launch_id_group(const IdGroupDesc* d_desc, int nd, int group, double eps,
                            int* d_status, cudaStream_t s, int max_m, int max_n) {
  if (nd <= 0) return cudaSuccess;
  size_t smem = (size_t)std::max(max_m, 2 * max_n) * sizeof(double) + 64;
  if (smem > 48 * 1024) ensure_smem((const void*)k_id_group, smem);
  int grid = nd * group;
  if (group > 1) {
    // co-residency of the whole grid is required by the group barriers; the
    // cooperative launch guarantees it or fails without running
    void* args[] = {(void*)&d_desc, (void*)&group, (void*)&eps, (void*)&d_status};
    return cudaLaunchCooperativeKernel((const void*)k_id_group, dim3(grid), dim3(512), args, smem,
                                       s);
  }
  k_id_group<<<grid, 512, smem, s>>>(d_desc, group, eps, d_status);
  return cudaGetLastError();
}

void launch_id(const IdDesc* d_desc, int nd, int max_n, double eps, int* d_status,
               cudaStream_t s, long long max_mn) {
  if (nd <= 0) return;
  size_t smem = (size_t)max_n * 2 * sizeof(double) + 64 * sizeof(double) +
                (size_t)max_n * 3 * sizeof(int) + 32 * sizeof(int);
  // faces that fit run from shared memory (the Householder updates then read
  // and write the face on chip instead of through L2)
  int stage_off = 0;
  const size_t off = (smem + sizeof(double) - 1) / sizeof(double);
  if (max_mn > 0 && (off + (size_t)max_mn) * sizeof(double) <= (size_t)200 * 1024) {
    stage_off = (int)off;
    smem = (off + (size_t)max_mn) * sizeof(double);
  }
  // narrow faces: fewer threads per face, more faces per SM
  const int threads = max_n <= 16 ? 128 : 512;
  if (smem > 48 * 1024) ensure_smem((const void*)k_id, smem);
  k_id<<<nd, threads, smem, s>>>(d_desc, eps, d_status, stage_off);
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

// Transposing copy through a shared-memory tile (coalesced on both sides).
__global__ void __launch_bounds__(256) k_tcopy(const TCopyDesc* __restrict__ descs,
                                               const int* __restrict__ tile_off, int nd) {
  const int di = find_desc(tile_off, nd, blockIdx.x);
  const TCopyDesc c = descs[di];
  const int local = blockIdx.x - tile_off[di];
  const int tm = (c.m + 31) / 32;
  const int i0 = (local % tm) * 32, j0 = (local / tm) * 32;
  __shared__ double t[32][33];
  // read: consecutive threads take consecutive j (contiguous in src)
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
    const int jj = e & 31, ii = e >> 5;
    const int i = i0 + ii, j = j0 + jj;
    t[jj][ii] = (i < c.m && j < c.n) ? c.src[j + (long long)i * c.lds] : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
    const int ii = e & 31, jj = e >> 5;
    const int i = i0 + ii, j = j0 + jj;
    if (i < c.m && j < c.n) c.dst[i + (long long)j * c.ldd] = c.alpha * t[jj][ii];
  }
}

void launch_tcopy(const TCopyDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                  cudaStream_t s) {
  if (total_tiles <= 0) return;
  k_tcopy<<<total_tiles, 256, 0, s>>>(d_desc, d_tile_off, nd);
}

// ===========================================================================
// Row compression: blocked Householder QR panels (one CTA per face)
// ===========================================================================
__global__ void __launch_bounds__(512) k_qr_panel(const QrDesc* __restrict__ descs,
                                                  const int* __restrict__ active, int k0,
                                                  int vrow0) {
  const QrDesc d = descs[active[blockIdx.x]];
  const int m = d.m, kb = min(kQrNB, d.n - k0);
  double* Vout = d.V + (long long)(k0 - vrow0) * m;  // this sub-panel's columns of V
  double* M = d.M;
  __shared__ double s_tau[kQrNB];
  __shared__ double scratch[64];
  __shared__ double T[kQrNB * kQrNB];
  __shared__ double Wd[kQrNB * kQrNB];
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int nw = nthr >> 5;
  for (int j = 0; j < kb; ++j) {
    const int col = k0 + j;
    double* cc = M + (long long)col * m;
    double xs = 0.0;
    for (int r = col + 1 + tid; r < m; r += nthr) xs = fma(cc[r], cc[r], xs);
    const double xnorm = sqrt(block_sum(xs, scratch));
    const double alpha = cc[col];
    double tau = 0.0, beta = alpha;
    if (xnorm != 0.0) {
      beta = -copysign(hypot(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      const double scal = 1.0 / (alpha - beta);
      for (int r = col + 1 + tid; r < m; r += nthr) cc[r] *= scal;
    }
    __syncthreads();
    if (tid == 0) {
      cc[col] = beta;
      s_tau[j] = tau;
    }
    __syncthreads();
    if (tau != 0.0) {
      for (int c = col + 1 + warp; c < k0 + kb; c += nw) {
        double* cj = M + (long long)c * m;
        double w = (lane == 0) ? cj[col] : 0.0;
        for (int r = col + 1 + lane; r < m; r += 32) w = fma(cc[r], cj[r], w);
        w = warp_sum(w) * tau;
        if (lane == 0) cj[col] -= w;
        for (int r = col + 1 + lane; r < m; r += 32) cj[r] = fma(-w, cc[r], cj[r]);
      }
    }
    __syncthreads();
  }
  // explicit V (unit diagonal, zeros above) for rows vrow0..m-1
  const int mt = m - vrow0;
  for (long long e = tid; e < (long long)mt * kb; e += nthr) {
    const int rr = (int)(e % mt), j = (int)(e / mt);
    const int r = vrow0 + rr;
    double v = 0.0;
    if (r == k0 + j) v = 1.0;
    else if (r > k0 + j) v = M[r + (long long)(k0 + j) * m];
    Vout[r + (long long)j * m] = v;
  }
  for (int j = tid; j < kb; j += nthr) d.tau[k0 - vrow0 + j] = s_tau[j];
  __syncthreads();
  // Wd = V^T V in one pass over the rows: lane c holds V[r, c]; the products
  // with every other column come by shuffle. Warps add their partial sums in
  // warp order (deterministic).
  {
    double acc[kQrNB];
#pragma unroll
    for (int i = 0; i < kQrNB; ++i) acc[i] = 0.0;
    for (int r = k0 + warp; r < m; r += nw) {
      const double v = (lane < kb) ? Vout[r + (long long)lane * m] : 0.0;
#pragma unroll
      for (int i = 0; i < kQrNB; ++i) acc[i] = fma(__shfl_sync(0xffffffffu, v, i), v, acc[i]);
    }
    for (int e = tid; e < kQrNB * kQrNB; e += nthr) Wd[e] = 0.0;
    __syncthreads();
    for (int w = 0; w < nw; ++w) {
      if (warp == w) {
#pragma unroll
        for (int i = 0; i < kQrNB; ++i) Wd[i + lane * kQrNB] += acc[i];
      }
      __syncthreads();
    }
  }
  // T (forward, columnwise): T[j,j] = tau_j, T[0:j, j] = -tau_j T[0:j,0:j] Wd[0:j, j]
  for (int j = 0; j < kb; ++j) {
    if (tid < j) {
      double acc = 0.0;
      for (int l = tid; l < j; ++l) acc = fma(T[tid + l * kQrNB], Wd[l + j * kQrNB], acc);
      T[tid + j * kQrNB] = -s_tau[j] * acc;
    }
    if (tid == 0) T[j + j * kQrNB] = s_tau[j];
    for (int i = j + 1 + tid; i < kQrNB; i += nthr) T[i + j * kQrNB] = 0.0;
    __syncthreads();
  }
  for (int e = tid; e < kQrNB * kQrNB; e += nthr) {
    const int i = e % kQrNB, j = e / kQrNB;
    d.T[e] = (i < kb && j < kb) ? T[e] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// The same sub-panel factorization by a thread-block cluster per face: the
// cluster's CTAs split the panel's rows (at most kQrcRows each) and keep them
// in shared memory for the whole panel. Per column, every CTA sums over its
// rows the squared norm below the diagonal and the products of the column with
// the columns to its right; the owner of the diagonal row adds that row's
// entries. One cluster barrier, then every CTA adds the CTAs' partial vectors
// in rank order (identical sums everywhere, deterministic), forms the
// reflector (beta, tau) exactly as the single-CTA kernel does and updates its
// rows. Partial vectors alternate between two buffers, so one barrier per
// column orders both the reads of step j and the writes of step j + 2.
// ---------------------------------------------------------------------------
namespace cg = cooperative_groups;
constexpr int kQrcRows = 768;
constexpr int kQrcSlots = 2 * kQrNB + 2;  // [norm^2 | x.A_c (32) | alpha | A[col, c] (32)]

__global__ void __launch_bounds__(512) k_qr_panel_cluster(const QrDesc* __restrict__ descs,
                                                          const int* __restrict__ active,
                                                          int k1, int vrow0) {
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const QrDesc d = descs[active[blockIdx.x / C]];
  const int m = d.m, kb = min(kQrNB, d.n - k1), mt = m - k1;
  const int chunk = (mt + C - 1) / C;
  const int r0 = k1 + rank * chunk, r1 = min(m, r0 + chunk), nr = max(0, r1 - r0);
  const int ld = chunk | 1;  // odd: lanes reading one row of 32 columns hit distinct banks
  extern __shared__ double P[];  // nr x kQrNB, ld ld (local rows r0..r1)
  __shared__ double red[2][kQrcSlots];
  __shared__ double wpart[16][kQrcSlots];
  __shared__ double tot[kQrcSlots];
  __shared__ double gram[kQrNB * kQrNB];
  __shared__ double s_tau[kQrNB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthr = blockDim.x;
  double* M = d.M;
  for (int e = tid; e < nr * kQrNB; e += nthr) {
    const int i = e % nr, c = e / nr;
    P[i + c * ld] = (c < kb) ? M[(r0 + i) + (long long)(k1 + c) * m] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < kb; ++j) {
    const int col = k1 + j;
    // partial sums over local rows below the diagonal
    double acc[kQrNB + 1];
#pragma unroll
    for (int c = 0; c <= kQrNB; ++c) acc[c] = 0.0;
    for (int i = tid; i < nr; i += nthr) {
      if (r0 + i <= col) continue;
      const double x = P[i + j * ld];
      acc[0] = fma(x, x, acc[0]);
#pragma unroll
      for (int c = 0; c < kQrNB; ++c)
        if (c > j) acc[1 + c] = fma(x, P[i + c * ld], acc[1 + c]);
    }
    // warp reduce-scatter of acc[1..32] (5 halving exchanges, 31 shuffles):
    // afterwards lane c holds the warp's total of acc[1 + c]; acc[0] by warp_sum
    {
      const double n2 = warp_sum(acc[0]);
      if (lane == 0) wpart[warp][0] = n2;
#pragma unroll
      for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & h) != 0;
#pragma unroll
        for (int c = 0; c < h; ++c) {
          // keep the half selected by this lane's bit, send the other half
          const double send = upper ? acc[1 + c] : acc[1 + c + h];
          const double keep = upper ? acc[1 + c + h] : acc[1 + c];
          acc[1 + c] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
      }
      // the kept halves follow the lane's bits from high to low: acc[1] of lane c
      // is the warp's total for column c
      wpart[warp][1 + lane] = acc[1];
    }
    __syncthreads();
    double* rb = red[j & 1];
    if (tid <= kQrNB) {
      double sacc = 0.0;
      for (int w = 0; w < (nthr >> 5); ++w) sacc += wpart[w][tid];
      rb[tid] = sacc;
    } else if (tid <= 2 * kQrNB + 1) {
      // diagonal-row entries (alpha and A[col, c]) from the CTA that owns the row
      const int c = tid - (kQrNB + 1);  // 0 -> alpha, 1 + c' -> A[col, c']
      double v = 0.0;
      if (col >= r0 && col < r1) {
        const int cc = (c == 0) ? j : c - 1;
        if (c == 0 || (cc > j && cc < kb)) v = P[(col - r0) + cc * ld];
      }
      rb[tid] = v;
    }
    cl.sync();
    if (tid < kQrcSlots) {
      double v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = (q < C) ? cl.map_shared_rank(rb, q)[tid] : 0.0;
      double sacc = 0.0;
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (q < C) sacc += v[q];
      tot[tid] = sacc;
    }
    __syncthreads();
    const double xnorm = sqrt(tot[0]);
    const double alpha = tot[kQrNB + 1];
    double tau = 0.0, beta = alpha, scal = 1.0;
    if (xnorm != 0.0) {
      beta = -copysign(hypot(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    // update the local rows: v = x * scal below the diagonal, w_c = tau (A[col, c] + v . A_c)
    for (int i = tid; i < nr; i += nthr) {
      const int r = r0 + i;
      if (r < col) continue;
      if (r == col) {
        P[i + j * ld] = beta;
        for (int c = j + 1; c < kb; ++c) {
          const double w = tau * (tot[kQrNB + 2 + c] + scal * tot[1 + c]);
          P[i + c * ld] -= w;
        }
      } else {
        const double v = (xnorm != 0.0) ? P[i + j * ld] * scal : P[i + j * ld];
        P[i + j * ld] = v;
        for (int c = j + 1; c < kb; ++c) {
          const double w = tau * (tot[kQrNB + 2 + c] + scal * tot[1 + c]);
          P[i + c * ld] = fma(-w, v, P[i + c * ld]);
        }
      }
    }
    if (tid == 0) s_tau[j] = tau;
    __syncthreads();
  }
  // results: the panel back to M, V (unit diagonal, zeros above) for rows
  // vrow0.., tau
  double* Vout = d.V + (long long)(k1 - vrow0) * m;
  for (int e = tid; e < nr * kb; e += nthr) {
    const int i = e % nr, c = e / nr;
    const int r = r0 + i;
    const double p = P[i + c * ld];
    M[r + (long long)(k1 + c) * m] = p;
    Vout[r + (long long)c * m] = (r == k1 + c) ? 1.0 : (r > k1 + c ? p : 0.0);
  }
  if (rank == 0) {
    for (int e = tid; e < (k1 - vrow0) * kb; e += nthr) {
      const int i = e % (k1 - vrow0), c = e / (k1 - vrow0);
      Vout[vrow0 + i + (long long)c * m] = 0.0;
    }
    for (int j = tid; j < kb; j += nthr) d.tau[k1 - vrow0 + j] = s_tau[j];
  }
  // W = V^T V: local partial Gram (lane c holds column c; products with every
  // other column by shuffle), warps added in warp order, CTAs summed by rank 0
  // in rank order
  {
    double accg[kQrNB];
#pragma unroll
    for (int a = 0; a < kQrNB; ++a) accg[a] = 0.0;
    for (int i = warp; i < nr; i += (nthr >> 5)) {
      const int r = r0 + i;
      const double v = (lane < kb) ? (r == k1 + lane ? 1.0 : (r > k1 + lane ? P[i + lane * ld] : 0.0))
                                   : 0.0;
#pragma unroll
      for (int a = 0; a < kQrNB; ++a) accg[a] = fma(__shfl_sync(0xffffffffu, v, a), v, accg[a]);
    }
    for (int e = tid; e < kQrNB * kQrNB; e += nthr) gram[e] = 0.0;
    __syncthreads();
    for (int w = 0; w < (nthr >> 5); ++w) {
      if (warp == w) {
#pragma unroll
        for (int a = 0; a < kQrNB; ++a) gram[a + lane * kQrNB] += accg[a];
      }
      __syncthreads();
    }
  }
  cl.sync();
  if (rank == 0) {
    // the panel rows are no longer needed: W and T live in their space
    double* Wsum = P;
    double* Tl = P + kQrNB * kQrNB;
    for (int e = tid; e < kQrNB * kQrNB; e += nthr) {
      double g = 0.0;
      for (int q = 0; q < C; ++q) g += cl.map_shared_rank(gram, q)[e];
      Wsum[e] = g;
      Tl[e] = 0.0;
    }
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
      if (tid < j) {
        double a = 0.0;
        for (int l = tid; l < j; ++l) a = fma(Tl[tid + l * kQrNB], Wsum[l + j * kQrNB], a);
        Tl[tid + j * kQrNB] = -s_tau[j] * a;
      }
      if (tid == 0) Tl[j + j * kQrNB] = s_tau[j];
      __syncthreads();
    }
    for (int e = tid; e < kQrNB * kQrNB; e += nthr) d.T[e] = Tl[e];
  }
  cl.sync();  // no CTA leaves while rank 0 reads its shared memory
}

void launch_qr_panel(const QrDesc* d_desc, const int* d_active, int nact, int k1, int k0,
                     cudaStream_t s) {
  if (nact <= 0) return;
  k_qr_panel<<<nact, 512, 0, s>>>(d_desc, d_active, k1, k0);
}

int qr_cluster_max_rows() {
  // per device: the attributes and the cluster occupancy belong to the device
  static std::mutex mu;
  static std::map<int, int> caps;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  int& cap = caps.emplace(dev, -1).first->second;
  if (cap < 0) {
    ensure_smem((const void*)k_qr_panel_cluster, (kQrcRows + 1) * kQrNB * 8);
    cudaFuncSetAttribute(k_qr_panel_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    // the largest cluster the device can place with this kernel's footprint
    int best = 1;
    for (int c : {16, 8}) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(c, 1, 1);
      cfg.blockDim = dim3(512, 1, 1);
      cfg.dynamicSmemBytes = (kQrcRows + 1) * kQrNB * 8;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = c;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, k_qr_panel_cluster, &cfg) == cudaSuccess && n > 0) {
        best = c;
        break;
      }
      cudaGetLastError();
    }
    cap = best * kQrcRows;
  }
  return cap;
}

void launch_qr_panel_cluster(const QrDesc* d_desc, const int* d_active, int nact, int k1,
                             int k0, int max_rows, cudaStream_t s) {
  if (nact <= 0) return;
  const int C = std::max(1, (max_rows + kQrcRows - 1) / kQrcRows);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nact * C, 1, 1);
  cfg.blockDim = dim3(512, 1, 1);
  cfg.dynamicSmemBytes = (kQrcRows + 1) * kQrNB * 8;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_qr_panel_cluster, d_desc, d_active, k1, k0);
}

// One CTA per outer panel: the forward column recurrence for T over kQrNB2
// reflectors (T kept in shared memory, 128 KB).
__global__ void __launch_bounds__(256) k_qr_tfactor(const TFactorDesc* __restrict__ descs) {
  const TFactorDesc d = descs[blockIdx.x];
  extern __shared__ double Ts[];  // kQrNB2 x kQrNB2
  const int nb = d.nb, tid = threadIdx.x;
  for (int e = tid; e < kQrNB2 * kQrNB2; e += blockDim.x) Ts[e] = 0.0;
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const double tj = d.tau[j];
    for (int i = tid; i < j; i += blockDim.x) {
      double acc = 0.0;
      for (int l = i; l < j; ++l) acc = fma(Ts[i + l * kQrNB2], d.W[l + j * kQrNB2], acc);
      Ts[i + j * kQrNB2] = -tj * acc;
    }
    if (tid == 0) Ts[j + j * kQrNB2] = tj;
    __syncthreads();
  }
  for (int e = tid; e < kQrNB2 * kQrNB2; e += blockDim.x) d.T[e] = Ts[e];
}

void launch_qr_tfactor(const TFactorDesc* d_desc, int nd, cudaStream_t s) {
  if (nd <= 0) return;
  ensure_smem((const void*)k_qr_tfactor, kQrNB2 * kQrNB2 * 8);
  k_qr_tfactor<<<nd, 256, kQrNB2 * kQrNB2 * 8, s>>>(d_desc);
}

__global__ void k_triu(const TriuDesc* __restrict__ descs) {
  const TriuDesc d = descs[blockIdx.y];
  const long long nn = (long long)d.n * d.n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % d.n), j = (int)(e / d.n);
    d.dst[i + j * d.ldd] = (i <= j) ? d.src[i + j * d.lds] : 0.0;
  }
}

void launch_triu(const TriuDesc* d_desc, int nd, cudaStream_t s) {
  if (nd <= 0) return;
  dim3 grid(64, nd);
  k_triu<<<grid, 256, 0, s>>>(d_desc);
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
// Pivoted Cholesky ID (mixed precision mode), one CTA per face.
// ===========================================================================
__global__ void __launch_bounds__(512) k_pchol_panel(const PcholDesc* __restrict__ descs,
                                                     const int* __restrict__ active, int i0,
                                                     int nb, double eps, int* __restrict__ status) {
  const PcholDesc P = descs[active[blockIdx.x]];
  const int n = P.id.n, tid = threadIdx.x, nthr = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nthr >> 5;
  extern __shared__ double pc_sm[];
  double* d = pc_sm;                              // current Schur diagonal
  int* ch = reinterpret_cast<int*>(pc_sm + n);    // chosen flags
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ double pcol[64];                     // R[l, p] for the panel's rows
  __shared__ int s_p, s_stop;
  __shared__ double s_dp, s_d0;
  const double* G = P.G;
  double* R = P.R;
  if (P.info[1]) return;
  if (i0 == 0) {
    double mx = 0.0;
    for (int j = tid; j < n; j += nthr) {
      const double v = G[j + (long long)j * n];
      d[j] = v;
      ch[j] = 0;
      mx = fmax(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red_v[warp] = mx;
    __syncthreads();
    if (tid == 0) {
      double m0 = 0.0;
      for (int w = 0; w < nw; ++w) m0 = fmax(m0, red_v[w]);
      s_d0 = m0;
      *P.d0 = m0;
      if (!(m0 > 0.0)) atomicOr(status, kStatusIdZero);
    }
  } else {
    for (int j = tid; j < n; j += nthr) {
      const int c = P.chosen[j];
      ch[j] = c;
      d[j] = c ? 0.0 : G[j + (long long)j * n];
    }
    if (tid == 0) s_d0 = *P.d0;
  }
  if (tid == 0) s_stop = 0;
  __syncthreads();
  const double thr = eps * eps * s_d0;
  const int iend = min(n, i0 + nb);
  int i = i0;
  for (; i < iend; ++i) {
    // pivot: largest remaining diagonal, smallest index on ties
    double best = -1.0;
    int bi = INT_MAX;
    for (int j = tid; j < n; j += nthr)
      if (!ch[j] && (d[j] > best || (d[j] == best && j < bi))) { best = d[j]; bi = j; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (lane == 0) { red_v[warp] = best; red_i[warp] = bi; }
    __syncthreads();
    if (tid == 0) {
      double b = red_v[0];
      int bb = red_i[0];
      for (int w = 1; w < nw; ++w)
        if (red_v[w] > b || (red_v[w] == b && red_i[w] < bb)) { b = red_v[w]; bb = red_i[w]; }
      s_p = bb;
      s_dp = b;
      // R_ii <= eps R_00 (or nothing left): the rank is i
      if (bb == INT_MAX || !(b > thr)) s_stop = 1;
      else P.piv[i] = bb;
    }
    __syncthreads();
    if (s_stop) break;
    const int p = s_p;
    const double rii = sqrt(s_dp);
    for (int l = tid; l < i - i0; l += nthr) pcol[l] = R[(long long)(i0 + l) * n + p];
    __syncthreads();
    double* Ri = R + (long long)i * n;
    for (int j = tid; j < n; j += nthr) {
      if (ch[j]) { Ri[j] = 0.0; continue; }
      if (j == p) { Ri[j] = rii; continue; }
      // only the lower triangle of G is kept: G[j, p] for j > p, G[p, j] above
      double sacc = (j > p) ? G[j + (long long)p * n] : G[p + (long long)j * n];
      for (int l = 0; l < i - i0; ++l) sacc = fma(-pcol[l], R[(long long)(i0 + l) * n + j], sacc);
      const double r = sacc / rii;
      Ri[j] = r;
      d[j] = fma(-r, r, d[j]);
    }
    __syncthreads();
    if (tid == 0) ch[p] = 1;
    __syncthreads();
  }
  for (int j = tid; j < n; j += nthr) P.chosen[j] = ch[j];
  if (tid == 0) {
    P.info[0] = i;
    if (s_stop || i == n) P.info[1] = 1;
  }
}

void launch_pchol_panel(const PcholDesc* d_desc, const int* d_active, int nact, int i0, int nb,
                        double eps, int max_n, int* d_status, cudaStream_t s) {
  if (nact <= 0) return;
  const size_t smem = (size_t)max_n * (sizeof(double) + sizeof(int));
  if (smem > 48 * 1024) ensure_smem((const void*)k_pchol_panel, smem);
  k_pchol_panel<<<nact, 512, smem, s>>>(d_desc, d_active, i0, nb, eps, d_status);
}

__global__ void __launch_bounds__(512) k_pchol_finish(const PcholDesc* __restrict__ descs) {
  const PcholDesc P = descs[blockIdx.x];
  const int n = P.id.n, tid = threadIdx.x, nthr = blockDim.x;
  extern __shared__ int pf_sm[];  // order: n
  __shared__ int s_k;
  if (tid == 0) {
    const int k = P.info[0];
    int q = 0;
    for (int i = 0; i < k; ++i) pf_sm[q++] = P.piv[i];
    for (int j = 0; j < n; ++j)
      if (!P.chosen[j]) pf_sm[q++] = j;
    s_k = k;
    *P.id.rank = k;
  }
  __syncthreads();
  const int k = s_k;
  const double* R = P.R;
  for (int i = tid; i < n; i += nthr) {
    P.id.jpvt[i] = pf_sm[i];
    P.id.keep[i] = i < k;
    P.id.rdiag[i] = (i < k) ? R[(long long)i * n + pf_sm[i]] : 0.0;
  }
  // R11 (k x k, ld k, upper) into G's space; R12 into W (k x (n - k), ld k)
  double* R11 = P.G;
  for (long long e = tid; e < (long long)k * k; e += nthr) {
    const int a = (int)(e % k), b = (int)(e / k);
    R11[e] = (b >= a) ? R[(long long)a * n + pf_sm[b]] : 0.0;
  }
  const int nr = n - k;
  for (long long e = tid; e < (long long)k * nr; e += nthr) {
    const int a = (int)(e % k), c = (int)(e / k);
    P.id.W[e] = R[(long long)a * n + pf_sm[k + c]];
  }
}

void launch_pchol_finish(const PcholDesc* d_desc, int nd, int max_n, cudaStream_t s) {
  if (nd <= 0) return;
  const size_t smem = (size_t)max_n * sizeof(int);
  if (smem > 48 * 1024) ensure_smem((const void*)k_pchol_finish, smem);
  k_pchol_finish<<<nd, 512, smem, s>>>(d_desc);
}

// One CTA per (face, 128 columns): the diagonal block of R11 in shared memory,
// one column of W per thread, back substitution over the block's rows.
__global__ void __launch_bounds__(128) k_trsm_block(const TrsmBlockDesc* __restrict__ descs,
                                                    int chunks) {
  const TrsmBlockDesc t = descs[blockIdx.x / chunks];
  const int c = (blockIdx.x % chunks) * 128 + threadIdx.x;
  const int bs = t.a1 - t.a0;
  extern __shared__ double tb_sm[];
  double* Rb = tb_sm;                    // kTrsmNB x kTrsmNB
  double* X = tb_sm + kTrsmNB * kTrsmNB;  // kTrsmNB x 128
  if (bs <= 0) return;
  for (int e = threadIdx.x; e < bs * bs; e += blockDim.x) {
    const int a = e % bs, b = e / bs;
    Rb[a + b * kTrsmNB] = t.R[(t.a0 + a) + (long long)(t.a0 + b) * t.k];
  }
  const bool live = c < t.ncols;
  if (live)
    for (int a = 0; a < bs; ++a)
      X[a * 128 + threadIdx.x] = t.W[(t.a0 + a) + (long long)c * t.k];
  __syncthreads();
  if (!live) return;
  for (int a = bs - 1; a >= 0; --a) {
    const double xa = X[a * 128 + threadIdx.x] / Rb[a + a * kTrsmNB];
    X[a * 128 + threadIdx.x] = xa;
    for (int r = 0; r < a; ++r)
      X[r * 128 + threadIdx.x] = fma(-Rb[r + a * kTrsmNB], xa, X[r * 128 + threadIdx.x]);
  }
  for (int a = 0; a < bs; ++a) t.W[(t.a0 + a) + (long long)c * t.k] = X[a * 128 + threadIdx.x];
}

void launch_trsm_block(const TrsmBlockDesc* d_desc, int nd, int max_cols, cudaStream_t s) {
  if (nd <= 0 || max_cols <= 0) return;
  const int chunks = (max_cols + 127) / 128;
  const int smem = (kTrsmNB * kTrsmNB + kTrsmNB * 128) * (int)sizeof(double);
  ensure_smem((const void*)k_trsm_block, smem);
  k_trsm_block<<<nd * chunks, 128, smem, s>>>(d_desc, chunks);
}

// ===========================================================================
// Source membership (one CTA per cell / face)
// ===========================================================================
__global__ void k_member_cells(const int* __restrict__ skel, const long long* __restrict__ off,
                               const int* __restrict__ src, int cpd, int w, int NC,
                               int* __restrict__ dof_src) {
  const int b = blockIdx.x;
  const int id = src[b];
  if (id < 0) return;
  const long long n3 = (long long)NC * NC * NC;
  const int c[3] = {b / (cpd * cpd), (b / cpd) % cpd, b % cpd};
  const long long o = off[b], s = off[b + 1] - o;
  for (long long t = threadIdx.x; t < s; t += blockDim.x) {
    const int p = skel[o + t];
    const int x[3] = {p % NC, (p / NC) % NC, p / (NC * NC)};
    int slot = 1;  // high face
    for (int a = 0; a < 3; ++a)
      if (x[a] % w == 0 && x[a] == w * c[a]) slot = 0;  // low face
    dof_src[(2 * slot) * n3 + p] = id;
    dof_src[(2 * slot + 1) * n3 + p] = (int)t;
  }
}

void launch_member_cells(const int* d_skel, const long long* d_off, const int* d_src, int ncell,
                         int cpd, int w, int NC, int* d_dof_src, cudaStream_t s) {
  if (ncell <= 0) return;
  k_member_cells<<<ncell, 128, 0, s>>>(d_skel, d_off, d_src, cpd, w, NC, d_dof_src);
}

__global__ void k_member_faces(const int* __restrict__ skel, const long long* __restrict__ off,
                               const int* __restrict__ cnt, const int* __restrict__ src,
                               long long n3, int* __restrict__ dof_src) {
  const int q = blockIdx.x;
  const long long o = off[q];
  for (int t = threadIdx.x; t < cnt[q]; t += blockDim.x) {
    const int p = skel[o + t];
    dof_src[4 * n3 + p] = src[q];
    dof_src[5 * n3 + p] = t;
  }
}

void launch_member_faces(const int* d_skel, const long long* d_off, const int* d_cnt,
                         const int* d_src, int nq, long long n3, int* d_dof_src, cudaStream_t s) {
  if (nq <= 0) return;
  k_member_faces<<<nq, 128, 0, s>>>(d_skel, d_off, d_cnt, d_src, n3, d_dof_src);
}

// ===========================================================================
// Apply: batched gather - GEMV - scatter over right-hand sides.
// trans = 0: 256 output rows per CTA, one row per thread (coalesced along M's
//            columns); trans = 1: 32 output columns per CTA, one warp per
//            column (coalesced down the column).
// ===========================================================================
constexpr int kRhsGroup = 4;
constexpr int kXChunk = 256;


__device__ __forceinline__ void gemv_emit(const GemvDesc& g, int i, int c, double y,
                                          double* u_out, long long ldu, long long contrib_ld) {
  if (g.mode == 1) g.contrib[i + (long long)c * contrib_ld] = y;
  else if (g.mode == 0) u_out[g.out_idx[i] + (long long)c * ldu] += g.alpha * y;
  else u_out[g.out_idx[i] + (long long)c * ldu] = g.alpha * y;
}

// RG right-hand sides per pass: 4, or 1 for single-vector launches (fewer
// registers, so more CTAs and more loads in flight); a column of results is the
// same sequence of operations either way.
template <int RG>
__device__ __forceinline__ void gemv_tile(const GemvDesc& g0, int local,
                                          const double* __restrict__ u_in_k,
                                          double* __restrict__ u_out_k, int nrhs_k,
                                          long long ldu_k, long long contrib_ld_k) {
  GemvDesc g = g0;
  const double* u_in = g.uin ? g.uin : u_in_k;
  double* u_out = g.uin ? g.uout : u_out_k;
  const int nrhs = g.uin ? g.nrhs : nrhs_k;
  const long long ldu = g.uin ? g.ldu : ldu_k;
  const long long contrib_ld = g.uin ? g.cld : contrib_ld_k;
  __shared__ double xs[kXChunk][RG];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if constexpr (RG == 1) {
    // one vector: x is read where it is used (a broadcast load per column or
    // row) instead of being staged per chunk, so no barrier interrupts the
    // stream of M; the columns of each warp and the order of every sum are
    // those of the staged form, so the results are the same bit for bit
    if (g.trans == 0) {
      __shared__ double red1[8][32];
      const int i = local * 32 + lane;
      for (int c0 = 0; c0 < nrhs; ++c0) {
        double acc = 0.0;
        const int jend = g.tri ? min(g.n, (local + 1) * 32) : g.n;
        for (int j0 = 0; j0 < jend; j0 += kXChunk) {
          const int jb = warp * 32, cnt = min(32, min(kXChunk, jend - j0) - jb);
          if (i < g.m && cnt > 0) {
            const double* col = g.M + i + (long long)(j0 + jb) * g.ld;
            const int* idx = g.in_idx + j0 + jb;
            const double* x = u_in + (long long)c0 * ldu;
#pragma unroll 16
            for (int jj = 0; jj < cnt; ++jj)
              acc = fma(col[(long long)jj * g.ld], x[idx[jj]], acc);
          }
        }
        __syncthreads();  // the previous vector's sums have been read
        red1[warp][lane] = acc;
        __syncthreads();
        if (warp == 0 && i < g.m) {
          double y = red1[0][lane];
#pragma unroll
          for (int w = 1; w < 8; ++w) y += red1[w][lane];
          gemv_emit(g, i, c0, y, u_out, ldu, contrib_ld);
        }
      }
    } else {
      const int jw = local * 32 + warp * 4;
      const int ibeg = g.tri ? ((local * 32) / kXChunk) * kXChunk : 0;
      for (int c0 = 0; c0 < nrhs; ++c0) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        const double* x = u_in + (long long)c0 * ldu;
        for (int i0 = ibeg; i0 < g.m; i0 += kXChunk) {
          const int ni = min(kXChunk, g.m - i0);
#pragma unroll 2
          for (int ii = lane; ii < ni; ii += 32) {
            const double xv = x[g.in_idx[i0 + ii]];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const double mv = jw + q < g.n ? g.M[(long long)(jw + q) * g.ld + i0 + ii] : 0.0;
              acc[q] = fma(mv, xv, acc[q]);
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double y = warp_sum(acc[q]);
          if (lane == 0 && jw + q < g.n) gemv_emit(g, jw + q, c0, y, u_out, ldu, contrib_ld);
        }
      }
    }
    return;
  }
  if (g.trans == 0) {
    // 32-row strip, lane = row; of every staged chunk of x, warp w takes the
    // 32 columns [32 w, 32 w + 32), so that a warp's loads are whole 256-byte
    // column segments and several are in flight; the eight partial sums are
    // added in warp order
    __shared__ double red[8][32][RG];
    const int i = local * 32 + lane;
    for (int c0 = 0; c0 < nrhs; c0 += RG) {
      const int nc = min(RG, nrhs - c0);
      double acc[RG];
#pragma unroll
      for (int cc = 0; cc < RG; ++cc) acc[cc] = 0.0;
      // lower triangular: this strip's rows need no column right of its last row
      const int jend = g.tri ? min(g.n, (local + 1) * 32) : g.n;
      for (int j0 = 0; j0 < jend; j0 += kXChunk) {
        const int nj = min(kXChunk, jend - j0);
        __syncthreads();
        for (int e = tid; e < nj * RG; e += 256) {
          const int jj = e / RG, cc = e % RG;
          xs[jj][cc] = (cc < nc) ? u_in[g.in_idx[j0 + jj] + (long long)(c0 + cc) * ldu] : 0.0;
        }
        __syncthreads();
        const int jb = warp * 32, cnt = min(32, nj - jb);
        if (i < g.m && cnt > 0) {
          const double* col = g.M + i + (long long)(j0 + jb) * g.ld;
#pragma unroll 8
          for (int jj = 0; jj < cnt; ++jj) {
            const double mv = col[(long long)jj * g.ld];
#pragma unroll
            for (int cc = 0; cc < RG; ++cc)
              acc[cc] = fma(mv, xs[jb + jj][cc], acc[cc]);
          }
        }
      }
#pragma unroll
      for (int cc = 0; cc < RG; ++cc) red[warp][lane][cc] = acc[cc];
      __syncthreads();
      if (warp == 0 && i < g.m) {
        for (int cc = 0; cc < nc; ++cc) {
          double y = red[0][lane][cc];
#pragma unroll
          for (int w = 1; w < 8; ++w) y += red[w][lane][cc];
          gemv_emit(g, i, c0 + cc, y, u_out, ldu, contrib_ld);
        }
      }
    }
  } else {
    for (int c0 = 0; c0 < nrhs; c0 += RG) {
      const int nc = min(RG, nrhs - c0);
      double acc[4][RG];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < RG; ++cc) acc[q][cc] = 0.0;
      // lower triangular: these columns have no entry above their first column
      const int ibeg = g.tri ? ((local * 32) / kXChunk) * kXChunk : 0;
      const int jw = local * 32 + warp * 4;  // this warp's first column
      for (int i0 = ibeg; i0 < g.m; i0 += kXChunk) {
        const int ni = min(kXChunk, g.m - i0);
        __syncthreads();
        for (int e = tid; e < ni * RG; e += 256) {
          const int ii = e / RG, cc = e % RG;
          xs[ii][cc] = (cc < nc) ? u_in[g.in_idx[i0 + ii] + (long long)(c0 + cc) * ldu] : 0.0;
        }
        __syncthreads();
        // the warp's four columns at each row: four independent loads a step
#pragma unroll 2
        for (int ii = lane; ii < ni; ii += 32) {
          double mv[4];
#pragma unroll
          for (int q = 0; q < 4; ++q)
            mv[q] = jw + q < g.n ? g.M[(long long)(jw + q) * g.ld + i0 + ii] : 0.0;
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int cc = 0; cc < RG; ++cc) acc[q][cc] = fma(mv[q], xs[ii][cc], acc[q][cc]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = jw + q;
#pragma unroll
        for (int cc = 0; cc < RG; ++cc) {
          const double y = warp_sum(acc[q][cc]);
          if (lane == 0 && j < g.n && cc < nc) gemv_emit(g, j, c0 + cc, y, u_out, ldu, contrib_ld);
        }
      }
    }
  }
}

__device__ __forceinline__ int find_desc_ll(const long long* __restrict__ off, int nd,
                                            long long t) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_apply_gather(const ApplyGatherDesc* __restrict__ descs,
                               const long long* __restrict__ off, int nd, long long total,
                               const double* __restrict__ u, long long ldu) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int di = find_desc_ll(off, nd, t);
    const ApplyGatherDesc d = descs[di];
    const long long e = t - off[di];
    const int k = (int)(e % d.len);
    const long long c = e / d.len;
    d.dst[e] = u[d.idx[k] + c * ldu];
  }
}

void launch_apply_gather(const ApplyGatherDesc* d_desc, const long long* d_off, int nd,
                         long long total, const double* u, long long ldu, cudaStream_t s) {
  if (total <= 0) return;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  k_apply_gather<<<blocks, 256, 0, s>>>(d_desc, d_off, nd, total, u, ldu);
}

__global__ void k_apply_emit(const ApplyEmitDesc* __restrict__ descs,
                             const long long* __restrict__ off, int nd, long long total,
                             double* __restrict__ u, long long ldu, long long contrib_ld) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int di = find_desc_ll(off, nd, t);
    const ApplyEmitDesc d = descs[di];
    const long long e = t - off[di];
    const int i = (int)(e % d.rows);
    const long long c = e / d.rows;
    const double y = d.Y[e];
    if (d.mode == 1) d.contrib[i + c * contrib_ld] = y;
    else if (d.mode == 0) u[d.out_idx[i] + c * ldu] += d.alpha * y;
    else u[d.out_idx[i] + c * ldu] = d.alpha * y;
  }
}

void launch_apply_emit(const ApplyEmitDesc* d_desc, const long long* d_off, int nd,
                       long long total, double* u, long long ldu, long long contrib_ld,
                       cudaStream_t s) {
  if (total <= 0) return;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  k_apply_emit<<<blocks, 256, 0, s>>>(d_desc, d_off, nd, total, u, ldu, contrib_ld);
}

__global__ void k_reduce_seg(const ReduceSeg* __restrict__ segs, const int* __restrict__ seg_off,
                             int nseg) {
  const int total = seg_off[nseg];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int si = find_desc(seg_off, nseg, t);
    const ReduceSeg sg = segs[si];
    const int e = t - seg_off[si];
    const int d = e % sg.ndof, c = e / sg.ndof;
    double sum = 0.0;
    for (int q = sg.off[d]; q < sg.off[d + 1]; ++q) sum += sg.contrib[sg.slot[q] + (long long)c * sg.cld];
    sg.u[sg.dof[d] + (long long)c * sg.ldu] += sg.alpha * sum;
  }
}

void launch_reduce_seg(const ReduceSeg* d_segs, const int* d_seg_off, int nseg, int total,
                       cudaStream_t s) {
  if (total <= 0) return;
  const int blocks = std::min((total + 255) / 256, 4096);
  k_reduce_seg<<<blocks, 256, 0, s>>>(d_segs, d_seg_off, nseg);
}

// ---- apply GEMV, the plans' layouts ----------------------------------------
// A launch covers segments (one per operator / request: the serving loop runs
// several requests' stages in one launch), each a descriptor array and, for
// the larger layouts, a unit table; seg_off holds the units' prefix over
// segments. Every descriptor's own vectors (uin, uout, nrhs, ldu, cld) apply
// when set, else the launch's.
struct GemvCtx {
  const double* uin;
  double* uout;
  int nrhs;
  long long ldu, cld;
};
__device__ __forceinline__ GemvCtx gemv_ctx(const GemvDesc& g, const double* u_in, double* u_out,
                                            int nrhs, long long ldu, long long cld) {
  return g.uin ? GemvCtx{g.uin, g.uout, g.nrhs, g.ldu, g.cld}
               : GemvCtx{u_in, u_out, nrhs, ldu, cld};
}

// Small blocks (both dimensions at most 64): one warp per descriptor. y = M x:
// lane = row, columns in order. y = M^T x: lanes over rows, one warp sum per
// column (fixed shuffle order). Entries above the diagonal of a triangular M
// are not read.
__global__ void __launch_bounds__(256, 3) k_gemv_small(const GemvFastSeg* __restrict__ segs,
                                                    const int* __restrict__ seg_off, int nseg,
                                                    const double* __restrict__ u_in,
                                                    double* __restrict__ u_out, int nrhs_k,
                                                    long long ldu_k, long long cld_k) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int unit = blockIdx.x * 8 + warp;
  if (unit >= seg_off[nseg]) return;
  const int si = find_desc(seg_off, nseg, unit);
  const GemvDesc g = segs[si].desc[unit - seg_off[si]];
  const GemvCtx x = gemv_ctx(g, u_in, u_out, nrhs_k, ldu_k, cld_k);
  for (int c0 = 0; c0 < x.nrhs; c0 += kRhsGroup) {
    const int nc = min(kRhsGroup, x.nrhs - c0);
    if (g.trans == 0) {
      for (int i = lane; i < g.m; i += 32) {
        double acc[kRhsGroup] = {0.0, 0.0, 0.0, 0.0};
        const int jend = g.tri ? min(g.n, i + 1) : g.n;
        for (int j = 0; j < jend; ++j) {
          const double mv = g.M[i + (long long)j * g.ld];
          const long long xo = g.in_idx[j] + (long long)c0 * x.ldu;
#pragma unroll
          for (int cc = 0; cc < kRhsGroup; ++cc)
            if (cc < nc) acc[cc] = fma(mv, x.uin[xo + (long long)cc * x.ldu], acc[cc]);
        }
        for (int cc = 0; cc < nc; ++cc) gemv_emit(g, i, c0 + cc, acc[cc], x.uout, x.ldu, x.cld);
      }
    } else {
      double xr[2][kRhsGroup];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
#pragma unroll
        for (int cc = 0; cc < kRhsGroup; ++cc)
          xr[h][cc] = (i < g.m && cc < nc)
                          ? x.uin[g.in_idx[i] + (long long)(c0 + cc) * x.ldu] : 0.0;
      }
      for (int j = 0; j < g.n; ++j) {
        double acc[kRhsGroup] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int i = lane + 32 * h;
          if (i < g.m && (!g.tri || i >= j)) {
            const double mv = g.M[i + (long long)j * g.ld];
#pragma unroll
            for (int cc = 0; cc < kRhsGroup; ++cc) acc[cc] = fma(mv, xr[h][cc], acc[cc]);
          }
        }
#pragma unroll
        for (int cc = 0; cc < kRhsGroup; ++cc)
          if (cc < nc) acc[cc] = warp_sum(acc[cc]);  // nc is the same on every lane
        if (lane == 0)
          for (int cc = 0; cc < nc; ++cc) gemv_emit(g, j, c0 + cc, acc[cc], x.uout, x.ldu, x.cld);
      }
    }
  }
}

// Larger blocks: gemv_tile's tiles (y = M x: 32-row strips; y = M^T x:
// 32-column tiles), located from the unit table (descriptor, tile) rather than
// a search over tile offsets. Two CTAs per SM: each warp keeps eight column
// loads in flight, which covers the memory latency at this occupancy.
template <int RG>
__global__ void __launch_bounds__(256, RG == 1 ? 3 : 2)
    k_gemv_tiles(const GemvFastSeg* __restrict__ segs, const int* __restrict__ seg_off, int nseg,
                 const double* __restrict__ u_in, double* __restrict__ u_out, int nrhs,
                 long long ldu, long long contrib_ld) {
  const int si = find_desc(seg_off, nseg, blockIdx.x);
  const int2 t = segs[si].tab[blockIdx.x - seg_off[si]];
  gemv_tile<RG>(segs[si].desc[t.x], t.y, u_in, u_out, nrhs, ldu, contrib_ld);
}

int gemv_tile_count(int m, int n, int trans) {
  if (m <= 0 || n <= 0) return 0;
  // y = M x: 32-row strips; y = M^T x: 32-column tiles
  return ((trans == 0 ? m : n) + 31) / 32;
}

void launch_gemv_fast(const GemvFastSeg* d_segs, const int* d_seg_off, int nseg, int units,
                      int layout, const double* u_in, double* u_out, int nrhs, long long ldu,
                      long long contrib_ld, cudaStream_t s) {
  if (units <= 0) return;
  if (layout == kGemvSmall)
    k_gemv_small<<<(units + 7) / 8, 256, 0, s>>>(d_segs, d_seg_off, nseg, u_in, u_out, nrhs, ldu,
                                                 contrib_ld);
  else if (nrhs == 1)
    k_gemv_tiles<1><<<units, 256, 0, s>>>(d_segs, d_seg_off, nseg, u_in, u_out, nrhs, ldu,
                                          contrib_ld);
  else  // several vectors, or per-descriptor vectors (serving: nrhs 0)
    k_gemv_tiles<kRhsGroup><<<units, 256, 0, s>>>(d_segs, d_seg_off, nseg, u_in, u_out, nrhs,
                                                  ldu, contrib_ld);
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

// ---------------------------------------------------------------------------
// GMRES vector kernels. A Krylov basis of nb vectors per right-hand side is
// stored as V[(i * nrhs + c) * n + t] (vector i of column c); coefficient
// arrays as coef[i * nrhs + c]. Reductions run in a fixed order (per block,
// then over the kDotBlocks partials), so results are bit-reproducible.
// ---------------------------------------------------------------------------

// partial dots of w against basis vectors i0 .. i0 + nb - 1 (nb <= kGmresGroup):
// part[(q * nrhs + c) * gridDim.x + block]
__global__ void __launch_bounds__(256) k_gmres_dots(const double* __restrict__ V, int i0, int nb,
                                                    const double* __restrict__ w, long long n,
                                                    int nrhs, double* __restrict__ part) {
  const int c = blockIdx.y;
  const double* wc = w + (long long)c * n;
  double acc[kGmresGroup];
#pragma unroll
  for (int q = 0; q < kGmresGroup; ++q) acc[q] = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double wv = wc[t];
#pragma unroll
    for (int q = 0; q < kGmresGroup; ++q)
      if (q < nb) acc[q] = fma(V[((long long)(i0 + q) * nrhs + c) * n + t], wv, acc[q]);
  }
  __shared__ double sc[40];
#pragma unroll
  for (int q = 0; q < kGmresGroup; ++q) {
    if (q < nb) {  // nb is the same for the whole block: the barriers inside match
      const double tot = block_sum(acc[q], sc);
      if (threadIdx.x == 0) part[((long long)q * nrhs + c) * gridDim.x + blockIdx.x] = tot;
    }
  }
}

void launch_gmres_dots(const double* V, int nb, const double* w, long long n, int nrhs,
                       double* d_partial, double* d_out, cudaStream_t s) {
  for (int i0 = 0; i0 < nb; i0 += kGmresGroup) {
    const int g = nb - i0 < kGmresGroup ? nb - i0 : kGmresGroup;
    k_gmres_dots<<<dim3(kDotBlocks, nrhs), 256, 0, s>>>(V, i0, g, w, n, nrhs, d_partial);
    k_dot_final<<<g * nrhs, 256, 0, s>>>(d_partial, kDotBlocks, d_out + (long long)i0 * nrhs);
  }
}

// w[:, c] += sign * sum_{i < nb} coef[i * nrhs + c] V_i[:, c]
__global__ void __launch_bounds__(256) k_gmres_axpy(double* __restrict__ w,
                                                    const double* __restrict__ V, int nb,
                                                    const double* __restrict__ coef, double sign,
                                                    long long n, int nrhs) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (t >= n) return;
  double acc = 0.0;
  for (int i = 0; i < nb; ++i)
    acc = fma(coef[(long long)i * nrhs + c], V[((long long)i * nrhs + c) * n + t], acc);
  w[(long long)c * n + t] = fma(sign, acc, w[(long long)c * n + t]);
}

void launch_gmres_axpy(double* w, const double* V, int nb, const double* coef, double sign,
                       long long n, int nrhs, cudaStream_t s) {
  if (nb <= 0) return;
  k_gmres_axpy<<<dim3((unsigned)((n + 255) / 256), nrhs), 256, 0, s>>>(w, V, nb, coef, sign, n,
                                                                       nrhs);
}

// dst[:, c] = scale[c] * src[:, c]
__global__ void __launch_bounds__(256) k_gmres_scale(double* __restrict__ dst,
                                                     const double* __restrict__ src,
                                                     const double* __restrict__ scale,
                                                     long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (t >= n) return;
  dst[(long long)c * n + t] = scale[c] * src[(long long)c * n + t];
}

void launch_gmres_scale(double* dst, const double* src, const double* scale, long long n, int nrhs,
                        cudaStream_t s) {
  k_gmres_scale<<<dim3((unsigned)((n + 255) / 256), nrhs), 256, 0, s>>>(dst, src, scale, n);
}

}  // namespace hif
