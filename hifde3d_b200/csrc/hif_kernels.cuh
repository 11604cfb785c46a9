// Device kernels of the HIF factor / apply path (sm_100a, FP64).
//
// Every launcher takes device-resident descriptor arrays and a stream; the
// host engine (hif_engine.cpp) builds the descriptors per level phase.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hif {

// ---------------------------------------------------------------------------
// Status bits written by kernels (OR-ed into a device word per phase).
// ---------------------------------------------------------------------------
enum StatusBits : int {
  kStatusTinyPivot = 1,   // |pivot| <= 1e-300 or not finite in an elimination
  kStatusNonFinite = 2,   // NaN / Inf met in an output
  kStatusIdZero = 4,      // ID of an all-zero face block (every column redundant)
};

// A DOF's membership in one dense source block: source id and position.
struct CoverEntry {
  int src;  // < 0: unused slot
  int pos;
};
constexpr int kCover = 3;

// One dense "source" of the remaining operator (a Schur complement block).
struct SourceDesc {
  const double* ptr;
  long long ld;
};

// Assembly target: out(i, j) = A0(rows[i], cols[j]) + sum over the sources s
// that hold both DOFs rows[i] and cols[j] and are admitted for this target,
// of s(pos(rows[i]), pos(cols[j])).
//
// Source membership comes from per-DOF arrays (6 x NC^3 ints): for DOF p,
// dof_src[(2c) NC^3 + p] / dof_src[(2c+1) NC^3 + p] are (source, position)
// for slot c in {0: cell having p on its low face, 1: cell having p on its
// high face, 2: skeletonized face containing p}; source < 0 means none.
struct GatherTarget {
  double* out;
  long long ld;
  const int* rows;
  const int* cols;
  double* a22_out;  // optional copy of out[0:r, 0:r] (ld r)
  int m, n;
  int a0_skip;      // no stencil term where i >= a0_skip && j >= a0_skip
  int r;
  int mode;         // 0: sources with src_owner[s] == owner; 1: s in {allowA, allowB}; 2: none
  int owner;
  int allowA, allowB;
};

// C(m x n) = beta * C + alpha * op(A) * op(B); column-major.
struct GemmDesc {
  double* C;
  const double* A;
  const double* B;
  long long ldc, lda, ldb;
  int m, n, k;
  int transA, transB;
  double alpha, beta;
  int lower;  // 128 x 128 tiles only: skip the tiles above the diagonal (row tile < column tile)
  const int* skip;  // optional: the product is skipped when *skip != 0 (read on the device)
  int a_lower;  // op(A) is lower triangular (m = k): a row tile reads no k past its last row
  int b_lower;  // op(B) is lower triangular (k = n): a column tile reads no k before its first column
};

// Dense elimination block: B (n x n, ld n) in assembly order [red | skel].
// Gauss-Jordan: a22inv = A22^{-1}, X = A22^{-1} A21. Cholesky (symmetric
// positive definite A22): L = chol(A22) (lower, zeros above), a22inv = L^{-1}
// (lower), X = Y = L^{-1} A21; in both the skeleton block ends as
// A11 - A12 A22^{-1} A21 in B.
struct SweepDesc {
  double* B;
  double* a22inv;  // r x r, ld r  (compact copy written at the end)
  double* X;       // r x s, ld r
  int n, r;
  double* L;       // Cholesky only: r x r, ld r
};

// Interpolative decomposition of M (m x n, ld m) for one face.
struct IdDesc {
  double* M;
  const int* order;  // optional prescribed column order (replay), else null
  int* jpvt;         // n: 0-based pivot order
  double* rdiag;     // n: diagonal of R
  int* keep;         // n: 1 if |R_ii| > eps |R_00|
  int* rank;         // 1
  double* W;         // k x (n-k), ld k (written after the rank is known)
  int m, n;
};

// ---- Interpolative decomposition by pivoted Cholesky of G = M^T M (mixed
// precision mode). Column-pivoted QR of M and pivoted Cholesky of M^T M choose
// the same pivots and the same R in exact arithmetic (the pivot is the column
// with the largest norm orthogonal to the chosen ones, i.e. the largest
// remaining Schur diagonal); the factorization stops at the first pivot with
// R_ii <= eps R_00, so only the skeleton rows of R are formed.
struct PcholDesc {
  double* G;       // n x n, ld n: M^T M, updated after every panel
  double* R;       // n x n row-major: row i of R at R + i * n (original column order)
  int* chosen;     // n
  int* piv;        // n: pivot of step i
  int* info;       // [0] steps done, [1] 1 once the rank is known
  double* d0;      // R_00^2
  IdDesc id;       // outputs (jpvt, rdiag, keep, rank, W) and n
};
// nb steps from step i0 for the active faces; dynamic smem n doubles + n ints.
void launch_pchol_panel(const PcholDesc* d_desc, const int* d_active, int nact, int i0, int nb,
                        double eps, int max_n, int* d_status, cudaStream_t s);
// Outputs after the last panel: jpvt (skeleton pivots, then the redundant
// columns in increasing order), keep, rdiag, rank; R11 (k x k, ld k, upper) into
// G's space and R12 into W (k x (n - k), ld k) for the triangular solve.
void launch_pchol_finish(const PcholDesc* d_desc, int nd, int max_n, cudaStream_t s);
// Diagonal-block step of W := R11^{-1} W by blocks of kTrsmNB rows from the
// bottom: rows [a0, a1) of every face's W solved with R11's diagonal block.
constexpr int kTrsmNB = 64;
struct TrsmBlockDesc {
  const double* R;  // k x k, ld k, upper triangular
  double* W;        // k x ncols, ld k
  int k, ncols, a0, a1;
};
void launch_trsm_block(const TrsmBlockDesc* d_desc, int nd, int max_cols, cudaStream_t s);

// Source membership of the DOFs (the 6 x NC^3 arrays read by k_gather), built
// on the device. Cells: skeleton DOF t of cell b (cell_ids[b] >= 0) gets
// (source, t) in slot pair 0 (on the cell's low face along some axis) or 1.
void launch_member_cells(const int* d_skel, const long long* d_off, const int* d_src, int ncell,
                         int cpd, int w, int NC, int* d_dof_src, cudaStream_t s);
// Faces: skeleton DOF t of listed face q gets (d_src[q], t) in slot pair 2.
void launch_member_faces(const int* d_skel, const long long* d_off, const int* d_cnt,
                         const int* d_src, int nq, long long n3, int* d_dof_src, cudaStream_t s);

// Apply for many right-hand sides as gather / GEMM / emit: the input rows of a
// descriptor are gathered into a dense block (len x nrhs, ld len), multiplied
// by op(M) with the batched GEMM, and the result (rows x nrhs, ld rows) is
// emitted like the GEMV's output (mode 0: u[out] += alpha y; 1: contrib = y;
// 2: u[out] = alpha y). Element counts are prefix sums over descriptors.
struct ApplyGatherDesc {
  const int* idx;
  double* dst;
  int len;
};
struct ApplyEmitDesc {
  const double* Y;
  const int* out_idx;
  double* contrib;
  int rows, mode;
  double alpha;
};
void launch_apply_gather(const ApplyGatherDesc* d_desc, const long long* d_off, int nd,
                         long long total, const double* u, long long ldu, cudaStream_t s);
void launch_apply_emit(const ApplyEmitDesc* d_desc, const long long* d_off, int nd,
                       long long total, double* u, long long ldu, long long contrib_ld,
                       cudaStream_t s);
// Apply: y = op(M) x[in] with x, y gathered / scattered through DOF lists.
struct GemvDesc {
  const double* M;
  long long ld;
  const int* in_idx;
  const int* out_idx;   // mode 0 / 2
  double* contrib;      // mode 1: contribution slots (length = rows of op(M))
  int m, n;             // M is m x n
  int trans;            // 0: y = M x (len m), 1: y = M^T x (len n)
  int tri;              // 1: M is lower triangular (square); entries above the diagonal are not read
  double alpha;
  int mode;             // 0: u_out[out] += alpha y; 1: contrib = y; 2: u_out[out] = alpha y
  // Optional per-descriptor vectors (batched solves of several operators in one
  // launch); when uin is null the launch's vectors and sizes apply.
  const double* uin;
  double* uout;
  int nrhs;
  long long ldu, cld;
};

// The serving loop's batched reduce-scatter: one segment per request.
struct ReduceSeg {
  const int* dof;
  const int* off;
  const int* slot;
  const double* contrib;
  double* u;
  long long cld, ldu;
  int ndof, nrhs;
  double alpha;
};
// d_seg_off: prefix over segments of ndof * nrhs.
void launch_reduce_seg(const ReduceSeg* d_segs, const int* d_seg_off, int nseg, int total,
                       cudaStream_t s);

struct CopyDesc {
  const double* src;
  double* dst;
  long long lds, ldd;
  int m, n;
};
// dst (m x n, ld ldd) = alpha * src^T, src n x m (ld lds); 32 x 32 tiles.
struct TCopyDesc {
  const double* src;
  double* dst;
  long long lds, ldd;
  int m, n;
  double alpha;
};
void launch_tcopy(const TCopyDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                  cudaStream_t s);

// ---------------------------------------------------------------------------
// Launchers. Descriptor arrays live in device memory; tile_off (device) is
// the prefix sum of per-descriptor tile counts, total = tile_off[count].
// ---------------------------------------------------------------------------
void launch_gather(const GatherTarget* d_tg, const int* d_tile_off, int ntg, int total_tiles,
                   const SourceDesc* d_src, const int* d_src_owner, const int* d_dof_src,
                   const double* d_band, long long ncell3, int NC, cudaStream_t s);
int gather_tiles(int m, int n);

// tile: 64 (64x64x16, 4x4 per thread) or 128 (128x128x16, 8x8 per thread,
// 3-stage cp.async pipeline); tile offsets must be built with the same tile.
void launch_dgemm(const GemmDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                  cudaStream_t s, int tile = 64);
int dgemm_tiles(int m, int n, int tile = 64);

// Split-K reduction: C = alpha * sum_{s < S} P_s + beta * C, P_s = P + s * m * n
// (ld m), summed in order s = 0, 1, ... (deterministic).
struct SplitKDesc {
  double* C;
  const double* P;
  long long ldc;
  int m, n, S;
  double alpha, beta;
};
void launch_splitk_reduce(const SplitKDesc* d_desc, int nd, cudaStream_t s);

// Split-TF32 tensor-core GEMM (tcgen05, FP32 accumulation in tensor memory).
// Operands are first converted to TF32 (hi, lo) pairs in 128 x 32 tiles of
// kTcTileBytes each: element (i, kk) of an operand is op(X)[i, kk] for A and
// op(B)[kk, i] for B; tile (rt, kt) at out + (rt * ceil(kdim / 32) + kt) *
// kTcTileBytes.
constexpr int kTcTileBytes = 32768;
struct TcOperand {
  const double* X;
  long long ld;
  int trans;  // 0: element (i, kk) at X[i + kk ld]; 1: at X[kk + i ld]
  int rows, kdim;
  unsigned char* out;
};
// d_tile_off: prefix over operands of ceil(rows / 128) * ceil(kdim / 32).
void launch_tc_convert(const TcOperand* d_ops, const int* d_tile_off, int nops, int total_tiles,
                       cudaStream_t s);
// C = alpha A B^T-style product of converted operands (A rows m, B rows n,
// common kdim k) + beta C; 128 x 128 tiles counted by d_tile_off; bounded
// waits report kStatusTimeout in d_status.
struct TcGemm {
  const unsigned char* A;
  const unsigned char* B;
  double* C;
  long long ldc;
  int m, n, k;
  double alpha, beta;
  int lower;  // skip the tiles above the diagonal
};
void launch_gemm_tc(const TcGemm* d_desc, const int* d_tile_off, int nd, int total_tiles,
                    int* d_status, cudaStream_t s);

// FP64 products on the int8 tensor cores (Ozaki scheme). Every operand row
// (a row of op(A), a column of op(B)) gets a power-of-two exponent e (its
// largest magnitude is below 2^e) and S signed 7-bit slices q_s with
// x = 2^e sum_s q_s 2^{-7(s+1)} + r, |r| < 2^{e - 7S}. Converted operands are
// tiles of 128 rows x 64 values of k: tile (rt, kt) holds S slices of
// kOzPart bytes at out + ((rt * ceil(kdim / 64) + kt) * S + s) * kOzPart.
constexpr int kOzK = 64, kOzPart = 128 * kOzK, kOzMaxS = 8;
// Largest k of one product: every diagonal sum of slice products stays exact in
// int32 ((d + 1) k 127^2 < 2^31 for d < kOzMaxS).
constexpr int kOzMaxK = 16384;
struct OzOperand {
  const double* X;
  long long ld;
  int trans;  // 0: element (i, kk) at X[i + kk ld]; 1: at X[kk + i ld]
  int rows, kdim;
  signed char* out;
  int* rexp;  // per-row exponent, rows entries
};
// d_tile_off: prefix over operands of ceil(rows / 128) * ceil(kdim / 64).
// Every rexp lies in [d_rexp, d_rexp + n_rexp): it is cleared, then the
// exponents are taken (one pass over the operands), then the slices (a second).
void launch_oz_convert(const OzOperand* d_ops, const int* d_tile_off, int nops, int total_tiles,
                       int slices, int* d_rexp, long long n_rexp, cudaStream_t s);
struct OzGemm {
  const signed char* A;  // converted op(A): rows m
  const signed char* B;  // converted op(B)^T: rows n
  const int* ea;
  const int* eb;
  double* C;
  long long ldc;
  int m, n;
  int kt_total;     // k tiles of the converted operands
  int kt0, kt_cnt;  // k tiles of this product (kt_cnt * kOzK <= kOzMaxK)
  double alpha, beta;
  int lower;  // skip the tiles entirely above the diagonal
  int a_lower;  // op(A) lower triangular: a 128-row tile reads no k tile past its last row
  int b_lower;  // op(B) lower triangular: a column tile reads no k tile before its first column
};
// C = alpha op(A) op(B) + beta C from converted operands with `slices` slices
// (2..kOzMaxS); d_tile_off counts tiles of 128 x oz_tile_n(slices) columns.
int oz_tile_n(int slices);
void launch_gemm_oz(const OzGemm* d_desc, const int* d_tile_off, int nd, int total_tiles,
                    int slices, int* d_status, cudaStream_t s);

// In-shared-memory Gauss-Jordan sweep of the first r pivots (n <= kSmallSweepN).
constexpr int kSmallSweepN = 160;
void launch_sweep_small(const SweepDesc* d_desc, int nd, int max_n, int* d_status,
                        cudaStream_t s);

// Blocked sweep, one pivot block [k0, k0+nbk) of every active block.
constexpr int kSweepNB = 128;
void launch_sweep_diag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                       double* d_dinv, int* d_status, cudaStream_t s, int sym = 0);
// Cholesky elimination of symmetric positive definite interiors (lower
// triangles only). Small blocks whole in shared memory: L, L^{-1}, Y and the
// Schur complement in one launch.
void launch_chol_small(const SweepDesc* d_desc, int nd, int max_n, int* d_status,
                       cudaStream_t s);
// Pivot block K = [k0, k0 + 128) of the blocked factorization: L_KK = chol(B[K, K])
// written over B[K, K] (zeros above its diagonal) and L_KK^{-1} (lower, zeros
// above) into dinv (128 x 128 per active block, ld = its width).
void launch_chol_diag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                      double* d_dinv, int* d_status, cudaStream_t s);
void launch_sweep_setdiag(const SweepDesc* d_desc, const int* d_active, int nact, int k0,
                          const double* d_dinv, cudaStream_t s);

// Column-pivoted Householder QR + rank + interpolation matrix, one CTA per face.
// W is written to IdDesc::W, which must hold at least n*n/4 + n doubles.
void launch_id(const IdDesc* d_desc, int nd, int max_n, double eps, int* d_status,
               cudaStream_t s, long long max_mn = 0);

void launch_copy(const CopyDesc* d_desc, const int* d_tile_off, int nd, int total_tiles,
                 cudaStream_t s);

// Grouped interpolative decomposition: `group` CTAs cooperate on one face,
// owning its columns cyclically (column j belongs to CTA j % group). Per
// column step: candidates -> group barrier -> the pivot column's owner swaps
// and builds the reflector -> group barrier -> every CTA updates its columns.
// Cross-CTA data goes through L2; barrier waits are bounded (a timeout sets
// kStatusTimeout and the kernel returns). Results equal k_id's. Needs all CTAs
// co-resident: launched cooperatively when group > 1.
// work: per face 4 * n doubles + 64 ints of scratch (norms, pivots, barrier).
enum { kStatusTimeout = 8 };
struct IdGroupDesc {
  IdDesc id;
  double* norms;  // 2n (vn1, vn2)
  int* sync;      // 64 ints: barrier count / generation, candidates
  double* cand;   // group doubles
  double* tau;    // 1
};
cudaError_t launch_id_group(const IdGroupDesc* d_desc, int nd, int group, double eps,
                            int* d_status, cudaStream_t s, int max_m, int max_n);

// Row compression of a tall face block before its pivoted QR: blocked
// Householder QR (no pivoting) in 32-column panels. For panel [k0, k0+kb) the
// panel kernel factors M[k0:m, k0:k0+kb) in place and writes the explicit
// reflector block V (unit diagonal, zeros above; m x 32, ld m, rows below k0
// unused) and T, the upper triangular factor of the compact WY form
// Q = I - V T V^T (32 x 32, ld 32). The trailing columns C are then updated by
// batched GEMMs: Z = V^T C, Z = T^T Z, C -= V Z.
constexpr int kQrNB = 32;
// Two-level blocked Householder: outer panels of kQrNB2 columns, each
// factored by kQrNB-wide sub-panels.
constexpr int kQrNB2 = 128;
struct QrDesc {
  double* M;    // m x n, ld m
  double* V;    // m x kQrNB2, ld m: reflectors of the current outer panel
  double* T;    // kQrNB x kQrNB: compact-WY factor of the current sub-panel
  double* tau;  // kQrNB2: Householder scalars of the current outer panel
  int m, n;
};
// Sub-panel at columns [k1, k1 + kQrNB) of the outer panel starting at k0: V's
// columns k1 - k0 .. are written for rows k0 .. m - 1 (zeros above the unit
// diagonal), tau likewise, T for the sub-panel.
void launch_qr_panel(const QrDesc* d_desc, const int* d_active, int nact, int k1, int k0,
                     cudaStream_t s);
// The same by one thread-block cluster per face with the panel rows held in
// shared memory: for faces with at most qr_cluster_max_rows() rows below k1;
// max_rows = the largest m - k1 among the active faces (sets the cluster size).
int qr_cluster_max_rows();
void launch_qr_panel_cluster(const QrDesc* d_desc, const int* d_active, int nact, int k1,
                             int k0, int max_rows, cudaStream_t s);
// T (nb x nb, ld kQrNB2) of the outer panel from W = V^T V (ld kQrNB2) and tau:
// T[j, j] = tau_j, T[0:j, j] = -tau_j T[0:j, 0:j] W[0:j, j].
struct TFactorDesc {
  const double* W;
  const double* tau;
  double* T;
  int nb;
};
void launch_qr_tfactor(const TFactorDesc* d_desc, int nd, cudaStream_t s);
// dst (n x n, ld ldd) = upper triangle of src (ld lds), zeros below.
struct TriuDesc {
  const double* src;
  double* dst;
  long long lds, ldd;
  int n;
};
void launch_triu(const TriuDesc* d_desc, int nd, cudaStream_t s);

// Solve R X = B in place (R: k x k upper triangular, non-unit; B: k x nb), one
// right-hand side column per thread (the reference's dtrsm('L','U','N','N') call,
// src/InterpDecomp.cpp:213-231).
void launch_trsm_upper(const double* R, long long ldr, int k, double* B, long long ldb, int nb,
                       cudaStream_t s);
int copy_tiles(int m, int n);

// contrib_ld: stride between right-hand sides in the contribution buffer.
// The apply's GEMV launches (the engine's plans and the serving loop's batched
// stages). Layouts: kGemvSmall, one warp per descriptor (both dimensions <=
// kGemvSmallMax; units = descriptors); kGemvTiles, y = M x by 32-row strips or
// y = M^T x by 32-column tiles (units = entries (descriptor, tile) of the
// segment's table, gemv_tile_count tiles per descriptor). A launch covers
// segments (one per operator or request) of one layout; seg_off: prefix of the
// units over the segments.
constexpr int kGemvSmall = 0, kGemvTiles = 1, kGemvLayouts = 2;
int gemv_tile_count(int m, int n, int trans);
constexpr int kGemvSmallMax = 64;
struct GemvFastSeg {
  const GemvDesc* desc;
  const int2* tab;  // null for kGemvSmall
};
void launch_gemv_fast(const GemvFastSeg* d_segs, const int* d_seg_off, int nseg, int units,
                      int layout, const double* u_in, double* u_out, int nrhs, long long ldu,
                      long long contrib_ld, cudaStream_t s);

// u[dof[d]] += alpha * sum_{t in [off[d], off[d+1])} contrib[slot[t]], in order.
void launch_reduce_scatter(const int* d_dof, const int* d_off, const int* d_slot,
                           const double* d_contrib, int ndof, long long contrib_ld,
                           double alpha, double* u, int nrhs, long long ldu, cudaStream_t s);

// Operators and vectors.
void launch_setup_node(const double* d_A, const double* d_V, int N, double h, double* d_band,
                       cudaStream_t s);
void launch_setup_faces(const double* d_ax, const double* d_ay, const double* d_az,
                        const double* d_V, int N, double h, double* d_band, cudaStream_t s);
void launch_stencil_apply(const double* d_band, int NC, const double* x, double* y, int nrhs,
                          long long ldx, int transpose, cudaStream_t s);
void launch_zero_boundary(double* u, int NC, int nrhs, long long ldu, cudaStream_t s);

// Deterministic dot products: out[c] = sum_i x[i + c ld] y[i + c ld] (per rhs c).
void launch_dot(const double* x, const double* y, long long n, int nrhs, long long ld,
                double* d_partial, double* d_out, cudaStream_t s);
constexpr int kDotBlocks = 296;

// PCG vector updates (all per rhs column c, scalars from device arrays):
//   x += a p; r -= a q with a = rz / pq
void launch_pcg_update_xr(double* x, double* r, const double* p, const double* q,
                          const double* rz, const double* pq, long long n, int nrhs,
                          long long ld, cudaStream_t s);
//   p = z + (rz_new / rz_old) p
void launch_pcg_update_p(double* p, const double* z, const double* rz_new,
                         const double* rz_old, long long n, int nrhs, long long ld,
                         cudaStream_t s);

// GMRES (basis vector i of rhs c at V + (i * nrhs + c) * n, coefficients at
// coef[i * nrhs + c]; all deterministic):
//   out[i * nrhs + c] = <V_i[:, c], w[:, c]> for i < nb (partial: kGmresGroup *
//   nrhs * kDotBlocks doubles)
constexpr int kGmresGroup = 16;
void launch_gmres_dots(const double* V, int nb, const double* w, long long n, int nrhs,
                       double* d_partial, double* d_out, cudaStream_t s);
//   w[:, c] += sign * sum_{i < nb} coef[i * nrhs + c] V_i[:, c]
void launch_gmres_axpy(double* w, const double* V, int nb, const double* coef, double sign,
                       long long n, int nrhs, cudaStream_t s);
//   dst[:, c] = scale[c] src[:, c]
void launch_gmres_scale(double* dst, const double* src, const double* scale, long long n, int nrhs,
                        cudaStream_t s);

}  // namespace hif
