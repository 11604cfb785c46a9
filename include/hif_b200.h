/*
 * hif_b200.h -- C ABI of the B200 implementation of HIFDE3D's hierarchical
 * interpolative factorization (HIF) for 3D 7-point elliptic operators.
 *
 * The reference (arbenson/HIFDE3D) exposes a C++ template API; each entry
 * point below replaces one call of it for Scalar = double. All functions
 * return an int status (HIF_OK = 0). Handles are not thread-safe; one handle
 * drives one CUDA device (the device current at hif_create) and one stream.
 *
 * Host-pointer entry points copy their inputs to the GPU and their results
 * back; *_device entry points take device pointers on that device and do not
 * synchronise the stream unless stated.
 *
 * Vector layout everywhere: NC^3 entries (NC = N + 1), DOF id
 * i + NC*j + NC^2*k for i, j, k in [0, N]; entries with i, j or k equal to 0 are
 * the Dirichlet planes and are ignored / zeroed (src/Factor.cpp:79-89,977-990).
 * Several right-hand sides are stored column-major with leading dimension ldu.
 */
#ifndef HIF_B200_H_
#define HIF_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hif_factor_s* hif_handle;

enum hif_status {
  HIF_OK = 0,
  HIF_ERR_ARG = 1,        /* invalid argument */
  HIF_ERR_CUDA = 2,       /* CUDA runtime error (message: hif_last_error) */
  HIF_ERR_NOMEM = 3,      /* device allocation failed */
  HIF_ERR_SINGULAR = 4,   /* zero / non-finite pivot in an elimination */
  HIF_ERR_STATE = 5,      /* call out of order (e.g. Apply before Factor) */
  HIF_ERR_NODEVICE = 6,   /* no CUDA device / kernels not loadable */
  HIF_ERR_BUDGET = 7,     /* would exceed the handle's memory budget */
  HIF_ERR_IO = 8          /* factor file unreadable, unwritable, truncated or corrupt */
};

enum hif_partition {
  HIF_PARTITION_REFERENCE = 0, /* cells_per_dir = NC / width (src/Factor.cpp:52-53) */
  HIF_PARTITION_CLIPPED = 1    /* ceil(NC / width), last cell clipped at N */
};

/* HIFFactor<double>(int N, int P, double epsilon) -- include/Factor.hpp:12-13. */
int hif_create(int N, int P, double epsilon, int partition, hif_handle* out);
/* ~HIFFactor -- include/Factor.hpp:15. */
int hif_destroy(hif_handle h);

/* Stream used by every call on this handle (a cudaStream_t; 0 = the handle's own). */
int hif_set_stream(hif_handle h, void* stream);

/* SetupStencil(factor, N, h, A, V) -- include/setup_stencil.hpp:6-76.
 * A, V: (N+2)^3 float64 tensors in NumTns order (i fastest, include/numtns.hpp:99). */
int hif_setup_stencil(hif_handle h, int N, double hstep, const double* A, const double* V);
int hif_setup_stencil_device(hif_handle h, int N, double hstep, const double* dA,
                             const double* dV);
/* Symmetric flux form -div(a grad u) + V u with face coefficients (no reference
 * counterpart; the reference's node form is non-symmetric for variable a).
 * ax(i,j,k) couples (i,j,k)-(i+1,j,k); ay, az likewise; all (N+2)^3, i fastest. */
int hif_setup_stencil_faces(hif_handle h, int N, double hstep, const double* ax,
                            const double* ay, const double* az, const double* V);
int hif_setup_stencil_faces_device(hif_handle h, int N, double hstep, const double* dax,
                                   const double* day, const double* daz, const double* dV);

/* HIFFactor::Initialize -- src/Factor.cpp:6-39. */
int hif_initialize(hif_handle h);
/* HIFFactor::Factor -- src/Factor.cpp:41-63. */
int hif_factor(hif_handle h);

/* Factor save / load. No counterpart in the reference, whose factor data
 * (FactorData / IndexData per block, include/data.hpp:11-62,84-110) lives only in
 * the HIFFactor object. hif_save_factor writes the factorization held by h (after
 * hif_factor or hif_load_factor) to `path`: every level's index data, the matrices
 * the apply reads (A22, A22^{-1}, X, W) and, when h has one, the operator, so
 * that hif_solve_pcg works after a load. The file is written as path + ".tmp"
 * and renamed when complete. hif_load_factor reads such a file into a handle
 * created with the same N, P, epsilon and partition (HIF_ERR_ARG otherwise),
 * replacing any factorization it held; afterwards hif_apply / hif_solve_pcg give
 * the results of the saved factorization bit for bit. Schur complements kept
 * with HIF_OPT_KEEP_SCHUR are not saved. A file that is missing, truncated,
 * corrupt (sizes, offsets or DOF ids out of range, checksum) or written on a
 * machine of the other byte order returns HIF_ERR_IO and leaves h without a
 * factorization. Both synchronise the handle's stream. */
int hif_save_factor(hif_handle h, const char* path);
int hif_load_factor(hif_handle h, const char* path);

/* HIFFactor::Apply(u, apply_inverse) -- src/Factor.cpp:992-1081, in place. */
int hif_apply(hif_handle h, double* u, int nrhs, long long ldu, int apply_inverse);
int hif_apply_device(hif_handle h, double* du, int nrhs, long long ldu, int apply_inverse);

/* SpMV(sp_matrix, x, y) -- src/Factor.cpp:1099-1113: y = A^T x (the reference walks
 * columns); transpose = 0 gives y = A x. The operator is the one set up, kept intact
 * by hif_factor (the reference consumes its sparse matrix). */
int hif_spmv(hif_handle h, const double* x, double* y, int nrhs, long long ld, int transpose);
int hif_spmv_device(hif_handle h, const double* dx, double* dy, int nrhs, long long ld,
                    int transpose);

/* Preconditioned CG on A x = b with the factor's inverse apply as preconditioner and
 * an FP64 residual on the operator (the reference has no iterative solver; its driver
 * only reports e_a / e_s, tests/HIFDE3D/main.cpp:121-134). x is an output (x0 = 0).
 * iters, relres: per right-hand side. */
int hif_solve_pcg(hif_handle h, const double* b, double* x, int nrhs, long long ld,
                  double tol, int maxit, int* iters, double* relres);
int hif_solve_pcg_device(hif_handle h, const double* db, double* dx, int nrhs, long long ld,
                         double tol, int maxit, int* iters, double* relres);

/* Restarted GMRES(restart) on A x = b with the factor's inverse apply as right
 * preconditioner, so the residual it minimises and reports is the true FP64
 * residual |b - A x| / |b| on the operator. No counterpart in the reference (it has
 * no iterative solver); this is the solver for its node-coefficient operator
 * (SetupStencil, include/setup_stencil.hpp:6-76), which is not symmetric for
 * variable coefficients. x is an output (x0 = 0); restart in 1..64; maxit bounds
 * the Arnoldi steps (one preconditioner and one operator apply each) per
 * right-hand side; iters / relres per right-hand side. Bit-reproducible. */
int hif_solve_gmres(hif_handle h, const double* b, double* x, int nrhs, long long ld,
                    double tol, int maxit, int restart, int* iters, double* relres);
int hif_solve_gmres_device(hif_handle h, const double* db, double* dx, int nrhs, long long ld,
                           double tol, int maxit, int restart, int* iters, double* relres);

/* ---- the reference's free functions on the hot path -----------------------------
 * Schur(matrix, data) -- include/Schur.hpp:72-100: eliminate the redundant DOFs of a
 * dense block. matrix: m x m (ld); red / skel: positions (redundant_inds /
 * skeleton_inds). Outputs (any may be NULL): A22 (nr x nr), A22^{-1} (nr x nr),
 * X = A22^{-1} A21 (nr x ns), S = -A12 X (ns x ns), column-major, ld = rows. */
int hif_schur(const double* matrix, int m, long long ld, const int* red, int nr,
              const int* skel, int ns, double* A22, double* A22inv, double* X, double* S);
/* The same on device memory, block given in [redundant | skeleton] order (n x n,
 * ld n; r redundant): writes A22^{-1}, X and S. Allocates device workspace. */
int hif_schur_device(const double* dB, int n, int r, double* dA22inv, double* dX, double* dS);
/* Allocation-free variant of hif_schur_device; it has no counterpart in the reference.
 * For callers that cannot allocate device memory: a process whose framework allocator
 * already holds the whole GPU, or a loop that must not call into the allocator between
 * its own kernels. All scratch lives in one fixed device array inside the library
 * (about 2 MiB per GPU, held from library load until process exit), so blocks are limited
 * to n <= 512 (larger ones return HIF_ERR_ARG). Inputs and outputs are the caller's
 * device buffers; work is queued on `stream` (a cudaStream_t, NULL = legacy default).
 * Every call ends by copying the pivot status to the host and synchronising `stream`,
 * so it returns only after its kernels have finished. Every call on a device shares the
 * scratch array: calls whose kernels may overlap on the GPU race and must be
 * serialised by the caller. The first call on a device looks up the array's device
 * address with that device current; make that first call before any stream capture
 * begins on the device. The address is kept for the process's life: do
 * not use the library on a device after cudaDeviceReset. n = 0 is a no-op returning
 * HIF_OK. */
int hif_schur_device_noalloc(const double* dB, int n, int r, double* dA22inv, double* dX,
                             double* dS, void* stream);
/* InterpDecomp(M, W, skel, red, eps) -- src/InterpDecomp.cpp:86-138: column-pivoted
 * QR of M (m x n, m >= n; overwritten, R on and above the diagonal), skeleton =
 * {i : |R_ii| > eps |R_00|}, W = R11^{-1} R12 on the redundant columns. W holds
 * rank x (n - rank) (room for n*n/4 + n doubles); skeleton_cols / redundant_cols in
 * pivot order, 0-based. */
int hif_interp_decomp(double* M, int m, int n, long long ldm, double eps, double* W,
                      int* skeleton_cols, int* redundant_cols, int* rank);
/* PivotedQRWrapper(A, jpvt) -- src/InterpDecomp.cpp:198-211 (geqp3; jpvt 0-based). */
int hif_pivoted_qr(double* A, int m, int n, long long lda, int* jpvt);
/* TriangularSolveWrapper(R, B) -- src/InterpDecomp.cpp:213-231: B := R^{-1} B with R
 * upper triangular, non-unit (k x k), B k x nb. */
int hif_triangular_solve(const double* R, int k, long long ldr, double* B, int nb,
                         long long ldb);

/* ---- introspection (schur_level_data / skel_level_data, include/Factor.hpp:50-51,
 *      declared but not defined by the reference) --------------------------------- */
int hif_num_levels(hif_handle h, int* levels);
/* kind: 0 = Schur (cell interiors), 1 = skeletonization (faces). */
int hif_num_blocks(hif_handle h, int level, int kind, int* nblocks);
/* Sizes of block b: |global_inds|, |redundant_inds|, |skeleton_inds| and the face
 * (data.hpp enum, -1 for Schur blocks). */
int hif_block_info(hif_handle h, int level, int kind, int b, int* ng, int* nr, int* ns,
                   int* face);
/* Index data exactly as the reference's IndexData (include/data.hpp:11-62). */
int hif_block_indices(hif_handle h, int level, int kind, int b, int* global_inds,
                      int* redundant_inds, int* skeleton_inds);
/* which: 0 A_22, 1 A_22^{-1}, 2 X = A_22^{-1} A_21, 3 W (skeletonization only),
 * 4 Schur complement S (only with HIF_OPT_KEEP_SCHUR); for phases eliminated by
 * Cholesky (HIF_OPT_ELIMINATION) 0-2 are formed from the stored factors and
 * 5 L, 6 L^{-1}, 7 Y = L^{-1} A_21 are the stored ones. Column-major, rows / columns
 * ordered as redundant_inds / skeleton_inds. */
int hif_block_matrix(hif_handle h, int level, int kind, int b, int which, double* out);
/* Pivot order (0-based, n entries) and R diagonal of a skeletonized face's ID. */
int hif_block_pivots(hif_handle h, int level, int b, int* jpvt, double* rdiag);
/* For every DOF id p in [0, NC^3): the phase that eliminated it, 2 * level + kind
 * (kind 0 = Schur, 1 = skeletonization), or -1 for the index-0 planes. The union of
 * the redundant_inds of every block (UpdateRemainingDOFs, src/Factor.cpp:91-111);
 * used to state errors per level. */
int hif_dof_levels(hif_handle h, int* phase_of_dof);

enum hif_option {
  HIF_OPT_KEEP_SCHUR = 1,    /* keep every Schur complement for hif_block_matrix(which=4) */
  HIF_OPT_VERBOSE = 2,       /* 1: per-phase wall times on stderr (synchronising);
                                2: per-phase host and device times, no synchronisation */
  HIF_OPT_MEM_BUDGET_MB = 3, /* refuse factorizations whose device memory exceeds this */
  HIF_OPT_PROFILE = 4,       /* time every launch with CUDA events (resets the counters) */
  HIF_OPT_ID_GROUP_MIN_N = 5, /* faces with at least this many columns get a CTA group (default 512) */
  HIF_OPT_PRECISION = 6,      /* HIF_PRECISION_FP64 (default) or HIF_PRECISION_MIXED */
  HIF_OPT_AUTOTUNE = 7,       /* 1: tune online: the tile shape of the batched FP64
                                 products per batch signature, and in mixed precision on
                                 a symmetric operator (HIF_ELIM_AUTO) the elimination
                                 method per phase; each candidate runs once on the first
                                 factorizations, then the faster is kept; results may then
                                 differ in the last bits between those factorizations */
  HIF_OPT_SCHUR_SLICES = 8,   /* MIXED: int8 slices (2..8) of the Schur-complement products
                                 S = A11 - A12 X (default 5); 0: split TF32 */
  HIF_OPT_X_SLICES = 9,       /* MIXED, Gauss-Jordan elimination: int8 slices (2..8) of
                                 X = A22^{-1} A21 (default 7); 0: FP64 */
  HIF_OPT_ELIMINATION = 10,   /* enum hif_elimination (default HIF_ELIM_AUTO) */
  HIF_OPT_Y_SLICES = 11,      /* MIXED, Cholesky elimination: int8 slices (2..8) of
                                 Y = L^{-1} A21 (default 6); 0: FP64 */
  HIF_OPT_GRAM_MIN_N = 12,    /* MIXED: faces with more columns than this (and more rows
                                 than columns) take the Gram-matrix ID (default 32) */
  HIF_OPT_GRAM_SLICES = 13,   /* MIXED: the Gram matrices M^T M of that ID from int8 slices
                                 (2..8); 0 (default): FP64 products */
  HIF_OPT_CHOL_SLICES = 14    /* MIXED, Cholesky elimination: int8 slices (2..8) of the
                                 products forming L^{-1} (default 7); 0: FP64. The
                                 rank-128 updates of the pivot-block factorization stay
                                 FP64 (too short a k for the slices) */
};
/* Arithmetic of the factorization. MIXED: the long-K products of the eliminations
 * (S = A11 - A12 X, and X or Y) are FP64 products formed from exact int8 slice
 * products on the tcgen05 tensor cores (HIF_OPT_SCHUR_SLICES 0 selects split TF32 for
 * S); the interpolative decompositions of the large faces use the pivoted Cholesky of
 * M^T M (FP64) instead of the column-pivoted QR when epsilon >= 1e-7; the diagonal-block
 * factorization, the factor storage, the apply and the PCG residual stay FP64. */
enum hif_precision { HIF_PRECISION_FP64 = 0, HIF_PRECISION_MIXED = 1 };
/* Elimination of the redundant DOFs of each block.
 * GAUSS_JORDAN: explicit A22^{-1}, X = A22^{-1} A21, S = A11 - A12 X (the reference's
 *   Schur(): getrf + getri, include/Schur.hpp:72-100).
 * CHOLESKY (symmetric operators, hif_setup_stencil_faces): A22 = L L^T,
 *   Y = L^{-1} A21, S = A11 - Y^T Y; the factor keeps L, L^{-1} and Y. Same operator
 *   to rounding (X = L^{-T} Y, A22^{-1} = L^{-T} L^{-1}); hif_block_matrix still
 *   returns A22, A22^{-1} and X, formed from them.
 * AUTO: CHOLESKY for symmetric operators in MIXED precision, else GAUSS_JORDAN. */
enum hif_elimination { HIF_ELIM_AUTO = 0, HIF_ELIM_GAUSS_JORDAN = 1, HIF_ELIM_CHOLESKY = 2 };
int hif_set_option(hif_handle h, int option, long long value);

/* Test hook: prescribe the ID column order of every face of one level (replay of
 * another implementation's pivot decisions). offsets: nfaces+1 prefix offsets into
 * orders. Pass nfaces = 0 to clear. */
int hif_set_replay_pivots(hif_handle h, int level, int nfaces, const int* offsets,
                          const int* orders);

/* Timings of the last hif_factor in seconds: total, and per phase kind (gather,
 * elimination, ID, host partition). */
int hif_factor_stats(hif_handle h, double* total_s, double* gather_s, double* elim_s,
                     double* id_s, double* host_s, long long* device_bytes);

/* ---- host-only test hooks of the partitioner (no GPU needed) ---------------------
 * Index data over a caller-given remaining-DOF mask (NC^3 bytes, DOF order).
 * hif_partition_cell: InteriorCellIndexData (src/Factor.cpp:359-392); counts[3] =
 * {|global|, |red|, |skel|}. hif_partition_face: SkelInteractionIndexData
 * (src/Factor.cpp:645-755) for face TOP / LEFT / FRONT; rows[0], cols[0] hold the
 * counts, entries follow. Output arrays must hold NC^3 (+1) ints. reserved: 0. */
int hif_partition_cell(int N, int P, int level, int ci, int cj, int ck, int reserved,
                       const unsigned char* mask, int* global_inds, int* redundant_inds,
                       int* skeleton_inds, int* counts);
int hif_partition_face(int N, int P, int level, int ci, int cj, int ck, int face,
                       int reserved, const unsigned char* mask, int* rows, int* cols);

/* Kernel classes of hif_kernel_stats. */
enum hif_kernel_class {
  HIF_KCLASS_GATHER = 0,      /* block assembly from the stencil + Schur complement blocks */
  HIF_KCLASS_GEMM = 1,        /* batched FP64 GEMM (elimination updates, ID rotations) */
  HIF_KCLASS_SWEEP_SMALL = 2, /* whole-block elimination in shared memory */
  HIF_KCLASS_SWEEP_PANEL = 3, /* pivot-block inverse and panels of the blocked elimination */
  HIF_KCLASS_ID = 4,          /* pivoted-QR interpolative decomposition */
  HIF_KCLASS_GEMV = 5,        /* apply sweeps */
  HIF_KCLASS_COPY = 6,        /* compact copies of factor blocks */
  HIF_KCLASS_VECTOR = 7,      /* reductions / vector updates of the apply */
  HIF_KCLASS_QR = 8,          /* blocked Householder row compression of face blocks */
  HIF_KCLASS_GEMM_MIXED = 9,  /* split-TF32 tensor-core Schur-complement updates */
  HIF_KCLASS_GEMM_INT8 = 10,  /* FP64 products from int8 slices on the tensor cores (flops:
                                 the int8 operations of the slice products) */
  HIF_KCLASS_COUNT = 11
};
/* Accumulated launches, milliseconds (CUDA events on the handle's stream), algorithmic
 * flops and bytes of one kernel class since HIF_OPT_PROFILE was last set. */
int hif_kernel_stats(hif_handle h, int kclass, long long* launches, double* ms, double* flops,
                     double* bytes);

/* State of the HIF_OPT_AUTOTUNE tuner: batch signatures seen, signatures with a
 * decision, and how many of those chose the 128 x 128 tensor-core tile. */
int hif_autotune_stats(hif_handle h, int* signatures, int* decided, int* chose_128);
/* The tuner's per-phase elimination choices (mixed precision, symmetric operator,
 * HIF_ELIM_AUTO): phase signatures seen, decided, and how many chose Cholesky over
 * Gauss-Jordan. No reference counterpart. */
int hif_autotune_elimination(hif_handle h, int* signatures, int* decided, int* chose_cholesky);

/* Device memory held by the handle: the factor (kept until the next hif_factor or
 * hif_destroy) and the factorization workspace (kept for reuse by later
 * factorizations; hif_trim returns it to the device). */
int hif_memory(hif_handle h, long long* factor_bytes, long long* workspace_bytes);
int hif_trim(hif_handle h);
/* Temporaries freed by any handle stay reserved in the current device's default
 * memory pool for reuse (handles raise its release threshold); this returns the
 * unused part to the device. Synchronises the device. */
int hif_trim_device_pool(void);

/* Mixed-precision GEMM on device pointers, the kernel of the HIF_PRECISION_MIXED
 * Schur-complement updates: C = alpha op(A) op(B) + beta C (column-major; op(A) is
 * m x k, op(B) k x n) with each FP64 operand split into a TF32 pair and the products
 * hi*hi + hi*lo + lo*hi accumulated in FP32 on the tcgen05 tensor cores; relative
 * error of order 1e-6 of |A| |B|. No reference counterpart (the reference's products
 * are hmat_tools::Multiply dgemm calls, include/Schur.hpp:97-99). Runs on the calling thread's default
 * per-thread stream and returns after completion. */
int hif_gemm_mixed_device(int transA, int transB, int m, int n, int k, double alpha,
                          const double* dA, long long lda, const double* dB, long long ldb,
                          double beta, double* dC, long long ldc);

/* FP64 GEMM on device pointers from exact int8 products on the tcgen05 tensor cores
 * (Ozaki scheme): every row of op(A) and column of op(B) is scaled by a power of two
 * and cut into `slices` (2..8) signed 7-bit pieces; the slice products with
 * s + t < slices are accumulated exactly in int32 and summed in FP64. The error is
 * of order k 2^(-7 slices) max|row of op(A)| max|column of op(B)|; the result does
 * not depend on the order of the products. C = alpha op(A) op(B) + beta C,
 * column-major. No reference counterpart (the reference's products are
 * hmat_tools::Multiply dgemm calls, include/Schur.hpp:97-99). Runs on the calling
 * thread's default per-thread stream and returns after completion. */
int hif_gemm_int8_device(int transA, int transB, int m, int n, int k, double alpha,
                         const double* dA, long long lda, const double* dB, long long ldb,
                         double beta, double* dC, long long ldc, int slices);

/* ---- Serving: many operators resident on one GPU ------------------------------
 * No reference counterpart (the reference factors one operator per process,
 * tests/HIFDE3D/main.cpp). A server keeps factored operators in device memory and
 * runs requests from any host thread:
 *   - factor requests (face-coefficient operator, as hif_setup_stencil_faces) run on
 *     worker threads, each on its operator's own stream; one is admitted when its
 *     expected device footprint fits in budget_bytes beside the resident factors and
 *     the factorizations running; one whose expected footprint exceeds budget_bytes
 *     itself is refused with HIF_ERR_BUDGET (and so are the solves submitted for it);
 *   - solve requests (PCG preconditioned by the inverse apply, as hif_solve_pcg)
 *     are batched across operators at every iteration: up to max_active_solves run
 *     together, one launch per apply stage for all of them; requests join and
 *     leave between iterations. A request's result equals hif_solve_pcg's on the
 *     same operator and right-hand sides, bit for bit, whatever else runs with it.
 * Submitting returns a request id at once; hif_server_wait blocks until it ends.
 * x_out (NC^3 x nrhs, host) must stay valid until then. Operator ids are chosen by
 * the caller; a solve may be submitted while its operator is still being factored.
 * Destroy the server only after every request has been waited for. */
typedef struct hif_server_s* hif_server;
int hif_server_create(long long budget_bytes, int max_active_solves, int factor_workers,
                      hif_server* out);
int hif_server_destroy(hif_server s);
int hif_server_submit_factor(hif_server s, int op_id, int N, int P, double epsilon,
                             int partition, int precision, double hstep, const double* ax,
                             const double* ay, const double* az, const double* V,
                             long long* request_id);
int hif_server_submit_solve(hif_server s, int op_id, const double* b, int nrhs, double tol,
                            int maxit, double* x_out, long long* request_id);
/* status: HIF_OK or the request's error; iters / relres: the largest over its
 * right-hand sides; latency_ms: submit to completion. */
int hif_server_wait(hif_server s, long long request_id, int* status, int* iters,
                    double* relres, double* latency_ms);
/* hif_server_wait plus queue_ms: submit until the request was admitted (a factor
 * request by the memory budget and a free worker; a solve into the active set, which
 * needs its operator factored, a free slot and memory); latency_ms - queue_ms is the
 * time in service. */
int hif_server_wait_detail(hif_server s, long long request_id, int* status, int* iters,
                           double* relres, double* latency_ms, double* queue_ms);
/* Waits for the operator's solves in flight, then frees its factor. */
int hif_server_release(hif_server s, int op_id);
int hif_server_stats(hif_server s, long long* device_bytes, long long* resident_ops,
                     long long* completed, long long* iterations, long long* batched_launches);

/* Message of the last error on this thread. */
const char* hif_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* HIF_B200_H_ */
