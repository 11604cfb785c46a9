// Host engine of the B200 HIF factorization and the C ABI (include/hif_b200.h).
//
// Mirrors HIFFactor<double> of arbenson/HIFDE3D (include/Factor.hpp,
// src/Factor.cpp). The reference keeps the remaining operator in one global
// std::map sparse matrix, gathers every dense block from it and scatters every
// Schur complement back (UpdateMatrixAndDOFs, src/Factor.cpp:262-311). Here the
// remaining operator is never formed. It is the 7-point stencil (7 bands in
// HBM) plus the live dense Schur-complement blocks ("sources") of the previous
// phase; each phase assembles its dense blocks directly from those on the GPU:
//
//   after Schur(l):  operator = A0 + sum_c T_c, T_c on the face DOFs of cell c,
//                    T_c = (sources inherited by c)(skel, skel) + S_c;
//   skel(l):         face f between cells c (owner) and c': M and A_ff read
//                    A0, T_c and T_c'; S_f becomes a source;
//   Schur(l+1):      cell C reads A0 and the sources it owns (its 8 children's
//                    T_c and the S_f of faces owned by its children); the
//                    skeleton-skeleton part of what it read plus S_C is T_C.
//
// Every source is summed into exactly one later T, so the assembled blocks
// equal the reference's DenseSubmatrix of its updated sparse matrix. Only the
// partition and the small ID decisions cross PCIe; one host sync per phase.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdint>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <atomic>
#include <memory>
#include <string>
#include <exception>
#include <future>
#include <thread>
#include <vector>

#include "../../include/hif_b200.h"
#include "hif_kernels.cuh"
#include "hif_partition.hpp"

namespace hif {

thread_local std::string g_last_error;

struct Error {
  int code;
  std::string msg;
};

namespace {

#define HIF_CK(call)                                                                      \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      throw ::hif::Error{e_ == cudaErrorMemoryAllocation ? HIF_ERR_NOMEM : HIF_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_)};                    \
    }                                                                                     \
  } while (0)

double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Device allocation helpers on the engine stream (stream-ordered allocator).
template <class T>
T* dalloc(size_t count, cudaStream_t s) {
  if (count == 0) count = 1;
  void* p = nullptr;
  HIF_CK(cudaMallocAsync(&p, count * sizeof(T), s));
  return static_cast<T*>(p);
}

void dfree(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// Pinned host staging for the host -> device copies of a factorization. A copy
// from pageable memory may make the driver wait for the stream before staging
// it, which would stall the host behind the GPU at every descriptor upload;
// from pinned memory the copy is queued and the host goes on. The staging is
// bump-allocated in chunks kept for the owner's life and reused from the start
// once the owner has synchronised (its copies are then complete).
struct PinnedStage {
  struct Chunk {
    char* p;
    size_t size, used;
  };
  std::vector<Chunk> chunks;
  size_t cur = 0;
  static constexpr size_t kMinChunk = size_t(32) << 20;
  void* get(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    for (; cur < chunks.size(); ++cur) {
      Chunk& c = chunks[cur];
      if (c.size - c.used >= bytes) {
        void* r = c.p + c.used;
        c.used += bytes;
        return r;
      }
    }
    const size_t sz = std::max(bytes, kMinChunk);
    void* p = nullptr;
    HIF_CK(cudaHostAlloc(&p, sz, cudaHostAllocDefault));
    chunks.push_back(Chunk{static_cast<char*>(p), sz, bytes});
    cur = chunks.size() - 1;
    return p;
  }
  void reset() {
    for (Chunk& c : chunks) c.used = 0;
    cur = 0;
  }
  void release() {
    for (Chunk& c : chunks) cudaFreeHost(c.p);
    chunks.clear();
    cur = 0;
  }
  ~PinnedStage() { release(); }
};
// Staging used by upload() on this thread (set while a factorization runs).
thread_local PinnedStage* t_stage = nullptr;

struct Arena;
// Arena for the large temporaries of gemm_batch on this thread (the engine's
// current level workspace while a factorization runs), else the pool.
thread_local Arena* t_scratch = nullptr;

void copy_to_device(void* d, const void* h, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (t_stage) {
    void* p = t_stage->get(bytes);
    std::memcpy(p, h, bytes);
    HIF_CK(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, s));
  } else {
    HIF_CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
  }
}

template <class T>
T* desc_alloc(size_t count, cudaStream_t s);

template <class T>
T* upload(const std::vector<T>& v, cudaStream_t s) {
  T* d = desc_alloc<T>(v.size(), s);
  copy_to_device(d, v.data(), v.size() * sizeof(T), s);
  return d;
}

// A caller's host array copied straight to a new stream-ordered device buffer
// (freed with dfree): no intermediate host copy. The runtime stages a pageable
// source itself, so the array may be reused once the copy call has returned.
template <class T>
T* upload_host(const T* src, long long count, cudaStream_t s) {
  T* d = dalloc<T>((size_t)count, s);
  if (count > 0)
    HIF_CK(cudaMemcpyAsync(d, src, (size_t)count * sizeof(T), cudaMemcpyHostToDevice, s));
  return d;
}

// Host worker pool for parallel_for, started on first use and kept for the
// process (several host threads run parallel loops at once: a factorization's
// partition threads, the serving loop's factor workers). A loop is a job on
// its caller's stack; idle workers take 64-index chunks of any open job, the
// caller takes chunks too, and it returns once every chunk has run and no
// worker holds the job. Workers are created once, not per loop: the lower
// levels run dozens of loops per factorization.
class HostPool {
 public:
  struct Job {
    const std::function<void(int)>* f;
    int n;
    std::atomic<int> next{0};
    int holders = 0;  // workers inside the job (guarded by mu_)
  };
  static HostPool& get() {
    static HostPool* p = new HostPool;  // never destroyed: workers live for the process
    return *p;
  }
  int workers() const { return (int)workers_.size(); }
  void run(Job& job) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      jobs_.push_back(&job);
    }
    cv_.notify_all();
    work(job);
    std::unique_lock<std::mutex> lk(mu_);
    jobs_.erase(std::find(jobs_.begin(), jobs_.end(), &job));
    done_cv_.wait(lk, [&] { return job.holders == 0; });
  }

 private:
  HostPool() {
    const int nt = std::min<int>(std::max(1u, std::thread::hardware_concurrency()), 32) - 1;
    for (int t = 0; t < nt; ++t) workers_.emplace_back([this] { loop(); });
  }
  static void work(Job& j) {
    for (;;) {
      const int i0 = j.next.fetch_add(64);
      if (i0 >= j.n) break;
      const int i1 = std::min(j.n, i0 + 64);
      for (int i = i0; i < i1; ++i) (*j.f)(i);
    }
  }
  // the open job with the fewest workers: concurrent loops (a partition thread's
  // long one, the factorization thread's short ones) share the pool instead of
  // the first one taking every worker
  Job* open_job() {
    Job* best = nullptr;
    for (Job* j : jobs_)
      if (j->next.load() < j->n && (!best || j->holders < best->holders)) best = j;
    return best;
  }
  void loop() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      // the job found by the wait is the one taken: `next` moves without the
      // lock, so a second search could find none
      Job* j = nullptr;
      cv_.wait(lk, [&] { return (j = open_job()) != nullptr; });
      ++j->holders;
      lk.unlock();
      work(*j);
      lk.lock();
      if (--j->holders == 0) done_cv_.notify_all();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::vector<Job*> jobs_;
  std::vector<std::thread> workers_;
};

// Host parallel loop over [0, n) in chunks (partitioning of cells / faces).
template <class F>
void parallel_for(int n, F&& f) {
  if (n < 256) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  HostPool& pool = HostPool::get();
  if (pool.workers() == 0) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  const std::function<void(int)> fn = [&](int i) { f(i); };
  HostPool::Job job;
  job.f = &fn;
  job.n = n;
  pool.run(job);
}

// Keeps device buffers of one phase alive until released together.
struct Arena;
// Device memory for the small uploads of a factorization (descriptor arrays,
// index lists): bump-allocated from chunks kept for the handle's life and
// given back all at once when the next factorization starts, instead of one
// stream-ordered allocation and free per upload (several driver calls per
// launch, which set the pace of the many short launches of the lower levels).
thread_local Arena* t_desc = nullptr;
bool desc_owned(const void* x);

struct BufList {
  std::vector<void*> p;
  template <class T>
  T* add(T* x) {
    if (!desc_owned(x)) p.push_back(x);
    return x;
  }
  void release(cudaStream_t s) {
    for (void* x : p) dfree(x, s);
    p.clear();
  }
};

// Device memory for the factorization's big buffers: chunks obtained from
// cudaMalloc once and kept for the life of the handle, bump-allocated, and
// made free again by reset(). All users are on one stream, so a reset followed
// by new allocations is ordered after the previous users' kernels. Successive
// factorizations of one size request the same sequence, so after the first the
// chunks are reused as they are and no allocator call is made.
struct Arena {
  struct Chunk {
    char* p;
    size_t size, used;
  };
  std::vector<Chunk> chunks;
  size_t cur = 0;
  double grow_s = 0;  // host time spent in cudaMalloc for new chunks
  static constexpr size_t kMinChunk = size_t(256) << 20;

  template <class T>
  T* alloc(size_t count) {
    size_t bytes = (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~size_t(255);
    for (; cur < chunks.size(); ++cur) {
      Chunk& c = chunks[cur];
      if (c.size - c.used >= bytes) {
        void* r = c.p + c.used;
        c.used += bytes;
        return static_cast<T*>(r);
      }
    }
    const size_t sz = std::max(bytes, kMinChunk);
    void* p = nullptr;
    const double t0 = wall();
    HIF_CK(cudaMalloc(&p, sz));
    grow_s += wall() - t0;
    chunks.push_back(Chunk{static_cast<char*>(p), sz, bytes});
    cur = chunks.size() - 1;
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& v, cudaStream_t s) {
    T* d = alloc<T>(v.size());
    copy_to_device(d, v.data(), v.size() * sizeof(T), s);
    return d;
  }
  void reset() {
    size_t u = 0;
    for (Chunk& c : chunks) {
      u += c.used;
      c.used = 0;
    }
    hw_cycle = std::max(hw_cycle, u);
    cur = 0;
  }
  // Chunks are sized by the requests that first outgrew them, so a handle whose
  // block sizes change (another precision, a refactorization with other
  // skeleton ranks) can end with chunks none of which fits a later request.
  // At a point where nothing on the device uses the arena, consolidate():
  // when it holds several chunks, they are replaced by one of the largest
  // total the arena was asked for in a cycle since the last consolidation.
  size_t hw_cycle = 0;
  void consolidate() {
    size_t u = 0;
    for (const Chunk& c : chunks) u += c.used;
    hw_cycle = std::max(hw_cycle, u);
    if (chunks.size() > 1 && hw_cycle > 0) {
      release();
      const size_t sz = ((hw_cycle + hw_cycle / 16) + 255) & ~size_t(255);
      void* p = nullptr;
      const double t0 = wall();
      if (cudaMalloc(&p, sz) == cudaSuccess) {
        chunks.push_back(Chunk{static_cast<char*>(p), sz, 0});
      } else {
        cudaGetLastError();  // leave it empty: alloc() grows it on demand
      }
      grow_s += wall() - t0;
    }
    for (Chunk& c : chunks) c.used = 0;
    cur = 0;
    hw_cycle = 0;
  }
  // Stack discipline for temporaries: everything allocated after mark() is
  // given back by rewind(). Users are on one stream, so memory handed out
  // again after a rewind is written only by work ordered after the old users.
  struct Mark {
    size_t cur, used;
  };
  Mark mark() const { return Mark{cur, chunks.empty() ? 0 : chunks[cur].used}; }
  void rewind(const Mark& m) {
    for (size_t q = m.cur + 1; q < chunks.size(); ++q) chunks[q].used = 0;
    if (!chunks.empty()) chunks[m.cur].used = m.used;
    cur = m.cur;
  }
  size_t reserved() const {
    size_t t = 0;
    for (const Chunk& c : chunks) t += c.size;
    return t;
  }
  bool owns(const void* x) const {
    const char* q = static_cast<const char*>(x);
    for (const Chunk& c : chunks)
      if (q >= c.p && q < c.p + c.size) return true;
    return false;
  }
  void release() {
    for (Chunk& c : chunks) cudaFree(c.p);
    chunks.clear();
    cur = 0;
  }
};

bool desc_owned(const void* x) { return t_desc != nullptr && t_desc->owns(x); }

template <class T>
T* desc_alloc(size_t count, cudaStream_t s) {
  return t_desc ? t_desc->alloc<T>(count) : dalloc<T>(count, s);
}

}  // namespace

// ---------------------------------------------------------------------------
// Factor data of one block (FactorData, include/data.hpp:84-110)
// ---------------------------------------------------------------------------
struct BlockInfo {
  std::vector<int> global;    // global_inds (reference order)
  std::vector<int> red_pos;   // redundant_inds
  std::vector<int> skel_pos;  // skeleton_inds
  int face = -1;
  int cell = -1;  // cell index (ci * cpd + cj) * cpd + ck
  int nbr = -1;   // skeletonization: neighbour cell index
  int r() const { return (int)red_pos.size(); }
  int s() const { return (int)skel_pos.size(); }
  std::vector<int> jpvt;  // skeletonization: pivot order over global
  std::vector<double> rdiag;
  std::vector<double> S;  // kept Schur complement (option)
};

struct StepData {
  int level = 0;
  bool skel = false;
  // elimination by Cholesky: the A22 / A22^{-1} / X slots hold L, L^{-1} and
  // Y = L^{-1} A21 instead (see chol_blocks)
  bool chol = false;
  int cpd = 0;
  std::vector<BlockInfo> blocks;
  double* arena = nullptr;  // A22 | A22inv | X | W per block
  std::vector<long long> o_a22, o_inv, o_x, o_w;
  int* d_red = nullptr;
  int* d_skel = nullptr;
  std::vector<long long> o_red, o_skel;
  long long n_red = 0, n_skel = 0;
};

// One launch of the apply sweep.
struct ApplyLaunch {
  double bytes = 0;  // matrix bytes streamed per right-hand-side group
  long long key = 0;  // stage order shared by all operators (batched solves)
  std::vector<GemvDesc> hdesc;  // host copy of the descriptors
  int type = 0;  // 0 gemv, 1 reduce-scatter
  GemvDesc* d_desc = nullptr;
  int nd = 0;
  int in_vec = 0, out_vec = 0;  // 0 = ua, 1 = ub, 2 = uc (Cholesky phases' L^{-1} u_r)
  // GEMV layout (launch_gemv_fast) and its unit table; the serving loop binds
  // the descriptors to a request's vectors and reuses the table
  int layout = 0;
  int2* d_tab = nullptr;
  int units = 0;
  GemvFastSeg* d_seg = nullptr;  // one segment: this launch's descriptors and table
  int* d_segoff = nullptr;
  int* d_dof = nullptr;
  int* d_off = nullptr;
  int* d_slot = nullptr;
  int ndof = 0;
  double alpha = 0.0;
};

struct ApplyPlan {
  std::vector<ApplyLaunch> launches;
  BufList bufs;
  long long contrib_slots = 0;
};

// Live Schur complement blocks feeding the next phase.
struct Sources {
  std::vector<SourceDesc> desc;
  std::vector<int> owner;      // target cell (next Schur phase) that sums this source
  // the 6 x NC^3 membership arrays (see GatherTarget) live on the device,
  // in Engine::d_dof_src, one set at a time
  std::vector<int> cell_src;   // cell index -> source id (T_c), -1 if none
  BufList bufs;                // device memory holding the blocks
};

// One batched GEMM launch; 128x128 tiles when most of the work sits in
// problems at least that large (or when forced: in-place panel products rely on
// a single output tile along the aliased dimension), else 64x64. Problems with
// a reduction much longer than their output dimensions are split along k into
// partial products and summed in a fixed order.
// Online tile-shape tuner for the batched FP64 products (HIF_OPT_AUTOTUNE).
// A batch is keyed by its class and the log2 buckets of its work and mean
// shape; until both candidate tiles (64 x 64 FFMA, 128 x 128 DMMA) have run
// once for a key, the next untried one runs with events around it; after that
// the faster is kept. Events are read when the factorization synchronises.
struct GemmTuner {
  struct Rec {
    double ms[2] = {0.0, 0.0};
    int runs[2] = {0, 0};
    int choice = -1;
  };
  struct Pending {
    long long key;
    int cand;
    cudaEvent_t a, b;
  };
  std::map<long long, Rec> recs;
  std::vector<Pending> pending;
  static constexpr int kTiles[2] = {64, 128};
  ~GemmTuner() {
    for (Pending& p : pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
  }
  void resolve() {
    for (Pending& p : pending) {
      float ms = 0;
      if (cudaEventSynchronize(p.b) == cudaSuccess &&
          cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
        Rec& r = recs[p.key];
        r.ms[p.cand] += ms;
        r.runs[p.cand] += 1;
        if (r.runs[0] > 0 && r.runs[1] > 0)
          r.choice = (r.ms[0] / r.runs[0] <= r.ms[1] / r.runs[1]) ? 0 : 1;
      }
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    pending.clear();
  }
};
thread_local GemmTuner* t_tuner = nullptr;

int ilog2_bucket(double x) {
  int b = 0;
  while (x >= 2.0 && b < 62) {
    x *= 0.5;
    ++b;
  }
  return b;
}

// Temporaries of one call: from t_scratch (given back when the scope ends) or
// from the pool (released with tmp).
struct ScratchScope {
  Arena* a;
  Arena::Mark m{};
  ScratchScope() : a(t_scratch) {
    if (a) m = a->mark();
  }
  ~ScratchScope() {
    if (a) a->rewind(m);
  }
};
template <class T>
T* scratch_alloc(size_t count, BufList& tmp, cudaStream_t s) {
  return t_scratch ? t_scratch->alloc<T>(count) : tmp.add(dalloc<T>(count, s));
}

template <class Timed>
void gemm_batch(const std::vector<GemmDesc>& gin, BufList& tmp, cudaStream_t stream, int cls,
                Timed&& timed, int force_tile = 0, int* mixed_status = nullptr) {
  if (gin.empty()) return;
  ScratchScope scope;
  if (mixed_status) {  // split-TF32 tensor-core path (Schur-complement updates)
    double fl = 0;
    long long tiles = 0;
    for (const GemmDesc& x : gin) {
      if (x.m <= 0 || x.n <= 0) continue;
      const long long kt = (x.k + 31) / 32;
      tiles += ((x.m + 127) / 128 + (x.n + 127) / 128) * kt;
    }
    unsigned char* cbuf =
        scratch_alloc<unsigned char>(std::max(1LL, tiles) * kTcTileBytes, tmp, stream);
    std::vector<TcOperand> ops;
    std::vector<int> ooff(1, 0);
    std::vector<TcGemm> tg;
    std::vector<int> toff(1, 0);
    long long used = 0;
    for (const GemmDesc& x : gin) {
      if (x.m <= 0 || x.n <= 0) continue;
      fl += 2.0 * x.m * x.n * x.k;
      const int kt = (x.k + 31) / 32;
      const int ta = (x.m + 127) / 128 * kt, tb = (x.n + 127) / 128 * kt;
      unsigned char* pa = cbuf + used * kTcTileBytes;
      unsigned char* pb = cbuf + (used + ta) * kTcTileBytes;
      used += ta + tb;
      // A: element (i, kk) = op(A)[i, kk]; B: element (j, kk) = op(B)[kk, j]
      ops.push_back(TcOperand{x.A, x.lda, x.transA, x.m, x.k, pa});
      ooff.push_back(ooff.back() + ta);
      ops.push_back(TcOperand{x.B, x.ldb, x.transB ? 0 : 1, x.n, x.k, pb});
      ooff.push_back(ooff.back() + tb);
      tg.push_back(TcGemm{pa, pb, x.C, x.ldc, x.m, x.n, x.k, x.alpha, x.beta, x.lower});
      toff.push_back(toff.back() + (x.m + 127) / 128 * ((x.n + 127) / 128));
    }
    if (toff.back() == 0) return;
    TcOperand* dops = tmp.add(upload(ops, stream));
    int* doo = tmp.add(upload(ooff, stream));
    TcGemm* dg = tmp.add(upload(tg, stream));
    int* dt = tmp.add(upload(toff, stream));
    timed(HIF_KCLASS_GEMM_MIXED, fl, 0.0, [&] {
      launch_tc_convert(dops, doo, (int)ops.size(), ooff.back(), stream);
      launch_gemm_tc(dg, dt, (int)tg.size(), toff.back(), mixed_status, stream);
    }, 2);
    HIF_CK(cudaGetLastError());
    return;
  }
  std::vector<GemmDesc> g;
  std::vector<SplitKDesc> red;
  double fl = 0;
  long long psz = 0;
  struct Split {
    size_t idx;
    int S;
  };
  std::vector<Split> splits;
  for (size_t q = 0; q < gin.size(); ++q) {
    const GemmDesc& x = gin[q];
    fl += (x.a_lower || x.b_lower) ? 1.0 * x.m * x.n * (x.k + 1) : 2.0 * x.m * x.n * x.k;
    const int big = std::max(x.m, x.n);
    if (force_tile == 0 && !x.lower && !x.a_lower && !x.b_lower && x.k >= 2048 &&
        x.k >= 8 * big) {
      const int S = std::min(32, (x.k + 1023) / 1024);
      splits.push_back(Split{q, S});
      psz += (long long)S * x.m * x.n;
    } else {
      g.push_back(x);
    }
  }
  double* P = psz ? scratch_alloc<double>(psz, tmp, stream) : nullptr;
  long long po = 0;
  for (const Split& sp : splits) {
    const GemmDesc& x = gin[sp.idx];
    const int chunk = (x.k + sp.S - 1) / sp.S;
    for (int q = 0; q < sp.S; ++q) {
      const int k0 = q * chunk, kk = std::min(chunk, x.k - k0);
      GemmDesc y = x;
      y.C = P + po + (long long)q * x.m * x.n;
      y.ldc = x.m;
      y.k = std::max(kk, 0);
      y.A = x.transA == 0 ? x.A + (long long)k0 * x.lda : x.A + k0;
      y.B = x.transB == 0 ? x.B + k0 : x.B + (long long)k0 * x.ldb;
      y.alpha = 1.0;
      y.beta = 0.0;
      g.push_back(y);
    }
    red.push_back(SplitKDesc{x.C, P + po, x.ldc, x.m, x.n, sp.S, x.alpha, x.beta});
    po += (long long)sp.S * x.m * x.n;
  }
  double big = 0, all = 0;
  for (const GemmDesc& x : g) {
    const double w = (double)x.m * x.n;
    all += w;
    if (x.m >= 96 && x.n >= 96) big += w;
  }
  bool lower = false;  // lower-triangle products are tiled by 128 x 128
  for (const GemmDesc& x : g) lower = lower || x.lower;
  int tile = force_tile ? force_tile : ((lower || big >= 0.5 * all) ? 128 : 64);
  GemmTuner::Pending tp{0, -1, nullptr, nullptr};
  if (t_tuner && !force_tile && !lower && !g.empty()) {
    double sm = 0, sn = 0, sk = 0;
    for (const GemmDesc& x : g) {
      sm += x.m;
      sn += x.n;
      sk += x.k;
    }
    const double cnt = (double)g.size();
    const long long key = ((long long)cls << 40) | ((long long)ilog2_bucket(fl) << 30) |
                          ((long long)ilog2_bucket(sm / cnt) << 20) |
                          ((long long)ilog2_bucket(sn / cnt) << 10) | ilog2_bucket(sk / cnt);
    GemmTuner::Rec& r = t_tuner->recs[key];
    if (r.choice >= 0) {
      tile = GemmTuner::kTiles[r.choice];
    } else {
      const int cand = r.runs[0] == 0 ? 0 : 1;
      tile = GemmTuner::kTiles[cand];
      tp.key = key;
      tp.cand = cand;
    }
  }
  std::vector<int> toff(1, 0);
  for (const GemmDesc& x : g) toff.push_back(toff.back() + dgemm_tiles(x.m, x.n, tile));
  if (toff.back() == 0 && red.empty()) return;
  GemmDesc* dg = tmp.add(upload(g, stream));
  int* dt = tmp.add(upload(toff, stream));
  if (tp.cand >= 0) {
    HIF_CK(cudaEventCreate(&tp.a));
    HIF_CK(cudaEventCreate(&tp.b));
    HIF_CK(cudaEventRecord(tp.a, stream));
  }
  timed(cls, fl, 0.0, [&] { launch_dgemm(dg, dt, (int)g.size(), toff.back(), stream, tile); }, 1);
  if (tp.cand >= 0) {
    HIF_CK(cudaEventRecord(tp.b, stream));
    t_tuner->pending.push_back(tp);
  }
  if (!red.empty()) {
    SplitKDesc* dr = tmp.add(upload(red, stream));
    timed(cls, 0.0, 0.0, [&] { launch_splitk_reduce(dr, (int)red.size(), stream); }, 1);
  }
  HIF_CK(cudaGetLastError());
}

// FP64 products of a batch from int8 slices (Ozaki scheme, `slices` pieces per
// operand value): the operands are converted once, then products whose k
// exceeds kOzMaxK run as consecutive launches over k ranges (beta = 1 after
// the first), which keeps every diagonal sum exact in int32.
template <class Timed>
void gemm_batch_int8(const std::vector<GemmDesc>& gin, BufList& tmp, cudaStream_t stream,
                     Timed&& timed, int slices, int* status) {
  if (gin.empty()) return;
  ScratchScope scope;
  const int bn = oz_tile_n(slices);
  constexpr int kChunkTiles = kOzMaxK / kOzK;
  // op(B)^T = op(A) (S = A11 - Y^T Y, and the Cholesky updates P P^T): B's
  // converted rows are A's
  auto same_operand = [](const GemmDesc& x) {
    return x.A == x.B && x.lda == x.ldb && x.m == x.n &&
           ((x.transA == 1 && x.transB == 0) || (x.transA == 0 && x.transB == 1));
  };
  long long parts = 0, nexp = 0;
  for (const GemmDesc& x : gin) {
    if (x.m <= 0 || x.n <= 0) continue;
    const long long kt = (x.k + kOzK - 1) / kOzK;
    const bool same = same_operand(x);
    parts += ((x.m + 127) / 128 + (same ? 0 : (x.n + 127) / 128)) * kt * slices;
    nexp += x.m + (same ? 0 : x.n);
  }
  if (nexp == 0) return;
  signed char* cbuf = scratch_alloc<signed char>(std::max(1LL, parts) * kOzPart, tmp, stream);
  int* ebuf = scratch_alloc<int>(nexp, tmp, stream);
  std::vector<OzOperand> ops;
  std::vector<int> ooff(1, 0);
  std::vector<std::vector<OzGemm>> launches;
  long long used = 0, eo = 0;
  double fl = 0;
  // work counted as the tensor cores' int8 operations: slices (slices + 1) / 2
  // products of the padded tile shape, for the tiles computed
  const double pairs = 0.5 * slices * (slices + 1);
  for (const GemmDesc& x : gin) {
    if (x.m <= 0 || x.n <= 0) continue;
    const int kt = (x.k + kOzK - 1) / kOzK;
    {
      const int tm = (x.m + 127) / 128, tn = (x.n + bn - 1) / bn;
      // k tiles run, over the tiles computed
      double tk = 0;
      for (int i = 0; i < tm; ++i) {
        const int cols = x.lower ? std::min(tn, (i * 128 + 128 + bn - 1) / bn) : tn;
        const int kti = x.a_lower ? std::min(kt, (i * 128 + 128 + kOzK - 1) / kOzK) : kt;
        if (x.b_lower)
          for (int j = 0; j < cols; ++j) tk += std::max(0, kti - j * bn / kOzK);
        else
          tk += (double)cols * kti;
      }
      fl += pairs * 2.0 * 128.0 * bn * kOzK * tk;
    }
    const bool same = same_operand(x);
    const int ta = (x.m + 127) / 128 * kt, tb = same ? 0 : (x.n + 127) / 128 * kt;
    signed char* pa = cbuf + used * kOzPart;
    signed char* pb = same ? pa : cbuf + (used + (long long)ta * slices) * kOzPart;
    used += (long long)(ta + tb) * slices;
    int* ea = ebuf + eo;
    int* eb = same ? ea : ea + x.m;
    eo += x.m + (same ? 0 : x.n);
    if (kt > 0) {
      // A: element (i, kk) = op(A)[i, kk]; B: element (j, kk) = op(B)[kk, j]
      ops.push_back(OzOperand{x.A, x.lda, x.transA, x.m, x.k, pa, ea});
      ooff.push_back(ooff.back() + ta);
      if (!same) {
        ops.push_back(OzOperand{x.B, x.ldb, x.transB ? 0 : 1, x.n, x.k, pb, eb});
        ooff.push_back(ooff.back() + tb);
      }
    }
    for (int c = 0, kt0 = 0; kt0 < kt || c == 0; ++c, kt0 += kChunkTiles) {
      if ((int)launches.size() <= c) launches.emplace_back();
      launches[c].push_back(OzGemm{pa, pb, ea, eb, x.C, x.ldc, x.m, x.n, kt, kt0,
                                   std::min(kChunkTiles, std::max(0, kt - kt0)), x.alpha,
                                   c == 0 ? x.beta : 1.0, x.lower, x.a_lower, x.b_lower});
    }
  }
  timed(HIF_KCLASS_GEMM_INT8, fl, 0.0, [&] {
    if (!ops.empty()) {
      OzOperand* dops = tmp.add(upload(ops, stream));
      int* doo = tmp.add(upload(ooff, stream));
      launch_oz_convert(dops, doo, (int)ops.size(), ooff.back(), slices, ebuf, nexp, stream);
    } else {
      HIF_CK(cudaMemsetAsync(ebuf, 0x80, (size_t)nexp * sizeof(int), stream));
    }
    for (const std::vector<OzGemm>& lg : launches) {
      std::vector<int> toff(1, 0);
      for (const OzGemm& y : lg)
        toff.push_back(toff.back() + (y.m + 127) / 128 * ((y.n + bn - 1) / bn));
      OzGemm* dg = tmp.add(upload(lg, stream));
      int* dt = tmp.add(upload(toff, stream));
      launch_gemm_oz(dg, dt, (int)lg.size(), toff.back(), slices, status, stream);
    }
  }, (int)launches.size() + (ops.empty() ? 0 : 2));
  HIF_CK(cudaGetLastError());
}

// Dense elimination of a batch of blocks: descs[b].B holds [A22 A21; A12 A11]
// (ld n); on return the compact A22^{-1}, X are written and B's trailing block
// holds A11 - A12 X. Blocks up to kSmallSweepN are eliminated whole in shared
// memory; larger ones by 64-wide pivot blocks with batched GEMM updates.
// `timed(kernel class, flops, bytes, launch, launches)` wraps every launch.
// Arithmetic of the products of an elimination. schur: S = A11 - A12 X in FP64
// (-1), split TF32 (0) or from `schur` int8 slices; x: X = A22^{-1} A21 in FP64
// (0) or from `x` int8 slices. The Gauss-Jordan updates of A22^{-1} are rank-128
// products, bound by the traffic of their target rather than by arithmetic, and
// stay FP64.
// chol: in the Cholesky elimination, the products forming L^{-1} (long k) in
// FP64 (0) or from `chol` int8 slices; the pivot-block updates stay FP64.
struct ElimArith {
  int schur = -1;
  int x = 0;
  int chol = 0;
};

// Cholesky elimination of a batch of symmetric positive definite interiors
// (lower triangles only): writes L (descs[b].L), L^{-1} (a22inv) and
// Y = L^{-1} A21 (X); B's trailing block ends as A11 - Y^T Y, mirrored.
//   small blocks: k_chol_small, whole in shared memory;
//   large blocks: right-looking over 128-pivot blocks of A22 only:
//     L_KK = chol(B[K, K]) and L_KK^{-1} (k_chol_diag),
//     panel  B[K1:r, K] = B[K1:r, K] L_KK^{-T},
//     update B[K1:r, K1:r] -= panel panel^T (lower tiles),
//     L_KK^{-1} into the diagonal block K of L^{-1};
//   then the rest of L^{-1} by a halving of the 128-blocks (X21 = -X22 L21 X11,
//   bottom up, every node of a depth in two batched products),
//   then Y = L^{-1} A21 and S = A11 - Y^T Y as long-K products (FP64, or from
//   int8 slices in mixed precision: ar.x slices for Y, ar.schur for S).
// 2r^3/3 + 2r^2 s + r s^2 flops against the Gauss-Jordan path's
// r^3 + 2r^2 s + r s^2 (symmetric), with Y's product entries bounded by
// about sqrt(cond(A22)) times A21's rather than cond(A22) times.
template <class Timed>
void chol_blocks(const std::vector<SweepDesc>& descs, BufList& tmp, cudaStream_t stream,
                 int* d_status, Timed&& timed, ElimArith ar, Arena* scratch) {
  auto big = [&](size_t count) -> double* {
    return scratch ? scratch->alloc<double>(count) : tmp.add(dalloc<double>(count, stream));
  };
  std::vector<SweepDesc> small, large;
  int max_small = 0;
  for (const SweepDesc& d : descs) {
    if (d.r <= 0) continue;
    if (d.n <= kSmallSweepN) {
      small.push_back(d);
      max_small = std::max(max_small, d.n);
    } else {
      large.push_back(d);
    }
  }
  if (!small.empty()) {
    SweepDesc* dd = tmp.add(upload(small, stream));
    double fl = 0, by = 0;
    for (const SweepDesc& d : small) {
      const double r = d.r, sk = d.n - d.r;
      fl += 2.0 / 3.0 * r * r * r + 2 * r * r * sk + 2 * r * sk * sk;
      by += 8.0 * d.n * d.n + 8.0 * (2 * r * r + r * sk + sk * sk);
    }
    timed(HIF_KCLASS_SWEEP_SMALL, fl, by, [&] {
      launch_chol_small(dd, (int)small.size(), max_small, d_status, stream);
    });
    HIF_CK(cudaGetLastError());
  }
  if (large.empty()) return;
  const int nl = (int)large.size();
  SweepDesc* dd = tmp.add(upload(large, stream));
  double* dinv = big((size_t)nl * kSweepNB * kSweepNB);
  int maxr = 0;
  std::vector<long long> oq(nl);
  long long qsz = 0;
  for (int b = 0; b < nl; ++b) {
    maxr = std::max(maxr, large[b].r);
    oq[b] = qsz;
    qsz += (long long)large[b].r * kSweepNB;
  }
  double* Qb = big(qsz);  // per block: old panel (r x 128, ld r)
  // L and L^{-1} read as zero above their diagonals
  {
    std::vector<GemmDesc> z;
    for (const SweepDesc& d : large)
      for (double* C : {d.L, d.a22inv}) {
        GemmDesc g{};
        g.C = C;
        g.A = g.B = C;
        g.ldc = g.lda = g.ldb = d.r;
        g.m = g.n = d.r;
        g.k = 0;
        z.push_back(g);
      }
    gemm_batch(z, tmp, stream, HIF_KCLASS_COPY, timed);
  }
  for (int k0 = 0; k0 < maxr; k0 += kSweepNB) {
    std::vector<int> active;
    std::vector<CopyDesc> cq, cdg;
    std::vector<int> ocq(1, 0), ocd(1, 0);
    std::vector<GemmDesc> gp, gu;
    for (int b = 0; b < nl; ++b) {
      const SweepDesc& d = large[b];
      if (d.r <= k0) continue;
      active.push_back(b);
      const int r = d.r, k1 = std::min(r, k0 + kSweepNB), nbk = k1 - k0;
      const double* Dv = dinv + (long long)b * kSweepNB * kSweepNB;  // nbk x nbk, ld nbk
      double* Q = Qb + oq[b];
      double* P = d.B + k1 + (long long)k0 * d.n;  // panel rows k1..r of column block K
      if (r > k1) {
        cq.push_back(CopyDesc{P, Q, d.n, r, r - k1, nbk});
        ocq.push_back(ocq.back() + copy_tiles(r - k1, nbk));
        GemmDesc g{};
        g.C = P;
        g.ldc = d.n;
        g.A = Q;
        g.lda = r;
        g.B = Dv;
        g.ldb = nbk;
        g.transB = 1;
        g.m = r - k1;
        g.n = nbk;
        g.k = nbk;
        g.alpha = 1.0;
        gp.push_back(g);
        GemmDesc u{};
        u.C = d.B + k1 + (long long)k1 * d.n;
        u.ldc = d.n;
        u.A = P;
        u.lda = d.n;
        u.B = P;
        u.ldb = d.n;
        u.transB = 1;
        u.m = u.n = r - k1;
        u.k = nbk;
        u.alpha = -1.0;
        u.beta = 1.0;
        u.lower = 1;
        gu.push_back(u);
      }
      cdg.push_back(CopyDesc{Dv, d.a22inv + k0 + (long long)k0 * r, nbk, r, nbk, nbk});
      ocd.push_back(ocd.back() + copy_tiles(nbk, nbk));
    }
    BufList step;
    int* dact = step.add(upload(active, stream));
    timed(HIF_KCLASS_SWEEP_PANEL, 0, 0, [&] {
      launch_chol_diag(dd, dact, (int)active.size(), k0, dinv, d_status, stream);
    });
    if (!cq.empty()) {
      CopyDesc* dq = step.add(upload(cq, stream));
      int* doq = step.add(upload(ocq, stream));
      timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(dq, doq, (int)cq.size(), ocq.back(), stream); });
    }
    gemm_batch(gp, step, stream, HIF_KCLASS_SWEEP_PANEL, timed);
    // rank-128 updates: FP64 (from int8 slices they are bound by their C traffic)
    gemm_batch(gu, step, stream, HIF_KCLASS_GEMM, timed, 128);
    {
      CopyDesc* dc = step.add(upload(cdg, stream));
      int* doc = step.add(upload(ocd, stream));
      timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(dc, doc, (int)cdg.size(), ocd.back(), stream); });
    }
    HIF_CK(cudaGetLastError());
    step.release(stream);
  }
  // L: the block-lower column strips of B[0:r, 0:r] (its diagonal tiles already
  // hold zeros above the diagonal; the tiles above them still hold A22)
  {
    std::vector<CopyDesc> cl;
    std::vector<int> ocl(1, 0);
    for (const SweepDesc& d : large)
      for (int j0 = 0; j0 < d.r; j0 += kSweepNB) {
        const int nbj = std::min(kSweepNB, d.r - j0);
        cl.push_back(CopyDesc{d.B + j0 + (long long)j0 * d.n, d.L + j0 + (long long)j0 * d.r,
                              d.n, d.r, d.r - j0, nbj});
        ocl.push_back(ocl.back() + copy_tiles(d.r - j0, nbj));
      }
    CopyDesc* dc = tmp.add(upload(cl, stream));
    int* doc = tmp.add(upload(ocl, stream));
    timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(dc, doc, (int)cl.size(), ocl.back(), stream); });
    HIF_CK(cudaGetLastError());
  }
  // L^{-1} off the diagonal blocks (which hold L_KK^{-1}), bottom up over a
  // halving of each block's 128-blocks: for a node [b0, b1) split at mid,
  //   X21 = -X22 (L21 X11),
  // X11 and X22 being the inverses of its halves, done one depth before. The
  // nodes of one depth, over all blocks, are two batched products.
  {
    struct Node {
      int b, o1, r1, o2, r2;  // block, first row / size of each half
    };
    std::vector<std::vector<Node>> depth;
    std::function<void(int, int, int, int)> split = [&](int b, int b0, int b1, int dep) {
      if (b1 - b0 < 2) return;
      const int mid = b0 + (b1 - b0) / 2, r = large[b].r;
      if ((int)depth.size() <= dep) depth.resize(dep + 1);
      depth[dep].push_back(Node{b, b0 * kSweepNB, (mid - b0) * kSweepNB, mid * kSweepNB,
                                std::min(r, b1 * kSweepNB) - mid * kSweepNB});
      split(b, b0, mid, dep + 1);
      split(b, mid, b1, dep + 1);
    };
    for (int b = 0; b < nl; ++b) split(b, 0, (large[b].r + kSweepNB - 1) / kSweepNB, 0);
    long long tmax = 0;
    for (const std::vector<Node>& v : depth) {
      long long t = 0;
      for (const Node& q : v) t += (long long)q.r1 * q.r2;
      tmax = std::max(tmax, t);
    }
    double* Tsc = tmax ? big(tmax) : nullptr;
    for (int dep = (int)depth.size() - 1; dep >= 0; --dep) {
      std::vector<GemmDesc> g1, g2;
      long long to = 0;
      for (const Node& q : depth[dep]) {
        const SweepDesc& d = large[q.b];
        double* T = Tsc + to;  // r2 x r1, ld r2
        to += (long long)q.r1 * q.r2;
        GemmDesc t{};  // T = L21 X11 (X11 lower triangular)
        t.C = T;
        t.ldc = q.r2;
        t.A = d.B + q.o2 + (long long)q.o1 * d.n;
        t.lda = d.n;
        t.B = d.a22inv + q.o1 + (long long)q.o1 * d.r;
        t.ldb = d.r;
        t.b_lower = 1;
        t.m = q.r2;
        t.n = q.r1;
        t.k = q.r1;
        t.alpha = 1.0;
        g1.push_back(t);
        GemmDesc x{};  // X21 = -X22 T (X22 lower triangular)
        x.C = d.a22inv + q.o2 + (long long)q.o1 * d.r;
        x.ldc = d.r;
        x.A = d.a22inv + q.o2 + (long long)q.o2 * d.r;
        x.lda = d.r;
        x.a_lower = 1;
        x.B = T;
        x.ldb = q.r2;
        x.m = q.r2;
        x.n = q.r1;
        x.k = q.r2;
        x.alpha = -1.0;
        g2.push_back(x);
      }
      if (ar.chol > 0) {
        gemm_batch_int8(g1, tmp, stream, timed, ar.chol, d_status);
        gemm_batch_int8(g2, tmp, stream, timed, ar.chol, d_status);
      } else {
        gemm_batch(g1, tmp, stream, HIF_KCLASS_SWEEP_PANEL, timed);
        gemm_batch(g2, tmp, stream, HIF_KCLASS_SWEEP_PANEL, timed);
      }
    }
  }
  // Y = L^{-1} A21 and S = A11 - Y^T Y
  std::vector<GemmDesc> gy, gs;
  for (const SweepDesc& d : large) {
    const int r = d.r, sk = d.n - d.r;
    if (sk == 0) continue;
    GemmDesc y{};
    y.C = d.X;
    y.ldc = r;
    y.A = d.a22inv;
    y.a_lower = 1;  // L^{-1}: half the product
    y.lda = r;
    y.B = d.B + (long long)r * d.n;
    y.ldb = d.n;
    y.m = r;
    y.n = sk;
    y.k = r;
    y.alpha = 1.0;
    gy.push_back(y);
    GemmDesc g{};
    g.C = d.B + r + (long long)r * d.n;
    g.ldc = d.n;
    g.A = d.X;
    g.lda = r;
    g.transA = 1;
    g.B = d.X;
    g.ldb = r;
    g.m = g.n = sk;
    g.k = r;
    g.alpha = -1.0;
    g.beta = 1.0;
    g.lower = 1;
    gs.push_back(g);
  }
  if (ar.x > 0) gemm_batch_int8(gy, tmp, stream, timed, ar.x, d_status);
  else gemm_batch(gy, tmp, stream, HIF_KCLASS_GEMM, timed);
  if (ar.schur > 0) gemm_batch_int8(gs, tmp, stream, timed, ar.schur, d_status);
  else if (ar.schur == 0) gemm_batch(gs, tmp, stream, HIF_KCLASS_GEMM_MIXED, timed, 128, d_status);
  else gemm_batch(gs, tmp, stream, HIF_KCLASS_GEMM, timed, 128);
  std::vector<TCopyDesc> tm;
  std::vector<int> otm(1, 0);
  for (const SweepDesc& d : large) {
    const int sk = d.n - d.r;
    double* S = d.B + d.r + (long long)d.r * d.n;
    for (int j0 = 128; j0 < sk; j0 += 128) {
      const int j1 = std::min(sk, j0 + 128);
      tm.push_back(TCopyDesc{S + j0, S + (long long)j0 * d.n, d.n, d.n, j0, j1 - j0, 1.0});
      otm.push_back(otm.back() + copy_tiles(j0, j1 - j0));
    }
  }
  if (!tm.empty()) {
    TCopyDesc* dm = tmp.add(upload(tm, stream));
    int* dom = tmp.add(upload(otm, stream));
    timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_tcopy(dm, dom, (int)tm.size(), otm.back(), stream); });
    HIF_CK(cudaGetLastError());
  }
}

template <class Timed>
void sweep_blocks(const std::vector<SweepDesc>& descs, BufList& tmp, cudaStream_t stream,
                int* d_status, Timed&& timed, ElimArith ar = {}, bool sym = false,
                Arena* scratch = nullptr) {
  // large per-call scratch from the caller's arena when it has one (no pool
  // traffic), else from the stream-ordered pool
  auto big = [&](size_t count) -> double* {
    return scratch ? scratch->alloc<double>(count) : tmp.add(dalloc<double>(count, stream));
  };
  std::vector<SweepDesc> small, large;
  int max_small = 0;
  for (const SweepDesc& d : descs) {
    if (d.r <= 0) continue;
    if (d.n <= kSmallSweepN) {
      small.push_back(d);
      max_small = std::max(max_small, d.n);
    } else {
      large.push_back(d);
    }
  }
  if (!small.empty()) {
    SweepDesc* dd = tmp.add(upload(small, stream));
    double fl = 0, by = 0;
    for (const SweepDesc& d : small) {
      const double r = d.r, sk = d.n - d.r;
      fl += 2 * r * r * r + 2 * r * r * sk + 2 * r * sk * sk;
      by += 8.0 * d.n * d.n + 8.0 * (r * r + r * sk + sk * sk);
    }
    timed(HIF_KCLASS_SWEEP_SMALL, fl, by, [&] {
      launch_sweep_small(dd, (int)small.size(), max_small, d_status, stream);
    });
    HIF_CK(cudaGetLastError());
  }
  if (large.empty()) return;
  // Large blocks (include/Schur.hpp:72-100 in the reference's order):
  //   1. A22^{-1} in place by a blocked Gauss-Jordan sweep over the r x r block
  //      only (FP64 in every arithmetic: the diagonal-block factorization);
  //   2. X = A22^{-1} A21, one product with k = r, written to the compact X;
  //   3. S = A11 - A12 X, one product with k = r, in place in the trailing block.
  const int nl = (int)large.size();
  SweepDesc* dd = tmp.add(upload(large, stream));
  double* dinv = big((size_t)nl * kSweepNB * kSweepNB);
  int maxr = 0;
  for (const SweepDesc& d : large) maxr = std::max(maxr, d.r);
  if (sym) {
    // Symmetric A22 (the face operator): only the block-lower triangle is
    // kept. After the pivot blocks before K, entry (i, j) equals +(j, i) when
    // i and j are both pivoted or both not, -(j, i) otherwise. Step K with
    // Q = the old column block K (rows above K from row block K, negated),
    // W = -Q D^{-1}: new column block K = W (rows below K), new row block K
    // = W^T (columns left of K), and lower tile (I, J) += tau_J W_I Q_J^T with
    // tau_J = -1 left of K, +1 right of K. At the end every pivot is taken,
    // the inverse is symmetric and the upper tiles are mirrored from the lower.
    // 2r^3 -> r^3 flops.
    std::vector<long long> oq(nl);
    long long qsz = 0;
    for (int b = 0; b < nl; ++b) {
      oq[b] = qsz;
      qsz += (long long)large[b].r * kSweepNB;
    }
    double* Qb = big(qsz);
    double* Wb = big(qsz);
    for (int k0 = 0; k0 < maxr; k0 += kSweepNB) {
      std::vector<int> active;
      std::vector<CopyDesc> cq, cw;
      std::vector<int> ocq(1, 0), ocw(1, 0);
      std::vector<TCopyDesc> tq, tw;
      std::vector<int> otq(1, 0), otw(1, 0);
      std::vector<GemmDesc> gw, gu;
      for (int b = 0; b < nl; ++b) {
        const SweepDesc& d = large[b];
        if (d.r <= k0) continue;
        active.push_back(b);
        const int k1 = std::min(d.r, k0 + kSweepNB), nbk = k1 - k0, r = d.r;
        const double* Dv = dinv + (long long)b * kSweepNB * kSweepNB;
        double* Q = Qb + oq[b];
        double* W = Wb + oq[b];
        if (r > k1) {
          cq.push_back(CopyDesc{d.B + k1 + (long long)k0 * d.n, Q + k1, d.n, r, r - k1, nbk});
          ocq.push_back(ocq.back() + copy_tiles(r - k1, nbk));
          cw.push_back(CopyDesc{W + k1, d.B + k1 + (long long)k0 * d.n, r, d.n, r - k1, nbk});
          ocw.push_back(ocw.back() + copy_tiles(r - k1, nbk));
        }
        if (k0 > 0) {
          tq.push_back(TCopyDesc{d.B + k0, Q, d.n, r, k0, nbk, -1.0});
          otq.push_back(otq.back() + copy_tiles(k0, nbk));
          tw.push_back(TCopyDesc{W, d.B + k0, r, d.n, nbk, k0, 1.0});
          otw.push_back(otw.back() + copy_tiles(nbk, k0));
        }
        auto wg = [&](int r0, int r1) {
          if (r1 <= r0) return;
          GemmDesc g{};
          g.C = W + r0;
          g.ldc = r;
          g.A = Q + r0;
          g.lda = r;
          g.B = Dv;
          g.ldb = nbk;
          g.m = r1 - r0;
          g.n = nbk;
          g.k = nbk;
          g.alpha = -1.0;
          g.beta = 0.0;
          gw.push_back(g);
        };
        wg(0, k0);
        wg(k1, r);
        for (int j0 = 0; j0 < r; j0 += kSweepNB) {
          if (j0 == k0) continue;
          const int j1 = std::min(r, j0 + kSweepNB);
          const double tau = j0 < k0 ? -1.0 : 1.0;
          auto ug = [&](int r0, int r1) {
            if (r1 <= r0) return;
            GemmDesc g{};
            g.C = d.B + r0 + (long long)j0 * d.n;
            g.ldc = d.n;
            g.A = W + r0;
            g.lda = r;
            g.B = Q + j0;
            g.ldb = r;
            g.transB = 1;
            g.m = r1 - r0;
            g.n = j1 - j0;
            g.k = nbk;
            g.alpha = tau;
            g.beta = 1.0;
            gu.push_back(g);
          };
          if (j0 < k0) {
            ug(j0, k0);
            ug(k1, r);
          } else {
            ug(j0, r);
          }
        }
      }
      BufList step;
      int* dact = step.add(upload(active, stream));
      timed(HIF_KCLASS_SWEEP_PANEL, 0, 0, [&] {
        launch_sweep_diag(dd, dact, (int)active.size(), k0, dinv, d_status, stream, 1);
      });
      if (!cq.empty()) {
        CopyDesc* dq = step.add(upload(cq, stream));
        int* doq = step.add(upload(ocq, stream));
        timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(dq, doq, (int)cq.size(), ocq.back(), stream); });
      }
      if (!tq.empty()) {
        TCopyDesc* dq = step.add(upload(tq, stream));
        int* doq = step.add(upload(otq, stream));
        timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_tcopy(dq, doq, (int)tq.size(), otq.back(), stream); });
      }
      gemm_batch(gw, step, stream, HIF_KCLASS_SWEEP_PANEL, timed);
      gemm_batch(gu, step, stream, HIF_KCLASS_GEMM, timed);
      if (!cw.empty()) {
        CopyDesc* dw = step.add(upload(cw, stream));
        int* dow = step.add(upload(ocw, stream));
        timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(dw, dow, (int)cw.size(), ocw.back(), stream); });
      }
      if (!tw.empty()) {
        TCopyDesc* dw = step.add(upload(tw, stream));
        int* dow = step.add(upload(otw, stream));
        timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_tcopy(dw, dow, (int)tw.size(), otw.back(), stream); });
      }
      timed(HIF_KCLASS_SWEEP_PANEL, 0, 0, [&] {
        launch_sweep_setdiag(dd, dact, (int)active.size(), k0, dinv, stream);
      });
      HIF_CK(cudaGetLastError());
      step.release(stream);
    }
    // upper tiles of A22^{-1} from the lower ones
    std::vector<TCopyDesc> tm;
    std::vector<int> otm(1, 0);
    for (const SweepDesc& d : large)
      for (int j0 = kSweepNB; j0 < d.r; j0 += kSweepNB) {
        const int j1 = std::min(d.r, j0 + kSweepNB);
        tm.push_back(TCopyDesc{d.B + j0, d.B + (long long)j0 * d.n, d.n, d.n, j0, j1 - j0, 1.0});
        otm.push_back(otm.back() + copy_tiles(j0, j1 - j0));
      }
    if (!tm.empty()) {
      TCopyDesc* dm = tmp.add(upload(tm, stream));
      int* dom = tmp.add(upload(otm, stream));
      timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_tcopy(dm, dom, (int)tm.size(), otm.back(), stream); });
      HIF_CK(cudaGetLastError());
    }
  } else {
    for (int k0 = 0; k0 < maxr; k0 += kSweepNB) {
      std::vector<int> active;
      std::vector<GemmDesc> gd, rowg, colg;
      for (int b = 0; b < nl; ++b) {
        const SweepDesc& d = large[b];
        if (d.r <= k0) continue;
        active.push_back(b);
        const int k1 = std::min(d.r, k0 + kSweepNB);
        const int nbk = k1 - k0;
        const double* Dv = dinv + (long long)b * kSweepNB * kSweepNB;  // nbk x nbk, ld nbk
        // row panel B[K, c0:c1) = Dinv B[K, c0:c1), in place: one 128-row tile
        auto rowp = [&](int c0, int c1) {
          if (c1 <= c0) return;
          GemmDesc g{};
          g.C = d.B + k0 + (long long)c0 * d.n;
          g.A = Dv;
          g.B = g.C;
          g.ldc = g.ldb = d.n;
          g.lda = nbk;
          g.m = nbk;
          g.n = c1 - c0;
          g.k = nbk;
          g.alpha = 1.0;
          g.beta = 0.0;
          rowg.push_back(g);
        };
        // column panel B[r0:r1, K] = -B[r0:r1, K] Dinv, in place: one 128-column tile
        auto colp = [&](int r0, int r1) {
          if (r1 <= r0) return;
          GemmDesc g{};
          g.C = d.B + r0 + (long long)k0 * d.n;
          g.A = g.C;
          g.B = Dv;
          g.ldc = g.lda = d.n;
          g.ldb = nbk;
          g.m = r1 - r0;
          g.n = nbk;
          g.k = nbk;
          g.alpha = -1.0;
          g.beta = 0.0;
          colg.push_back(g);
        };
        rowp(0, k0);
        rowp(k1, d.r);
        colp(0, k0);
        colp(k1, d.r);
        auto gemm = [&](int r0, int r1, int c0, int c1) {
          if (r1 <= r0 || c1 <= c0) return;
          GemmDesc g{};
          g.C = d.B + r0 + (long long)c0 * d.n;
          g.A = d.B + r0 + (long long)k0 * d.n;
          g.B = d.B + k0 + (long long)c0 * d.n;
          g.ldc = g.lda = g.ldb = d.n;
          g.m = r1 - r0;
          g.n = c1 - c0;
          g.k = nbk;
          g.alpha = -1.0;
          g.beta = 1.0;
          gd.push_back(g);
        };
        gemm(0, k0, 0, k0);
        gemm(0, k0, k1, d.r);
        gemm(k1, d.r, 0, k0);
        gemm(k1, d.r, k1, d.r);
      }
      BufList step;
      int* dact = step.add(upload(active, stream));
      timed(HIF_KCLASS_SWEEP_PANEL, 0, 0, [&] {
        launch_sweep_diag(dd, dact, (int)active.size(), k0, dinv, d_status, stream);
      });
      gemm_batch(rowg, step, stream, HIF_KCLASS_SWEEP_PANEL, timed, 128);
      gemm_batch(gd, step, stream, HIF_KCLASS_GEMM, timed);
      gemm_batch(colg, step, stream, HIF_KCLASS_SWEEP_PANEL, timed, 128);
      timed(HIF_KCLASS_SWEEP_PANEL, 0, 0, [&] {
        launch_sweep_setdiag(dd, dact, (int)active.size(), k0, dinv, stream);
      });
      HIF_CK(cudaGetLastError());
      step.release(stream);
    }
  }
  // X = A22^{-1} A21 and S = A11 - A12 X
  std::vector<GemmDesc> gx, gs;
  for (const SweepDesc& d : large) {
    const int r = d.r, sk = d.n - d.r;
    if (sk == 0) continue;
    GemmDesc x{};
    x.C = d.X;
    x.ldc = r;
    x.A = d.B;
    x.lda = d.n;
    x.B = d.B + (long long)r * d.n;
    x.ldb = d.n;
    x.m = r;
    x.n = sk;
    x.k = r;
    x.alpha = 1.0;
    x.beta = 0.0;
    gx.push_back(x);
    GemmDesc y{};
    y.C = d.B + r + (long long)r * d.n;
    y.ldc = d.n;
    y.A = d.B + r;
    y.lda = d.n;
    y.B = d.X;
    y.ldb = r;
    y.m = sk;
    y.n = sk;
    y.k = r;
    y.alpha = -1.0;
    y.beta = 1.0;
    y.lower = sym ? 1 : 0;  // S is symmetric: the tiles above the diagonal are mirrored
    gs.push_back(y);
  }
  // X comes from the explicit inverse, whose entries exceed X's by about
  // cond(A22): a TF32-level product would lose that factor in X, so it is FP64
  // or from enough int8 slices to be close to it.
  if (ar.x > 0) gemm_batch_int8(gx, tmp, stream, timed, ar.x, d_status);
  else gemm_batch(gx, tmp, stream, HIF_KCLASS_GEMM, timed);
  if (ar.schur > 0) gemm_batch_int8(gs, tmp, stream, timed, ar.schur, d_status);
  else if (ar.schur == 0) gemm_batch(gs, tmp, stream, HIF_KCLASS_GEMM_MIXED, timed, 128, d_status);
  else gemm_batch(gs, tmp, stream, HIF_KCLASS_GEMM, timed, sym ? 128 : 0);
  if (sym) {
    std::vector<TCopyDesc> tm;
    std::vector<int> otm(1, 0);
    for (const SweepDesc& d : large) {
      const int sk = d.n - d.r;
      double* S = d.B + d.r + (long long)d.r * d.n;
      for (int j0 = 128; j0 < sk; j0 += 128) {
        const int j1 = std::min(sk, j0 + 128);
        tm.push_back(TCopyDesc{S + j0, S + (long long)j0 * d.n, d.n, d.n, j0, j1 - j0, 1.0});
        otm.push_back(otm.back() + copy_tiles(j0, j1 - j0));
      }
    }
    if (!tm.empty()) {
      TCopyDesc* dm = tmp.add(upload(tm, stream));
      int* dom = tmp.add(upload(otm, stream));
      timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_tcopy(dm, dom, (int)tm.size(), otm.back(), stream); });
      HIF_CK(cudaGetLastError());
    }
  }
  // compact copy of A22^{-1}
  std::vector<CopyDesc> cd;
  std::vector<int> coff(1, 0);
  for (const SweepDesc& d : large) {
    CopyDesc a{d.B, d.a22inv, d.n, d.r, d.r, d.r};
    cd.push_back(a);
    coff.push_back(coff.back() + copy_tiles(d.r, d.r));
  }
  CopyDesc* dcd = tmp.add(upload(cd, stream));
  int* dco = tmp.add(upload(coff, stream));
  timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(dcd, dco, (int)cd.size(), coff.back(), stream); });
  HIF_CK(cudaGetLastError());
}


class Engine {
 public:
  int N, P, NC, partition;
  double eps;
  long long n3;
  int L = 0;
  cudaStream_t stream = nullptr;      // stream every launch goes to
  cudaStream_t own_stream = nullptr;  // created by the handle
  double* d_band = nullptr;
  bool have_op = false, initialized = false, factored = false;
  std::vector<uint8_t> rem;
  std::vector<StepData> steps;
  // factor storage (persistent) and per-level workspace (alternating by level);
  // arena_desc: the factorization's uploads (see t_desc), its apply plans' too
  Arena arena_factor, arena_work[2], arena_desc;
  Arena* cur_work = &arena_work[0];
  bool keep_schur = false, verbose = false;
  int verbose_mode = 0;
  int precision = HIF_PRECISION_FP64;
  int factor_precision = HIF_PRECISION_FP64;  // the precision the held factor was made in
  long long budget_mb = 0;
  std::map<int, std::vector<std::vector<int>>> replay;
  double t_total = 0, t_gather = 0, t_elim = 0, t_id = 0, t_host = 0, t_plan = 0;
  long long peak_bytes = 0, cur_bytes = 0;
  int* d_status = nullptr;
  int* d_dof_src = nullptr;  // source membership, 6 x NC^3 (see Sources)
  // the operator is symmetric (face-coefficient form): eliminations keep only
  // the lower triangle of A22
  bool symmetric = false;

  // ---- per-kernel-class timing (HIF_OPT_PROFILE): CUDA events on the engine
  // stream around each launch, with the launch's algorithmic flops / bytes.
  struct KStat {
    long long launches = 0;
    double ms = 0, flops = 0, bytes = 0;
  };
  struct Pending {
    int cls;
    cudaEvent_t a, b;
    double flops, bytes;
    int nlaunch;
  };
  bool profile = false;
  KStat kstat[HIF_KCLASS_COUNT];
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> ev_pool;

  cudaEvent_t get_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    HIF_CK(cudaEventCreate(&e));
    return e;
  }

  template <class F>
  void timed(int cls, double flops, double bytes, F&& launch, int nlaunch = 1) {
    if (!profile) {
      launch();
      return;
    }
    Pending pd{cls, get_event(), get_event(), flops, bytes, nlaunch};
    HIF_CK(cudaEventRecord(pd.a, stream));
    launch();
    HIF_CK(cudaEventRecord(pd.b, stream));
    pending.push_back(pd);
  }

  void resolve_profile() {
    for (Pending& pd : pending) {
      HIF_CK(cudaEventSynchronize(pd.b));
      float ms = 0;
      HIF_CK(cudaEventElapsedTime(&ms, pd.a, pd.b));
      KStat& k = kstat[pd.cls];
      k.launches += pd.nlaunch;
      k.ms += ms;
      k.flops += pd.flops;
      k.bytes += pd.bytes;
      ev_pool.push_back(pd.a);
      ev_pool.push_back(pd.b);
    }
    pending.clear();
  }

  void reset_profile() {
    resolve_profile();
    for (KStat& k : kstat) k = KStat{};
  }

  // apply / solve workspace
  double* d_ua = nullptr;
  double* d_ub = nullptr;
  double* d_uc = nullptr;
  double* d_contrib = nullptr;
  int ws_nrhs = 0;
  ApplyPlan plan_inv, plan_fwd;
  bool plans_built = false;
  // PCG workspace
  double* d_pcg = nullptr;
  int pcg_nrhs = 0;

  Engine(int N_, int P_, double eps_, int part)
      : N(N_), P(P_), NC(N_ + 1), partition(part), eps(eps_) {
    n3 = (long long)NC * NC * NC;
    HIF_CK(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;
    // keep freed pool memory reserved: factorizations reallocate the same
    // workspace sizes, and growing the pool again costs more than the kernels
    int dev = 0;
    HIF_CK(cudaGetDevice(&dev));
    cudaMemPool_t pool;
    HIF_CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    unsigned long long keep = ~0ull;
    HIF_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    d_status = dalloc<int>(4, stream);
    HIF_CK(cudaMemsetAsync(d_status, 0, 4 * sizeof(int), stream));
    d_band = dalloc<double>(7 * n3, stream);
    HIF_CK(cudaMemsetAsync(d_band, 0, 7 * n3 * sizeof(double), stream));
  }

  ~Engine() {
    join_face_partition();
    join_cell_partition();
    sync_quiet();
    for (Pending& pd : pending) {
      cudaEventDestroy(pd.a);
      cudaEventDestroy(pd.b);
    }
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    release_factor();
    join_reaper();
    release_workspace();
    sync_quiet();
    arena_factor.release();
    arena_work[0].release();
    arena_work[1].release();
    arena_desc.release();
    dfree(cell0.d_red, stream);
    dfree(cell0.d_skel, stream);
    dfree(cell0.d_rows, stream);
    dfree(face0_didx, stream);
    dfree(d_band, stream);
    dfree(d_status, stream);
    dfree(d_dof_src, stream);
    cudaStreamSynchronize(stream);
    cudaStreamSynchronize(own_stream);
    cudaStreamDestroy(own_stream);
  }

  void sync() { HIF_CK(cudaStreamSynchronize(stream)); }
  // verbose: print the time since the last mark (after a stream sync)
  double mark_t = 0;
  // verbose 1: synchronise at every mark and print the phase's wall time;
  // verbose 2: no synchronisation; an event per mark, and at the end of the
  // factorization each phase's host time (issue) beside its device time
  struct Mark {
    const char* what;
    int level;
    double host;
    cudaEvent_t ev;
  };
  std::vector<Mark> marks;
  void mark(const char* what, int level) {
    if (!verbose) return;
    if (verbose_mode == 2) {
      Mark m{what, level, wall(), get_event()};
      HIF_CK(cudaEventRecord(m.ev, stream));
      marks.push_back(m);
      return;
    }
    sync();
    const double t = wall();
    if (mark_t > 0) std::fprintf(stderr, "[hif]   L%d %-22s %9.3f ms\n", level, what, 1e3 * (t - mark_t));
    mark_t = t;
  }
  void report_marks() {
    if (marks.empty()) return;
    sync();
    for (size_t q = 1; q < marks.size(); ++q) {
      float ms = 0;
      HIF_CK(cudaEventElapsedTime(&ms, marks[q - 1].ev, marks[q].ev));
      std::fprintf(stderr, "[hif]   L%d %-22s host %9.3f ms  device %9.3f ms\n", marks[q].level,
                   marks[q].what, 1e3 * (marks[q].host - marks[q - 1].host), ms);
    }
    for (Mark& m : marks) ev_pool.push_back(m.ev);
    marks.clear();
    std::fprintf(stderr, "[hif]   arenas: factor %zu chunks %.1f GB, work %zu + %zu chunks %.1f GB, "
                 "cudaMalloc %.1f ms so far\n", arena_factor.chunks.size(),
                 arena_factor.reserved() / 1e9, arena_work[0].chunks.size(),
                 arena_work[1].chunks.size(),
                 (arena_work[0].reserved() + arena_work[1].reserved()) / 1e9,
                 1e3 * (arena_factor.grow_s + arena_work[0].grow_s + arena_work[1].grow_s));
  }
  void sync_quiet() { cudaStreamSynchronize(stream); }

  void release_workspace() {
    drop_graphs();
    dfree(d_ua, stream);
    dfree(d_ub, stream);
    dfree(d_uc, stream);
    dfree(d_pcg, stream);
    d_ua = d_ub = d_uc = d_pcg = nullptr;
    ws_nrhs = pcg_nrhs = 0;
  }

  // CUDA graphs of the apply sweep (boundary zeroing, output clearing and every
  // launch of the plan), one per (direction, right-hand-side count); valid
  // while the plans and the apply workspace stay as they were captured
  std::map<std::pair<int, int>, cudaGraphExec_t> apply_graphs;
  void drop_graphs() {
    for (auto& kv : apply_graphs) cudaGraphExecDestroy(kv.second);
    apply_graphs.clear();
    for (auto& kv : gemm_plans) kv.second.bufs.release(stream);
    gemm_plans.clear();
  }

  // ---- apply for many right-hand sides: every GEMV launch of a plan as gather /
  // GEMM / emit, so each factor matrix is read once per apply instead of once
  // per 4 right-hand sides. Built per (direction, RHS count) from the plan's
  // descriptors; launches only, so the sweep is still captured in a graph.
  static constexpr int kGemmApplyMinRhs = 16;
  struct GemmStage {
    size_t launch = 0;  // plan launch (reduce-scatter launches are run as they are)
    ApplyGatherDesc* d_gather = nullptr;
    long long* d_goff = nullptr;
    int ng = 0;
    long long gtotal = 0;
    GemmDesc* d_gemm = nullptr;
    int* d_toff = nullptr;
    int tiles = 0, tile = 64;
    ApplyEmitDesc* d_emit = nullptr;
    long long* d_eoff = nullptr;
    long long etotal = 0;
    double flops = 0;
  };
  struct GemmPlan {
    std::vector<GemmStage> stages;
    BufList bufs;
  };
  std::map<std::pair<int, int>, GemmPlan> gemm_plans;

  GemmPlan& gemm_plan(ApplyPlan& plan, int inverse, int nrhs) {
    const std::pair<int, int> key(inverse, nrhs);
    auto it = gemm_plans.find(key);
    if (it != gemm_plans.end()) return it->second;
    GemmPlan gp;
    long long xmax = 1, ymax = 1;
    for (const ApplyLaunch& l : plan.launches) {
      if (l.type != 0) continue;
      long long xs = 0, ys = 0;
      for (const GemvDesc& g : l.hdesc) {
        xs += (long long)(g.trans ? g.m : g.n) * nrhs;
        ys += (long long)(g.trans ? g.n : g.m) * nrhs;
      }
      xmax = std::max(xmax, xs);
      ymax = std::max(ymax, ys);
    }
    double* xin = gp.bufs.add(dalloc<double>(xmax, stream));
    double* yout = gp.bufs.add(dalloc<double>(ymax, stream));
    for (size_t q = 0; q < plan.launches.size(); ++q) {
      const ApplyLaunch& l = plan.launches[q];
      GemmStage st;
      st.launch = q;
      if (l.type == 0) {
        std::vector<ApplyGatherDesc> gd;
        std::vector<ApplyEmitDesc> ed;
        std::vector<GemmDesc> gm;
        std::vector<long long> goff(1, 0), eoff(1, 0);
        std::vector<int> toff(1, 0);
        long long ox = 0, oy = 0;
        const int tile = nrhs >= 48 ? 128 : 64;
        for (const GemvDesc& g : l.hdesc) {
          const int len = g.trans ? g.m : g.n, rows = g.trans ? g.n : g.m;
          gd.push_back(ApplyGatherDesc{g.in_idx, xin + ox, len});
          goff.push_back(goff.back() + (long long)len * nrhs);
          GemmDesc m{};
          m.C = yout + oy;
          m.ldc = rows;
          m.A = g.M;
          m.lda = g.ld;
          m.transA = g.trans;
          m.B = xin + ox;
          m.ldb = len;
          m.m = rows;
          m.n = nrhs;
          m.k = len;
          m.alpha = 1.0;
          m.beta = 0.0;
          gm.push_back(m);
          toff.push_back(toff.back() + dgemm_tiles(rows, nrhs, tile));
          ed.push_back(ApplyEmitDesc{yout + oy, g.out_idx, g.contrib, rows, g.mode, g.alpha});
          eoff.push_back(eoff.back() + (long long)rows * nrhs);
          st.flops += 2.0 * rows * len * nrhs;
          ox += (long long)len * nrhs;
          oy += (long long)rows * nrhs;
        }
        st.d_gather = gp.bufs.add(upload(gd, stream));
        st.d_goff = gp.bufs.add(upload(goff, stream));
        st.ng = (int)gd.size();
        st.gtotal = goff.back();
        st.d_gemm = gp.bufs.add(upload(gm, stream));
        st.d_toff = gp.bufs.add(upload(toff, stream));
        st.tiles = toff.back();
        st.tile = tile;
        st.d_emit = gp.bufs.add(upload(ed, stream));
        st.d_eoff = gp.bufs.add(upload(eoff, stream));
        st.etotal = eoff.back();
      }
      gp.stages.push_back(st);
    }
    return gemm_plans.emplace(key, std::move(gp)).first->second;
  }

  void run_gemm_plan(ApplyPlan& plan, GemmPlan& gp, int nrhs) {
    double* vec[3] = {d_ua, d_ub, d_uc};
    for (GemmStage& st : gp.stages) {
      ApplyLaunch& l = plan.launches[st.launch];
      if (l.type == 0) {
        timed(HIF_KCLASS_VECTOR, 0, 0, [&] {
          launch_apply_gather(st.d_gather, st.d_goff, st.ng, st.gtotal, vec[l.in_vec], n3,
                              stream);
        });
        timed(HIF_KCLASS_GEMV, st.flops, l.bytes, [&] {
          launch_dgemm(st.d_gemm, st.d_toff, st.ng, st.tiles, stream, st.tile);
        });
        timed(HIF_KCLASS_VECTOR, 0, 0, [&] {
          launch_apply_emit(st.d_emit, st.d_eoff, st.ng, st.etotal, vec[l.out_vec], n3,
                            contrib_ld, stream);
        });
      } else {
        timed(HIF_KCLASS_VECTOR, 0, 0, [&] {
          launch_reduce_scatter(l.d_dof, l.d_off, l.d_slot, d_contrib, l.ndof, contrib_ld,
                                l.alpha, vec[l.out_vec], nrhs, n3, stream);
        });
      }
      HIF_CK(cudaGetLastError());
    }
  }

  void release_plans() {
    drop_graphs();
    reduce_bufs.release(stream);
    reduce_lists.clear();
    plan_inv.bufs.release(stream);
    plan_fwd.bufs.release(stream);
    plan_inv.launches.clear();
    plan_fwd.launches.clear();
    plans_built = false;
  }

  void release_factor() {
    release_plans();
    for (auto& kv : reduce_pending)
      if (kv.second.valid()) kv.second.wait();
    reduce_pending.clear();
    dfree(d_contrib, stream);
    d_contrib = nullptr;
    contrib_cap = 0;
    // the released factor's host structures (some 10^5 small vectors at
    // n = 128, ~25 ms to free) are destroyed on a thread of their own, off the
    // next factorization's critical path; they hold no device resources
    join_reaper();
    if (!steps.empty()) {
      auto* old = new std::vector<StepData>(std::move(steps));
      steps.clear();
      reaper_ = std::thread([old] { delete old; });
    }
    arena_factor.reset();
    factored = false;
  }
  std::thread reaper_;
  void join_reaper() {
    if (reaper_.joinable()) reaper_.join();
  }

  int levels_for() const {
    if (partition == HIF_PARTITION_REFERENCE) {
      // src/Factor.cpp:36: round(log2(NC / P)) + 1 with integer NC / P
      return (int)std::lround(std::log2((double)(NC / P))) + 1;
    }
    int l = 0;
    while ((long long)P << l < NC) ++l;
    return l + 1;
  }

  int cells_per_dir(int level) const {
    const int w = (1 << level) * P;
    return partition == HIF_PARTITION_REFERENCE ? NC / w : (NC + w - 1) / w;
  }

  // ---- operator setup ----------------------------------------------------
  void setup_node_device(const double* dA, const double* dV, double hstep) {
    launch_setup_node(dA, dV, N, hstep, d_band, stream);
    HIF_CK(cudaGetLastError());
    have_op = true;
    symmetric = false;  // the node form is not symmetric for variable A
  }

  // ---- Initialize (src/Factor.cpp:6-39) -----------------------------------
  void initialize() {
    release_factor();
    // every DOF with all three indices in [1, NC) remains: one run of NC - 1
    // bytes per (j, k) row
    rem.assign(n3, 0);
    for (int k = 1; k < NC; ++k)
      for (int j = 1; j < NC; ++j)
        std::memset(rem.data() + 1 + (long long)NC * j + (long long)NC * NC * k, 1, NC - 1);
    L = levels_for();
    initialized = true;
  }

  void track(long long bytes) {
    cur_bytes += bytes;
    peak_bytes = std::max(peak_bytes, cur_bytes);
    if (budget_mb > 0 && cur_bytes > budget_mb * (1LL << 20))
      throw Error{HIF_ERR_BUDGET, "device memory budget exceeded"};
  }

  // ---- dense elimination of a batch of blocks ---------------------------
  // descs[b].B holds [A22 A21; A12 A11] (ld n); on return the compact
  // A22^{-1}, X are written and B's trailing block holds A11 - A12 X.
  // Elimination of one phase's blocks. With HIF_OPT_AUTOTUNE in mixed precision
  // on a symmetric operator (and HIF_ELIM_AUTO), the method is tuned per phase
  // signature (kind, level, log2 buckets of the block count and mean size):
  // the first factorizations run it once with each method, timed by CUDA
  // events, and the faster is kept. st.chol records the method used.
  static constexpr long long kTuneElimKey = 1LL << 62;
  void run_sweep(const std::vector<SweepDesc>& descs, BufList& tmp, StepData& st) {
    bool chol = use_chol;
    GemmTuner::Pending tp{0, -1, nullptr, nullptr};
    if (t_tuner && symmetric && precision == HIF_PRECISION_MIXED &&
        elimination == HIF_ELIM_AUTO && !descs.empty()) {
      double sn = 0;
      for (const SweepDesc& d : descs) sn += d.n;
      const long long key = kTuneElimKey | ((long long)(st.skel ? 1 : 0) << 40) |
                            ((long long)st.level << 32) |
                            ((long long)ilog2_bucket((double)descs.size()) << 16) |
                            ilog2_bucket(sn / descs.size());
      GemmTuner::Rec& r = t_tuner->recs[key];
      if (r.choice >= 0) {
        chol = r.choice == 1;
      } else {
        tp.key = key;
        tp.cand = r.runs[0] == 0 ? 0 : 1;
        chol = tp.cand == 1;
        HIF_CK(cudaEventCreate(&tp.a));
        HIF_CK(cudaEventCreate(&tp.b));
        HIF_CK(cudaEventRecord(tp.a, stream));
      }
    }
    st.chol = chol;
    ElimArith ar;
    if (precision == HIF_PRECISION_MIXED) {
      ar.schur = schur_slices;
      ar.x = chol ? y_slices : x_slices;
      ar.chol = chol ? chol_slices : 0;
    }
    auto tm = [&](int cls, double fl, double by, auto&& f, int n = 1) { timed(cls, fl, by, f, n); };
    if (chol) chol_blocks(descs, tmp, stream, d_status, tm, ar, cur_work);
    else sweep_blocks(descs, tmp, stream, d_status, tm, ar, symmetric, cur_work);
    if (tp.cand >= 0) {
      HIF_CK(cudaEventRecord(tp.b, stream));
      t_tuner->pending.push_back(tp);
    }
  }

  void gather(std::vector<GatherTarget>& tg, const Sources& src, const int* d_src_owner,
              const SourceDesc* d_srcdesc, const int* d_dof_src, BufList& tmp) {
    std::vector<int> toff(1, 0);
    double by = 0;
    for (const GatherTarget& g : tg) {
      toff.push_back(toff.back() + gather_tiles(g.m, g.n));
      by += 8.0 * g.m * g.n;
    }
    if (toff.back() == 0) return;
    GatherTarget* dt = tmp.add(upload(tg, stream));
    int* dto = tmp.add(upload(toff, stream));
    timed(HIF_KCLASS_GATHER, 0, by, [&] {
      launch_gather(dt, dto, (int)tg.size(), toff.back(), d_srcdesc, d_src_owner, d_dof_src,
                    d_band, n3, NC, stream);
    });
    HIF_CK(cudaGetLastError());
    (void)src;
  }

  // Upload the source tables of a phase; the membership arrays are shared by
  // every gather of that phase.
  void upload_sources(const Sources& s, BufList& tmp, SourceDesc** d_desc, int** d_owner,
                      int** d_dof) {
    *d_desc = tmp.add(upload(s.desc, stream));
    *d_owner = tmp.add(upload(s.owner, stream));
    *d_dof = d_dof_src;
  }

  // Stream-ordered after every gather that read the previous membership.
  void empty_sources(Sources& s, int ncells) {
    s.desc.clear();
    s.owner.clear();
    s.cell_src.assign(ncells, -1);
    if (!d_dof_src) d_dof_src = dalloc<int>(6 * n3, stream);
    HIF_CK(cudaMemsetAsync(d_dof_src, 0xFF, 6 * n3 * sizeof(int), stream));
  }

  // ---- Schur phase (LevelFactorSchur, src/Factor.cpp:184-213) ------------
  struct Cell0Layout {
    bool cached = false;
    std::vector<BlockInfo> blocks;
    std::vector<int> red_all, skel_all, rows_all;
    std::vector<long long> o_B, o_rows, o_a22, o_inv, o_x, o_red, o_skel;
    long long bsz = 0, asz = 0;
    // device copies of red_all / skel_all / rows_all, made by the second
    // factorization (the first one's uploads live in its arenas); read-only
    int* d_red = nullptr;
    int* d_skel = nullptr;
    int* d_rows = nullptr;
  };
  // A device copy of `count` ints at src that lives with the handle.
  int* keep_on_device(const int* src, size_t count) {
    int* d = dalloc<int>(std::max<size_t>(count, 1), stream);
    if (count)
      HIF_CK(cudaMemcpyAsync(d, src, count * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    return d;
  }
  Cell0Layout cell0;
  void schur_phase(int level, Sources& in, Sources& out) {
    double th = wall();
    const int cpd = cells_per_dir(level);
    const int w = (1 << level) * P;
    StepData st;
    st.level = level;
    st.skel = false;
    st.chol = use_chol;
    st.cpd = cpd;
    Partitioner part{N, P, NC, rem.data()};
    const int ncell = cpd * cpd * cpd;
    // level 0's cells see the initial DOF mask, so their blocks, offsets and
    // index lists are the grid's alone: kept from the handle's first
    // factorization (cell0) and reused by the later ones
    const bool cell0_hit = level == 0 && cell0.cached;
    if (cell0_hit) {
      st.blocks.resize(ncell);
      parallel_for(ncell, [&](int idx) { st.blocks[idx] = cell0.blocks[idx]; });
    } else if (take_cell_partition(level, st.blocks)) {
      // built before the last skeletonization's DOFs were removed: drop them
      // (the scan order and the classification of the rest do not change).
      // Every position is either redundant or skeleton and red_pos ascends,
      // so one walk compacts the three lists in place (each write index
      // trails its read index).
      parallel_for(ncell, [&](int idx) {
        BlockInfo& b = st.blocks[idx];
        int* gl = b.global.data();
        int* rp = b.red_pos.data();
        int* sp = b.skel_pos.data();
        const size_t ng_in = b.global.size(), nr_in = b.red_pos.size();
        size_t ri = 0, nr = 0, ns = 0, ng = 0;
        for (size_t t = 0; t < ng_in; ++t) {
          const bool is_red = ri < nr_in && rp[ri] == (int)t;
          ri += is_red;
          const int gid = gl[t];
          if (!rem[gid]) continue;
          if (is_red)
            rp[nr++] = (int)ng;
          else
            sp[ns++] = (int)ng;
          gl[ng++] = gid;
        }
        b.global.resize(ng);
        b.red_pos.resize(nr);
        b.skel_pos.resize(ns);
      });
    } else {
      st.blocks.resize(ncell);
      parallel_for(ncell, [&](int idx) {
        const int c[3] = {idx / (cpd * cpd), (idx / cpd) % cpd, idx % cpd};
        BlockInfo& b = st.blocks[idx];
        part.cell_index(level, c, b.global, b.red_pos, b.skel_pos);
        b.cell = idx;
      });
    }
    mark("schur cell partition", level);
    // sizes and device layout (the flat lists reuse the handle's host buffers:
    // their pages are touched once, not at every factorization)
    std::vector<int>& red_all = cell0_hit ? cell0.red_all : h_red_all;
    std::vector<int>& skel_all = cell0_hit ? cell0.skel_all : h_skel_all;
    std::vector<int>& rows_all = cell0_hit ? cell0.rows_all : h_rows_all;
    long long bsz = 0, asz = 0;
    std::vector<long long> o_B(ncell);
    std::vector<long long> o_rows(ncell);
    st.o_w.assign(ncell, 0);
    if (cell0_hit) {
      bsz = cell0.bsz;
      asz = cell0.asz;
      o_B = cell0.o_B;
      o_rows = cell0.o_rows;
      st.o_a22 = cell0.o_a22;
      st.o_inv = cell0.o_inv;
      st.o_x = cell0.o_x;
      st.o_red = cell0.o_red;
      st.o_skel = cell0.o_skel;
    } else {
      st.o_a22.resize(ncell);
      st.o_inv.resize(ncell);
      st.o_x.resize(ncell);
      st.o_red.resize(ncell);
      st.o_skel.resize(ncell);
      long long nred = 0, nskel = 0;
      for (int b = 0; b < ncell; ++b) {
        const BlockInfo& bi = st.blocks[b];
        const long long n = bi.global.size(), r = bi.r(), s = bi.s();
        o_B[b] = bsz;
        bsz += n * n;
        st.o_a22[b] = asz;
        asz += r * r;
        st.o_inv[b] = asz;
        asz += r * r;
        st.o_x[b] = asz;
        asz += r * s;
        st.o_red[b] = nred;
        st.o_skel[b] = nskel;
        o_rows[b] = nred + nskel;
        nred += r;
        nskel += s;
      }
      red_all.resize(nred);
      skel_all.resize(nskel);
      rows_all.resize(nred + nskel);
      parallel_for(ncell, [&](int b) {
        const BlockInfo& bi = st.blocks[b];
        long long q = o_rows[b];
        for (size_t t = 0; t < bi.red_pos.size(); ++t) {
          const int g = bi.global[bi.red_pos[t]];
          red_all[st.o_red[b] + t] = g;
          rows_all[q++] = g;
        }
        for (size_t t = 0; t < bi.skel_pos.size(); ++t) {
          const int g = bi.global[bi.skel_pos[t]];
          skel_all[st.o_skel[b] + t] = g;
          rows_all[q++] = g;
        }
      });
      if (level == 0) {
        cell0.blocks = st.blocks;
        cell0.red_all = red_all;
        cell0.skel_all = skel_all;
        cell0.rows_all = rows_all;
        cell0.o_B = o_B;
        cell0.o_rows = o_rows;
        cell0.o_a22 = st.o_a22;
        cell0.o_inv = st.o_inv;
        cell0.o_x = st.o_x;
        cell0.o_red = st.o_red;
        cell0.o_skel = st.o_skel;
        cell0.bsz = bsz;
        cell0.asz = asz;
        cell0.cached = true;
      }
    }
    st.n_red = red_all.size();
    st.n_skel = skel_all.size();
    if (level > 0) start_face_partition(level, red_all);
    mark("schur index lists", level);
    t_host += wall() - th;

    track((bsz + asz) * 8);
    // this level's workspace: what it held (level - 2) is no longer read
    Arena& work = arena_work[level & 1];
    work.reset();
    cur_work = &work;
    t_scratch = &work;
    double* dB = work.alloc<double>(bsz);
    st.arena = arena_factor.alloc<double>(asz);
    BufList tmp;
    int* drows;
    if (cell0_hit && cell0.d_rows) {
      st.d_red = cell0.d_red;
      st.d_skel = cell0.d_skel;
      drows = cell0.d_rows;
    } else {
      st.d_red = arena_factor.upload(red_all, stream);
      st.d_skel = arena_factor.upload(skel_all, stream);
      drows = work.upload(rows_all, stream);
      if (cell0_hit) {
        cell0.d_red = keep_on_device(st.d_red, red_all.size());
        cell0.d_skel = keep_on_device(st.d_skel, skel_all.size());
        cell0.d_rows = keep_on_device(drows, rows_all.size());
      }
    }

    // gather every cell block
    double tg0 = wall();
    SourceDesc* d_sd;
    int *d_own, *d_dof;
    upload_sources(in, tmp, &d_sd, &d_own, &d_dof);
    std::vector<GatherTarget> tg(ncell);
    for (int b = 0; b < ncell; ++b) {
      const BlockInfo& bi = st.blocks[b];
      GatherTarget& g = tg[b];
      g.out = dB + o_B[b];
      g.ld = bi.global.size();
      g.rows = g.cols = drows + o_rows[b];
      g.a22_out = st.arena + st.o_a22[b];
      g.m = g.n = (int)bi.global.size();
      g.a0_skip = bi.r();  // the skeleton-skeleton stencil part stays in A0
      g.r = bi.r();
      g.mode = level == 0 ? 2 : 0;
      g.owner = b;
      g.allowA = g.allowB = -1;
    }
    mark("schur partition+upload", level);
    gather(tg, in, d_own, d_sd, d_dof, tmp);
    if (verbose && verbose_mode != 2) sync();
    t_gather += wall() - tg0;
    mark("schur gather", level);

    // sources consumed: free them once the gather has run (stream order)
    in.bufs.release(stream);

    // keep-Schur option: remember what was gathered on the skeleton block
    std::vector<double> side_all;
    if (keep_schur) {
      sync();
      for (int b = 0; b < ncell; ++b) {
        BlockInfo& bi = st.blocks[b];
        const int n = bi.global.size(), r = bi.r(), s = bi.s();
        bi.S.assign((size_t)s * s, 0.0);
        std::vector<double> full((size_t)n * n);
        HIF_CK(cudaMemcpy(full.data(), dB + o_B[b], full.size() * 8, cudaMemcpyDeviceToHost));
        for (int j = 0; j < s; ++j)
          for (int i = 0; i < s; ++i) bi.S[i + (size_t)j * s] = -full[(r + i) + (size_t)(r + j) * n];
      }
    }

    // eliminate
    double te0 = wall();
    std::vector<SweepDesc> sd;
    for (int b = 0; b < ncell; ++b) {
      const BlockInfo& bi = st.blocks[b];
      SweepDesc d{};
      d.B = dB + o_B[b];
      d.a22inv = st.arena + st.o_inv[b];
      d.X = st.arena + st.o_x[b];
      d.L = st.arena + st.o_a22[b];
      d.n = bi.global.size();
      d.r = bi.r();
      sd.push_back(d);
    }
    run_sweep(sd, tmp, st);
    if (verbose && verbose_mode != 2) sync();
    t_elim += wall() - te0;
    mark("schur eliminate", level);

    if (keep_schur) {
      sync();
      for (int b = 0; b < ncell; ++b) {
        BlockInfo& bi = st.blocks[b];
        const int n = bi.global.size(), r = bi.r(), s = bi.s();
        std::vector<double> full((size_t)n * n);
        HIF_CK(cudaMemcpy(full.data(), dB + o_B[b], full.size() * 8, cudaMemcpyDeviceToHost));
        for (int j = 0; j < s; ++j)
          for (int i = 0; i < s; ++i) bi.S[i + (size_t)j * s] += full[(r + i) + (size_t)(r + j) * n];
      }
    }

    // new sources T_c = B(skel, skel); membership by low / high face of the cell
    th = wall();
    const int cpd_next = cells_per_dir(level + 1);
    empty_sources(out, ncell);
    for (int b = 0; b < ncell; ++b) {
      const BlockInfo& bi = st.blocks[b];
      const int s = bi.s(), r = bi.r(), n = bi.global.size();
      if (s == 0) continue;
      const int id = (int)out.desc.size();
      out.desc.push_back(SourceDesc{dB + o_B[b] + r + (long long)r * n, (long long)n});
      const int ci = b / (cpd * cpd), cj = (b / cpd) % cpd, ck = b % cpd;
      const int parent = cpd_next > 0 ? ((ci / 2) * cpd_next + cj / 2) * cpd_next + ck / 2 : -1;
      out.owner.push_back(parent);
      out.cell_src[b] = id;
    }
    {
      std::vector<long long> off(st.o_skel.begin(), st.o_skel.end());
      off.push_back(st.n_skel);
      long long* d_off = tmp.add(upload(off, stream));
      int* d_src = tmp.add(upload(out.cell_src, stream));
      launch_member_cells(st.d_skel, d_off, d_src, ncell, cpd, w, NC, d_dof_src, stream);
      HIF_CK(cudaGetLastError());
    }
    // remove eliminated DOFs (UpdateRemainingDOFs, src/Factor.cpp:91-111)
    for (int p : red_all) rem[p] = 0;
    tmp.release(stream);
    if (level < L - 1) start_reduce_lists(st, skel_all);
    steps.push_back(std::move(st));
    t_host += wall() - th;
  }

  // ---- skeletonization phase (LevelFactorSkel, src/Factor.cpp:232-260) -----
  // SkelInteractionIndexData for every TOP / FRONT / LEFT face of the level
  // (src/Factor.cpp:645-755), over the given remaining-DOF mask.
  void partition_faces(int level, const uint8_t* mask, std::vector<BlockInfo>& blocks,
                       std::vector<std::vector<int>>& rows_l) const {
    const int cpd = cells_per_dir(level);
    Partitioner part{N, P, NC, mask};
    const int ncell = cpd * cpd * cpd;
    std::vector<std::vector<BlockInfo>> pb(ncell);
    std::vector<std::vector<std::vector<int>>> pr(ncell);
    parallel_for(ncell, [&](int idx) {
      const int c[3] = {idx / (cpd * cpd), (idx / cpd) % cpd, idx % cpd};
      std::vector<int> rw, cl;
      for (int face : {TOP, FRONT, LEFT}) {
        int nb[3];
        if (!part.skel_interaction(level, c, face, rw, cl, nb)) continue;
        if (cl.empty()) continue;
        BlockInfo b;
        b.face = face;
        b.global = std::move(cl);
        b.cell = idx;
        b.nbr = (nb[0] * cpd + nb[1]) * cpd + nb[2];
        pb[idx].push_back(std::move(b));
        pr[idx].push_back(std::move(rw));
        rw.clear();
        cl.clear();
      }
    });
    // cell order, merged in parallel into place
    std::vector<int> off(ncell + 1, 0);
    for (int idx = 0; idx < ncell; ++idx) off[idx + 1] = off[idx] + (int)pb[idx].size();
    const size_t base = blocks.size();
    blocks.resize(base + off[ncell]);
    rows_l.resize(base + off[ncell]);
    parallel_for(ncell, [&](int idx) {
      for (size_t q = 0; q < pb[idx].size(); ++q) {
        blocks[base + off[idx] + q] = std::move(pb[idx][q]);
        rows_l[base + off[idx] + q] = std::move(pr[idx][q]);
      }
    });
  }

  // The face partition of a level depends only on the DOFs left after that
  // level's cell eliminations, which are known once its cell partition is: it
  // runs on a host thread while the cell phase is assembled and eliminated.
  struct FacePartition {
    int level = -1;
    std::vector<uint8_t> mask;
    std::vector<BlockInfo> blocks;
    std::vector<std::vector<int>> rows_l;
    std::exception_ptr err;
  };
  FacePartition face_pre;
  std::thread face_thread;
  void start_face_partition(int level, const std::vector<int>& red) {
    join_face_partition();
    if (level >= L - 1) return;
    face_pre = FacePartition{};
    face_pre.level = level;
    face_pre.mask = rem;
    for (int p : red) face_pre.mask[p] = 0;
    face_thread = std::thread([this, level] {
      try {
        partition_faces(level, face_pre.mask.data(), face_pre.blocks, face_pre.rows_l);
      } catch (...) {
        face_pre.err = std::current_exception();
      }
    });
  }
  void join_face_partition() {
    if (face_thread.joinable()) face_thread.join();
  }
  // The next level's cell partition, built on a host thread while a
  // skeletonization phase runs on the device: over the DOFs left before that
  // phase, to be filtered by the ones it eliminates (take_cell_partition's
  // caller does that).
  struct CellPartition {
    int level = -1;
    std::vector<uint8_t> mask;
    std::vector<BlockInfo> blocks;
    std::exception_ptr err;
  };
  CellPartition cell_pre;
  std::thread cell_thread;
  void start_cell_partition(int level) {
    join_cell_partition();
    if (level >= L) return;
    cell_pre = CellPartition{};
    cell_pre.level = level;
    cell_pre.mask = rem;
    cell_thread = std::thread([this, level] {
      try {
        Partitioner part{N, P, NC, cell_pre.mask.data()};
        const int cpd = cells_per_dir(level);
        const int ncell = cpd * cpd * cpd;
        cell_pre.blocks.resize(ncell);
        parallel_for(ncell, [&](int idx) {
          const int c[3] = {idx / (cpd * cpd), (idx / cpd) % cpd, idx % cpd};
          BlockInfo& b = cell_pre.blocks[idx];
          part.cell_index(level, c, b.global, b.red_pos, b.skel_pos);
          b.cell = idx;
        });
      } catch (...) {
        cell_pre.err = std::current_exception();
      }
    });
  }
  void join_cell_partition() {
    if (cell_thread.joinable()) cell_thread.join();
  }
  bool take_cell_partition(int level, std::vector<BlockInfo>& blocks) {
    join_cell_partition();
    if (cell_pre.level != level) return false;
    cell_pre.level = -1;
    if (cell_pre.err) std::rethrow_exception(cell_pre.err);
    blocks = std::move(cell_pre.blocks);
    return true;
  }

  // Level 0's face partition depends on the grid alone: its DOF mask is the
  // initial one less every DOF strictly inside a level-0 cell (all three
  // coordinates interior to the cell width, src/Factor.cpp:314-320), which is
  // exactly what level 0's cell phase eliminates. It starts at once, so the
  // host thread builds it while the cell phase is assembled and eliminated.
  // Being the grid's alone, it is built once per handle: the first
  // factorization keeps it (face0_*); later ones copy its blocks on a host
  // thread while level 0's cell phase runs and read its row lists in place, so
  // the partition is not rebuilt and no partition loop competes with level 0's
  // host work for the worker pool.
  std::vector<BlockInfo> face0_blocks;
  std::vector<std::vector<int>> face0_rows;
  bool face0_cached = false;
  int* face0_didx = nullptr;  // its row and column lists on the device (read-only)
  void start_face_partition0() {
    join_face_partition();
    if (L <= 1) return;
    face_pre = FacePartition{};
    face_pre.level = 0;
    if (face0_cached) {
      // the factor keeps its own copy of the blocks (pivots and index sets are
      // added to them): made here, while level 0's cell phase runs
      face_thread = std::thread([this] {
        try {
          face_pre.blocks.resize(face0_blocks.size());
          parallel_for((int)face0_blocks.size(),
                       [&](int f) { face_pre.blocks[f] = face0_blocks[f]; });
        } catch (...) {
          face_pre.err = std::current_exception();
        }
      });
      return;
    }
    face_pre.mask = rem;
    face_thread = std::thread([this] {
      try {
        uint8_t* m = face_pre.mask.data();
        Partitioner part{N, P, NC, m};
        const int w = part.width(0);
        parallel_for(NC, [&](int k) {
          if (!part.interior(w, k)) return;
          for (int j = 1; j < NC; ++j) {
            if (!part.interior(w, j)) continue;
            for (int i = 1; i < NC; ++i)
              if (part.interior(w, i)) m[part.lin(i, j, k)] = 0;
          }
        });
        partition_faces(0, m, face_pre.blocks, face_pre.rows_l);
      } catch (...) {
        face_pre.err = std::current_exception();
      }
    });
  }
  // rows: set to the row lists to read (rows_l, or level 0's kept lists).
  bool take_face_partition(int level, std::vector<BlockInfo>& blocks,
                           std::vector<std::vector<int>>& rows_l,
                           const std::vector<std::vector<int>>** rows) {
    join_face_partition();
    if (face_pre.level != level) return false;
    face_pre.level = -1;
    if (face_pre.err) std::rethrow_exception(face_pre.err);
    if (level == 0) {
      if (face0_cached) {
        blocks = std::move(face_pre.blocks);
      } else {
        face0_blocks = std::move(face_pre.blocks);
        face0_rows = std::move(face_pre.rows_l);
        face0_cached = true;
        blocks.resize(face0_blocks.size());
        parallel_for((int)face0_blocks.size(), [&](int f) { blocks[f] = face0_blocks[f]; });
      }
      *rows = &face0_rows;
      return true;
    }
    blocks = std::move(face_pre.blocks);
    rows_l = std::move(face_pre.rows_l);
    *rows = &rows_l;
    return true;
  }

  void skel_phase(int level, Sources& cells, Sources& out) {
    double th = wall();
    const int cpd = cells_per_dir(level);
    StepData st;
    st.level = level;
    st.skel = true;
    st.chol = use_chol;
    st.cpd = cpd;
    std::vector<std::vector<int>> rows_own;
    const std::vector<std::vector<int>>* rows_p = &rows_own;
    std::vector<BlockInfo>& blocks = st.blocks;
    if (!take_face_partition(level, blocks, rows_own, &rows_p))
      partition_faces(level, rem.data(), blocks, rows_own);
    const std::vector<std::vector<int>>& rows_l = *rows_p;
    start_cell_partition(level + 1);
    mark("skel face partition", level);
    const int nf = (int)blocks.size();
    // M blocks (rows x cols) and ID workspace
    std::vector<long long> o_rows(nf), o_cols(nf), o_M(nf), o_W(nf), o_i(nf);
    long long msz = 0, wsz = 0, isz = 0, xsz = 0;
    int max_n = 0;
    for (int f = 0; f < nf; ++f) {
      const int m = rows_l[f].size(), n = blocks[f].global.size();
      if (m < n) throw Error{HIF_ERR_STATE, "face with fewer interaction rows than columns"};
      o_rows[f] = xsz;
      o_cols[f] = xsz + m;
      xsz += m + n;
      o_M[f] = msz;
      msz += (long long)m * n;
      o_W[f] = wsz;
      wsz += (long long)n * n / 4 + n + 1;
      o_i[f] = isz;
      isz += n;
      max_n = std::max(max_n, n);
    }
    // row and column lists of every face, filled in parallel
    // written straight into pinned staging memory: no host array to zero-fill
    // and page in, and no second copy before the upload. Level 0's are the
    // grid's alone: from a handle's second factorization on, the device copy
    // it keeps is read instead
    const bool face0_hit = rows_p == &face0_rows;
    const bool idx_kept = face0_hit && face0_didx != nullptr;
    int* idx_all = nullptr;
    if (!idx_kept) {
      idx_all = static_cast<int*>(stage.get(std::max<long long>(xsz, 1) * sizeof(int)));
      parallel_for(nf, [&](int f) {
        std::copy(rows_l[f].begin(), rows_l[f].end(), idx_all + o_rows[f]);
        std::copy(blocks[f].global.begin(), blocks[f].global.end(), idx_all + o_cols[f]);
      });
    }
    mark("skel index lists", level);
    t_host += wall() - th;

    BufList tmp;
    track((msz + wsz) * 8);
    Arena& work = arena_work[level & 1];
    cur_work = &work;
    t_scratch = &work;
    double* dM = work.alloc<double>(msz);
    double* dWs = work.alloc<double>(wsz);
    int* didx;
    if (idx_kept) {
      didx = face0_didx;
    } else {
      didx = tmp.add(desc_alloc<int>(xsz, stream));
      if (xsz)
        HIF_CK(cudaMemcpyAsync(didx, idx_all, xsz * sizeof(int), cudaMemcpyHostToDevice, stream));
      if (face0_hit) face0_didx = keep_on_device(didx, xsz);
    }
    int* d_jp = tmp.add(dalloc<int>(isz + 1, stream));
    int* d_keep = tmp.add(dalloc<int>(isz + 1, stream));
    int* d_rank = tmp.add(dalloc<int>(nf + 1, stream));
    double* d_rd = tmp.add(dalloc<double>(isz + 1, stream));

    double tg0 = wall();
    SourceDesc* d_sd;
    int *d_own, *d_dof;
    upload_sources(cells, tmp, &d_sd, &d_own, &d_dof);
    std::vector<GatherTarget> tg(nf);
    for (int f = 0; f < nf; ++f) {
      GatherTarget& g = tg[f];
      g.out = dM + o_M[f];
      g.m = rows_l[f].size();
      g.n = blocks[f].global.size();
      g.ld = g.m;
      g.rows = didx + o_rows[f];
      g.cols = didx + o_cols[f];
      g.a22_out = nullptr;
      g.a0_skip = INT_MAX;
      g.r = 0;
      g.mode = 1;
      g.owner = -1;
      g.allowA = cells.cell_src[blocks[f].cell];
      g.allowB = cells.cell_src[blocks[f].nbr];
    }
    mark("skel partition+upload", level);
    gather(tg, cells, d_own, d_sd, d_dof, tmp);
    if (verbose && verbose_mode != 2) sync();
    t_gather += wall() - tg0;
    mark("skel gather M", level);

    // interpolative decompositions
    double ti0 = wall();
    std::vector<int> orders;
    std::vector<long long> o_ord(nf, -1);
    auto rp = replay.find(level);
    if (rp != replay.end()) {
      if ((int)rp->second.size() != nf)
        throw Error{HIF_ERR_ARG, "replay pivots: face count differs"};
      for (int f = 0; f < nf; ++f) {
        if ((int)rp->second[f].size() != (int)blocks[f].global.size())
          throw Error{HIF_ERR_ARG, "replay pivots: face size differs"};
        o_ord[f] = orders.size();
        orders.insert(orders.end(), rp->second[f].begin(), rp->second[f].end());
      }
    }
    int* d_ord = orders.empty() ? nullptr : tmp.add(upload(orders, stream));
    // Tall faces are first reduced to their triangular factor R0 (n x n) by an
    // unpivoted blocked Householder QR; the pivoted QR of R0 makes the same
    // pivot choices and yields the same R as that of M in exact arithmetic
    // (both depend on M only through M^T M = R0^T R0).
    std::vector<double*> idM(nf);
    std::vector<int> idm(nf);
    for (int f = 0; f < nf; ++f) {
      idM[f] = dM + o_M[f];
      idm[f] = rows_l[f].size();
    }
    // mixed precision: tall faces go to the pivoted Cholesky ID instead (no
    // compression; replayed pivot orders keep the QR path). The Gram matrix
    // M^T M resolves a column's remaining norm only down to about sqrt(u) ||M||
    // = 1.5e-8 ||M||, so the rank test R_ii <= eps R_00 needs eps well above
    // that: below kGramMinEps the faces take the FP64 pivoted QR as in FP64 mode.
    const bool chol = precision == HIF_PRECISION_MIXED && d_ord == nullptr && eps >= kGramMinEps;
    if (!chol) compress_faces(blocks, rows_l, dM, o_M, idM, idm, tmp);
    mark("skel row compression", level);
    std::vector<IdDesc> idd(nf);
    for (int f = 0; f < nf; ++f) {
      IdDesc& d = idd[f];
      d.M = idM[f];
      d.order = d_ord ? d_ord + o_ord[f] : nullptr;
      d.jpvt = d_jp + o_i[f];
      d.rdiag = d_rd + o_i[f];
      d.keep = d_keep + o_i[f];
      d.rank = d_rank + f;
      d.W = dWs + o_W[f];
      d.m = idm[f];
      d.n = blocks[f].global.size();
    }
    // small faces: one CTA each (k_id); compressed faces: grouped ID, several
    // CTAs per face for the largest ones
    std::vector<IdDesc> small_id, chol_id;
    std::vector<IdGroupDesc> g1, gbig;
    int small_n = 0, g1_m = 0, g1_n = 0, big_m = 0, big_n = 0;
    for (int f = 0; f < nf; ++f) {
      const bool compressed = idM[f] != dM + o_M[f];
      const int n = idd[f].n;
      if (chol && n > gram_min_n && idd[f].m > n) {
        chol_id.push_back(idd[f]);
        continue;
      }
      if (!compressed) {
        small_id.push_back(idd[f]);
        small_n = std::max(small_n, n);
        continue;
      }
      IdGroupDesc gd{};
      gd.id = idd[f];
      (n >= kGroupMinN ? gbig : g1).push_back(gd);
      if (n >= kGroupMinN) {
        big_m = std::max(big_m, idd[f].m);
        big_n = std::max(big_n, n);
      } else {
        g1_m = std::max(g1_m, idd[f].m);
        g1_n = std::max(g1_n, n);
      }
    }
    const int group = gbig.empty() ? 1 : std::max(1, std::min(16, 148 / (int)gbig.size()));
    auto scratch_for = [&](std::vector<IdGroupDesc>& v, int grp) {
      long long nd = 0, ni = 0;
      for (const IdGroupDesc& g : v) nd += 2LL * g.id.n + grp + 2;
      ni = 64LL * v.size();
      double* dsc = tmp.add(dalloc<double>(nd, stream));
      int* isc = tmp.add(dalloc<int>(ni, stream));
      HIF_CK(cudaMemsetAsync(isc, 0, ni * sizeof(int), stream));
      long long od = 0;
      for (size_t q = 0; q < v.size(); ++q) {
        v[q].norms = dsc + od;
        v[q].cand = dsc + od + 2LL * v[q].id.n;
        v[q].tau = dsc + od + 2LL * v[q].id.n + grp;
        od += 2LL * v[q].id.n + grp + 2;
        v[q].sync = isc + 64 * q;
      }
    };
    double idfl = 0;
    for (const IdDesc& d : idd) idfl += 4.0 * d.m * d.n * d.n - 4.0 / 3.0 * d.n * d.n * (double)d.n;
    if (!small_id.empty()) {
      IdDesc* d_idd = tmp.add(upload(small_id, stream));
      long long max_mn = 0;
      for (const IdDesc& d : small_id) max_mn = std::max(max_mn, (long long)d.m * d.n);
      timed(HIF_KCLASS_ID, idfl, 0, [&] {
        launch_id(d_idd, (int)small_id.size(), small_n, eps, d_status, stream, max_mn);
      });
      idfl = 0;
    }
    if (!chol_id.empty()) id_cholesky(chol_id, tmp);
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<IdGroupDesc>& v = pass == 0 ? g1 : gbig;
      if (v.empty()) continue;
      const int grp = pass == 0 ? 1 : group;
      scratch_for(v, grp);
      IdGroupDesc* dg = tmp.add(upload(v, stream));
      cudaError_t le = cudaSuccess;
      timed(HIF_KCLASS_ID, idfl, 0, [&] {
        le = launch_id_group(dg, (int)v.size(), grp, eps, d_status, stream,
                             pass == 0 ? g1_m : big_m, pass == 0 ? g1_n : big_n);
      });
      idfl = 0;
      if (le != cudaSuccess)
        throw Error{HIF_ERR_CUDA, std::string("grouped ID launch: ") + cudaGetErrorString(le)};
    }
    HIF_CK(cudaGetLastError());
    // pivots, kept flags and |R_ii| read back into pinned staging: the copies
    // run at full link speed right after the IDs, and no host array is
    // zero-filled first
    int* h_jp = static_cast<int*>(stage.get((isz + 1) * sizeof(int)));
    int* h_keep = static_cast<int*>(stage.get((isz + 1) * sizeof(int)));
    double* h_rd = static_cast<double*>(stage.get((isz + 1) * sizeof(double)));
    HIF_CK(cudaMemcpyAsync(h_jp, d_jp, isz * sizeof(int), cudaMemcpyDeviceToHost, stream));
    HIF_CK(cudaMemcpyAsync(h_keep, d_keep, isz * sizeof(int), cudaMemcpyDeviceToHost, stream));
    HIF_CK(cudaMemcpyAsync(h_rd, d_rd, isz * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    t_id += wall() - ti0;
    mark("skel pivoted QR", level);

    // skeleton / redundant sets (InterpDecomp.cpp:102-110), internal order
    th = wall();
    std::vector<int>& red_all = h_red_all;
    std::vector<int>& skel_all = h_skel_all;
    std::vector<int>& rows2 = h_rows_all;
    std::vector<long long> o_B(nf), o_r2(nf);
    long long bsz = 0, asz = 0;
    st.o_a22.resize(nf);
    st.o_inv.resize(nf);
    st.o_x.resize(nf);
    st.o_w.resize(nf);
    st.o_red.resize(nf);
    st.o_skel.resize(nf);
    parallel_for(nf, [&](int f) {
      BlockInfo& b = blocks[f];
      const int n = b.global.size();
      b.jpvt.assign(h_jp + o_i[f], h_jp + o_i[f] + n);
      b.rdiag.assign(h_rd + o_i[f], h_rd + o_i[f] + n);
      int k = 0;
      for (int i = 0; i < n; ++i) k += h_keep[o_i[f] + i] != 0;
      b.skel_pos.reserve(k);
      b.red_pos.reserve(n - k);
      for (int i = 0; i < n; ++i) {
        if (h_keep[o_i[f] + i]) b.skel_pos.push_back(b.jpvt[i]);
        else b.red_pos.push_back(b.jpvt[i]);
      }
    });
    long long nred = 0, nskel = 0;
    for (int f = 0; f < nf; ++f) {
      const BlockInfo& b = blocks[f];
      const int n = b.global.size();
      const long long r = b.r(), k = b.s();
      o_B[f] = bsz;
      bsz += (long long)n * n;
      st.o_a22[f] = asz;
      asz += r * r;
      st.o_inv[f] = asz;
      asz += r * r;
      st.o_x[f] = asz;
      asz += r * k;
      st.o_w[f] = asz;
      asz += k * r;
      st.o_red[f] = nred;
      st.o_skel[f] = nskel;
      o_r2[f] = nred + nskel;
      nred += r;
      nskel += k;
    }
    red_all.resize(nred);
    skel_all.resize(nskel);
    rows2.resize(nred + nskel);
    parallel_for(nf, [&](int f) {
      const BlockInfo& b = blocks[f];
      long long q = o_r2[f];
      for (size_t t = 0; t < b.red_pos.size(); ++t) {
        const int g = b.global[b.red_pos[t]];
        red_all[st.o_red[f] + t] = g;
        rows2[q++] = g;
      }
      for (size_t t = 0; t < b.skel_pos.size(); ++t) {
        const int g = b.global[b.skel_pos[t]];
        skel_all[st.o_skel[f] + t] = g;
        rows2[q++] = g;
      }
    });
    st.n_red = red_all.size();
    st.n_skel = skel_all.size();
    mark("skel ID index lists", level);
    t_host += wall() - th;

    track((bsz + asz) * 8);
    double* dB = work.alloc<double>(bsz);
    st.arena = arena_factor.alloc<double>(asz);
    st.d_red = arena_factor.upload(red_all, stream);
    st.d_skel = arena_factor.upload(skel_all, stream);
    int* drows2 = work.upload(rows2, stream);

    // A_ff in [red | skel] order (SchurAfterID, src/Factor.cpp:113-153)
    tg0 = wall();
    std::vector<GatherTarget> tg2;
    std::vector<int> act;
    for (int f = 0; f < nf; ++f) {
      const BlockInfo& b = blocks[f];
      if (b.r() == 0) continue;
      act.push_back(f);
      GatherTarget g{};
      g.out = dB + o_B[f];
      g.m = g.n = b.global.size();
      g.ld = g.m;
      g.rows = g.cols = drows2 + o_r2[f];
      g.a22_out = nullptr;
      g.a0_skip = INT_MAX;
      g.r = 0;
      g.mode = 1;
      g.owner = -1;
      g.allowA = cells.cell_src[b.cell];
      g.allowB = cells.cell_src[b.nbr];
      tg2.push_back(g);
    }
    gather(tg2, cells, d_own, d_sd, d_dof, tmp);
    if (verbose && verbose_mode != 2) sync();
    t_gather += wall() - tg0;
    mark("skel gather A_ff", level);

    // rotation by the ID: B(red,:) -= W^T B(skel,:); B(:,red) -= B(:,skel) W; B(skel,skel) = 0
    te_rot_and_sweep(st, act, dB, o_B, dWs, o_W, tmp);
    mark("skel rotate+eliminate", level);

    // keep-Schur: S_f = B(skel, skel) after the sweep
    if (keep_schur) {
      sync();
      for (int f : act) {
        BlockInfo& b = blocks[f];
        const int n = b.global.size(), r = b.r(), k = b.s();
        std::vector<double> full((size_t)n * n);
        HIF_CK(cudaMemcpy(full.data(), dB + o_B[f], full.size() * 8, cudaMemcpyDeviceToHost));
        b.S.assign((size_t)k * k, 0.0);
        for (int j = 0; j < k; ++j)
          for (int i = 0; i < k; ++i) b.S[i + (size_t)j * k] = full[(r + i) + (size_t)(r + j) * n];
      }
    }

    // new sources: S_f of faces that eliminated something
    th = wall();
    const int cpd_next = cells_per_dir(level + 1);
    // cell memberships stay (T_c are still live): slots 0-3 of d_dof_src
    out.desc = cells.desc;
    out.owner = cells.owner;
    out.cell_src = cells.cell_src;
    std::vector<long long> mo;
    std::vector<int> mc, ms;
    for (int f : act) {
      const BlockInfo& b = blocks[f];
      const int r = b.r(), k = b.s(), n = b.global.size();
      if (k == 0) continue;
      const int id = (int)out.desc.size();
      out.desc.push_back(SourceDesc{dB + o_B[f] + r + (long long)r * n, (long long)n});
      const int ci = b.cell / (cpd * cpd), cj = (b.cell / cpd) % cpd, ck = b.cell % cpd;
      out.owner.push_back(((ci / 2) * cpd_next + cj / 2) * cpd_next + ck / 2);
      mo.push_back(st.o_skel[f]);
      mc.push_back(k);
      ms.push_back(id);
    }
    if (!mo.empty()) {
      long long* d_mo = tmp.add(upload(mo, stream));
      int* d_mc = tmp.add(upload(mc, stream));
      int* d_ms = tmp.add(upload(ms, stream));
      launch_member_faces(st.d_skel, d_mo, d_mc, d_ms, (int)mo.size(), n3, d_dof_src, stream);
      HIF_CK(cudaGetLastError());
    }
    // T_c buffers move to the output set; add this phase's B
    out.bufs.p = cells.bufs.p;
    cells.bufs.p.clear();
    for (int p : red_all) rem[p] = 0;
    tmp.release(stream);
    steps.push_back(std::move(st));
    t_host += wall() - th;
  }

  // ID of the tall faces in mixed precision: G = M^T M (FP64 product), then a
  // pivoted Cholesky of G by panels of kPcholNB steps (one CTA per face per
  // panel, the trailing G updated by an FP64 product after each panel) until
  // R_ii <= eps R_00, then W = R11^{-1} R12 by blocks of kTrsmNB rows. Pivot
  // choices equal column-pivoted QR's in exact arithmetic (InterpDecomp.cpp:
  // 86-138); the skeleton test is the reference's |R_ii| > eps |R_00|.
  static constexpr int kPcholNB = 32;
  static constexpr double kGramMinEps = 1e-7;
  // mixed precision: faces wider than this (and taller than wide) take the
  // Gram-matrix ID; narrower ones the one-CTA pivoted QR (HIF_OPT_GRAM_MIN_N)
  int gram_min_n = 32;
  int gram_slices = 0;  // HIF_OPT_GRAM_SLICES
  void id_cholesky(const std::vector<IdDesc>& v, BufList& tmp) {
    Arena& work = *cur_work;
    const int nd = (int)v.size();
    long long gsz = 0, isz = 0;
    int max_n = 0;
    for (const IdDesc& d : v) {
      gsz += (long long)d.n * d.n;
      isz += 2LL * d.n;
      max_n = std::max(max_n, d.n);
    }
    double* G = work.alloc<double>(gsz);
    double* R = work.alloc<double>(gsz);
    int* ibuf = work.alloc<int>(isz + 2LL * nd);
    double* d0 = work.alloc<double>(nd);
    HIF_CK(cudaMemsetAsync(ibuf + isz, 0, 2 * nd * sizeof(int), stream));
    std::vector<PcholDesc> pd(nd);
    std::vector<GemmDesc> gram;
    long long og = 0, oi = 0;
    for (int q = 0; q < nd; ++q) {
      const IdDesc& d = v[q];
      PcholDesc& p = pd[q];
      p.G = G + og;
      p.R = R + og;
      p.chosen = ibuf + oi;
      p.piv = ibuf + oi + d.n;
      p.info = ibuf + isz + 2 * q;
      p.d0 = d0 + q;
      p.id = d;
      og += (long long)d.n * d.n;
      oi += 2LL * d.n;
      GemmDesc g{};  // G = M^T M
      g.C = p.G;
      g.ldc = d.n;
      g.A = d.M;
      g.lda = d.m;
      g.B = d.M;
      g.ldb = d.m;
      g.m = g.n = d.n;
      g.k = d.m;
      g.transA = 1;
      g.alpha = 1.0;
      g.beta = 0.0;
      g.lower = 1;  // G is symmetric: the panels read its lower triangle only
      gram.push_back(g);
    }
    auto tm = [&](int cls, double fl, double by, auto&& f, int n) { timed(cls, fl, by, f, n); };
    // G in FP64 on DMMA, or (HIF_OPT_GRAM_SLICES) from int8 slices: with 8
    // slices the product's error, about k 2^-56 max|M|^2, is below an FP64
    // product's k u |M|^2 bound, so the pivots and rank see FP64 accuracy
    if (gram_slices > 0) gemm_batch_int8(gram, tmp, stream, tm, gram_slices, d_status);
    else gemm_batch(gram, tmp, stream, HIF_KCLASS_QR, tm, 128);
    PcholDesc* dpd = tmp.add(upload(pd, stream));
    // a fixed sequence of panels without host synchronisation: a face whose
    // rank is known skips its later panels and updates on the device
    std::vector<int> info(2 * nd);
    for (int i0 = 0; i0 < max_n; i0 += kPcholNB) {
      std::vector<int> active;
      std::vector<GemmDesc> upd;
      for (int q = 0; q < nd; ++q) {
        const int n = pd[q].id.n;
        if (n <= i0) continue;
        active.push_back(q);
        if (n <= i0 + kPcholNB) continue;  // no columns left after this panel
        GemmDesc g{};  // G -= Y Y^T, Y = the panel's rows of R as an n x nb matrix
        g.C = pd[q].G;
        g.ldc = n;
        g.A = pd[q].R + (long long)i0 * n;
        g.lda = n;
        g.B = g.A;
        g.ldb = n;
        g.transB = 1;
        g.m = g.n = n;
        g.k = kPcholNB;
        g.alpha = -1.0;
        g.beta = 1.0;
        g.lower = 1;
        g.skip = pd[q].info + 1;
        upd.push_back(g);
      }
      BufList step;
      int* da = step.add(upload(active, stream));
      timed(HIF_KCLASS_ID, 0, 0, [&] {
        launch_pchol_panel(dpd, da, (int)active.size(), i0, kPcholNB, eps, max_n, d_status,
                           stream);
      });
      HIF_CK(cudaGetLastError());
      gemm_batch(upd, step, stream, HIF_KCLASS_ID, tm, 128);
      HIF_CK(cudaGetLastError());
      step.release(stream);
    }
    HIF_CK(cudaMemcpyAsync(info.data(), ibuf + isz, 2 * nd * sizeof(int), cudaMemcpyDeviceToHost,
                           stream));
    sync();
    timed(HIF_KCLASS_ID, 0, 0, [&] { launch_pchol_finish(dpd, nd, max_n, stream); });
    HIF_CK(cudaGetLastError());
    // W := R11^{-1} R12, diagonal blocks from the bottom, products above them
    int kmax = 0;
    for (int q = 0; q < nd; ++q) kmax = std::max(kmax, info[2 * q]);
    for (int b = 0; b * kTrsmNB < kmax; ++b) {
      std::vector<TrsmBlockDesc> tb;
      std::vector<GemmDesc> up;
      int maxc = 0;
      for (int q = 0; q < nd; ++q) {
        const int k = info[2 * q], nc = pd[q].id.n - k;
        const int a1 = k - b * kTrsmNB, a0 = std::max(0, a1 - kTrsmNB);
        if (a1 <= 0 || nc <= 0) continue;
        tb.push_back(TrsmBlockDesc{pd[q].G, pd[q].id.W, k, nc, a0, a1});
        maxc = std::max(maxc, nc);
        if (a0 > 0) {
          GemmDesc g{};
          g.C = pd[q].id.W;
          g.ldc = k;
          g.A = pd[q].G + (long long)a0 * k;
          g.lda = k;
          g.B = pd[q].id.W + a0;
          g.ldb = k;
          g.m = a0;
          g.n = nc;
          g.k = a1 - a0;
          g.alpha = -1.0;
          g.beta = 1.0;
          up.push_back(g);
        }
      }
      if (tb.empty()) continue;
      BufList step;
      TrsmBlockDesc* dtb = step.add(upload(tb, stream));
      timed(HIF_KCLASS_ID, 0, 0, [&] { launch_trsm_block(dtb, (int)tb.size(), maxc, stream); });
      gemm_batch(up, step, stream, HIF_KCLASS_ID, tm);
      HIF_CK(cudaGetLastError());
      step.release(stream);
    }
  }

  // Blocked Householder row compression of the faces with more than
  // kCompressMinN columns: on return idM[f] / idm[f] point at R0 (n x n, ld n).
  // Two levels of blocking: kQrNB2-column outer panels, each factored by
  // kQrNB-column sub-panels that update only the rest of the outer panel; the
  // columns right of the outer panel get one compact-WY update with all of its
  // kQrNB2 reflectors (T from V^T V).
  static constexpr int kCompressMinN = 64;
  int kGroupMinN = 512;  // faces this wide get a CTA group (HIF_OPT_ID_GROUP_MIN_N)
  void compress_faces(const std::vector<BlockInfo>& blocks,
                      const std::vector<std::vector<int>>& rows_l, double* dM,
                      const std::vector<long long>& o_M, std::vector<double*>& idM,
                      std::vector<int>& idm, BufList& tmp) {
    std::vector<int> list;
    long long vsz = 0, wsz = 0, rsz = 0;
    int maxn = 0;
    for (size_t f = 0; f < blocks.size(); ++f) {
      const int n = blocks[f].global.size(), m = rows_l[f].size();
      if (n > kCompressMinN && m > n) {
        list.push_back(f);
        vsz += (long long)m * kQrNB2;
        wsz += (long long)kQrNB2 * n;
        rsz += (long long)n * n;
        maxn = std::max(maxn, n);
      }
    }
    if (list.empty()) return;
    Arena& work = *cur_work;
    const size_t nl = list.size();
    double* V = work.alloc<double>(vsz);
    double* Tm = work.alloc<double>(nl * kQrNB * kQrNB);
    double* T2 = work.alloc<double>(nl * kQrNB2 * kQrNB2);
    double* Wv = work.alloc<double>(nl * kQrNB2 * kQrNB2);
    double* tau = work.alloc<double>(nl * kQrNB2);
    double* Z = work.alloc<double>(wsz);
    double* Z2 = work.alloc<double>(wsz);
    double* R0 = work.alloc<double>(rsz);
    std::vector<QrDesc> qd;
    std::vector<long long> o_w, o_r;
    long long ov = 0, ow = 0, orr = 0;
    for (size_t q = 0; q < nl; ++q) {
      const int f = list[q];
      const int n = blocks[f].global.size(), m = rows_l[f].size();
      qd.push_back(QrDesc{dM + o_M[f], V + ov, Tm + (long long)q * kQrNB * kQrNB,
                          tau + (long long)q * kQrNB2, m, n});
      o_w.push_back(ow);
      o_r.push_back(orr);
      ov += (long long)m * kQrNB2;
      ow += (long long)kQrNB2 * n;
      orr += (long long)n * n;
    }
    QrDesc* dq = tmp.add(upload(qd, stream));
    const int qr_cap = qr_cluster_max_rows();
    if (verbose) {
      long long sm = 0, sn = 0;
      int mm = 0, mn = 0, ncl = 0;
      for (const QrDesc& d : qd) {
        sm += d.m;
        sn += d.n;
        mm = std::max(mm, d.m);
        mn = std::max(mn, d.n);
        ncl += d.m <= qr_cap;
      }
      std::fprintf(stderr,
                   "[hif]     compression: %zu faces, m avg %lld max %d, n avg %lld max %d, "
                   "cluster rows cap %d (%d faces fit from the first panel)\n",
                   qd.size(), sm / (long long)qd.size(), mm, sn / (long long)qd.size(), mn, qr_cap,
                   ncl);
    }
    auto tm = [&](int cls, double fl, double by, auto&& f, int n) { timed(cls, fl, by, f, n); };
    // C (rows k.. of columns c0..c1) -= V T^T V^T C with V the kb reflectors at
    // V + voff (ld m), T ld ldt: three products
    auto wy_update = [&](std::vector<GemmDesc>& g1, std::vector<GemmDesc>& g2,
                         std::vector<GemmDesc>& g3, size_t q, const double* Vq, const double* Tq,
                         int ldt, int k, int kb, int c0, int c1) {
      const QrDesc& d = qd[q];
      const int mt = d.m - k, nt = c1 - c0;
      if (nt <= 0 || kb <= 0) return;
      double* C = d.M + k + (long long)c0 * d.m;
      GemmDesc a{};  // Z = V^T C
      a.C = Z + o_w[q];
      a.A = Vq;
      a.B = C;
      a.ldc = kQrNB2;
      a.lda = d.m;
      a.ldb = d.m;
      a.m = kb;
      a.n = nt;
      a.k = mt;
      a.transA = 1;
      a.alpha = 1.0;
      a.beta = 0.0;
      g1.push_back(a);
      GemmDesc t{};  // Z2 = T^T Z
      t.C = Z2 + o_w[q];
      t.A = Tq;
      t.B = Z + o_w[q];
      t.ldc = kQrNB2;
      t.lda = ldt;
      t.ldb = kQrNB2;
      t.m = kb;
      t.n = nt;
      t.k = kb;
      t.transA = 1;
      t.alpha = 1.0;
      t.beta = 0.0;
      g2.push_back(t);
      GemmDesc c{};  // C -= V Z2
      c.C = C;
      c.A = Vq;
      c.B = Z2 + o_w[q];
      c.ldc = d.m;
      c.lda = d.m;
      c.ldb = kQrNB2;
      c.m = mt;
      c.n = nt;
      c.k = kb;
      c.alpha = -1.0;
      c.beta = 1.0;
      g3.push_back(c);
    };
    for (int k0 = 0; k0 < maxn; k0 += kQrNB2) {
      // sub-panels of the outer panel, each applied to the rest of the panel
      for (int k1 = k0; k1 < std::min(maxn, k0 + kQrNB2); k1 += kQrNB) {
        std::vector<int> act, actc;  // single-CTA / cluster panels
        int maxc = 0;
        std::vector<GemmDesc> g1, g2, g3;
        for (size_t q = 0; q < nl; ++q) {
          const QrDesc& d = qd[q];
          if (d.n <= k1) continue;
          if (d.m - k1 <= qr_cap) {
            actc.push_back(q);
            maxc = std::max(maxc, d.m - k1);
          } else {
            act.push_back(q);
          }
          const int kb = std::min(kQrNB, d.n - k1);
          const double* Vq = d.V + (long long)(k1 - k0) * d.m + k1;
          wy_update(g1, g2, g3, q, Vq, d.T, kQrNB, k1, kb, k1 + kb, std::min(d.n, k0 + kQrNB2));
        }
        BufList step;
        if (!act.empty()) {
          int* da = step.add(upload(act, stream));
          timed(HIF_KCLASS_QR, 0, 0,
                [&] { launch_qr_panel(dq, da, (int)act.size(), k1, k0, stream); });
        }
        if (!actc.empty()) {
          int* dc = step.add(upload(actc, stream));
          timed(HIF_KCLASS_QR, 0, 0, [&] {
            launch_qr_panel_cluster(dq, dc, (int)actc.size(), k1, k0, maxc, stream);
          });
        }
        gemm_batch(g1, step, stream, HIF_KCLASS_QR, tm);
        gemm_batch(g2, step, stream, HIF_KCLASS_QR, tm);
        gemm_batch(g3, step, stream, HIF_KCLASS_QR, tm);
        HIF_CK(cudaGetLastError());
        step.release(stream);
      }
      // outer panel: T from V^T V, then one update of the trailing columns
      std::vector<GemmDesc> gw, g1, g2, g3;
      std::vector<TFactorDesc> tf;
      for (size_t q = 0; q < nl; ++q) {
        const QrDesc& d = qd[q];
        const int nb = std::min(kQrNB2, d.n - k0);
        if (nb <= 0 || d.n <= k0 + kQrNB2) continue;
        const double* Vq = d.V + k0;
        double* Wq = Wv + (long long)q * kQrNB2 * kQrNB2;
        double* Tq = T2 + (long long)q * kQrNB2 * kQrNB2;
        GemmDesc w{};  // W = V^T V
        w.C = Wq;
        w.A = Vq;
        w.B = Vq;
        w.ldc = kQrNB2;
        w.lda = w.ldb = d.m;
        w.m = w.n = nb;
        w.k = d.m - k0;
        w.transA = 1;
        w.alpha = 1.0;
        w.beta = 0.0;
        gw.push_back(w);
        tf.push_back(TFactorDesc{Wq, d.tau, Tq, nb});
        wy_update(g1, g2, g3, q, Vq, Tq, kQrNB2, k0, nb, k0 + nb, d.n);
      }
      if (tf.empty()) continue;
      BufList step;
      gemm_batch(gw, step, stream, HIF_KCLASS_QR, tm);
      TFactorDesc* dtf = step.add(upload(tf, stream));
      timed(HIF_KCLASS_QR, 0, 0, [&] { launch_qr_tfactor(dtf, (int)tf.size(), stream); });
      gemm_batch(g1, step, stream, HIF_KCLASS_QR, tm);
      gemm_batch(g2, step, stream, HIF_KCLASS_QR, tm);
      gemm_batch(g3, step, stream, HIF_KCLASS_QR, tm);
      HIF_CK(cudaGetLastError());
      step.release(stream);
    }
    std::vector<TriuDesc> td;
    for (size_t q = 0; q < qd.size(); ++q) {
      const int f = list[q], n = qd[q].n;
      td.push_back(TriuDesc{qd[q].M, R0 + o_r[q], qd[q].m, n, n});
      idM[f] = R0 + o_r[q];
      idm[f] = n;
    }
    TriuDesc* dtd = tmp.add(upload(td, stream));
    timed(HIF_KCLASS_QR, 0, 0, [&] { launch_triu(dtd, (int)td.size(), stream); });
    HIF_CK(cudaGetLastError());
  }

  void te_rot_and_sweep(StepData& st, const std::vector<int>& act, double* dB,
                        const std::vector<long long>& o_B, double* dWs,
                        const std::vector<long long>& o_W, BufList& tmp) {
    double te0 = wall();
    std::vector<GemmDesc> g1, g2, g3;
    std::vector<int> t1(1, 0), t2(1, 0), t3(1, 0);
    std::vector<CopyDesc> cw, ca;
    std::vector<int> tw(1, 0), ta(1, 0);
    for (int f : act) {
      const BlockInfo& b = st.blocks[f];
      const int n = b.global.size(), r = b.r(), k = b.s();
      double* B = dB + o_B[f];
      const double* W = dWs + o_W[f];
      if (k > 0) {
        GemmDesc a{};
        a.C = B;
        a.A = W;
        a.B = B + r;
        a.ldc = n;
        a.lda = k;
        a.ldb = n;
        a.m = r;
        a.n = n;
        a.k = k;
        a.transA = 1;
        a.alpha = -1.0;
        a.beta = 1.0;
        g1.push_back(a);
        t1.push_back(t1.back() + dgemm_tiles(a.m, a.n));
        GemmDesc c{};
        c.C = B;
        c.A = B + (long long)r * n;
        c.B = W;
        c.ldc = n;
        c.lda = n;
        c.ldb = k;
        c.m = n;
        c.n = r;
        c.k = k;
        c.alpha = -1.0;
        c.beta = 1.0;
        g2.push_back(c);
        t2.push_back(t2.back() + dgemm_tiles(c.m, c.n));
        GemmDesc z{};
        z.C = B + r + (long long)r * n;
        z.A = z.B = B;
        z.ldc = n;
        z.lda = z.ldb = n;
        z.m = k;
        z.n = k;
        z.k = 0;
        z.alpha = 0.0;
        z.beta = 0.0;
        g3.push_back(z);
        t3.push_back(t3.back() + dgemm_tiles(k, k));
        cw.push_back(CopyDesc{W, st.arena + st.o_w[f], k, k, k, r});
        tw.push_back(tw.back() + copy_tiles(k, r));
      }
      ca.push_back(CopyDesc{B, st.arena + st.o_a22[f], n, r, r, r});
      ta.push_back(ta.back() + copy_tiles(r, r));
    }
    auto run_gemm = [&](std::vector<GemmDesc>& g, std::vector<int>&) {
      gemm_batch(g, tmp, stream, HIF_KCLASS_GEMM,
                 [&](int cls, double fl, double by, auto&& f, int n) { timed(cls, fl, by, f, n); });
    };
    auto run_copy = [&](std::vector<CopyDesc>& c, std::vector<int>& t) {
      if (c.empty()) return;
      CopyDesc* d = tmp.add(upload(c, stream));
      int* to = tmp.add(upload(t, stream));
      timed(HIF_KCLASS_COPY, 0, 0, [&] { launch_copy(d, to, (int)c.size(), t.back(), stream); });
      HIF_CK(cudaGetLastError());
    };
    run_gemm(g1, t1);
    run_gemm(g2, t2);
    run_gemm(g3, t3);
    run_copy(cw, tw);
    run_copy(ca, ta);
    std::vector<SweepDesc> sd;
    for (int f : act) {
      const BlockInfo& b = st.blocks[f];
      SweepDesc d{};
      d.B = dB + o_B[f];
      d.a22inv = st.arena + st.o_inv[f];
      d.X = st.arena + st.o_x[f];
      d.L = st.arena + st.o_a22[f];
      d.n = b.global.size();
      d.r = b.r();
      sd.push_back(d);
    }
    run_sweep(sd, tmp, st);
    if (verbose && verbose_mode != 2) sync();
    t_elim += wall() - te0;
  }

  // ---- Factor (src/Factor.cpp:41-63) --------------------------------------
  PinnedStage stage;  // host staging of this handle's factorization uploads
  GemmTuner tuner;
  bool autotune = false;
  // HIF_PRECISION_MIXED: int8 slices of the Schur products (0: split TF32) and
  // of the X products (0: FP64)
  int schur_slices = 5, x_slices = 7, y_slices = 6, chol_slices = 7;
  // host index lists of the phase being built, kept across phases and
  // factorizations
  std::vector<int> h_red_all, h_skel_all, h_rows_all;
  // HIF_OPT_ELIMINATION, and the choice made for the factorization in progress
  int elimination = HIF_ELIM_AUTO;
  bool use_chol = false;
  struct StageScope {
    PinnedStage* prev;
    Arena* prev_scratch;
    GemmTuner* prev_tuner;
    Arena* prev_desc;
    StageScope(PinnedStage* s, GemmTuner* tu, Arena* desc)
        : prev(t_stage), prev_scratch(t_scratch), prev_tuner(t_tuner), prev_desc(t_desc) {
      t_stage = s;
      t_tuner = tu;
      t_desc = desc;
    }
    ~StageScope() {
      t_stage = prev;
      t_scratch = prev_scratch;
      t_tuner = prev_tuner;
      t_desc = prev_desc;
    }
  };

  void factor() {
    if (!have_op) throw Error{HIF_ERR_STATE, "no operator: call hif_setup_stencil first"};
    // the previous factorization ended with a synchronisation: its staged
    // copies are complete
    sync();
    stage.reset();
    StageScope scope(&stage, autotune ? &tuner : nullptr, &arena_desc);
    join_face_partition();
    face_pre.level = -1;
    join_cell_partition();
    cell_pre.level = -1;
    if (partition == HIF_PARTITION_CLIPPED && NC % P != 0)
      throw Error{HIF_ERR_ARG, "clipped partition needs (N+1) divisible by P"};
    initialize();
    // the previous factorization's descriptors (its apply plans included) were
    // dropped with it, after the synchronisation above: nothing on the device
    // uses the arenas now
    arena_factor.consolidate();
    arena_work[0].consolidate();
    arena_work[1].consolidate();
    arena_desc.consolidate();
    start_face_partition0();
    // Cholesky elimination for symmetric operators: by default in mixed
    // precision; the FP64 default keeps the reference's explicit inverse
    // (getrf + getri, include/Schur.hpp:86)
    if (elimination == HIF_ELIM_CHOLESKY && !symmetric)
      throw Error{HIF_ERR_ARG, "Cholesky elimination needs a symmetric operator "
                               "(hif_setup_stencil_faces)"};
    use_chol = symmetric && (elimination == HIF_ELIM_CHOLESKY ||
                             (elimination == HIF_ELIM_AUTO && precision == HIF_PRECISION_MIXED));
    t_total = t_gather = t_elim = t_id = t_host = 0;
    cur_bytes = peak_bytes = 0;
    HIF_CK(cudaMemsetAsync(d_status, 0, 4 * sizeof(int), stream));
    const double t0 = wall();
    mark_t = 0;
    mark("start", -1);
    Sources a, b;
    empty_sources(a, 0);
    for (int level = 0; level < L; ++level) {
      const double tl = wall();
      schur_phase(level, a, b);
      if (level < L - 1) {
        skel_phase(level, b, a);
      } else {
        b.bufs.release(stream);
      }
      if (verbose && verbose_mode != 2) {
        sync();
        std::fprintf(stderr, "[hif] level %d: %.3f ms\n", level, 1e3 * (wall() - tl));
      }
    }
    mark("end", L);
    // The apply sweeps are part of the factorization's output. Their plans
    // depend on the index data and the factor's addresses only, all known on
    // the host now: they are built while the device finishes the last levels.
    const double tp = wall();
    ensure_workspace(1);
    t_plan = wall() - tp;
    sync();
    t_total = wall() - t0;
    tuner.resolve();
    report_marks();
    if (verbose) std::fprintf(stderr, "[hif]   apply plans built in %.3f ms (host)\n", 1e3 * t_plan);
    int st = 0;
    HIF_CK(cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost));
    factored = true;
    factor_precision = precision;
    if (st & kStatusTinyPivot) throw Error{HIF_ERR_SINGULAR, "zero or non-finite pivot"};
    if (st & kStatusTimeout)
      throw Error{HIF_ERR_CUDA, "a bounded device wait timed out (grouped ID barrier or tensor-core "
                                "pipeline)"};
    if (profile) resolve_profile();
  }

  // ---- Apply (src/Factor.cpp:992-1081) ------------------------------------
  // Builds the launch list of one sweep. Matrices: X (r x s, ld r),
  // W (k x r, ld k), A22 / A22^{-1} (r x r, ld r).
  long long plan_key = 0;  // stage key for the next launches added to a plan
  void add_gemv(ApplyPlan& plan, const StepData& st, int which, int trans, bool in_red,
                bool out_red, double alpha, int mode, int in_vec, int out_vec, int tri = 0) {
    const long long my_key = plan_key++;  // taken even when the launch is empty
    std::vector<GemvDesc> dd;
    double mbytes = 0;
    for (size_t b = 0; b < st.blocks.size(); ++b) {
      const BlockInfo& bi = st.blocks[b];
      const int r = bi.r(), s = bi.s();
      if (r == 0 || (which < 2 && s == 0)) continue;
      GemvDesc g{};
      if (which == 0) {  // X: r x s
        g.M = st.arena + st.o_x[b];
        g.ld = r;
        g.m = r;
        g.n = s;
      } else if (which == 1) {  // W: k x r
        g.M = st.arena + st.o_w[b];
        g.ld = s;
        g.m = s;
        g.n = r;
      } else {  // 2: A22, 3: A22^{-1}
        g.M = st.arena + (which == 2 ? st.o_a22[b] : st.o_inv[b]);
        g.ld = r;
        g.m = r;
        g.n = r;
      }
      g.in_idx = in_red ? st.d_red + st.o_red[b] : st.d_skel + st.o_skel[b];
      g.out_idx = out_red ? st.d_red + st.o_red[b] : st.d_skel + st.o_skel[b];
      g.trans = trans;
      g.tri = tri;
      g.alpha = alpha;
      g.mode = mode;
      g.contrib = (mode == 1) ? d_contrib + st.o_skel[b] : nullptr;
      mbytes += 8.0 * g.m * g.n;
      dd.push_back(g);
    }
    if (dd.empty()) return;
    ApplyLaunch l;
    l.type = 0;
    l.bytes = mbytes;
    l.nd = dd.size();
    l.in_vec = in_vec;
    l.out_vec = out_vec;
    l.d_desc = plan.bufs.add(upload(dd, stream));
    int big = 0;
    for (const GemvDesc& g : dd) big = std::max(big, std::max(g.m, g.n));
    if (big <= kGemvSmallMax) {
      l.layout = kGemvSmall;
      l.units = (int)dd.size();
    } else {
      l.layout = kGemvTiles;
      std::vector<int2> tab;
      for (size_t q = 0; q < dd.size(); ++q) {
        const int nt = gemv_tile_count(dd[q].m, dd[q].n, trans);
        for (int t = 0; t < nt; ++t) tab.push_back(make_int2((int)q, t));
      }
      l.units = (int)tab.size();
      l.d_tab = plan.bufs.add(upload(tab, stream));
    }
    l.d_seg = plan.bufs.add(upload(std::vector<GemvFastSeg>{{l.d_desc, l.d_tab}}, stream));
    l.d_segoff = plan.bufs.add(upload(std::vector<int>{0, l.units}, stream));
    l.hdesc = std::move(dd);
    l.key = my_key;
    plan.launches.push_back(std::move(l));
  }

  // A22 = L L^T, A22^{-1} = L^{-T} L^{-1} or X = L^{-T} Y (which 0 / 1 / 2) of
  // block b of a Cholesky phase, formed on the device, copied to `out`.
  void chol_readback(const StepData& st, int b, int which, double* out) {
    const BlockInfo& bi = st.blocks[b];
    const int r = bi.r(), k = bi.s();
    const int ncol = which == 2 ? k : r;
    BufList tmp;
    double* C = tmp.add(dalloc<double>((size_t)r * ncol, stream));
    GemmDesc g{};
    g.C = C;
    g.ldc = r;
    g.m = r;
    g.n = ncol;
    g.k = r;
    g.alpha = 1.0;
    g.lda = g.ldb = r;
    if (which == 0) {
      g.A = g.B = st.arena + st.o_a22[b];
      g.transB = 1;
    } else {
      g.A = st.arena + st.o_inv[b];
      g.transA = 1;
      g.B = which == 1 ? st.arena + st.o_inv[b] : st.arena + st.o_x[b];
    }
    std::vector<GemmDesc> v(1, g);
    gemm_batch(v, tmp, stream, HIF_KCLASS_GEMM,
               [&](int, double, double, auto&& f, int = 1) { f(); }, 128);
    HIF_CK(cudaGetLastError());
    sync();
    HIF_CK(cudaMemcpy(out, C, (size_t)r * ncol * 8, cudaMemcpyDeviceToHost));
    tmp.release(stream);
    sync();
  }

  // Host part of a Schur phase's reduction lists: every skeleton DOF of the
  // level (blocks with redundant DOFs, in block order) with its contribution
  // slots. Computed on a worker thread while the factorization goes on (the
  // inputs are the phase's skeleton DOF list, its offsets and which blocks
  // eliminate anything), so that the plans at the end only upload them.
  struct ReduceHost {
    std::vector<int> dof, off, slot;
  };
  static ReduceHost reduce_host(long long n3, std::vector<int> skel_all,
                                std::vector<long long> o_skel, std::vector<char> has_r) {
    ReduceHost h;
    std::vector<int> head(n3, -1), cnt;
    const size_t nb = o_skel.size();
    auto range = [&](size_t b) {
      const long long a = o_skel[b];
      const long long e = b + 1 < nb ? o_skel[b + 1] : (long long)skel_all.size();
      return std::make_pair(a, e);
    };
    for (size_t b = 0; b < nb; ++b) {
      if (!has_r[b]) continue;
      const auto re = range(b);
      for (long long t = re.first; t < re.second; ++t) {
        const int p = skel_all[t];
        if (head[p] < 0) {
          head[p] = (int)h.dof.size();
          h.dof.push_back(p);
          cnt.push_back(0);
        }
        ++cnt[head[p]];
      }
    }
    if (h.dof.empty()) return h;
    h.off.assign(h.dof.size() + 1, 0);
    for (size_t d = 0; d < h.dof.size(); ++d) h.off[d + 1] = h.off[d] + cnt[d];
    h.slot.resize(h.off.back());
    std::vector<int> cur(h.off.begin(), h.off.end() - 1);
    for (size_t b = 0; b < nb; ++b) {
      if (!has_r[b]) continue;
      const auto re = range(b);
      for (long long t = re.first; t < re.second; ++t) h.slot[cur[head[skel_all[t]]]++] = (int)t;
    }
    return h;
  }
  std::map<int, std::future<ReduceHost>> reduce_pending;  // Schur phase level -> lists
  void start_reduce_lists(const StepData& st, const std::vector<int>& skel_all) {
    std::vector<char> has_r(st.blocks.size());
    for (size_t b = 0; b < st.blocks.size(); ++b) has_r[b] = st.blocks[b].r() > 0;
    reduce_pending[st.level] = std::async(std::launch::async, reduce_host, n3, skel_all,
                                          st.o_skel, std::move(has_r));
  }

  // Reduction lists of a Schur phase (every skeleton DOF of the level with its
  // contribution slots, in block order), built once per phase and shared by
  // both plans.
  struct ReduceLists {
    int* d_dof = nullptr;
    int* d_off = nullptr;
    int* d_slot = nullptr;
    int ndof = 0;
  };
  std::map<const StepData*, ReduceLists> reduce_lists;
  std::vector<int> reduce_head;  // n3, all -1 between uses
  BufList reduce_bufs;

  const ReduceLists& reduce_lists_for(const StepData& st) {
    auto it = reduce_lists.find(&st);
    if (it != reduce_lists.end()) return it->second;
    auto pend = reduce_pending.find(st.level);
    if (!st.skel && pend != reduce_pending.end() && pend->second.valid()) {
      ReduceHost h = pend->second.get();
      reduce_pending.erase(pend);
      ReduceLists rl;
      if (!h.dof.empty()) {
        rl.d_dof = reduce_bufs.add(upload(h.dof, stream));
        rl.d_off = reduce_bufs.add(upload(h.off, stream));
        rl.d_slot = reduce_bufs.add(upload(h.slot, stream));
        rl.ndof = (int)h.dof.size();
      }
      return reduce_lists.emplace(&st, rl).first->second;
    }
    if ((long long)reduce_head.size() != n3) reduce_head.assign(n3, -1);
    std::vector<int>& head = reduce_head;
    std::vector<int> dof, cnt;
    for (size_t b = 0; b < st.blocks.size(); ++b) {
      const BlockInfo& bi = st.blocks[b];
      if (bi.r() == 0) continue;
      for (int t = 0; t < bi.s(); ++t) {
        const int p = bi.global[bi.skel_pos[t]];
        if (head[p] < 0) {
          head[p] = (int)dof.size();
          dof.push_back(p);
          cnt.push_back(0);
        }
        ++cnt[head[p]];
      }
    }
    ReduceLists rl;
    if (!dof.empty()) {
      std::vector<int> off(dof.size() + 1, 0);
      for (size_t d = 0; d < dof.size(); ++d) off[d + 1] = off[d] + cnt[d];
      std::vector<int> slot(off.back()), cur(off.begin(), off.end() - 1);
      for (size_t b = 0; b < st.blocks.size(); ++b) {
        const BlockInfo& bi = st.blocks[b];
        if (bi.r() == 0) continue;
        for (int t = 0; t < bi.s(); ++t) {
          const int p = bi.global[bi.skel_pos[t]];
          slot[cur[head[p]]++] = (int)(st.o_skel[b] + t);
        }
      }
      rl.d_dof = reduce_bufs.add(upload(dof, stream));
      rl.d_off = reduce_bufs.add(upload(off, stream));
      rl.d_slot = reduce_bufs.add(upload(slot, stream));
      rl.ndof = (int)dof.size();
    }
    for (int p : dof) head[p] = -1;
    return reduce_lists.emplace(&st, rl).first->second;
  }

  void add_reduce(ApplyPlan& plan, const StepData& st, double alpha, int vec) {
    const long long my_key = plan_key++;
    const ReduceLists& rl = reduce_lists_for(st);
    if (rl.ndof == 0) return;
    ApplyLaunch l;
    l.type = 1;
    l.d_dof = rl.d_dof;
    l.d_off = rl.d_off;
    l.d_slot = rl.d_slot;
    l.ndof = rl.ndof;
    l.alpha = alpha;
    l.out_vec = vec;
    l.key = my_key;
    plan.launches.push_back(l);
  }

  // Contribution buffer: max over phases of the skeleton slots, times the
  // right-hand-side capacity; GEMV descriptors point into it directly.
  long long contrib_ld = 1;
  int contrib_cap = 0;

  void build_plans(int nrhs_cap) {
    release_plans();
    long long max_slots = 1;
    for (const StepData& st : steps) max_slots = std::max(max_slots, st.n_skel);
    contrib_ld = max_slots;
    dfree(d_contrib, stream);
    d_contrib = dalloc<double>(max_slots * nrhs_cap, stream);
    contrib_cap = nrhs_cap;
    plan_inv.contrib_slots = plan_fwd.contrib_slots = max_slots;
    // index steps by (level, kind)
    std::vector<const StepData*> sch(L, nullptr), skl(L, nullptr);
    for (const StepData& st : steps) (st.skel ? skl : sch)[st.level] = &st;
    // Stage keys: forward sweeps (segment 0, level ascending), diagonal
    // (segment 1), backward sweeps (segment 2, level descending); within a
    // stage the launch order. Every operator's own launch order is increasing in
    // key, so launches of several operators with equal keys can share a launch.
    auto key = [](int seg, int lev, int sub) {
      return ((long long)seg << 32) | ((long long)lev << 8) | sub;
    };
    // Vectors: 0 = ua (input, forward sweeps), 1 = ub (output, backward
    // sweeps), 2 = uc. A Gauss-Jordan phase (A22^{-1}, X) follows
    // src/Factor.cpp:992-1081: forward u_s -= X^T u_r, diagonal u_r = A22^{-1} u_r
    // (ua -> ub), backward u_r -= X u_s. A Cholesky phase (L, L^{-1}, Y) splits
    // A22^{-1} = L^{-T} L^{-1} around the sweeps: forward v_r = L^{-1} u_r
    // (ua -> uc), u_s -= Y^T v_r; backward v_r -= Y u_s (uc), u_r = L^{-T} v_r
    // (uc -> ub); no diagonal step (the top phase, which has no skeleton, does
    // both triangles there). Each phase's redundant entries of uc are its own.
    // inverse
    {
      ApplyPlan& p = plan_inv;
      for (int l = 0; l < L - 1; ++l) {
        if (sch[l]) {
          plan_key = key(0, l, 0);
          if (sch[l]->chol) {
            add_gemv(p, *sch[l], 3, 0, true, true, 1.0, 2, 0, 2, 1);
            add_gemv(p, *sch[l], 0, 1, true, false, 1.0, 1, 2, 0);
          } else {
            add_gemv(p, *sch[l], 0, 1, true, false, 1.0, 1, 0, 0);
          }
          add_reduce(p, *sch[l], -1.0, 0);
        }
        if (skl[l]) {
          plan_key = key(0, l, 4);
          add_gemv(p, *skl[l], 1, 1, false, true, -1.0, 0, 0, 0);
          if (skl[l]->chol) {
            add_gemv(p, *skl[l], 3, 0, true, true, 1.0, 2, 0, 2, 1);
            add_gemv(p, *skl[l], 0, 1, true, false, -1.0, 0, 2, 0);
          } else {
            add_gemv(p, *skl[l], 0, 1, true, false, -1.0, 0, 0, 0);
          }
        }
      }
      for (int l = 0; l < L; ++l) {
        for (const StepData* st : {sch[l], skl[l]}) {
          if (!st) continue;
          plan_key = key(1, l, st->skel ? 4 : 0);
          if (!st->chol) {
            add_gemv(p, *st, 3, 0, true, true, 1.0, 2, 0, 1);
          } else if (l == L - 1) {
            add_gemv(p, *st, 3, 0, true, true, 1.0, 2, 0, 2, 1);
            add_gemv(p, *st, 3, 1, true, true, 1.0, 2, 2, 1, 1);
          }
        }
      }
      for (int l = L - 2; l >= 0; --l) {
        if (skl[l]) {
          plan_key = key(2, 255 - l, 0);
          if (skl[l]->chol) {
            add_gemv(p, *skl[l], 0, 0, false, true, -1.0, 0, 1, 2);
            add_gemv(p, *skl[l], 3, 1, true, true, 1.0, 2, 2, 1, 1);
          } else {
            add_gemv(p, *skl[l], 0, 0, false, true, -1.0, 0, 1, 1);
          }
          add_gemv(p, *skl[l], 1, 0, true, false, -1.0, 0, 1, 1);
        }
        plan_key = key(2, 255 - l, 4);
        if (sch[l]) {
          if (sch[l]->chol) {
            add_gemv(p, *sch[l], 0, 0, false, true, -1.0, 0, 1, 2);
            add_gemv(p, *sch[l], 3, 1, true, true, 1.0, 2, 2, 1, 1);
          } else {
            add_gemv(p, *sch[l], 0, 0, false, true, -1.0, 0, 1, 1);
          }
        }
      }
    }
    // forward (F u). Gauss-Jordan phase: u_r += X u_s, u_r = A22 u_r, u_s += X^T u_r.
    // Cholesky phase, F = [L 0; Y^T I] [I 0; 0 S] [L^T Y; 0 I]: w_r = L^T u_r + Y u_s
    // (ua -> uc), then u_s += Y^T w_r and u_r = L w_r (uc -> ub).
    {
      ApplyPlan& p = plan_fwd;
      for (int l = 0; l < L - 1; ++l) {
        if (sch[l]) {
          if (sch[l]->chol) {
            add_gemv(p, *sch[l], 2, 1, true, true, 1.0, 2, 0, 2, 1);
            add_gemv(p, *sch[l], 0, 0, false, true, 1.0, 0, 0, 2);
          } else {
            add_gemv(p, *sch[l], 0, 0, false, true, 1.0, 0, 0, 0);
          }
        }
        if (skl[l]) {
          add_gemv(p, *skl[l], 1, 0, true, false, 1.0, 0, 0, 0);
          if (skl[l]->chol) {
            add_gemv(p, *skl[l], 2, 1, true, true, 1.0, 2, 0, 2, 1);
            add_gemv(p, *skl[l], 0, 0, false, true, 1.0, 0, 0, 2);
          } else {
            add_gemv(p, *skl[l], 0, 0, false, true, 1.0, 0, 0, 0);
          }
        }
      }
      for (int l = 0; l < L; ++l) {
        for (const StepData* st : {sch[l], skl[l]}) {
          if (!st) continue;
          if (!st->chol) {
            add_gemv(p, *st, 2, 0, true, true, 1.0, 2, 0, 1);
          } else if (l == L - 1) {
            add_gemv(p, *st, 2, 1, true, true, 1.0, 2, 0, 2, 1);
            add_gemv(p, *st, 2, 0, true, true, 1.0, 2, 2, 1, 1);
          }
        }
      }
      for (int l = L - 2; l >= 0; --l) {
        if (skl[l]) {
          if (skl[l]->chol) {
            add_gemv(p, *skl[l], 0, 1, true, false, 1.0, 0, 2, 1);
            add_gemv(p, *skl[l], 2, 0, true, true, 1.0, 2, 2, 1, 1);
          } else {
            add_gemv(p, *skl[l], 0, 1, true, false, 1.0, 0, 1, 1);
          }
          add_gemv(p, *skl[l], 1, 1, false, true, 1.0, 0, 1, 1);
        }
        if (sch[l]) {
          if (sch[l]->chol) {
            add_gemv(p, *sch[l], 0, 1, true, false, 1.0, 1, 2, 1);
            add_reduce(p, *sch[l], 1.0, 1);
            add_gemv(p, *sch[l], 2, 0, true, true, 1.0, 2, 2, 1, 1);
          } else {
            add_gemv(p, *sch[l], 0, 1, true, false, 1.0, 1, 1, 1);
            add_reduce(p, *sch[l], 1.0, 1);
          }
        }
      }
    }
    plans_built = true;
  }

  void ensure_workspace(int nrhs) {
    if (!plans_built || contrib_cap < nrhs) build_plans(std::max(nrhs, contrib_cap));
    if (ws_nrhs >= nrhs && d_ua) return;
    drop_graphs();
    dfree(d_ua, stream);
    dfree(d_ub, stream);
    dfree(d_uc, stream);
    d_ua = dalloc<double>(n3 * nrhs, stream);
    d_ub = dalloc<double>(n3 * nrhs, stream);
    d_uc = dalloc<double>(n3 * nrhs, stream);
    ws_nrhs = nrhs;
  }

  void run_plan(ApplyPlan& plan, int nrhs) {
    double* vec[3] = {d_ua, d_ub, d_uc};
    for (ApplyLaunch& l : plan.launches) {
      if (l.type == 0) {
        const double by = l.bytes * ((nrhs + 3) / 4);
        timed(HIF_KCLASS_GEMV, 2.0 * l.bytes / 8 * nrhs, by, [&] {
          launch_gemv_fast(l.d_seg, l.d_segoff, 1, l.units, l.layout, vec[l.in_vec],
                           vec[l.out_vec], nrhs, n3, contrib_ld, stream);
        });
      } else {
        timed(HIF_KCLASS_VECTOR, 0, 0, [&] {
          launch_reduce_scatter(l.d_dof, l.d_off, l.d_slot, d_contrib, l.ndof, contrib_ld,
                                l.alpha, vec[l.out_vec], nrhs, n3, stream);
        });
      }
      HIF_CK(cudaGetLastError());
    }
  }

  void apply_device(double* du, int nrhs, long long ldu, bool inverse) {
    if (!factored) throw Error{HIF_ERR_STATE, "Apply before Factor"};
    if (nrhs <= 0 || ldu < n3) throw Error{HIF_ERR_ARG, "bad nrhs / ldu"};
    ensure_workspace(nrhs);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(d_ua + c * n3, du + c * ldu, n3 * 8, cudaMemcpyDeviceToDevice,
                             stream));
    ApplyPlan& plan = inverse ? plan_inv : plan_fwd;
    GemmPlan* gp = nrhs >= kGemmApplyMinRhs ? &gemm_plan(plan, inverse ? 1 : 0, nrhs) : nullptr;
    auto sweep = [&] {
      timed(HIF_KCLASS_VECTOR, 0, 8.0 * n3 * nrhs,
            [&] { launch_zero_boundary(d_ua, NC, nrhs, n3, stream); });
      HIF_CK(cudaMemsetAsync(d_ub, 0, n3 * nrhs * 8, stream));
      if (gp) run_gemm_plan(plan, *gp, nrhs);
      else run_plan(plan, nrhs);
    };
    if (profile) {
      sweep();  // per-launch events: no graph
    } else {
      const std::pair<int, int> key(inverse ? 1 : 0, nrhs);
      auto it = apply_graphs.find(key);
      if (it == apply_graphs.end()) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        HIF_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
          sweep();
        } catch (...) {
          cudaStreamEndCapture(stream, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        HIF_CK(cudaStreamEndCapture(stream, &g));
        const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        HIF_CK(ie);
        it = apply_graphs.emplace(key, ge).first;
      }
      HIF_CK(cudaGraphLaunch(it->second, stream));
    }
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(du + c * ldu, d_ub + c * n3, n3 * 8, cudaMemcpyDeviceToDevice,
                             stream));
  }

  // ---- PCG with the inverse apply as preconditioner -----------------------
  void solve_pcg_device(const double* db, double* dx, int nrhs, long long ld, double tol,
                        int maxit, int* iters, double* relres) {
    if (!factored) throw Error{HIF_ERR_STATE, "solve before Factor"};
    if (nrhs <= 0 || ld < n3) throw Error{HIF_ERR_ARG, "bad nrhs / ld"};
    if (pcg_nrhs < nrhs) {
      dfree(d_pcg, stream);
      d_pcg = dalloc<double>(5 * n3 * nrhs + 8 * nrhs + (size_t)kDotBlocks * nrhs, stream);
      pcg_nrhs = nrhs;
    }
    double* r = d_pcg;
    double* z = r + n3 * nrhs;
    double* p = z + n3 * nrhs;
    double* q = p + n3 * nrhs;
    double* x = q + n3 * nrhs;
    double* sc = x + n3 * nrhs;  // rz, rz_new, pq, rr, bb
    double* rz = sc;
    double* rz_new = sc + nrhs;
    double* pq = sc + 2 * nrhs;
    double* rr = sc + 3 * nrhs;
    double* bb = sc + 4 * nrhs;
    double* part = sc + 8 * nrhs;
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(r + c * n3, db + c * ld, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    const double vb = 8.0 * n3 * nrhs;
    timed(HIF_KCLASS_VECTOR, 0, vb, [&] { launch_zero_boundary(r, NC, nrhs, n3, stream); });
    HIF_CK(cudaMemsetAsync(x, 0, n3 * nrhs * 8, stream));
    timed(HIF_KCLASS_VECTOR, 0, vb, [&] { launch_dot(r, r, n3, nrhs, n3, part, bb, stream); }, 2);
    // z = M r
    auto precond = [&](double* in, double* outv) {
      if (outv != in)
        HIF_CK(cudaMemcpyAsync(outv, in, n3 * nrhs * 8, cudaMemcpyDeviceToDevice, stream));
      apply_device(outv, nrhs, n3, true);
    };
    precond(r, z);
    HIF_CK(cudaMemcpyAsync(p, z, n3 * nrhs * 8, cudaMemcpyDeviceToDevice, stream));
    timed(HIF_KCLASS_VECTOR, 0, 2 * vb, [&] { launch_dot(r, z, n3, nrhs, n3, part, rz, stream); }, 2);
    std::vector<double> h_bb(nrhs), h_rr(nrhs);
    HIF_CK(cudaMemcpyAsync(h_bb.data(), bb, nrhs * 8, cudaMemcpyDeviceToHost, stream));
    sync();
    std::vector<int> done(nrhs, 0);
    for (int c = 0; c < nrhs; ++c) {
      iters[c] = 0;
      relres[c] = h_bb[c] > 0 ? 1.0 : 0.0;
      if (h_bb[c] == 0) done[c] = 1;
    }
    for (int it = 1; it <= maxit; ++it) {
      bool all = true;
      for (int c = 0; c < nrhs; ++c) all = all && done[c];
      if (all) break;
      timed(HIF_KCLASS_VECTOR, 13.0 * n3 * nrhs, 9 * vb,
            [&] { launch_stencil_apply(d_band, NC, p, q, nrhs, n3, 0, stream); });
      timed(HIF_KCLASS_VECTOR, 0, 2 * vb, [&] { launch_dot(p, q, n3, nrhs, n3, part, pq, stream); }, 2);
      timed(HIF_KCLASS_VECTOR, 0, 6 * vb,
            [&] { launch_pcg_update_xr(x, r, p, q, rz, pq, n3, nrhs, n3, stream); });
      timed(HIF_KCLASS_VECTOR, 0, vb, [&] { launch_dot(r, r, n3, nrhs, n3, part, rr, stream); }, 2);
      HIF_CK(cudaMemcpyAsync(h_rr.data(), rr, nrhs * 8, cudaMemcpyDeviceToHost, stream));
      sync();
      bool all_now = true;
      for (int c = 0; c < nrhs; ++c) {
        if (done[c]) continue;
        relres[c] = std::sqrt(h_rr[c] / h_bb[c]);
        iters[c] = it;
        if (relres[c] <= tol) done[c] = 1;
        all_now = all_now && done[c];
      }
      if (all_now) break;
      precond(r, z);
      timed(HIF_KCLASS_VECTOR, 0, 2 * vb,
            [&] { launch_dot(r, z, n3, nrhs, n3, part, rz_new, stream); }, 2);
      timed(HIF_KCLASS_VECTOR, 0, 3 * vb,
            [&] { launch_pcg_update_p(p, z, rz_new, rz, n3, nrhs, n3, stream); });
      HIF_CK(cudaMemcpyAsync(rz, rz_new, nrhs * 8, cudaMemcpyDeviceToDevice, stream));
      HIF_CK(cudaGetLastError());
    }
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(dx + c * ld, x + c * n3, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    sync();
  }
};

#include "hif_factor_io.inl"
#include "hif_gmres.inl"

}  // namespace hif

// ===========================================================================
// C ABI
// ===========================================================================
struct hif_factor_s {
  std::unique_ptr<hif::Engine> e;
};

namespace {

template <class F>
int guarded(F&& f) {
  try {
    f();
    return HIF_OK;
  } catch (const hif::Error& e) {
    hif::g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    hif::g_last_error = "host allocation failed";
    return HIF_ERR_NOMEM;
  } catch (const std::exception& e) {
    hif::g_last_error = e.what();
    return HIF_ERR_CUDA;
  }
}

hif::StepData* find_step(hif_handle h, int level, int kind) {
  for (hif::StepData& s : h->e->steps)
    if (s.level == level && (int)s.skel == kind) return &s;
  return nullptr;
}

}  // namespace

extern "C" {

const char* hif_last_error(void) { return hif::g_last_error.c_str(); }

int hif_create(int N, int P, double epsilon, int partition, hif_handle* out) {
  if (!out || N < 1 || P < 1 || !(epsilon > 0) ||
      (partition != HIF_PARTITION_REFERENCE && partition != HIF_PARTITION_CLIPPED)) {
    hif::g_last_error = "hif_create: invalid argument";
    return HIF_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    hif::g_last_error = "no CUDA device";
    return HIF_ERR_NODEVICE;
  }
  return guarded([&] {
    auto* h = new hif_factor_s;
    try {
      h->e.reset(new hif::Engine(N, P, epsilon, partition));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int hif_destroy(hif_handle h) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] { delete h; });
}

int hif_set_stream(hif_handle h, void* stream) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] {
    h->e->sync();
    h->e->stream = stream ? static_cast<cudaStream_t>(stream) : h->e->own_stream;
  });
}

int hif_setup_stencil_device(hif_handle h, int N, double hstep, const double* dA,
                             const double* dV) {
  if (!h || !dA || !dV || N != h->e->N || !(hstep > 0)) return HIF_ERR_ARG;
  return guarded([&] { h->e->setup_node_device(dA, dV, hstep); });
}

int hif_setup_stencil(hif_handle h, int N, double hstep, const double* A, const double* V) {
  if (!h || !A || !V || N != h->e->N || !(hstep > 0)) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    const long long nt = (long long)(N + 2) * (N + 2) * (N + 2);
    double* dA = hif::upload_host(A, nt, e.stream);
    double* dV = hif::upload_host(V, nt, e.stream);
    e.setup_node_device(dA, dV, hstep);
    hif::dfree(dA, e.stream);
    hif::dfree(dV, e.stream);
    e.sync();
  });
}

int hif_setup_stencil_faces(hif_handle h, int N, double hstep, const double* ax,
                            const double* ay, const double* az, const double* V) {
  if (!h || !ax || !ay || !az || !V || N != h->e->N || !(hstep > 0)) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    const long long nt = (long long)(N + 2) * (N + 2) * (N + 2);
    double* dx = hif::upload_host(ax, nt, e.stream);
    double* dy = hif::upload_host(ay, nt, e.stream);
    double* dz = hif::upload_host(az, nt, e.stream);
    double* dv = hif::upload_host(V, nt, e.stream);
    hif::launch_setup_faces(dx, dy, dz, dv, N, hstep, e.d_band, e.stream);
    HIF_CK(cudaGetLastError());
    hif::dfree(dx, e.stream);
    hif::dfree(dy, e.stream);
    hif::dfree(dz, e.stream);
    hif::dfree(dv, e.stream);
    e.have_op = true;
    e.symmetric = true;
    e.sync();
  });
}

int hif_setup_stencil_faces_device(hif_handle h, int N, double hstep, const double* dax,
                                   const double* day, const double* daz, const double* dV) {
  if (!h || !dax || !day || !daz || !dV || N != h->e->N || !(hstep > 0)) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    e.timed(HIF_KCLASS_VECTOR, 0, 11.0 * 8 * e.n3, [&] {
      hif::launch_setup_faces(dax, day, daz, dV, N, hstep, e.d_band, e.stream);
    });
    HIF_CK(cudaGetLastError());
    e.have_op = true;
    e.symmetric = true;
  });
}

int hif_initialize(hif_handle h) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] { h->e->initialize(); });
}

int hif_factor(hif_handle h) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] { h->e->factor(); });
}

int hif_save_factor(hif_handle h, const char* path) {
  if (!h || !path || !*path) return HIF_ERR_ARG;
  return guarded([&] { hif::save_factor(*h->e, path); });
}

int hif_load_factor(hif_handle h, const char* path) {
  if (!h || !path || !*path) return HIF_ERR_ARG;
  return guarded([&] { hif::load_factor(*h->e, path); });
}

int hif_apply_device(hif_handle h, double* du, int nrhs, long long ldu, int apply_inverse) {
  if (!h || !du) return HIF_ERR_ARG;
  return guarded([&] { h->e->apply_device(du, nrhs, ldu, apply_inverse != 0); });
}

int hif_apply(hif_handle h, double* u, int nrhs, long long ldu, int apply_inverse) {
  if (!h || !u || nrhs <= 0) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    if (ldu < e.n3) throw hif::Error{HIF_ERR_ARG, "ldu < (N+1)^3"};
    double* d = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(d + c * e.n3, u + c * ldu, e.n3 * 8, cudaMemcpyHostToDevice, e.stream));
    e.apply_device(d, nrhs, e.n3, apply_inverse != 0);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(u + c * ldu, d + c * e.n3, e.n3 * 8, cudaMemcpyDeviceToHost, e.stream));
    hif::dfree(d, e.stream);
    e.sync();
  });
}

int hif_spmv_device(hif_handle h, const double* dx, double* dy, int nrhs, long long ld,
                    int transpose) {
  if (!h || !dx || !dy || nrhs <= 0) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    if (!e.have_op) throw hif::Error{HIF_ERR_STATE, "no operator"};
    if (ld < e.n3) throw hif::Error{HIF_ERR_ARG, "ld < (N+1)^3"};
    hif::launch_stencil_apply(e.d_band, e.NC, dx, dy, nrhs, ld, transpose, e.stream);
    HIF_CK(cudaGetLastError());
  });
}

int hif_spmv(hif_handle h, const double* x, double* y, int nrhs, long long ld, int transpose) {
  if (!h || !x || !y || nrhs <= 0) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    if (!e.have_op) throw hif::Error{HIF_ERR_STATE, "no operator"};
    if (ld < e.n3) throw hif::Error{HIF_ERR_ARG, "ld < (N+1)^3"};
    double* dx = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    double* dy = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(dx + c * e.n3, x + c * ld, e.n3 * 8, cudaMemcpyHostToDevice, e.stream));
    hif::launch_stencil_apply(e.d_band, e.NC, dx, dy, nrhs, e.n3, transpose, e.stream);
    HIF_CK(cudaGetLastError());
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(y + c * ld, dy + c * e.n3, e.n3 * 8, cudaMemcpyDeviceToHost, e.stream));
    hif::dfree(dx, e.stream);
    hif::dfree(dy, e.stream);
    e.sync();
  });
}

int hif_solve_pcg_device(hif_handle h, const double* db, double* dx, int nrhs, long long ld,
                         double tol, int maxit, int* iters, double* relres) {
  if (!h || !db || !dx || !iters || !relres || nrhs <= 0 || maxit < 0) return HIF_ERR_ARG;
  return guarded([&] { h->e->solve_pcg_device(db, dx, nrhs, ld, tol, maxit, iters, relres); });
}

int hif_solve_pcg(hif_handle h, const double* b, double* x, int nrhs, long long ld, double tol,
                  int maxit, int* iters, double* relres) {
  if (!h || !b || !x || !iters || !relres || nrhs <= 0 || maxit < 0) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    if (ld < e.n3) throw hif::Error{HIF_ERR_ARG, "ld < (N+1)^3"};
    double* db = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    double* dx = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(db + c * e.n3, b + c * ld, e.n3 * 8, cudaMemcpyHostToDevice, e.stream));
    e.solve_pcg_device(db, dx, nrhs, e.n3, tol, maxit, iters, relres);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(x + c * ld, dx + c * e.n3, e.n3 * 8, cudaMemcpyDeviceToHost, e.stream));
    hif::dfree(db, e.stream);
    hif::dfree(dx, e.stream);
    e.sync();
  });
}

int hif_solve_gmres_device(hif_handle h, const double* db, double* dx, int nrhs, long long ld,
                           double tol, int maxit, int restart, int* iters, double* relres) {
  if (!h || !db || !dx || !iters || !relres || nrhs <= 0 || maxit < 0) return HIF_ERR_ARG;
  return guarded([&] {
    hif::solve_gmres_device(*h->e, db, dx, nrhs, ld, tol, maxit, restart, iters, relres);
  });
}

int hif_solve_gmres(hif_handle h, const double* b, double* x, int nrhs, long long ld, double tol,
                    int maxit, int restart, int* iters, double* relres) {
  if (!h || !b || !x || !iters || !relres || nrhs <= 0 || maxit < 0) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Engine& e = *h->e;
    if (ld < e.n3) throw hif::Error{HIF_ERR_ARG, "ld < (N+1)^3"};
    double* db = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    double* dx = hif::dalloc<double>(e.n3 * nrhs, e.stream);
    struct Free {
      double *a, *b;
      cudaStream_t s;
      ~Free() {
        hif::dfree(a, s);
        hif::dfree(b, s);
      }
    } guard{db, dx, e.stream};
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(db + c * e.n3, b + c * ld, e.n3 * 8, cudaMemcpyHostToDevice, e.stream));
    hif::solve_gmres_device(e, db, dx, nrhs, e.n3, tol, maxit, restart, iters, relres);
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(x + c * ld, dx + c * e.n3, e.n3 * 8, cudaMemcpyDeviceToHost, e.stream));
    e.sync();
  });
}

int hif_num_levels(hif_handle h, int* levels) {
  if (!h || !levels) return HIF_ERR_ARG;
  *levels = h->e->initialized ? h->e->L : h->e->levels_for();
  return HIF_OK;
}

int hif_num_blocks(hif_handle h, int level, int kind, int* nblocks) {
  if (!h || !nblocks) return HIF_ERR_ARG;
  hif::StepData* s = find_step(h, level, kind);
  *nblocks = s ? (int)s->blocks.size() : 0;
  return HIF_OK;
}

int hif_block_info(hif_handle h, int level, int kind, int b, int* ng, int* nr, int* ns,
                   int* face) {
  if (!h) return HIF_ERR_ARG;
  hif::StepData* s = find_step(h, level, kind);
  if (!s || b < 0 || b >= (int)s->blocks.size()) return HIF_ERR_ARG;
  const hif::BlockInfo& bi = s->blocks[b];
  if (ng) *ng = bi.global.size();
  if (nr) *nr = bi.r();
  if (ns) *ns = bi.s();
  if (face) *face = bi.face;
  return HIF_OK;
}

int hif_block_indices(hif_handle h, int level, int kind, int b, int* g, int* r, int* s_) {
  if (!h) return HIF_ERR_ARG;
  hif::StepData* s = find_step(h, level, kind);
  if (!s || b < 0 || b >= (int)s->blocks.size()) return HIF_ERR_ARG;
  const hif::BlockInfo& bi = s->blocks[b];
  if (g) std::copy(bi.global.begin(), bi.global.end(), g);
  if (r) std::copy(bi.red_pos.begin(), bi.red_pos.end(), r);
  if (s_) std::copy(bi.skel_pos.begin(), bi.skel_pos.end(), s_);
  return HIF_OK;
}

int hif_block_matrix(hif_handle h, int level, int kind, int b, int which, double* out) {
  if (!h || !out) return HIF_ERR_ARG;
  hif::StepData* s = find_step(h, level, kind);
  if (!s || b < 0 || b >= (int)s->blocks.size()) return HIF_ERR_ARG;
  return guarded([&] {
    const hif::BlockInfo& bi = s->blocks[b];
    const long long r = bi.r(), k = bi.s();
    long long off = 0, cnt = 0;
    if (s->chol && which >= 0 && which <= 2) {
      // the reference's A22, A22^{-1}, X from the stored L, L^{-1}, Y
      if (r == 0 || (which == 2 && k == 0)) return;
      h->e->chol_readback(*s, b, which, out);
      return;
    }
    if (which >= 5 && which <= 7) {
      if (!s->chol) throw hif::Error{HIF_ERR_ARG, "which 5-7: Cholesky phases only"};
      which -= 5;
    }
    switch (which) {
      case 0: off = s->o_a22[b]; cnt = r * r; break;
      case 1: off = s->o_inv[b]; cnt = r * r; break;
      case 2: off = s->o_x[b]; cnt = r * k; break;
      case 3:
        if (!s->skel) throw hif::Error{HIF_ERR_ARG, "W exists for skeletonization blocks only"};
        off = s->o_w[b];
        cnt = k * r;
        break;
      case 4:
        if (!h->e->keep_schur) throw hif::Error{HIF_ERR_STATE, "enable HIF_OPT_KEEP_SCHUR"};
        if (r == 0) {
          std::fill(out, out + k * k, 0.0);
        } else {
          std::copy(bi.S.begin(), bi.S.end(), out);
        }
        return;
      default:
        throw hif::Error{HIF_ERR_ARG, "which"};
    }
    if (cnt == 0) return;
    h->e->sync();
    HIF_CK(cudaMemcpy(out, s->arena + off, cnt * 8, cudaMemcpyDeviceToHost));
  });
}

int hif_dof_levels(hif_handle h, int* phase_of_dof) {
  if (!h || !phase_of_dof) return HIF_ERR_ARG;
  if (!h->e->factored) {
    hif::g_last_error = "no factorization";
    return HIF_ERR_STATE;
  }
  std::fill(phase_of_dof, phase_of_dof + h->e->n3, -1);
  for (const hif::StepData& st : h->e->steps)
    for (const hif::BlockInfo& bi : st.blocks)
      for (int p : bi.red_pos) phase_of_dof[bi.global[p]] = 2 * st.level + (st.skel ? 1 : 0);
  return HIF_OK;
}

int hif_block_pivots(hif_handle h, int level, int b, int* jpvt, double* rdiag) {
  if (!h) return HIF_ERR_ARG;
  hif::StepData* s = find_step(h, level, 1);
  if (!s || b < 0 || b >= (int)s->blocks.size()) return HIF_ERR_ARG;
  const hif::BlockInfo& bi = s->blocks[b];
  if (jpvt) std::copy(bi.jpvt.begin(), bi.jpvt.end(), jpvt);
  if (rdiag) std::copy(bi.rdiag.begin(), bi.rdiag.end(), rdiag);
  return HIF_OK;
}

int hif_set_option(hif_handle h, int option, long long value) {
  if (!h) return HIF_ERR_ARG;
  switch (option) {
    case HIF_OPT_KEEP_SCHUR: h->e->keep_schur = value != 0; return HIF_OK;
    case HIF_OPT_VERBOSE:
      h->e->verbose = value != 0;
      h->e->verbose_mode = (int)value;
      return HIF_OK;
    case HIF_OPT_MEM_BUDGET_MB: h->e->budget_mb = value; return HIF_OK;
    case HIF_OPT_PRECISION:
      if (value != HIF_PRECISION_FP64 && value != HIF_PRECISION_MIXED) return HIF_ERR_ARG;
      h->e->precision = (int)value;
      return HIF_OK;
    case HIF_OPT_AUTOTUNE:
      h->e->autotune = value != 0;
      return HIF_OK;
    case HIF_OPT_SCHUR_SLICES:
      if (value != 0 && (value < 2 || value > hif::kOzMaxS)) return HIF_ERR_ARG;
      h->e->schur_slices = (int)value;
      return HIF_OK;
    case HIF_OPT_X_SLICES:
      if (value != 0 && (value < 2 || value > hif::kOzMaxS)) return HIF_ERR_ARG;
      h->e->x_slices = (int)value;
      return HIF_OK;
    case HIF_OPT_ELIMINATION:
      if (value != HIF_ELIM_AUTO && value != HIF_ELIM_GAUSS_JORDAN && value != HIF_ELIM_CHOLESKY)
        return HIF_ERR_ARG;
      h->e->elimination = (int)value;
      return HIF_OK;
    case HIF_OPT_Y_SLICES:
      if (value != 0 && (value < 2 || value > hif::kOzMaxS)) return HIF_ERR_ARG;
      h->e->y_slices = (int)value;
      return HIF_OK;
    case HIF_OPT_CHOL_SLICES:
      if (value != 0 && (value < 2 || value > hif::kOzMaxS)) return HIF_ERR_ARG;
      h->e->chol_slices = (int)value;
      return HIF_OK;
    case HIF_OPT_GRAM_SLICES:
      if (value != 0 && (value < 2 || value > hif::kOzMaxS)) return HIF_ERR_ARG;
      h->e->gram_slices = (int)value;
      return HIF_OK;
    case HIF_OPT_GRAM_MIN_N:
      if (value < 0) return HIF_ERR_ARG;
      h->e->gram_min_n = (int)value;
      return HIF_OK;
    case HIF_OPT_ID_GROUP_MIN_N:
      if (value < 2) return HIF_ERR_ARG;
      h->e->kGroupMinN = (int)value;
      return HIF_OK;
    case HIF_OPT_PROFILE:
      return guarded([&] {
        h->e->reset_profile();
        h->e->profile = value != 0;
      });
  }
  return HIF_ERR_ARG;
}

int hif_set_replay_pivots(hif_handle h, int level, int nfaces, const int* offsets,
                          const int* orders) {
  if (!h || level < 0 || nfaces < 0) return HIF_ERR_ARG;
  if (nfaces == 0) {
    h->e->replay.erase(level);
    return HIF_OK;
  }
  if (!offsets || !orders) return HIF_ERR_ARG;
  std::vector<std::vector<int>> v(nfaces);
  for (int f = 0; f < nfaces; ++f) v[f].assign(orders + offsets[f], orders + offsets[f + 1]);
  h->e->replay[level] = std::move(v);
  return HIF_OK;
}

int hif_factor_stats(hif_handle h, double* total_s, double* gather_s, double* elim_s,
                     double* id_s, double* host_s, long long* device_bytes) {
  if (!h) return HIF_ERR_ARG;
  hif::Engine& e = *h->e;
  if (total_s) *total_s = e.t_total;  // the apply plans included (built before its end)
  if (gather_s) *gather_s = e.t_gather;
  if (elim_s) *elim_s = e.t_elim;
  if (id_s) *id_s = e.t_id;
  if (host_s) *host_s = e.t_host;
  if (device_bytes)
    *device_bytes = (long long)(e.arena_factor.reserved() + e.arena_work[0].reserved() +
                                e.arena_work[1].reserved()) +
                    7LL * e.n3 * 8;
  return HIF_OK;
}

// ---- the reference's free functions -------------------------------------------
namespace {

struct FreeCtx {
  cudaStream_t stream = cudaStreamPerThread;
  int* d_status = nullptr;
  hif::BufList bufs;
  FreeCtx() {
    d_status = bufs.add(hif::dalloc<int>(4, stream));
    HIF_CK(cudaMemsetAsync(d_status, 0, 4 * sizeof(int), stream));
  }
  ~FreeCtx() {
    bufs.release(stream);
    cudaStreamSynchronize(stream);
  }
  int status() {
    int st = 0;
    HIF_CK(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    HIF_CK(cudaStreamSynchronize(stream));
    return st;
  }
};

int check_device() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    hif::g_last_error = "no CUDA device";
    return HIF_ERR_NODEVICE;
  }
  return HIF_OK;
}

// Eliminate the redundant DOFs of one device block given in [red | skel] order:
// writes A22^{-1} (r x r), X (r x s) and S = -A12 X (s x s), all ld = rows.
void schur_on_device(FreeCtx& c, const double* dB, int n, int r, double* dA22inv, double* dX,
                     double* dS) {
  const int s = n - r;
  double* W = c.bufs.add(hif::dalloc<double>((size_t)n * n, c.stream));
  HIF_CK(cudaMemcpyAsync(W, dB, (size_t)n * n * 8, cudaMemcpyDeviceToDevice, c.stream));
  if (s > 0) {  // S = -A12 X: eliminate with the skeleton block zeroed
    HIF_CK(cudaMemset2DAsync(W + r + (long long)r * n, (size_t)n * 8, 0, (size_t)s * 8, s, c.stream));
  }
  std::vector<hif::SweepDesc> sd(1);
  sd[0].B = W;
  sd[0].a22inv = dA22inv;
  sd[0].X = dX;
  sd[0].n = n;
  sd[0].r = r;
  hif::sweep_blocks(sd, c.bufs, c.stream, c.d_status,
                    [&](int, double, double, auto&& f, int = 1) { f(); });
  HIF_CK(cudaGetLastError());
  if (s > 0)
    HIF_CK(cudaMemcpy2DAsync(dS, (size_t)s * 8, W + r + (long long)r * n, (size_t)n * 8,
                             (size_t)s * 8, s, cudaMemcpyDeviceToDevice, c.stream));
}

}  // namespace

int hif_schur_device(const double* dB, int n, int r, double* dA22inv, double* dX, double* dS) {
  if (!dB || n < 0 || r < 0 || r > n || (r > 0 && (!dA22inv || (r < n && !dX))) ||
      (r < n && !dS))
    return HIF_ERR_ARG;
  if (int e = check_device()) return e;
  return guarded([&] {
    FreeCtx c;
    if (r == 0) {
      if (n > 0) HIF_CK(cudaMemsetAsync(dS, 0, (size_t)n * n * 8, c.stream));
    } else {
      schur_on_device(c, dB, n, r, dA22inv, dX, dS);
    }
    if (c.status() & hif::kStatusTinyPivot) throw hif::Error{HIF_ERR_SINGULAR, "zero pivot"};
  });
}

int hif_gemm_mixed_device(int transA, int transB, int m, int n, int k, double alpha,
                          const double* dA, long long lda, const double* dB, long long ldb,
                          double beta, double* dC, long long ldc) {
  if (m < 0 || n < 0 || k < 0 || (m && n && (!dC || ldc < m)) ||
      (m && n && k && (!dA || !dB || lda < (transA ? k : m) || ldb < (transB ? n : k))))
    return HIF_ERR_ARG;
  if (int e = check_device()) return e;
  return guarded([&] {
    if (m == 0 || n == 0) return;
    FreeCtx c;
    hif::GemmDesc g{};
    g.C = dC;
    g.A = dA;
    g.B = dB;
    g.ldc = ldc;
    g.lda = lda;
    g.ldb = ldb;
    g.m = m;
    g.n = n;
    g.k = k;
    g.transA = transA ? 1 : 0;
    g.transB = transB ? 1 : 0;
    g.alpha = alpha;
    g.beta = beta;
    hif::gemm_batch(std::vector<hif::GemmDesc>{g}, c.bufs, c.stream, HIF_KCLASS_GEMM_MIXED,
                    [&](int, double, double, auto&& f, int = 1) { f(); }, 128, c.d_status);
    if (c.status() & hif::kStatusTimeout)
      throw hif::Error{HIF_ERR_CUDA, "tensor-core pipeline wait timed out"};
  });
}

int hif_gemm_int8_device(int transA, int transB, int m, int n, int k, double alpha,
                         const double* dA, long long lda, const double* dB, long long ldb,
                         double beta, double* dC, long long ldc, int slices) {
  if (m < 0 || n < 0 || k < 0 || slices < 2 || slices > hif::kOzMaxS ||
      (m && n && (!dC || ldc < m)) ||
      (m && n && k && (!dA || !dB || lda < (transA ? k : m) || ldb < (transB ? n : k))))
    return HIF_ERR_ARG;
  if (int e = check_device()) return e;
  return guarded([&] {
    if (m == 0 || n == 0) return;
    FreeCtx c;
    hif::GemmDesc g{};
    g.C = dC;
    g.A = dA;
    g.B = dB;
    g.ldc = ldc;
    g.lda = lda;
    g.ldb = ldb;
    g.m = m;
    g.n = n;
    g.k = k;
    g.transA = transA ? 1 : 0;
    g.transB = transB ? 1 : 0;
    g.alpha = alpha;
    g.beta = beta;
    hif::gemm_batch_int8(std::vector<hif::GemmDesc>{g}, c.bufs, c.stream,
                         [&](int, double, double, auto&& f, int = 1) { f(); }, slices,
                         c.d_status);
    if (c.status() & hif::kStatusTimeout)
      throw hif::Error{HIF_ERR_CUDA, "tensor-core pipeline wait timed out"};
  });
}

int hif_schur(const double* matrix, int m, long long ld, const int* red, int nr, const int* skel,
              int ns, double* A22, double* A22inv, double* X, double* S) {
  if (!matrix || m < 0 || ld < m || nr < 0 || ns < 0 || nr + ns > m || (nr && !red) ||
      (ns && !skel))
    return HIF_ERR_ARG;
  if (int e = check_device()) return e;
  return guarded([&] {
    const int n = nr + ns;
    std::vector<int> ord(red, red + nr);
    ord.insert(ord.end(), skel, skel + ns);
    for (int p : ord)
      if (p < 0 || p >= m) throw hif::Error{HIF_ERR_ARG, "index out of range"};
    std::vector<double> B((size_t)n * n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) B[i + (size_t)j * n] = matrix[ord[i] + (long long)ord[j] * ld];
    if (A22)
      for (int j = 0; j < nr; ++j)
        for (int i = 0; i < nr; ++i) A22[i + (size_t)j * nr] = B[i + (size_t)j * n];
    FreeCtx c;
    double* dB = c.bufs.add(hif::upload(B, c.stream));
    double* dInv = c.bufs.add(hif::dalloc<double>((size_t)nr * nr, c.stream));
    double* dX = c.bufs.add(hif::dalloc<double>((size_t)nr * ns, c.stream));
    double* dS = c.bufs.add(hif::dalloc<double>((size_t)ns * ns, c.stream));
    if (nr == 0) {
      HIF_CK(cudaMemsetAsync(dS, 0, (size_t)ns * ns * 8, c.stream));
    } else {
      schur_on_device(c, dB, n, nr, dInv, dX, dS);
    }
    if (A22inv) HIF_CK(cudaMemcpyAsync(A22inv, dInv, (size_t)nr * nr * 8, cudaMemcpyDeviceToHost, c.stream));
    if (X) HIF_CK(cudaMemcpyAsync(X, dX, (size_t)nr * ns * 8, cudaMemcpyDeviceToHost, c.stream));
    if (S) HIF_CK(cudaMemcpyAsync(S, dS, (size_t)ns * ns * 8, cudaMemcpyDeviceToHost, c.stream));
    if (c.status() & hif::kStatusTinyPivot) throw hif::Error{HIF_ERR_SINGULAR, "zero pivot"};
  });
}

namespace {

// Pivoted QR + rank test + W of one host matrix on the device (the ID kernel).
// M is overwritten with the factorization (R on and above the diagonal).
void id_host(double* M, int m, int n, long long ldm, double eps, std::vector<int>& jpvt,
             std::vector<int>& keep, int& k, double* W) {
  FreeCtx c;
  double* dM = c.bufs.add(hif::dalloc<double>((size_t)m * n, c.stream));
  HIF_CK(cudaMemcpy2DAsync(dM, (size_t)m * 8, M, (size_t)ldm * 8, (size_t)m * 8, n,
                           cudaMemcpyHostToDevice, c.stream));
  int* dint = c.bufs.add(hif::dalloc<int>(2 * (size_t)n + 1, c.stream));
  double* drd = c.bufs.add(hif::dalloc<double>(n, c.stream));
  double* dW = c.bufs.add(hif::dalloc<double>((size_t)n * n / 4 + n + 1, c.stream));
  std::vector<hif::IdDesc> idd(1);
  idd[0].M = dM;
  idd[0].order = nullptr;
  idd[0].jpvt = dint;
  idd[0].keep = dint + n;
  idd[0].rank = dint + 2 * n;
  idd[0].rdiag = drd;
  idd[0].W = dW;
  idd[0].m = m;
  idd[0].n = n;
  hif::IdDesc* d_idd = c.bufs.add(hif::upload(idd, c.stream));
  hif::launch_id(d_idd, 1, n, eps, c.d_status, c.stream);
  HIF_CK(cudaGetLastError());
  std::vector<int> hi(2 * n + 1);
  HIF_CK(cudaMemcpyAsync(hi.data(), dint, (2 * (size_t)n + 1) * sizeof(int),
                         cudaMemcpyDeviceToHost, c.stream));
  HIF_CK(cudaMemcpy2DAsync(M, (size_t)ldm * 8, dM, (size_t)m * 8, (size_t)m * 8, n,
                           cudaMemcpyDeviceToHost, c.stream));
  HIF_CK(cudaStreamSynchronize(c.stream));
  jpvt.assign(hi.begin(), hi.begin() + n);
  keep.assign(hi.begin() + n, hi.begin() + 2 * n);
  k = hi[2 * n];
  if (W && k > 0 && k < n)
    HIF_CK(cudaMemcpyAsync(W, dW, (size_t)k * (n - k) * 8, cudaMemcpyDeviceToHost, c.stream));
  HIF_CK(cudaStreamSynchronize(c.stream));
}

}  // namespace

int hif_interp_decomp(double* M, int m, int n, long long ldm, double eps, double* W,
                      int* skeleton_cols, int* redundant_cols, int* rank) {
  if (!M || m < 1 || n < 1 || m < n || ldm < m || !(eps >= 0) || !rank) return HIF_ERR_ARG;
  if (int e = check_device()) return e;
  return guarded([&] {
    std::vector<int> jp, keep;
    int k = 0;
    id_host(M, m, n, ldm, eps, jp, keep, k, W);
    *rank = k;
    int a = 0, b = 0;
    for (int i = 0; i < n; ++i) {
      if (keep[i]) {
        if (skeleton_cols) skeleton_cols[a] = jp[i];
        ++a;
      } else {
        if (redundant_cols) redundant_cols[b] = jp[i];
        ++b;
      }
    }
  });
}

int hif_pivoted_qr(double* A, int m, int n, long long lda, int* jpvt) {
  if (!A || !jpvt || m < 1 || n < 1 || m < n || lda < m) return HIF_ERR_ARG;
  if (int e = check_device()) return e;
  return guarded([&] {
    std::vector<int> jp, keep;
    int k = 0;
    id_host(A, m, n, lda, 0.0, jp, keep, k, nullptr);
    std::copy(jp.begin(), jp.end(), jpvt);
  });
}

int hif_triangular_solve(const double* R, int k, long long ldr, double* B, int nb, long long ldb) {
  if (!R || !B || k < 0 || nb < 0 || ldr < k || ldb < k) return HIF_ERR_ARG;
  if (k == 0 || nb == 0) return HIF_OK;
  if (int e = check_device()) return e;
  return guarded([&] {
    FreeCtx c;
    double* dR = c.bufs.add(hif::dalloc<double>((size_t)k * k, c.stream));
    double* dB = c.bufs.add(hif::dalloc<double>((size_t)k * nb, c.stream));
    HIF_CK(cudaMemcpy2DAsync(dR, (size_t)k * 8, R, (size_t)ldr * 8, (size_t)k * 8, k,
                             cudaMemcpyHostToDevice, c.stream));
    HIF_CK(cudaMemcpy2DAsync(dB, (size_t)k * 8, B, (size_t)ldb * 8, (size_t)k * 8, nb,
                             cudaMemcpyHostToDevice, c.stream));
    hif::launch_trsm_upper(dR, k, k, dB, k, nb, c.stream);
    HIF_CK(cudaGetLastError());
    HIF_CK(cudaMemcpy2DAsync(B, (size_t)ldb * 8, dB, (size_t)k * 8, (size_t)k * 8, nb,
                             cudaMemcpyDeviceToHost, c.stream));
    HIF_CK(cudaStreamSynchronize(c.stream));
  });
}

int hif_trim(hif_handle h) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] {
    h->e->sync();
    h->e->arena_work[0].release();
    h->e->arena_work[1].release();
  });
}

int hif_trim_device_pool(void) {
  if (int e = check_device()) return e;
  return guarded([&] {
    int dev = 0;
    HIF_CK(cudaGetDevice(&dev));
    HIF_CK(cudaDeviceSynchronize());
    cudaMemPool_t pool;
    HIF_CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    HIF_CK(cudaMemPoolTrimTo(pool, 0));
  });
}

int hif_autotune_elimination(hif_handle h, int* signatures, int* decided, int* chose_cholesky) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] {
    h->e->sync();
    h->e->tuner.resolve();
    int n = 0, d = 0, c = 0;
    for (const auto& kv : h->e->tuner.recs) {
      if (!(kv.first & hif::Engine::kTuneElimKey)) continue;
      ++n;
      if (kv.second.choice >= 0) ++d;
      if (kv.second.choice == 1) ++c;
    }
    if (signatures) *signatures = n;
    if (decided) *decided = d;
    if (chose_cholesky) *chose_cholesky = c;
  });
}

int hif_memory(hif_handle h, long long* factor_bytes, long long* workspace_bytes) {
  if (!h) return HIF_ERR_ARG;
  // the factor and the descriptors its apply plans read
  if (factor_bytes)
    *factor_bytes = (long long)(h->e->arena_factor.reserved() + h->e->arena_desc.reserved());
  if (workspace_bytes)
    *workspace_bytes = (long long)(h->e->arena_work[0].reserved() + h->e->arena_work[1].reserved());
  return HIF_OK;
}

int hif_kernel_stats(hif_handle h, int kclass, long long* launches, double* ms, double* flops,
                     double* bytes) {
  if (!h || kclass < 0 || kclass >= HIF_KCLASS_COUNT) return HIF_ERR_ARG;
  return guarded([&] {
    h->e->sync();
    h->e->resolve_profile();
    const hif::Engine::KStat& k = h->e->kstat[kclass];
    if (launches) *launches = k.launches;
    if (ms) *ms = k.ms;
    if (flops) *flops = k.flops;
    if (bytes) *bytes = k.bytes;
  });
}

int hif_autotune_stats(hif_handle h, int* signatures, int* decided, int* chose_128) {
  if (!h) return HIF_ERR_ARG;
  return guarded([&] {
    h->e->sync();
    h->e->tuner.resolve();
    int n = 0, d = 0, c = 0;
    for (const auto& kv : h->e->tuner.recs) {
      if (kv.first & hif::Engine::kTuneElimKey) continue;
      ++n;
      if (kv.second.choice >= 0) ++d;
      if (kv.second.choice == 1) ++c;
    }
    if (signatures) *signatures = n;
    if (decided) *decided = d;
    if (chose_128) *chose_128 = c;
  });
}

int hif_partition_cell(int N, int P, int level, int ci, int cj, int ck, int reserved,
                       const unsigned char* mask, int* g, int* r, int* s_, int* counts) {
  if (N < 1 || P < 1 || level < 0 || !mask || !g || !r || !s_ || !counts || reserved != 0)
    return HIF_ERR_ARG;
  return guarded([&] {
    hif::Partitioner part{N, P, N + 1, mask};
    const int c[3] = {ci, cj, ck};
    std::vector<int> gg, rr, ss;
    part.cell_index(level, c, gg, rr, ss);
    std::copy(gg.begin(), gg.end(), g);
    std::copy(rr.begin(), rr.end(), r);
    std::copy(ss.begin(), ss.end(), s_);
    counts[0] = gg.size();
    counts[1] = rr.size();
    counts[2] = ss.size();
  });
}

int hif_partition_face(int N, int P, int level, int ci, int cj, int ck, int face, int reserved,
                       const unsigned char* mask, int* rows, int* cols) {
  if (N < 1 || P < 1 || level < 0 || !mask || !rows || !cols || reserved != 0) return HIF_ERR_ARG;
  if (face != hif::TOP && face != hif::LEFT && face != hif::FRONT) return HIF_ERR_ARG;
  return guarded([&] {
    hif::Partitioner part{N, P, N + 1, mask};
    const int c[3] = {ci, cj, ck};
    std::vector<int> rw, cl;
    int nb[3];
    if (!part.skel_interaction(level, c, face, rw, cl, nb)) {
      rw.clear();
      cl.clear();
    }
    rows[0] = rw.size();
    cols[0] = cl.size();
    std::copy(rw.begin(), rw.end(), rows + 1);
    std::copy(cl.begin(), cl.end(), cols + 1);
  });
}

}  // extern "C"

#include "hif_server.inl"
