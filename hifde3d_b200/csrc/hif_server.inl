// Serving loop: factored operators resident in HBM, new factorizations admitted
// by a device-memory budget, and solve requests of different operators and
// right-hand-side counts batched at the level of PCG iterations.
//
// Included at the end of hif_engine.cpp (needs the Engine internals, which
// live in that translation unit's anonymous namespace; the pragma below
// silences GCC's warning about using them from an included file).
#pragma GCC diagnostic ignored "-Wsubobject-linkage"
//
// Scheduling:
//   * factor requests run on worker threads, each on its operator's own stream,
//     so factorizations overlap with each other and with the solves on the GPU;
//     one is admitted when its memory estimate fits in the budget next to the
//     resident factors and the factorizations already running; after it
//     completes its workspace is returned and only the factor stays resident;
//   * solve requests join the active set between PCG iterations (continuous
//     batching) when a slot and memory are free; every iteration runs the
//     preconditioner applies of all active requests together: one launch per
//     apply stage covering every request (descriptor segments), instead of one
//     per request and stage; each request leaves the set when all its
//     right-hand sides reach the tolerance (or maxit).
// Every request performs the same arithmetic, in the same order, as
// hif_solve_pcg on its operator: results do not depend on the mix.

namespace hif {

class Server {
 public:
  struct Op {
    std::unique_ptr<Engine> e;
    int state = 0;  // 0 factoring, 1 ready, 2 failed, 3 released
    long long bytes = 0;
    long long n3 = 0;
    int active = 0;  // solves in flight
    std::string err;
  };
  struct Req {
    long long id = 0;
    int kind = 0;  // 0 factor, 1 solve
    int op = 0;
    // factor
    int N = 0, P = 4, partition = 0, precision = 0;
    double eps = 1e-6, hstep = 0;
    std::vector<double> ax, ay, az, V;
    // solve
    std::vector<double> b;
    int nrhs = 1, maxit = 100;
    double tol = 1e-10;
    double* xout = nullptr;
    // outcome
    int status = -1;
    int iters = 0;
    double relres = 0;
    double t_submit = 0, t_start = 0, t_done = 0;  // t_start: admitted (factor
                                                    // worker / active solve set)
    bool done = false;
    std::string err;
  };

  Server(long long budget, int slots, int factor_workers)
      : budget_(budget), slots_(std::max(1, slots)) {
    HIF_CK(cudaGetDevice(&device_));
    HIF_CK(cudaStreamCreateWithFlags(&sstream_, cudaStreamNonBlocking));
    stop_ = false;
    solver_ = std::thread([this] { solve_loop(); });
    for (int w = 0; w < std::max(1, factor_workers); ++w)
      workers_.emplace_back([this] { factor_loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    solver_.join();
    for (std::thread& t : workers_) t.join();
    ops_.clear();
    cudaStreamSynchronize(sstream_);
    cudaStreamDestroy(sstream_);
  }

  long long submit(std::unique_ptr<Req> r) {
    std::lock_guard<std::mutex> lk(mu_);
    r->id = ++next_id_;
    r->t_submit = wall();
    const long long id = r->id;
    if (r->kind == 0) {
      Op& o = ops_[r->op];
      if (o.e || (o.state == 0 && o.n3 > 0))
        throw Error{HIF_ERR_ARG, "operator id in use; release it first"};
      o = Op{};
      o.state = 0;
      o.n3 = (long long)(r->N + 1) * (r->N + 1) * (r->N + 1);
      fq_.push_back(r.get());
    } else {
      auto it = ops_.find(r->op);
      if (it == ops_.end() || it->second.state == 3) throw Error{HIF_ERR_ARG, "unknown operator"};
      if ((long long)r->b.size() != it->second.n3 * r->nrhs)
        throw Error{HIF_ERR_ARG, "right-hand side size does not match the operator"};
      sq_.push_back(r.get());
    }
    reqs_[id] = std::move(r);
    cv_.notify_all();
    return id;
  }

  // Blocks until the request completes; the request record is dropped.
  void wait(long long id, int* status, int* iters, double* relres, double* latency_ms,
            double* queue_ms = nullptr) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) throw Error{HIF_ERR_ARG, "unknown request"};
    Req* r = it->second.get();
    done_cv_.wait(lk, [&] { return r->done; });
    if (status) *status = r->status;
    if (iters) *iters = r->iters;
    if (relres) *relres = r->relres;
    if (latency_ms) *latency_ms = 1e3 * (r->t_done - r->t_submit);
    if (queue_ms) *queue_ms = 1e3 * ((r->t_start > 0 ? r->t_start : r->t_done) - r->t_submit);
    const std::string err = r->err;
    reqs_.erase(it);
    if (!err.empty()) g_last_error = err;
  }

  // DOFs of a registered operator (factoring or ready), 0 if unknown.
  long long dofs(int op) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = ops_.find(op);
    return it == ops_.end() ? 0 : it->second.n3;
  }

  void release(int op) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = ops_.find(op);
    if (it == ops_.end()) throw Error{HIF_ERR_ARG, "unknown operator"};
    done_cv_.wait(lk, [&] { return it->second.active == 0 && it->second.state != 0; });
    used_ -= it->second.bytes;
    std::unique_ptr<Engine> e = std::move(it->second.e);
    ops_.erase(it);
    lk.unlock();
    e.reset();
    cv_.notify_all();
  }

  void stats(long long* used, long long* resident_ops, long long* completed, long long* ticks,
             long long* batched_launches) {
    std::lock_guard<std::mutex> lk(mu_);
    if (used) *used = used_;
    if (resident_ops) *resident_ops = (long long)ops_.size();
    if (completed) *completed = completed_;
    if (ticks) *ticks = ticks_;
    if (batched_launches) *batched_launches = merged_launches_;
  }

 private:
  // Device bytes a factorization holds at its peak (factor plus workspace):
  // the footprint measured on an earlier factorization of the same size when
  // there is one, else a per-DOF bound with margin.
  long long estimate_bytes(int N) const {
    auto it = measured_.find(N);
    if (it != measured_.end()) return it->second + (64LL << 20);
    const double dofs = (double)(N + 1) * (N + 1) * (N + 1);
    return (long long)(dofs * 12.0 * 1024.0) + (256LL << 20);
  }

  // Device bytes of one active solve: x r z p q ua ub uc and the contribution
  // slots (the scalars are negligible).
  static long long solve_bytes(const Engine& e, int nrhs) {
    return 8LL * (8 * e.n3 * nrhs + e.contrib_ld * nrhs);
  }

  void finish(Req* r, int status, const std::string& err) {
    r->status = status;
    r->err = err;
    r->t_done = wall();
    r->done = true;
    ++completed_;
    done_cv_.notify_all();
  }

  // ---- factorizations -----------------------------------------------------
  void factor_loop() {
    cudaSetDevice(device_);
    for (;;) {
      Req* r = nullptr;
      long long need = 0;
      {
        std::unique_lock<std::mutex> lk(mu_);
        // the head request waits until its estimate fits beside what is
        // resident and running; one whose estimate exceeds the whole budget
        // can never fit and is refused
        cv_.wait(lk, [&] {
          if (stop_) return true;
          if (fq_.empty()) return false;
          need = estimate_bytes(fq_.front()->N);
          return need > budget_ || used_ + need <= budget_;
        });
        if (stop_) return;
        r = fq_.front();
        fq_.pop_front();
        r->t_start = wall();
        if (need > budget_) {
          Op& o = ops_[r->op];
          o.state = 2;
          o.err = "factorization needs an estimated " + std::to_string(need >> 20) +
                  " MiB, more than the server's budget of " + std::to_string(budget_ >> 20) +
                  " MiB";
          r->ax.clear();
          r->ay.clear();
          r->az.clear();
          r->V.clear();
          finish(r, HIF_ERR_BUDGET, o.err);
          cv_.notify_all();
          continue;
        }
        used_ += need;
      }
      std::unique_ptr<Engine> e;
      int st = HIF_OK;
      std::string err;
      long long keep = 0, peak = 0;
      try {
        e.reset(new Engine(r->N, r->P, r->eps, r->partition));
        e->precision = r->precision;
        const long long nt = (long long)(r->N + 2) * (r->N + 2) * (r->N + 2);
        double* d = dalloc<double>(4 * nt, e->stream);
        const std::vector<double>* src[4] = {&r->ax, &r->ay, &r->az, &r->V};
        for (int q = 0; q < 4; ++q)
          HIF_CK(cudaMemcpyAsync(d + q * nt, src[q]->data(), nt * 8, cudaMemcpyHostToDevice,
                                 e->stream));
        launch_setup_faces(d, d + nt, d + 2 * nt, d + 3 * nt, r->N, r->hstep, e->d_band,
                           e->stream);
        HIF_CK(cudaGetLastError());
        e->have_op = true;
        e->symmetric = true;
        dfree(d, e->stream);
        e->factor();
        e->sync();
        peak = (long long)(e->arena_factor.reserved() + e->arena_work[0].reserved() +
                           e->arena_work[1].reserved() + e->arena_desc.reserved());
        e->stage.release();
        e->arena_work[0].release();
        e->arena_work[1].release();
        e->release_workspace();  // solves use their own vectors
        keep = (long long)(e->arena_factor.reserved() + e->arena_desc.reserved()) +
               7LL * e->n3 * 8;
      } catch (const Error& x) {
        st = x.code;
        err = x.msg;
      } catch (const std::exception& x) {
        st = HIF_ERR_CUDA;
        err = x.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        Op& o = ops_[r->op];
        used_ -= need;
        if (st == HIF_OK) {
          long long& m = measured_[r->N];
          m = std::max(m, peak);
          o.e = std::move(e);
          o.bytes = keep;
          used_ += keep;
          o.state = 1;
        } else {
          o.state = 2;
          o.err = err;
        }
        r->ax.clear();
        r->ay.clear();
        r->az.clear();
        r->V.clear();
        finish(r, st, err);
      }
      cv_.notify_all();
    }
  }

  // ---- batched PCG ----------------------------------------------------------
  struct Active {
    Req* r;
    Engine* e;
    int nrhs;
    long long n3;
    double* mem = nullptr;  // x r z p q ua ub uc | contrib | scalars
    double *x, *rv, *z, *p, *q, *ua, *ub, *uc, *contrib, *sc;
    int it = 0;
    bool fresh = true;
    std::vector<double> bb, relres;
    std::vector<int> done, iters;
    // this request's apply launches (descriptors bound to its vectors)
    struct L {
      long long key;
      int type;
      GemvFastSeg gs;  // descriptors bound to this request's vectors
      int layout;
      ReduceSeg rs;
      int tiles;  // units of the GEMV layout, or reduced entries
    };
    std::vector<L> launches;
    BufList bufs;
  };

  void admit(Active& a, Op& o) {
    Engine& e = *o.e;
    a.e = &e;
    a.n3 = e.n3;
    a.nrhs = a.r->nrhs;
    const long long nv = a.n3 * a.nrhs;
    const long long cl = e.contrib_ld;
    const long long tot = 8 * nv + cl * a.nrhs + 8LL * a.nrhs + (long long)kDotBlocks * a.nrhs;
    a.mem = a.bufs.add(dalloc<double>(tot, sstream_));
    a.x = a.mem;
    a.rv = a.x + nv;
    a.z = a.rv + nv;
    a.p = a.z + nv;
    a.q = a.p + nv;
    a.ua = a.q + nv;
    a.ub = a.ua + nv;
    a.uc = a.ub + nv;
    a.contrib = a.uc + nv;
    a.sc = a.contrib + cl * a.nrhs;
    HIF_CK(cudaMemcpyAsync(a.rv, a.r->b.data(), nv * 8, cudaMemcpyHostToDevice, sstream_));
    a.r->b.clear();
    // bind the operator's inverse-apply plan to this request's vectors
    double* vec[3] = {a.ua, a.ub, a.uc};
    for (const ApplyLaunch& l : e.plan_inv.launches) {
      Active::L x{};
      x.key = l.key;
      x.type = l.type;
      if (l.type == 0) {
        std::vector<GemvDesc> dd = l.hdesc;
        for (GemvDesc& g : dd) {
          g.uin = vec[l.in_vec];
          g.uout = vec[l.out_vec];
          g.nrhs = a.nrhs;
          g.ldu = a.n3;
          g.cld = cl;
          if (g.mode == 1) g.contrib = a.contrib + (g.contrib - e.d_contrib);
        }
        x.gs.desc = a.bufs.add(upload(dd, sstream_));
        x.gs.tab = l.d_tab;
        x.layout = l.layout;
        x.tiles = l.units;
      } else {
        x.rs = ReduceSeg{l.d_dof, l.d_off, l.d_slot, a.contrib, vec[l.out_vec], cl, a.n3, l.ndof,
                         a.nrhs, l.alpha};
        x.tiles = l.ndof * a.nrhs;
      }
      a.launches.push_back(x);
    }
    a.bb.assign(a.nrhs, 0.0);
    a.relres.assign(a.nrhs, 0.0);
    a.done.assign(a.nrhs, 0);
    a.iters.assign(a.nrhs, 0);
  }

  // z = M^{-1} r for every request in `set`: per-request copies, then one launch
  // per stage key over all requests that have it.
  void batched_apply(std::vector<Active*>& set) {
    for (Active* a : set) {
      HIF_CK(cudaMemcpyAsync(a->ua, a->rv, a->n3 * a->nrhs * 8, cudaMemcpyDeviceToDevice, sstream_));
      launch_zero_boundary(a->ua, a->e->NC, a->nrhs, a->n3, sstream_);
      HIF_CK(cudaMemsetAsync(a->ub, 0, a->n3 * a->nrhs * 8, sstream_));
    }
    std::map<long long, std::vector<std::pair<Active*, size_t>>> stages;
    for (Active* a : set)
      for (size_t i = 0; i < a->launches.size(); ++i) stages[a->launches[i].key].push_back({a, i});
    BufList tick;
    for (auto& kv : stages) {
      // one launch per GEMV layout present at this stage (the same kernels as
      // hif_apply's, so each request computes exactly what it would alone)
      std::vector<GemvFastSeg> gs[kGemvLayouts];
      std::vector<int> goff[kGemvLayouts] = {{0}, {0}};
      std::vector<ReduceSeg> rs;
      std::vector<int> roff(1, 0);
      for (auto& pr : kv.second) {
        const Active::L& l = pr.first->launches[pr.second];
        if (l.type == 0) {
          gs[l.layout].push_back(l.gs);
          goff[l.layout].push_back(goff[l.layout].back() + l.tiles);
        } else {
          rs.push_back(l.rs);
          roff.push_back(roff.back() + l.tiles);
        }
      }
      for (int lay = 0; lay < kGemvLayouts; ++lay) {
        if (gs[lay].empty() || goff[lay].back() == 0) continue;
        GemvFastSeg* dg = tick.add(upload(gs[lay], sstream_));
        int* dgo = tick.add(upload(goff[lay], sstream_));
        launch_gemv_fast(dg, dgo, (int)gs[lay].size(), goff[lay].back(), lay, nullptr, nullptr, 0,
                         0, 0, sstream_);
        ++merged_launches_;
      }
      if (!rs.empty() && roff.back() > 0) {
        ReduceSeg* dr = tick.add(upload(rs, sstream_));
        int* dro = tick.add(upload(roff, sstream_));
        launch_reduce_seg(dr, dro, (int)rs.size(), roff.back(), sstream_);
        ++merged_launches_;
      }
      HIF_CK(cudaGetLastError());
    }
    for (Active* a : set)
      HIF_CK(cudaMemcpyAsync(a->z, a->ub, a->n3 * a->nrhs * 8, cudaMemcpyDeviceToDevice, sstream_));
    tick.release(sstream_);
  }

  void solve_loop() {
    cudaSetDevice(device_);
    std::vector<std::unique_ptr<Active>> act;
    for (;;) {
      // ---- admission (between iterations)
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] {
          if (stop_) return true;
          if (!act.empty()) return true;
          for (Req* r : sq_) {
            auto it = ops_.find(r->op);
            if (it != ops_.end() && it->second.state != 0) return true;
          }
          return false;
        });
        if (stop_ && act.empty()) return;
        for (auto it = sq_.begin(); it != sq_.end() && (int)act.size() < slots_;) {
          Req* r = *it;
          auto oi = ops_.find(r->op);
          if (oi == ops_.end() || oi->second.state == 3) {
            finish(r, HIF_ERR_ARG, "operator released");
            it = sq_.erase(it);
            continue;
          }
          Op& o = oi->second;
          if (o.state == 0) {
            ++it;
            continue;
          }
          if (o.state == 2) {
            finish(r, HIF_ERR_STATE, "operator factorization failed: " + o.err);
            it = sq_.erase(it);
            continue;
          }
          const long long need = solve_bytes(*o.e, r->nrhs);
          if (used_ + need > budget_ && !act.empty()) break;
          used_ += need;
          o.active += 1;
          r->t_start = wall();
          auto a = std::unique_ptr<Active>(new Active());
          a->r = r;
          try {
            admit(*a, o);
          } catch (const Error& x) {
            used_ -= need;
            o.active -= 1;
            finish(r, x.code, x.msg);
            it = sq_.erase(it);
            continue;
          }
          act.push_back(std::move(a));
          it = sq_.erase(it);
        }
      }
      if (act.empty()) continue;
      try {
        tick(act);
      } catch (const Error& x) {
        cudaStreamSynchronize(sstream_);
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& a : act) {
          ops_[a->r->op].active -= 1;
          used_ -= solve_bytes(*a->e, a->nrhs);
          a->bufs.release(sstream_);
          finish(a->r, x.code, x.msg);
        }
        act.clear();
        done_cv_.notify_all();
      }
    }
  }

  // One PCG iteration for every active request (see hif_solve_pcg for the scalar
  // form). Fresh requests take their first step: x = 0, r = b, z = M r, p = z.
  void tick(std::vector<std::unique_ptr<Active>>& act) {
    ++ticks_;
    for (auto& ap : act) {
      Active& a = *ap;
      const long long nv = a.n3 * a.nrhs;
      double* part = a.sc + 8 * a.nrhs;
      if (a.fresh) {
        launch_zero_boundary(a.rv, a.e->NC, a.nrhs, a.n3, sstream_);
        HIF_CK(cudaMemsetAsync(a.x, 0, nv * 8, sstream_));
        launch_dot(a.rv, a.rv, a.n3, a.nrhs, a.n3, part, a.sc + 4 * a.nrhs, sstream_);
      } else {
        double* rz = a.sc;
        double* pq = a.sc + 2 * a.nrhs;
        launch_stencil_apply(a.e->d_band, a.e->NC, a.p, a.q, a.nrhs, a.n3, 0, sstream_);
        launch_dot(a.p, a.q, a.n3, a.nrhs, a.n3, part, pq, sstream_);
        launch_pcg_update_xr(a.x, a.rv, a.p, a.q, rz, pq, a.n3, a.nrhs, a.n3, sstream_);
        launch_dot(a.rv, a.rv, a.n3, a.nrhs, a.n3, part, a.sc + 3 * a.nrhs, sstream_);
      }
    }
    // one host sync for the whole batch: residual norms
    std::vector<std::vector<double>> h(act.size());
    for (size_t i = 0; i < act.size(); ++i) {
      Active& a = *act[i];
      h[i].assign(2 * a.nrhs, 0.0);
      HIF_CK(cudaMemcpyAsync(h[i].data(), a.sc + 3 * a.nrhs, 2 * a.nrhs * 8,
                             cudaMemcpyDeviceToHost, sstream_));
    }
    HIF_CK(cudaStreamSynchronize(sstream_));
    std::vector<Active*> cont, retire;
    for (size_t i = 0; i < act.size(); ++i) {
      Active& a = *act[i];
      // per right-hand side, as hif_solve_pcg: a column that met the tolerance
      // keeps the iteration count and residual of that moment
      bool all = true;
      if (a.fresh) {
        a.bb.assign(h[i].begin() + a.nrhs, h[i].end());
        for (int c = 0; c < a.nrhs; ++c) {
          a.relres[c] = a.bb[c] > 0 ? 1.0 : 0.0;
          a.done[c] = a.bb[c] == 0;
          all = all && a.done[c];
        }
      } else {
        for (int c = 0; c < a.nrhs; ++c) {
          if (!a.done[c]) {
            a.relres[c] = std::sqrt(h[i][c] / a.bb[c]);
            a.iters[c] = a.it;
            if (a.relres[c] <= a.r->tol) a.done[c] = 1;
          }
          all = all && a.done[c];
        }
      }
      a.r->relres = *std::max_element(a.relres.begin(), a.relres.end());
      a.r->iters = *std::max_element(a.iters.begin(), a.iters.end());
      if (all || a.it >= a.r->maxit) retire.push_back(&a);
      else cont.push_back(&a);
    }
    if (!cont.empty()) batched_apply(cont);
    for (Active* a : cont) {
      double* part = a->sc + 8 * a->nrhs;
      double* rz = a->sc;
      double* rzn = a->sc + a->nrhs;
      launch_dot(a->rv, a->z, a->n3, a->nrhs, a->n3, part, rzn, sstream_);
      if (a->fresh) {
        HIF_CK(cudaMemcpyAsync(a->p, a->z, a->n3 * a->nrhs * 8, cudaMemcpyDeviceToDevice,
                               sstream_));
      } else {
        launch_pcg_update_p(a->p, a->z, rzn, rz, a->n3, a->nrhs, a->n3, sstream_);
      }
      HIF_CK(cudaMemcpyAsync(rz, rzn, a->nrhs * 8, cudaMemcpyDeviceToDevice, sstream_));
      a->fresh = false;
      a->it += 1;
    }
    HIF_CK(cudaGetLastError());
    if (!retire.empty()) {
      for (Active* a : retire)
        HIF_CK(cudaMemcpyAsync(a->r->xout, a->x, a->n3 * a->nrhs * 8, cudaMemcpyDeviceToHost,
                               sstream_));
      HIF_CK(cudaStreamSynchronize(sstream_));
      std::lock_guard<std::mutex> lk(mu_);
      for (Active* a : retire) {
        Op& o = ops_[a->r->op];
        o.active -= 1;
        used_ -= solve_bytes(*a->e, a->nrhs);
        a->bufs.release(sstream_);
        finish(a->r, HIF_OK, "");
      }
      act.erase(std::remove_if(act.begin(), act.end(),
                               [](const std::unique_ptr<Active>& a) { return a->r->done; }),
                act.end());
      done_cv_.notify_all();
      cv_.notify_all();
    }
  }

  long long budget_;
  int slots_;
  int device_ = 0;
  cudaStream_t sstream_ = nullptr;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  bool stop_ = false;
  std::map<int, Op> ops_;
  std::deque<Req*> fq_;
  std::list<Req*> sq_;
  std::map<long long, std::unique_ptr<Req>> reqs_;
  std::map<int, long long> measured_;  // grid size -> factorization footprint
  long long next_id_ = 0, used_ = 0, completed_ = 0, ticks_ = 0, merged_launches_ = 0;
  std::thread solver_;
  std::vector<std::thread> workers_;
};

}  // namespace hif

struct hif_server_s {
  std::unique_ptr<hif::Server> s;
};

extern "C" {

int hif_server_create(long long budget_bytes, int max_active_solves, int factor_workers,
                      hif_server* out) {
  if (!out || budget_bytes <= 0) return HIF_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    hif::g_last_error = "no CUDA device";
    return HIF_ERR_NODEVICE;
  }
  return guarded([&] {
    auto* h = new hif_server_s;
    h->s.reset(new hif::Server(budget_bytes, max_active_solves, factor_workers));
    *out = h;
  });
}

int hif_server_destroy(hif_server s) {
  if (!s) return HIF_ERR_ARG;
  return guarded([&] { delete s; });
}

int hif_server_submit_factor(hif_server s, int op_id, int N, int P, double epsilon,
                             int partition, int precision, double hstep, const double* ax,
                             const double* ay, const double* az, const double* V,
                             long long* request_id) {
  if (!s || !ax || !ay || !az || !V || !request_id || N < 1 || P < 1 || !(epsilon > 0) ||
      !(hstep > 0) || (precision != HIF_PRECISION_FP64 && precision != HIF_PRECISION_MIXED))
    return HIF_ERR_ARG;
  return guarded([&] {
    std::unique_ptr<hif::Server::Req> r(new hif::Server::Req());
    r->kind = 0;
    r->op = op_id;
    r->N = N;
    r->P = P;
    r->eps = epsilon;
    r->hstep = hstep;
    r->partition = partition;
    r->precision = precision;
    const long long nt = (long long)(N + 2) * (N + 2) * (N + 2);
    r->ax.assign(ax, ax + nt);
    r->ay.assign(ay, ay + nt);
    r->az.assign(az, az + nt);
    r->V.assign(V, V + nt);
    *request_id = s->s->submit(std::move(r));
  });
}

int hif_server_submit_solve(hif_server s, int op_id, const double* b, int nrhs, double tol,
                            int maxit, double* x_out, long long* request_id) {
  if (!s || !b || !x_out || !request_id || nrhs < 1 || !(tol > 0) || maxit < 0)
    return HIF_ERR_ARG;
  return guarded([&] {
    const long long n3 = s->s->dofs(op_id);
    if (n3 <= 0) throw hif::Error{HIF_ERR_ARG, "unknown operator"};
    std::unique_ptr<hif::Server::Req> r(new hif::Server::Req());
    r->kind = 1;
    r->op = op_id;
    r->nrhs = nrhs;
    r->tol = tol;
    r->maxit = maxit;
    r->xout = x_out;
    r->b.assign(b, b + n3 * nrhs);
    *request_id = s->s->submit(std::move(r));
  });
}

int hif_server_wait(hif_server s, long long request_id, int* status, int* iters, double* relres,
                    double* latency_ms) {
  if (!s) return HIF_ERR_ARG;
  return guarded([&] { s->s->wait(request_id, status, iters, relres, latency_ms); });
}

int hif_server_wait_detail(hif_server s, long long request_id, int* status, int* iters,
                           double* relres, double* latency_ms, double* queue_ms) {
  if (!s) return HIF_ERR_ARG;
  return guarded([&] { s->s->wait(request_id, status, iters, relres, latency_ms, queue_ms); });
}

int hif_server_release(hif_server s, int op_id) {
  if (!s) return HIF_ERR_ARG;
  return guarded([&] { s->s->release(op_id); });
}

int hif_server_stats(hif_server s, long long* device_bytes, long long* resident_ops,
                     long long* completed, long long* ticks, long long* batched_launches) {
  if (!s) return HIF_ERR_ARG;
  return guarded([&] { s->s->stats(device_bytes, resident_ops, completed, ticks, batched_launches); });
}

}  // extern "C"
