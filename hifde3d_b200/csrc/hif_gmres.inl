// Restarted GMRES(m) with the factor's inverse apply as right preconditioner:
// the Krylov space of A F^{-1} is built from r0 = b - A x0, and
// x = x0 + F^{-1} V y, so the residual the iteration minimises is the true
// FP64 residual b - A x on the operator (y = argmin |beta e1 - H y|, Givens
// rotations on the host). The reference has no iterative solver (its driver
// only reports e_a / e_s, tests/HIFDE3D/main.cpp:121-134); GMRES is the solver
// for its own node-coefficient operator (include/setup_stencil.hpp:6-76), which
// is not symmetric for variable coefficients, so CG does not apply to it.
//
// Orthogonalisation: classical Gram-Schmidt applied twice (CGS2), each pass one
// set of fused dot launches (w against every basis vector) and one fused update
// launch, so an Arnoldi step costs one preconditioner apply, one operator apply,
// two dot/update passes and one norm, with a single device-to-host read per step
// (the new Hessenberg column). Every right-hand side runs its own Arnoldi process
// in the same launches; a column that has converged (or reached maxit) is
// carried with zero basis vectors. All reductions have a fixed order, so the
// solve is bit-reproducible. Convergence is decided on the true residual
// recomputed at the end of each cycle; the Givens estimate only ends a cycle.

constexpr int kGmresMaxRestart = 64;

void solve_gmres_device(Engine& e, const double* db, double* dx, int nrhs, long long ld,
                        double tol, int maxit, int restart, int* iters, double* relres) {
  if (!e.factored) throw Error{HIF_ERR_STATE, "solve before Factor"};
  if (!e.have_op) throw Error{HIF_ERR_STATE, "no operator: call hif_setup_stencil first"};
  if (nrhs <= 0 || ld < e.n3) throw Error{HIF_ERR_ARG, "bad nrhs / ld"};
  if (restart < 1 || restart > kGmresMaxRestart)
    throw Error{HIF_ERR_ARG, "restart must be in 1.." + std::to_string(kGmresMaxRestart)};
  const long long n = e.n3;
  const int m = restart;
  cudaStream_t s = e.stream;
  const size_t vec = (size_t)n * nrhs;
  // V (m + 1 basis vectors) | z | w | r | x, then the small arrays
  double* work = dalloc<double>((size_t)(m + 5) * vec + (size_t)kGmresGroup * nrhs * kDotBlocks +
                                    (size_t)(3 * (m + 1) + 4) * nrhs,
                                s);
  double* V = work;
  double* z = V + (size_t)(m + 1) * vec;
  double* w = z + vec;
  double* r = w + vec;
  double* x = r + vec;
  double* part = x + vec;
  double* hd = part + (size_t)kGmresGroup * nrhs * kDotBlocks;  // first CGS pass, (m + 1) x nrhs
  double* gd = hd + (size_t)(m + 1) * nrhs;                        // second pass
  double* yd = gd + (size_t)(m + 1) * nrhs;                        // cycle solution, m x nrhs
  double* nd = yd + (size_t)(m + 1) * nrhs;                        // norms
  double* scd = nd + nrhs;                                         // per-column scale
  double* oned = scd + nrhs;                                       // ones
  struct Free {
    double* p;
    cudaStream_t s;
    ~Free() { dfree(p, s); }
  } guard{work, s};
  const double vb = 8.0 * n * nrhs;
  auto upload_small = [&](double* d, const std::vector<double>& h) {
    HIF_CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  };
  auto dot_self = [&](const double* a, std::vector<double>& out) {
    e.timed(HIF_KCLASS_VECTOR, 0, vb, [&] { launch_dot(a, a, n, nrhs, n, part, nd, s); }, 2);
    HIF_CK(cudaMemcpyAsync(out.data(), nd, nrhs * sizeof(double), cudaMemcpyDeviceToHost, s));
    e.sync();
  };
  // r = b - A x (boundary planes of b ignored, as in PCG)
  auto residual = [&](bool x_is_zero) {
    for (int c = 0; c < nrhs; ++c)
      HIF_CK(cudaMemcpyAsync(r + c * n, db + c * ld, n * 8, cudaMemcpyDeviceToDevice, s));
    e.timed(HIF_KCLASS_VECTOR, 0, vb, [&] { launch_zero_boundary(r, e.NC, nrhs, n, s); });
    if (x_is_zero) return;
    e.timed(HIF_KCLASS_VECTOR, 13.0 * vb / 8, 9 * vb,
            [&] { launch_stencil_apply(e.d_band, e.NC, x, w, nrhs, n, 0, s); });
    e.timed(HIF_KCLASS_VECTOR, 0, 3 * vb,
            [&] { launch_gmres_axpy(r, w, 1, oned, -1.0, n, nrhs, s); });
  };

  upload_small(oned, std::vector<double>(nrhs, 1.0));
  HIF_CK(cudaMemsetAsync(x, 0, vec * 8, s));
  residual(true);
  std::vector<double> bb(nrhs), rr(nrhs);
  dot_self(r, bb);
  rr = bb;
  std::vector<int> done(nrhs, 0), total(nrhs, 0);
  for (int c = 0; c < nrhs; ++c) {
    iters[c] = 0;
    relres[c] = bb[c] > 0 ? 1.0 : 0.0;
    done[c] = bb[c] > 0 ? 0 : 1;
  }
  // per-column Hessenberg factor R (column-major, (m + 1) x m), rotations, rhs
  std::vector<double> R((size_t)(m + 1) * m * nrhs), cs((size_t)m * nrhs), sn((size_t)m * nrhs),
      gv((size_t)(m + 1) * nrhs), hh((size_t)(m + 1) * nrhs), gg((size_t)(m + 1) * nrhs),
      nrm(nrhs), scale(nrhs), Y((size_t)m * nrhs);
  std::vector<int> steps(nrhs), live(nrhs);
  for (;;) {
    bool any = false;
    for (int c = 0; c < nrhs; ++c) {
      live[c] = !done[c] && total[c] < maxit && rr[c] > 0;
      any = any || live[c];
      const double beta = std::sqrt(rr[c]);
      scale[c] = live[c] ? 1.0 / beta : 0.0;
      gv[(size_t)c * (m + 1)] = live[c] ? beta : 0.0;
      steps[c] = 0;
    }
    if (!any) break;
    upload_small(scd, scale);
    e.timed(HIF_KCLASS_VECTOR, 0, 2 * vb, [&] { launch_gmres_scale(V, r, scd, n, nrhs, s); });
    int j = 0;
    for (; j < m; ++j) {
      bool active = false;
      for (int c = 0; c < nrhs; ++c) active = active || live[c];
      if (!active) break;
      double* Vj = V + (size_t)j * vec;
      // w = A F^{-1} v_j
      HIF_CK(cudaMemcpyAsync(z, Vj, vec * 8, cudaMemcpyDeviceToDevice, s));
      e.apply_device(z, nrhs, n, true);
      e.timed(HIF_KCLASS_VECTOR, 13.0 * vb / 8, 9 * vb,
              [&] { launch_stencil_apply(e.d_band, e.NC, z, w, nrhs, n, 0, s); });
      // two classical Gram-Schmidt passes against v_0 .. v_j
      for (int pass = 0; pass < 2; ++pass) {
        double* coef = pass == 0 ? hd : gd;
        e.timed(HIF_KCLASS_VECTOR, 2.0 * (j + 1) * vb / 8, (j + 2) * vb,
                [&] { launch_gmres_dots(V, j + 1, w, n, nrhs, part, coef, s); },
                2 * ((j + kGmresGroup) / kGmresGroup));
        e.timed(HIF_KCLASS_VECTOR, 2.0 * (j + 1) * vb / 8, (j + 3) * vb,
                [&] { launch_gmres_axpy(w, V, j + 1, coef, -1.0, n, nrhs, s); });
      }
      e.timed(HIF_KCLASS_VECTOR, 0, vb, [&] { launch_dot(w, w, n, nrhs, n, part, nd, s); }, 2);
      HIF_CK(cudaMemcpyAsync(hh.data(), hd, (size_t)(j + 1) * nrhs * 8, cudaMemcpyDeviceToHost, s));
      HIF_CK(cudaMemcpyAsync(gg.data(), gd, (size_t)(j + 1) * nrhs * 8, cudaMemcpyDeviceToHost, s));
      HIF_CK(cudaMemcpyAsync(nrm.data(), nd, nrhs * 8, cudaMemcpyDeviceToHost, s));
      e.sync();
      for (int c = 0; c < nrhs; ++c) {
        scale[c] = 0.0;
        if (!live[c]) continue;
        double* Rc = R.data() + (size_t)c * (m + 1) * m + (size_t)j * (m + 1);
        double* csc = cs.data() + (size_t)c * m;
        double* snc = sn.data() + (size_t)c * m;
        double* gc = gv.data() + (size_t)c * (m + 1);
        for (int i = 0; i <= j; ++i)
          Rc[i] = hh[(size_t)i * nrhs + c] + gg[(size_t)i * nrhs + c];
        const double hn = std::sqrt(std::max(nrm[c], 0.0));
        Rc[j + 1] = hn;
        for (int i = 0; i < j; ++i) {  // earlier rotations
          const double t = csc[i] * Rc[i] + snc[i] * Rc[i + 1];
          Rc[i + 1] = -snc[i] * Rc[i] + csc[i] * Rc[i + 1];
          Rc[i] = t;
        }
        const double den = std::hypot(Rc[j], Rc[j + 1]);
        csc[j] = den > 0 ? Rc[j] / den : 1.0;
        snc[j] = den > 0 ? Rc[j + 1] / den : 0.0;
        Rc[j] = den;
        Rc[j + 1] = 0.0;
        gc[j + 1] = -snc[j] * gc[j];
        gc[j] = csc[j] * gc[j];
        steps[c] = j + 1;
        total[c] += 1;
        const double est = std::fabs(gc[j + 1]) / std::sqrt(bb[c]);
        // a zero new direction (hn = 0) means the Krylov space holds the solution
        if (est <= tol || total[c] >= maxit || !(hn > 0) || den == 0) {
          live[c] = 0;
        } else {
          scale[c] = 1.0 / hn;
        }
      }
      upload_small(scd, scale);
      double* Vn = V + (size_t)(j + 1) * vec;
      e.timed(HIF_KCLASS_VECTOR, 0, 2 * vb, [&] { launch_gmres_scale(Vn, w, scd, n, nrhs, s); });
    }
    // y = R^{-1} g per column, then x += F^{-1} (V y)
    std::fill(Y.begin(), Y.end(), 0.0);
    int used = 0;
    for (int c = 0; c < nrhs; ++c) {
      const int k = steps[c];
      used = std::max(used, k);
      const double* Rc = R.data() + (size_t)c * (m + 1) * m;
      const double* gc = gv.data() + (size_t)c * (m + 1);
      for (int i = k - 1; i >= 0; --i) {
        double t = gc[i];
        for (int q = i + 1; q < k; ++q) t -= Rc[(size_t)q * (m + 1) + i] * Y[(size_t)q * nrhs + c];
        const double d = Rc[(size_t)i * (m + 1) + i];
        Y[(size_t)i * nrhs + c] = d != 0 ? t / d : 0.0;
      }
    }
    if (used == 0) break;
    upload_small(yd, Y);
    HIF_CK(cudaMemsetAsync(z, 0, vec * 8, s));
    e.timed(HIF_KCLASS_VECTOR, 2.0 * used * vb / 8, (used + 2) * vb,
            [&] { launch_gmres_axpy(z, V, used, yd, 1.0, n, nrhs, s); });
    e.apply_device(z, nrhs, n, true);
    e.timed(HIF_KCLASS_VECTOR, 0, 3 * vb, [&] { launch_gmres_axpy(x, z, 1, oned, 1.0, n, nrhs, s); });
    residual(false);
    dot_self(r, rr);
    for (int c = 0; c < nrhs; ++c) {
      if (bb[c] <= 0) continue;
      if (steps[c] > 0) {
        relres[c] = std::sqrt(std::max(rr[c], 0.0) / bb[c]);
        iters[c] = total[c];
      }
      if (relres[c] <= tol) done[c] = 1;
    }
  }
  for (int c = 0; c < nrhs; ++c)
    HIF_CK(cudaMemcpyAsync(dx + c * ld, x + c * n, n * 8, cudaMemcpyDeviceToDevice, s));
  e.sync();
}
