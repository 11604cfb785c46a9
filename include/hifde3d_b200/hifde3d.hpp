// Header-only drop-in for arbenson/HIFDE3D's C++ API (Scalar = double) on top of
// the B200 C ABI (hif_b200.h). A program written against the reference's
// include/hifde3d.hpp compiles unchanged with
//     -I <repo>/include/hifde3d_b200 -I <repo>/include  -L <lib dir> -lhif_b200
// and runs its factorization, apply and SpMV on the GPU.
//
// Provided (reference file:line of the interface each replaces):
//   Vector<T>               include/hifde3d/core/vector.hpp:20-58
//   Vec3T<T>, Index3        include/vec3t.hpp:10-197
//   NumTns<F>               include/numtns.hpp:9-170 (i-fastest storage)
//   Dense<T>                include/hifde3d/core/dense.hpp:24-660 (column-major, ldim)
//   IndexData, FactorData   include/data.hpp:11-110
//   HIFFactor<double>       include/Factor.hpp:8-203
//   SetupStencil            include/setup_stencil.hpp:6-76
//   Schur                   include/Schur.hpp:72-100
//   InterpDecomp, PivotedQRWrapper, TriangularSolveWrapper
//                           include/InterpDecomp.hpp:18-30
//   SpMV, RelativeErrorNorm2 include/Factor.hpp:205-209
//   DumpCallStack           src/global.cpp:27-35 (no call stack is kept)
// Errors: the C status codes are turned into std::runtime_error (the reference
// throws std::logic_error / std::runtime_error in non-RELEASE builds).
#ifndef HIFDE3D_B200_SHIM_HPP_
#define HIFDE3D_B200_SHIM_HPP_

#include <cassert>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../hif_b200.h"

namespace hifde3d {

inline void ThrowOnError(int status, const char* where) {
  if (status != HIF_OK) {
    throw std::runtime_error(std::string(where) + ": " + hif_last_error());
  }
}

inline void DumpCallStack() {}

inline int pow2(int l) { return 1 << l; }

template <typename T>
class Vector {
 public:
  Vector() {}
  explicit Vector(int height) : d_(height) {}
  Vector(int height, const T x) : d_(height, x) {}
  int Height() const { return (int)d_.size(); }
  int Size() const { return (int)d_.size(); }
  void Resize(int height) { d_.resize(height); }
  void Clear() { d_.clear(); }
  void Set(int i, T value) { d_[i] = value; }
  T Get(int i) const { return d_[i]; }
  T& operator[](int i) { return d_[i]; }
  const T& operator[](int i) const { return d_[i]; }
  void PushBack(T v) { d_.push_back(v); }
  T* Buffer() { return d_.data(); }
  const T* LockedBuffer() const { return d_.data(); }

 private:
  std::vector<T> d_;
};

template <class T>
class Vec3T {
 public:
  Vec3T() { v_[0] = v_[1] = v_[2] = T(0); }
  Vec3T(T a, T b, T c) {
    v_[0] = a;
    v_[1] = b;
    v_[2] = c;
  }
  T& operator()(int i) { return v_[i]; }
  const T& operator()(int i) const { return v_[i]; }
  T& operator[](int i) { return v_[i]; }
  const T& operator[](int i) const { return v_[i]; }

 private:
  T v_[3];
};
typedef Vec3T<int> Index3;

template <class F>
class NumTns {
 public:
  NumTns(int m = 0, int n = 0, int p = 0) : m_(m), n_(n), p_(p), d_((size_t)m * n * p) {}
  void resize(int m, int n, int p) {
    m_ = m;
    n_ = n;
    p_ = p;
    d_.assign((size_t)m * n * p, F());
  }
  F& operator()(int i, int j, int k) { return d_[i + (size_t)j * m_ + (size_t)k * m_ * n_]; }
  const F& operator()(int i, int j, int k) const {
    return d_[i + (size_t)j * m_ + (size_t)k * m_ * n_];
  }
  F& operator()(Index3 ind) { return (*this)(ind(0), ind(1), ind(2)); }
  const F& operator()(Index3 ind) const { return (*this)(ind(0), ind(1), ind(2)); }
  int m() const { return m_; }
  int n() const { return n_; }
  int p() const { return p_; }
  F* data() { return d_.data(); }
  const F* data() const { return d_.data(); }

 private:
  int m_, n_, p_;
  std::vector<F> d_;
};
typedef NumTns<int> IntNumTns;

template <typename T>
class Dense {
 public:
  Dense() : h_(0), w_(0) {}
  Dense(int h, int w) : h_(h), w_(w), d_((size_t)h * w) {}
  int Height() const { return h_; }
  int Width() const { return w_; }
  int LDim() const { return h_ > 0 ? h_ : 1; }
  void Resize(int h, int w) {
    h_ = h;
    w_ = w;
    d_.assign((size_t)h * w, T());
  }
  void Clear() { Resize(0, 0); }
  T Get(int i, int j) const { return d_[i + (size_t)j * h_]; }
  void Set(int i, int j, T v) { d_[i + (size_t)j * h_] = v; }
  T* Buffer(int i = 0, int j = 0) { return d_.data() + i + (size_t)j * h_; }
  const T* LockedBuffer(int i = 0, int j = 0) const { return d_.data() + i + (size_t)j * h_; }

 private:
  int h_, w_;
  std::vector<T> d_;
};

enum Face { TOP = 0, BOTTOM, RIGHT, LEFT, FRONT, BACK };

class IndexData {
 public:
  std::vector<int>& global_inds() { return g_; }
  std::vector<int>& redundant_inds() { return r_; }
  std::vector<int>& skeleton_inds() { return s_; }

 private:
  std::vector<int> g_, r_, s_;
};

template <typename Scalar>
class FactorData {
 public:
  Dense<Scalar>& A_22() { return a22_; }
  Dense<Scalar>& A_22_inv() { return inv_; }
  Dense<Scalar>& X_mat() { return x_; }
  Dense<Scalar>& Schur_comp() { return s_; }
  Dense<Scalar>& W_mat() { return w_; }
  int NumDOFsEliminated() { return (int)ind_.redundant_inds().size(); }
  IndexData& ind_data() { return ind_; }
  void set_face(Face f) { face_ = f; }
  Face face() { return face_; }

 private:
  IndexData ind_;
  Dense<Scalar> a22_, inv_, x_, s_, w_;
  Face face_ = TOP;
};

// sp_matrix(): the operator kept on the GPU (the reference's Sparse<Scalar>).
template <typename Scalar>
class SparseOperator {
 public:
  explicit SparseOperator(hif_handle h = nullptr) : h_(h) {}
  hif_handle handle() const { return h_; }

 private:
  hif_handle h_;
};

template <typename Scalar>
class HIFFactor;

template <>
class HIFFactor<double> {
 public:
  HIFFactor(int N, int P, double epsilon) : N_(N), P_(P), eps_(epsilon) {
    ThrowOnError(hif_create(N, P, epsilon, HIF_PARTITION_REFERENCE, &h_), "HIFFactor");
    op_ = SparseOperator<double>(h_);
  }
  ~HIFFactor() { hif_destroy(h_); }
  HIFFactor(const HIFFactor&) = delete;
  HIFFactor& operator=(const HIFFactor&) = delete;

  void Initialize() { ThrowOnError(hif_initialize(h_), "HIFFactor::Initialize"); }
  void Factor() { ThrowOnError(hif_factor(h_), "HIFFactor::Factor"); }

  Index3 Linear2TensorInd(int ind) {
    const int NC = N_ + 1;
    return Index3(ind % NC, (ind / NC) % NC, ind / (NC * NC));
  }
  int Tensor2LinearInd(Index3 ind) {
    const int NC = N_ + 1;
    return ind(0) + NC * ind(1) + NC * NC * ind(2);
  }
  void Apply(Vector<double>& u, bool apply_inverse = false) {
    ThrowOnError(hif_apply(h_, u.Buffer(), 1, u.Size(), apply_inverse ? 1 : 0),
                 "HIFFactor::Apply");
  }

  // ---- extensions (no counterpart in the reference) ----------------------
  // Iterative solves with the factor as preconditioner and an FP64 residual on the
  // operator, x0 = 0: PCG for the symmetric face-coefficient operator, GMRES for
  // SetupStencil's node operator (not symmetric for variable coefficients).
  // Return the iteration count; `relres` receives |b - A x| / |b|.
  int SolvePCG(const Vector<double>& b, Vector<double>& x, double tol = 1e-10,
               int maxit = 200, double* relres = nullptr) {
    x.Resize(b.Size());
    int it = 0;
    double rr = 0;
    ThrowOnError(hif_solve_pcg(h_, b.LockedBuffer(), x.Buffer(), 1, b.Size(), tol, maxit, &it,
                               &rr),
                 "HIFFactor::SolvePCG");
    if (relres) *relres = rr;
    return it;
  }
  int SolveGMRES(const Vector<double>& b, Vector<double>& x, double tol = 1e-10,
                 int maxit = 200, int restart = 30, double* relres = nullptr) {
    x.Resize(b.Size());
    int it = 0;
    double rr = 0;
    ThrowOnError(hif_solve_gmres(h_, b.LockedBuffer(), x.Buffer(), 1, b.Size(), tol, maxit,
                                 restart, &it, &rr),
                 "HIFFactor::SolveGMRES");
    if (relres) *relres = rr;
    return it;
  }
  // The factorization (and the operator) to / from a file; Load needs a
  // HIFFactor of the saved N, P and epsilon and replaces what it held.
  void Save(const std::string& path) {
    ThrowOnError(hif_save_factor(h_, path.c_str()), "HIFFactor::Save");
  }
  void Load(const std::string& path) {
    ThrowOnError(hif_load_factor(h_, path.c_str()), "HIFFactor::Load");
  }

  void set_N(int) { throw std::logic_error("set_N: recreate the HIFFactor"); }
  int N() { return N_; }
  void set_P(int) { throw std::logic_error("set_P: recreate the HIFFactor"); }
  int P() { return P_; }
  void set_epsilon(double) { throw std::logic_error("set_epsilon: recreate the HIFFactor"); }
  double epsilon() { return eps_; }
  SparseOperator<double>& sp_matrix() { return op_; }
  hif_handle handle() { return h_; }

 private:
  int N_, P_;
  double eps_;
  hif_handle h_ = nullptr;
  SparseOperator<double> op_;
};

inline void SetupStencil(HIFFactor<double>& factor, int N, double h, NumTns<double>& A,
                         NumTns<double>& V) {
  ThrowOnError(hif_setup_stencil(factor.handle(), N, h, A.data(), V.data()), "SetupStencil");
}

inline void SpMV(SparseOperator<double>& A, Vector<double>& x, Vector<double>& y) {
  ThrowOnError(hif_spmv(A.handle(), x.Buffer(), y.Buffer(), 1, x.Size(), 1), "SpMV");
}

inline double RelativeErrorNorm2(Vector<double>& x, Vector<double>& y) {
  double err = 0, norm = 0;
  for (int i = 0; i < x.Size(); ++i) {
    const double d = std::abs(x.Get(i) - y.Get(i));
    err += d * d;
    norm += std::abs(x.Get(i)) * std::abs(x.Get(i));
  }
  return std::sqrt(err / norm);
}

inline void Schur(Dense<double>& matrix, FactorData<double>& data) {
  std::vector<int>& r = data.ind_data().redundant_inds();
  std::vector<int>& s = data.ind_data().skeleton_inds();
  const int nr = (int)r.size(), ns = (int)s.size();
  data.A_22().Resize(nr, nr);
  data.A_22_inv().Resize(nr, nr);
  data.X_mat().Resize(nr, ns);
  data.Schur_comp().Resize(ns, ns);
  ThrowOnError(hif_schur(matrix.Buffer(), matrix.Height(), matrix.LDim(), r.data(), nr, s.data(),
                         ns, data.A_22().Buffer(), data.A_22_inv().Buffer(),
                         data.X_mat().Buffer(), data.Schur_comp().Buffer()),
               "Schur");
}

inline void InterpDecomp(Dense<double>& M, Dense<double>& W, std::vector<int>& skeleton_cols,
                         std::vector<int>& redundant_cols, double epsilon) {
  const int m = M.Height(), n = M.Width();
  std::vector<double> w((size_t)n * n / 4 + n + 1);
  std::vector<int> sk(n), rd(n);
  int k = 0;
  ThrowOnError(hif_interp_decomp(M.Buffer(), m, n, M.LDim(), epsilon, w.data(), sk.data(),
                                 rd.data(), &k),
               "InterpDecomp");
  skeleton_cols.insert(skeleton_cols.end(), sk.begin(), sk.begin() + k);
  redundant_cols.insert(redundant_cols.end(), rd.begin(), rd.begin() + (n - k));
  W.Resize(k, n - k);
  for (int j = 0; j < n - k; ++j)
    for (int i = 0; i < k; ++i) W.Set(i, j, w[i + (size_t)j * k]);
}

inline void PivotedQRWrapper(Dense<double>& A, std::vector<int>& jpvt) {
  jpvt.assign(A.Width(), 0);
  ThrowOnError(hif_pivoted_qr(A.Buffer(), A.Height(), A.Width(), A.LDim(), jpvt.data()),
               "PivotedQRWrapper");
}

inline void TriangularSolveWrapper(Dense<double>& R, Dense<double>& B) {
  ThrowOnError(hif_triangular_solve(R.Buffer(), B.Height(), R.LDim(), B.Buffer(), B.Width(),
                                    B.LDim()),
               "TriangularSolveWrapper");
}

}  // namespace hifde3d

#endif  // HIFDE3D_B200_SHIM_HPP_
