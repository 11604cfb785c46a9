// Test infrastructure: a driver compiled against the reference's own sources
// (src/Factor.cpp, src/InterpDecomp.cpp, src/hmat_tools/*.cpp) that records
// what the reference computes, so that the CPU restatement in hif_oracle.py and
// the CUDA path can be checked against it. It is never linked into the product.
//
// Modes
//   dump <N> <P> <eps> <A.bin> <V.bin> <u.bin> <out.bin>
//       Runs the reference's level loop (the same calls HIFFactor::Factor makes,
//       src/Factor.cpp:50-62) and writes, per level and per block, the index
//       data and the matrices A_22, A_22^{-1}, X, S (before UpdateMatrixAndDOFs
//       clears it, src/Factor.cpp:293) and W; then Apply(u,false), Apply(u,true)
//       (src/Factor.cpp:992-1081) and the driver's e_a / e_s check
//       (tests/HIFDE3D/main.cpp:88-134) on the v = 1 vector.
//   dumpf <N> <P> <eps> <ax.bin> <ay.bin> <az.bin> <V.bin> <u.bin> <out.bin>
//       dump on the face-coefficient operator (see timef).
//   time <N> <P> <eps> <max_levels> [A.bin V.bin]
//       Wall-clocks SetupStencil, each level's Schur / skeletonization / update
//       phase and one inverse Apply; prints one JSON object. max_levels < 0
//       runs the whole factorization. Each level's times are also written to
//       stderr as a "LEVEL {...}" line (flushed) the moment the level ends, so
//       that a run stopped by a wall-clock cap still records the levels it
//       reached.
//   timef <N> <P> <eps> <max_levels> <ax.bin> <ay.bin> <az.bin> <V.bin>
//       The same timings on the symmetric face-coefficient operator
//       -div(a grad u) + V u: the reference factors whatever its sparse matrix
//       holds, so the probe fills sp_matrix() through the reference's own
//       Sparse::Add (include/hifde3d/core/sparse.hpp:34), one row per DOF as
//       SetupStencil does (include/setup_stencil.hpp:17-70), with diagonal
//       V + sum of the six face coefficients / h^2 and -a_face / h^2 for each
//       interior neighbour. ax(i,j,k) couples nodes (i,j,k) and (i+1,j,k), ay
//       and az likewise; all four arrays are (NC+1)^3, i fastest.
//
// Input tensors are (NC+1)^3 float64 arrays in the reference's NumTns order
// (i fastest, include/numtns.hpp:99); u is NC^3 float64 in the DOF order
// i + NC*j + NC^2*k (src/Factor.cpp:79-89).

#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#define private public
#include "hifde3d.hpp"
#undef private

using namespace hifde3d;

namespace {

double now() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::vector<double> read_doubles(const char* path, size_t n) {
    std::vector<double> v(n);
    FILE* f = std::fopen(path, "rb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
    size_t got = std::fread(v.data(), sizeof(double), n, f);
    std::fclose(f);
    if (got != n) { std::fprintf(stderr, "short read %s\n", path); std::exit(2); }
    return v;
}

struct Out {
    FILE* f;
    void i32(int v) { std::fwrite(&v, 4, 1, f); }
    void f64(double v) { std::fwrite(&v, 8, 1, f); }
    void ivec(const std::vector<int>& v) {
        i32((int)v.size());
        if (!v.empty()) std::fwrite(v.data(), 4, v.size(), f);
    }
    void dense(Dense<double>& D) {
        i32(D.Height());
        i32(D.Width());
        for (int j = 0; j < D.Width(); ++j)
            for (int i = 0; i < D.Height(); ++i) f64(D.Get(i, j));
    }
    void vec(Vector<double>& v) {
        i32(v.Size());
        for (int i = 0; i < v.Size(); ++i) f64(v.Get(i));
    }
};

void dump_blocks(Out& o, std::vector<FactorData<double> >& blocks, bool skel) {
    // Skeletonization leaves unused trailing entries when a face is absent
    // (LevelFactorSkel sizes the vector for every possible face); keep only
    // the ones a face was written into.
    int n = 0;
    for (size_t b = 0; b < blocks.size(); ++b)
        if (!skel || !blocks[b].ind_data().global_inds().empty()) ++n;
    o.i32(n);
    for (size_t b = 0; b < blocks.size(); ++b) {
        FactorData<double>& d = blocks[b];
        if (skel && d.ind_data().global_inds().empty()) continue;
        o.i32(skel ? (int)d.face() : -1);
        o.ivec(d.ind_data().global_inds());
        o.ivec(d.ind_data().redundant_inds());
        o.ivec(d.ind_data().skeleton_inds());
        o.dense(d.A_22());
        o.dense(d.A_22_inv());
        o.dense(d.X_mat());
        o.dense(d.Schur_comp());
        o.dense(d.W_mat());
    }
}

void setup(HIFFactor<double>& f, int NC, NumTns<double>& A, NumTns<double>& V,
           const char* fa, const char* fv) {
    size_t nt = (size_t)(NC + 1) * (NC + 1) * (NC + 1);
    if (fa) {
        std::vector<double> a = read_doubles(fa, nt), v = read_doubles(fv, nt);
        for (size_t t = 0; t < nt; ++t) {
            A._data[t] = a[t];
            V._data[t] = v[t];
        }
    } else {
        for (size_t t = 0; t < nt; ++t) {
            A._data[t] = 1.0;
            V._data[t] = 0.0;
        }
    }
    SetupStencil(f, NC - 1, 1.0 / NC, A, V);
}

// Face-coefficient operator into the reference's sparse matrix (see timef).
void setup_faces(HIFFactor<double>& f, int NC, const char* fax, const char* fay,
                 const char* faz, const char* fv) {
    const size_t nt = (size_t)(NC + 1) * (NC + 1) * (NC + 1);
    std::vector<double> ax = read_doubles(fax, nt), ay = read_doubles(fay, nt),
                        az = read_doubles(faz, nt), vv = read_doubles(fv, nt);
    const int N = NC - 1, T = NC + 1;
    const double h = 1.0 / NC, hh = h * h;
    auto at = [T](const std::vector<double>& a, int i, int j, int k) {
        return a[i + (size_t)T * (j + (size_t)T * k)];
    };
    Sparse<double>& matrix = f.sp_matrix();
    for (int i = 1; i <= N; ++i)
        for (int j = 1; j <= N; ++j)
            for (int k = 1; k <= N; ++k) {
                const double w[6] = {at(ax, i - 1, j, k), at(ax, i, j, k), at(ay, i, j - 1, k),
                                     at(ay, i, j, k),     at(az, i, j, k - 1), at(az, i, j, k)};
                const int nb[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k},
                                      {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
                Vector<int> jidx;
                Vector<double> vals;
                double d = at(vv, i, j, k);
                for (int q = 0; q < 6; ++q) d += w[q] / hh;
                jidx.PushBack(f.Tensor2LinearInd(Index3(i, j, k)));
                vals.PushBack(d);
                for (int q = 0; q < 6; ++q) {
                    const int a = nb[q][0], b = nb[q][1], c = nb[q][2];
                    if (a < 1 || a > N || b < 1 || b > N || c < 1 || c > N) continue;
                    jidx.PushBack(f.Tensor2LinearInd(Index3(a, b, c)));
                    vals.PushBack(-w[q] / hh);
                }
                matrix.Add(f.Tensor2LinearInd(Index3(i, j, k)), jidx, vals);
            }
}

int mode_dump(int argc, char** argv, bool faces) {
    if (argc != (faces ? 11 : 9)) return 2;
    int N = std::atoi(argv[2]), P = std::atoi(argv[3]);
    double eps = std::atof(argv[4]);
    HIFFactor<double> f(N, P, eps);
    int NC = N + 1;
    NumTns<double> A(NC + 1, NC + 1, NC + 1), V(NC + 1, NC + 1, NC + 1);
    if (faces)
        setup_faces(f, NC, argv[5], argv[6], argv[7], argv[8]);
    else
        setup(f, NC, A, V, argv[5], argv[6]);
    const char* u_path = argv[faces ? 9 : 7];
    const char* out_path = argv[faces ? 10 : 8];
    std::vector<double> u0 = read_doubles(u_path, (size_t)NC * NC * NC);

    // Driver check vector (tests/HIFDE3D/main.cpp:88-103): v = 1 on DOFs.
    Vector<double> v(NC * NC * NC), w(NC * NC * NC);
    for (int k = 0; k < NC; ++k)
        for (int j = 0; j < NC; ++j)
            for (int i = 0; i < NC; ++i)
                v.Set(f.Tensor2LinearInd(Index3(i, j, k)), (i && j && k) ? 1.0 : 0.0);
    SpMV(f.sp_matrix(), v, w);
    Vector<double> Au(NC * NC * NC), uvec(NC * NC * NC);
    for (int t = 0; t < NC * NC * NC; ++t) uvec.Set(t, u0[t]);
    SpMV(f.sp_matrix(), uvec, Au);

    Out o{std::fopen(out_path, "wb")};
    if (!o.f) return 2;
    std::fwrite("HIFG", 1, 4, o.f);
    o.i32(1);
    f.Initialize();
    int L = (int)f.schur_level_data_.size();
    o.i32(N); o.i32(P); o.i32(L); o.f64(eps);
    for (int level = 0; level < L; ++level) {
        int width = pow2(level) * P, cpd = NC / width;
        f.LevelFactorSchur(cpd, level);
        dump_blocks(o, f.schur_level_data_[level], false);
        f.UpdateMatrixAndDOFs(f.schur_level_data_[level]);
        if (level < L - 1) {
            f.LevelFactorSkel(cpd, level);
            dump_blocks(o, f.skel_level_data_[level], true);
            f.UpdateMatrixAndDOFs(f.skel_level_data_[level]);
        } else {
            o.i32(0);
        }
    }
    Vector<double> fu(uvec), fiu(uvec), fiAu(Au);
    f.Apply(fu, false);
    f.Apply(fiu, true);
    f.Apply(fiAu, true);
    o.vec(Au);
    o.vec(fu);
    o.vec(fiu);
    o.vec(fiAu);
    Vector<double> u1(v);
    f.Apply(u1, false);
    double e_a = RelativeErrorNorm2(w, u1);
    f.Apply(w, true);
    double e_s = RelativeErrorNorm2(v, w);
    o.f64(e_a);
    o.f64(e_s);
    std::fclose(o.f);
    return 0;
}

int mode_time(int argc, char** argv, bool faces) {
    if (faces ? argc != 10 : (argc != 6 && argc != 8)) return 2;
    int N = std::atoi(argv[2]), P = std::atoi(argv[3]);
    double eps = std::atof(argv[4]);
    int max_levels = std::atoi(argv[5]);
    HIFFactor<double> f(N, P, eps);
    int NC = N + 1;
    NumTns<double> A(NC + 1, NC + 1, NC + 1), V(NC + 1, NC + 1, NC + 1);
    double t0 = now();
    if (faces)
        setup_faces(f, NC, argv[6], argv[7], argv[8], argv[9]);
    else
        setup(f, NC, A, V, argc == 8 ? argv[6] : nullptr, argc == 8 ? argv[7] : nullptr);
    double t_setup = now() - t0;
    f.Initialize();
    int L = (int)f.schur_level_data_.size();
    int run_levels = (max_levels < 0 || max_levels > L) ? L : max_levels;
    std::ostringstream lv;
    double t_schur = 0, t_skel = 0, t_upd = 0;
    double tf = now();
    for (int level = 0; level < run_levels; ++level) {
        int width = pow2(level) * P, cpd = NC / width;
        double a = now();
        f.LevelFactorSchur(cpd, level);
        double b = now();
        f.UpdateMatrixAndDOFs(f.schur_level_data_[level]);
        double c = now();
        double ks = 0, ku = 0;
        if (level < L - 1) {
            double d = now();
            f.LevelFactorSkel(cpd, level);
            double e = now();
            f.UpdateMatrixAndDOFs(f.skel_level_data_[level]);
            ks = e - d;
            ku = now() - e;
        }
        t_schur += b - a; t_upd += (c - b) + ku; t_skel += ks;
        std::ostringstream one;
        one << "{\"level\":" << level << ",\"schur_s\":" << (b - a) << ",\"skel_s\":" << ks
            << ",\"update_s\":" << (c - b) + ku << ",\"elapsed_s\":" << now() - tf << "}";
        lv << (level ? "," : "") << one.str();
        std::fprintf(stderr, "LEVEL %s\n", one.str().c_str());
        std::fflush(stderr);
    }
    double t_factor = now() - tf;
    double t_apply = -1;
    if (run_levels == L) {
        Vector<double> u(NC * NC * NC);
        for (int t = 0; t < NC * NC * NC; ++t) u.Set(t, 1.0);
        double a = now();
        f.Apply(u, true);
        t_apply = now() - a;
    }
    std::printf("{\"N\":%d,\"P\":%d,\"eps\":%g,\"levels\":%d,\"levels_run\":%d,"
                "\"setup_s\":%.6f,\"factor_s\":%.6f,\"schur_s\":%.6f,\"skel_s\":%.6f,"
                "\"update_s\":%.6f,\"apply_inv_s\":%.6f,\"per_level\":[%s]}\n",
                N, P, eps, L, run_levels, t_setup, t_factor, t_schur, t_skel, t_upd,
                t_apply, lv.str().c_str());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    // The reference prints progress lines on stdout (src/Factor.cpp:48,211,...);
    // send them to stderr so stdout carries only this probe's result.
    std::cout.rdbuf(std::cerr.rdbuf());
    if (argc < 2) return 2;
    std::string m = argv[1];
    if (m == "dump") return mode_dump(argc, argv, false);
    if (m == "dumpf") return mode_dump(argc, argv, true);
    if (m == "time") return mode_time(argc, argv, false);
    if (m == "timef") return mode_time(argc, argv, true);
    return 2;
}
