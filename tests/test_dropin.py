"""The reference's own drivers compile unchanged against the drop-in header.

tests/HIFDE3D/main.cpp and darcy.cpp of arbenson/HIFDE3D include "hifde3d.hpp"
and use HIFFactor<double>, NumTns, Vector, Index3, SetupStencil, SpMV,
Apply and RelativeErrorNorm2. Built against include/hifde3d_b200/hifde3d.hpp and
libhif_b200.so they must compile and link as they are (CPU-only check; the GPU
run is in test_gpu_dropin.py).
"""
import os
import subprocess

import pytest

from hifde3d_b200 import build as b

# the reference's source tree (HIFDE3D_REFERENCE overrides the default location)
REF = os.environ.get("HIFDE3D_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "tests", "HIFDE3D")),
                    reason="reference sources not present")
def test_reference_drivers_compile_against_shim():
    outs = b.build_drivers(REF)
    for o in outs:
        assert os.path.exists(o) and os.access(o, os.X_OK)


def test_shim_declares_reference_api():
    with open(os.path.join(os.path.dirname(b.HERE), "include", "hifde3d_b200", "hifde3d.hpp")) as f:
        text = f.read()
    for name in ("class HIFFactor<double>", "SetupStencil", "inline void Schur",
                 "inline void InterpDecomp", "PivotedQRWrapper", "TriangularSolveWrapper",
                 "inline void SpMV", "RelativeErrorNorm2", "class NumTns", "class Vector",
                 "typedef Vec3T<int> Index3", "class FactorData", "class Dense"):
        assert name in text, name


EXTENSIONS_PROGRAM = r"""
#include "hifde3d.hpp"
using namespace hifde3d;
int main(int argc, char** argv) {
  const int N = 15;
  HIFFactor<double> f(N, 4, 1e-6);
  NumTns<double> A(N + 2, N + 2, N + 2), V(N + 2, N + 2, N + 2);
  SetupStencil(f, N, 1.0 / (N + 1), A, V);
  f.Initialize();
  f.Factor();
  Vector<double> b((N + 1) * (N + 1) * (N + 1), 1.0), x;
  double rr = 0;
  int it = argc > 1 ? f.SolveGMRES(b, x, 1e-10, 100, 30, &rr) : f.SolvePCG(b, x, 1e-10, 100, &rr);
  f.Save(argv[0]);
  f.Load(argv[0]);
  return it > 0 && rr >= 0 ? 0 : 1;
}
"""


def test_shim_extensions_compile_and_link(tmp_path):
    """SolvePCG / SolveGMRES / Save / Load of the drop-in HIFFactor<double> compile
    and link against libhif_b200.so (CPU-only; the C ABI calls they forward to are
    exercised on the GPU by test_gpu_gmres.py and test_gpu_save_load.py)."""
    b.build()
    src = tmp_path / "ext.cpp"
    src.write_text(EXTENSIONS_PROGRAM)
    root = os.path.dirname(b.HERE)
    out = tmp_path / "ext"
    subprocess.run(["g++", "-std=c++14", "-O1", "-Wall", "-Werror",
                    "-I", os.path.join(root, "include", "hifde3d_b200"),
                    "-I", os.path.join(root, "include"), str(src), "-o", str(out),
                    "-L", b.HERE, "-lhif_b200"], check=True)
    assert out.exists()
