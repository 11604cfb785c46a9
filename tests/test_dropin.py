"""The reference's own drivers compile unchanged against the drop-in header.

tests/HIFDE3D/main.cpp and darcy.cpp of arbenson/HIFDE3D include "hifde3d.hpp"
and use HIFFactor<double>, NumTns, Vector, Index3, SetupStencil, SpMV,
Apply and RelativeErrorNorm2. Built against include/hifde3d_b200/hifde3d.hpp and
libhif_b200.so they must compile and link as they are (CPU-only check; the GPU
run is in test_gpu_dropin.py).
"""
import os

import pytest

from hifde3d_b200 import build as b

REF = "/root/reference"


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
