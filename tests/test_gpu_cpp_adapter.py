"""The C++ adapter (include/ibk.hpp) run on the GPU: a program built against
it and the library runs the reference's call forms -- spread(n, x, fl),
spread(n, x, fl, fe), interp(n, x, ue, ul) and interp(n, x, ue) -- on the
reference's test/grid.cc setup (periodic 10 um cube, fd::mac{16}, two points
at 5 um, unit forces and velocities) and on a walled channel with seeded
points.  Outputs against the oracle: interpolation bit for bit (both call
forms), spread within 1e-12 * sum |res w F| per face (both call forms: FP64
spreads agree with each other and the reference up to summation order)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _read_cases(path):
    raw = open(path, "rb").read()
    pos = 0

    def take(dtype, count):
        nonlocal pos
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=pos)
        pos += a.nbytes
        return a

    cases = []
    while pos < len(raw):
        dims = int(take(np.int32, 1)[0])
        n = int(take(np.int32, 1)[0])
        lengths = take(np.float64, 3)
        bounds = take(np.int32, 3)
        ref = int(take(np.int32, 1)[0])
        x = take(np.float64, 3 * n)
        fl = take(np.float64, 3 * n)
        ue, sizes = [], []
        for _ in range(dims):
            sz = int(take(np.int64, 1)[0])
            sizes.append(sz)
            ue.append(take(np.float64, sz))
        fe_new, fe_into = [], []
        for c in range(dims):
            fe_new.append(take(np.float64, sizes[c]))
            fe_into.append(take(np.float64, sizes[c]))
        ul_into = take(np.float64, dims * n)
        ul_new = take(np.float64, dims * n)
        cases.append(dict(dims=dims, n=n, lengths=lengths[:dims].tolist(), bounds=bounds[:dims].tolist(),
                          ref=ref, x=x, fl=fl, ue=ue, fe_new=fe_new, fe_into=fe_into, ul_into=ul_into,
                          ul_new=ul_new))
    return cases


def test_cpp_adapter_runs_reference_call_forms(ibk, oracle, cuda, tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    lib_dir = os.path.join(ROOT, "ib.cu_b200", "lib")
    exe = tmp_path / "adapter_run"
    r = subprocess.run([cxx, "-std=c++17", "-O1", os.path.join(ROOT, "tests", "cpp", "adapter_run.cc"),
                        "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
                        "-L" + lib_dir, "-libk", "-L/usr/local/cuda/lib64", "-lcudart",
                        "-Wl,-rpath," + lib_dir, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = tmp_path / "cases.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for case in _read_cases(str(out)):
        g = oracle.geometry(case["dims"], case["lengths"], case["bounds"], oracle.TAG_MAC, case["ref"])
        want_fe = oracle.spread(g, case["x"], case["fl"])
        absum = oracle.spread(g, case["x"], np.abs(case["fl"]))   # bspline<3>: weights >= 0
        want_ul = oracle.interpolate(g, case["x"], case["ue"])
        for c in range(case["dims"]):
            for got in (case["fe_new"][c], case["fe_into"][c]):
                assert np.all(np.abs(got - want_fe[c]) <= 1e-12 * absum[c] + 1e-300)
        assert np.array_equal(case["ul_into"], case["ul_new"])
        assert np.array_equal(case["ul_into"], want_ul)
