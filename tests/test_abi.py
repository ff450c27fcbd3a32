"""CPU checks of the C ABI: the library builds, loads without a GPU, and
exports every entry point include/*.h declares.  No compute call is made."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(ibk_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("ibk_plan_create", "ibk_spread", "ibk_interpolate", "ibk_plan_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol(ibk):
    ibk.build()
    lib = ctypes.CDLL(ibk.LIB_PATH)
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_lists_every_symbol(ibk):
    assert set(ibk.ABI_SYMBOLS) == declared_symbols()


def test_host_only_calls(ibk):
    """Calls that touch no device: version, status strings, null handling."""
    ibk.build()
    lib = ibk.lib()
    assert lib.ibk_version() == 100
    assert lib.ibk_status_string(0) == b"ok"
    assert lib.ibk_plan_destroy(None) == 0
    # n <= 0 returns before touching the plan's device state
    assert lib.ibk_spread(None, 0, None, None, None, None) == 1  # null plan is rejected first
    # batches: argument checks happen before any device work
    h = ctypes.c_void_p()
    assert lib.ibk_batch_create(0, None, ibk._Delta(), 0, 0, ctypes.byref(h)) == 1
    assert lib.ibk_batch_destroy(None) == 0
    assert lib.ibk_batch_run(None, ibk.OP_SPREAD, None) == 1
    assert lib.ibk_batch_bind(None, None, None) == 1


def test_cpp_adapter_compiles(tmp_path):
    """include/ibk.hpp (the reference-shaped C++ surface) compiles against
    the C ABI: operator objects, the allocating overloads and batches."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        import pytest
        pytest.skip("no host C++ compiler")
    src = tmp_path / "use_adapter.cc"
    src.write_text(r'''
#include "ibk.hpp"
int use(const double* x, const double* fl, const double* u0, const double* u1, const double* u2, int n)
{
    ibk::domain dom{ibk::dimension{3.2, ibk::periodic}, ibk::dimension{1.6, ibk::dirichlet},
                    ibk::dimension{3.2, ibk::periodic}};
    ibk::spread spread{ibk::mac{64}, dom, ibk::bspline<3>{}, IBK_PRECISION_FP32C};
    ibk::interpolate interp{ibk::mac{64}, dom, ibk::bspline<3>{}};
    auto fe = spread(n, x, fl);
    auto ul = interp(n, x, {u0, u1, u2});
    spread(n, x, fl, {fe[0].values(), fe[1].values(), fe[2].values()});
    std::vector<std::pair<ibk::mac, ibk::domain>> insts{{ibk::mac{32}, dom}, {ibk::mac{64}, dom}};
    ibk::batch b{insts, ibk_delta{IBK_DELTA_BSPLINE, 3}, IBK_PRECISION_FP32C, 2 * n};
    b.set_step(1e-3, 1e-3);
    return (int) ul.size();
}
''')
    inc = os.path.join(ROOT, "include")
    cuda_inc = "/usr/local/cuda/include"
    r = subprocess.run([cxx, "-std=c++17", "-c", str(src), "-I" + inc, "-I" + cuda_inc,
                        "-o", str(tmp_path / "use_adapter.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
