"""The C-ABI library: loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared_functions():
    names = set()
    for h in ("qvti.h", "Myfunctions.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;", text):
            name = m.group(1)
            if name not in ("sizeof",):
                names.add(name)
    return sorted(names)


def test_headers_declare_the_reference_abi():
    names = _declared_functions()
    for ref in ("getdevice", "cuda_forward_acoustic_3D", "cuda_Host_initialization", "cuda_Device_malloc",
                "cuda_Device_free", "getrik", "get_velQ"):
        assert ref in names
    assert "qvti_create" in names and "qvti_step" in names


def test_library_exports_every_declared_symbol(qvti):
    lib = ctypes.CDLL(qvti.LIB_PATH)
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts(qvti):
    # qvti_config is 12 4-byte fields
    assert ctypes.sizeof(qvti.Config) == 48


def test_getrik_matches_reference_formula(qvti):
    import numpy as np
    import qvti_cases as qc
    lib = ctypes.CDLL(qvti.LIB_PATH)
    nt = 300
    out = np.zeros(nt, np.float32)
    lib.getrik.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
    lib.getrik(nt, 1e-3, 25.0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert np.array_equal(out, qc.ricker(nt, 1e-3, 25.0))


def test_get_velq_pads_like_the_reference(qvti, tmp_path, monkeypatch):
    import numpy as np
    lib = ctypes.CDLL(qvti.LIB_PATH)
    pml, nx, ny, nz = 2, 3, 4, 5
    ntx, nty, ntz = nx + 2 * pml, ny + 2 * pml, nz + 2 * pml
    interior = np.arange(nx * ny * nz, dtype=np.float32).reshape(nx, ny, nz) + 1000
    f = tmp_path / "vp.bin"
    interior.tofile(f)
    monkeypatch.setenv("QVTI_VELP_FILE", str(f))
    arrs = [np.zeros((ntx, nty, ntz), np.float32) for _ in range(5)]
    P = ctypes.POINTER(ctypes.c_float)
    lib.get_velQ.argtypes = [ctypes.c_int] * 8 + [P] * 5
    lib.get_velQ(pml, ntx, nty, ntz, ntx * nty * ntz, nx, ny, nz, *[a.ctypes.data_as(P) for a in arrs])
    vp, qp, vs, qs, rho = arrs
    expect = np.pad(interior, pml, mode="edge")
    assert np.array_equal(vp, expect)
    assert np.allclose(vs, expect / np.float32(1.5)) and np.all(qp == 200) and np.all(qs == 150) and np.all(rho == 1800)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libqvti_ref.so")),
                    reason="reference build not present")
def test_reference_harness_exports():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libqvti_ref.so"))
    for n in ("qref_run", "cuda_forward_acoustic_3D", "cuda_Device_malloc", "cuda_Device_free",
              "cuda_Host_initialization", "getdevice"):
        assert hasattr(lib, n)


def test_host_driver_builds(qvti):
    """The C++ host driver with the reference's host surface compiles and
    links against the library (no GPU needed)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "q-vti_b200"), "driver"])
    assert os.access(os.path.join(ROOT, "q-vti_b200", "qvti_driver"), os.X_OK)


def test_per_device_once_logic(tmp_path):
    """Kernel attributes are per device: the once-per-device helper the
    engine and the allocation-free entry point use runs its set-up once for
    each device ordinal, retries after a failure and rejects ordinals out of
    range.  Plain C++, compiled and run here without a GPU."""
    import subprocess
    src = tmp_path / "t.cpp"
    src.write_text(r'''
#include <cstdio>
#include "per_device.h"
int main() {
    qvti::PerDeviceOnce<4> once;
    int calls[4] = {0, 0, 0, 0};
    int fail_next = 1;
    auto setup = [&](int d) { return [&, d] { ++calls[d]; if (d == 2 && fail_next) { fail_next = 0; return 7; } return 0; }; };
    int r0 = once.run(0, setup(0)), r0b = once.run(0, setup(0));
    int r1 = once.run(1, setup(1));
    int r2 = once.run(2, setup(2)), r2b = once.run(2, setup(2)), r2c = once.run(2, setup(2));
    int rbad = once.run(4, setup(0)), rneg = once.run(-1, setup(0));
    std::printf("%d %d %d %d %d %d %d %d | %d %d %d %d | %d %d %d\n", r0, r0b, r1, r2, r2b, r2c, rbad, rneg,
                calls[0], calls[1], calls[2], calls[3], (int)once.done(0), (int)once.done(2), (int)once.done(3));
    return 0;
}
''')
    exe = tmp_path / "t"
    subprocess.check_call(["g++", "-std=c++17", "-I", os.path.join(ROOT, "q-vti_b200", "csrc"), str(src), "-o", str(exe),
                           "-pthread"])
    out = subprocess.check_output([str(exe)], text=True).strip()
    # device 0 and 1 set up once; device 2 fails once, then succeeds once and is not run again
    assert out == "0 0 0 7 0 0 -1 -1 | 1 1 2 0 | 1 1 0", out
