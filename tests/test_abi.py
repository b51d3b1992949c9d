"""CPU checks of the drop-in boundary: the CUDA library loads, exports every
entry point declared in include/uaamg.h, and its host-side argument checks
answer without a GPU (no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(uaamg_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def cuda_lib():
    from uaamg_b200 import build
    build.build()
    from uaamg_b200 import _lib
    return _lib.lib()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "uaamg_poisson_create" in names and "uaamg_poisson_solve_pcg" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(cuda_lib):
    from uaamg_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT\s+(uaamg_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(cuda_lib, n)


def test_python_binding_covers_header():
    from uaamg_b200 import _lib
    bound = {name for name, _, _ in _lib.EXPORTS}
    assert set(declared_functions()) <= bound


def test_create_without_device_reports_error(cuda_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from uaamg_b200 import _lib
    g = _lib.LeafGridC()
    h = C.c_void_p()
    rc = cuda_lib.uaamg_poisson_create(C.byref(g), C.byref(g), 1.0, 0.1, C.byref(h))
    assert rc == -5  # UAAMG_ERR_NO_DEVICE
    assert b"device" in cuda_lib.uaamg_last_error()
    assert cuda_lib.uaamg_device_count() == 0


def test_null_arguments_are_rejected(cuda_lib):
    assert cuda_lib.uaamg_poisson_create(None, None, 1.0, 0.1, None) == -1
    assert cuda_lib.uaamg_poisson_set_smoother(None, 0) == -1
    assert cuda_lib.uaamg_poisson_destroy(None) == 0


def test_cpp_facade_compiles():
    """The header-only C++ facade (reference class names over the C ABI)."""
    src = os.path.join(ROOT, "include", "uaamg_simd.hpp")
    if not os.path.exists(src):
        pytest.skip("no C++ facade")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-x", "c++", "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_facade_links_and_checks_arguments(cuda_lib, tmp_path):
    """A C++ call site built against the facade links with the library and
    gets the library's argument errors as status codes (never exceptions: the
    program is built with -fno-exceptions); calls with nothing to do return
    without touching a device."""
    from uaamg_b200 import _lib
    prog = tmp_path / "facade.cpp"
    prog.write_text(r'''
#include "uaamg_simd.hpp"
#include <cstdio>
using namespace simd_uaamg_b200;
int main() {
    std::vector<int32_t> org = {0, 0, 0, 8, 0, 0};
    std::vector<float> vals(2 * 512, 0.f);
    std::vector<uint64_t> masks(2 * 8, 0);
    int ok = extrapolate_channel(3, org, vals, masks, {}, {});             // no voxel to fill
    int errors = 0;
    int rc = extrapolate_channel(3, org, vals, masks, {0, 0}, std::vector<uint64_t>(16, 1));  // a leaf listed twice
    errors += (rc == UAAMG_ERR_INVALID_ARGUMENT && lastError().find("twice") != std::string::npos);
    std::vector<int32_t> bad = {0, 0, 0, 4, 0, 0};
    rc = extrapolate_channel(3, bad, vals, masks, {1}, std::vector<uint64_t>(8, 1));
    errors += (rc == UAAMG_ERR_INVALID_ARGUMENT);
    LeafGrid solid;
    solid.background[0] = 1.f;
    int st = 1;
    std::vector<float> w = calculate_face_weights(solid, {}, {}, &st);  // empty topology
    LeafGrid liquid;
    std::vector<float> im = immerse_liquid_phi_values(solid, liquid, 0.1f);  // no liquid leaves
    LeafGrid phi;  // components 1, but the face weights need 3: a factory error, an empty pointer
    int cst = 0;
    LaplacianWithLevel::Ptr lap = LaplacianWithLevel::createPressurePoissonLaplacian(phi, phi, 1.f, 0.1f, &cst);
    errors += (!lap && cst < 0);
    PoissonSolver solver(lap);
    std::vector<float> p, b;
    errors += (solver.solveMultigridPCG(p, b) == UAAMG_ERR_INVALID_ARGUMENT);
    std::printf("%d %d %d %zu %zu\n", ok, errors, st, w.size(), im.size());
    return errors == 4 ? 0 : 1;
}
''')
    exe = tmp_path / "facade"
    libdir = os.path.dirname(_lib.LIB_PATH)
    r = subprocess.run(["g++", "-std=c++17", "-fno-exceptions", "-I", os.path.join(ROOT, "include"), str(prog),
                        "-o", str(exe), _lib.LIB_PATH, f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split() == ["0", "4", "0", "0", "0"]


def test_torch_ordering_detects_cuda_arguments():
    """The Python classes order a call with torch's stream when an argument is
    a CUDA tensor, a LeafGrid holding one, or a list of either; host data is
    not ordered (no torch calls)."""
    import torch
    from uaamg_b200 import _lib
    from uaamg_b200.grids import LeafGrid

    class FakeCuda:  # stands in for a CUDA tensor on a machine without a GPU
        is_cuda = True

    g = LeafGrid(origins=np.zeros((1, 3), np.int32), values=np.zeros((1, 512), np.float32), background=0.0)
    assert not _lib.is_cuda(g, np.zeros(3), torch.zeros(3), [torch.zeros(2)], None)
    assert _lib.is_cuda(FakeCuda())
    assert _lib.is_cuda([torch.zeros(1), FakeCuda()])
    g.values = FakeCuda()
    assert _lib.is_cuda(None, g)
    # nothing to order: the context manager neither loads torch.cuda state nor the library
    with _lib.torch_ordered("poisson", None, np.zeros(3), torch.zeros(3)):
        pass
    _lib.torch_inputs_ready(None, np.zeros(3), torch.zeros(3))
