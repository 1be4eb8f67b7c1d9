"""The C-ABI library: it builds, loads without a GPU, exports every symbol the headers declare,
and its struct layouts match the ctypes mirrors.  No compute calls (no GPU here)."""
import ctypes
import glob
import os
import re
import shutil
import subprocess

import pytest

from vlasov1d2v_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vl_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        if shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
            pytest.skip("library not built and nvcc unavailable")
        from vlasov1d2v_b200 import build

        build.build()
    return _lib.load()


def test_headers_exist():
    assert HEADERS, "include/*.h missing"


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"symbols declared but not exported: {missing}"


def test_binding_table_matches_header():
    assert set(_lib.EXPORTED) == set(declared_functions())


def test_abi_version(lib):
    assert lib.vl_abi_version() == _lib.ABI_VERSION


def test_null_arguments_are_rejected_without_a_gpu(lib):
    # argument validation happens before any CUDA call
    assert lib.vl_rhs(None, None, None, None, 0, None) == -1
    assert lib.vl_ctx_create(None, None) == -1
    assert b"null" in lib.vl_last_error()
    assert lib.vl_ctx_destroy(None) == 0
    assert lib.vl_state_elems(None) == 0


def test_config_validation_without_a_gpu(lib):
    cfg = _lib.VlConfig()
    cfg.abi_version = _lib.ABI_VERSION
    cfg.precision = 7
    h = ctypes.c_void_p()
    assert lib.vl_ctx_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    cfg.precision = 0
    cfg.n = 11
    assert lib.vl_ctx_create(ctypes.byref(cfg), ctypes.byref(h)) == -4
    cfg.n = 8
    cfg.nx, cfg.nu, cfg.nv = 100, 4, 4
    cfg.n_modes = 10
    assert lib.vl_ctx_create(ctypes.byref(cfg), ctypes.byref(h)) == -5
    assert not h.value


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc unavailable")
def test_struct_layout_matches_ctypes(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "vlasov1d2v.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(vl_config),"
        " offsetof(vl_config, courant), offsetof(vl_config, dft_qnode), sizeof(vl_run_state),"
        " offsetof(vl_run_state, hist_capacity), offsetof(vl_run_state, dt_hist));return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    C, R = _lib.VlConfig, _lib.VlRunState
    want = [ctypes.sizeof(C), C.courant.offset, C.dft_qnode.offset, ctypes.sizeof(R),
            R.hist_capacity.offset, R.dt_hist.offset]
    assert got == want


def test_gpu_entry_points_fail_loudly_without_cuda():
    import torch

    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    from vlasov1d2v_b200 import _device

    with pytest.raises(RuntimeError):
        _device.device()
