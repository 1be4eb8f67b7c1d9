"""Geometry of the fragment kernel and of the generic stage kernel's TMA form,
checked on the host (no GPU):
tensor-copy box widths and alignments, 128-byte staging offsets and shared-memory fit for every
compiled order and both precisions (tests/geometry/stage_geometry_check.cu, built with nvcc)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_generic_stage_geometry(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path / "stage_geometry_check"
    cmd = [nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "vlasov1d2v_b200", "csrc"),
           "-o", str(exe), os.path.join(HERE, "geometry", "stage_geometry_check.cu")]
    subprocess.run(cmd, check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and "ALL OK" in out.stdout, out.stdout


def test_field_prefetch_geometry(tmp_path):
    """The cluster field solve's table prefetch: copied and read entries inside their shared-memory
    regions and the global tables, region sizes against the launch's dynamic shared memory, for
    every order, element count and rank (tests/geometry/field_prefetch_check.cu)."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path / "field_prefetch_check"
    cmd = [nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "vlasov1d2v_b200", "csrc"),
           "-o", str(exe), os.path.join(HERE, "geometry", "field_prefetch_check.cu")]
    subprocess.run(cmd, check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and "ALL OK" in out.stdout, out.stdout
