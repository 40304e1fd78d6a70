"""Host-side row tiles of the shared-memory pair kernels (build_row_tiles in
repulsor_b200/csrc/host/tree_builder.cpp): tests/cpp/row_tiles_check.cpp checks coverage,
union caps, slots and row order on seeded random patterns (CPU only)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_row_tiles_invariants(tmp_path):
    exe = str(tmp_path / "row_tiles_check")
    src = os.path.join(ROOT, "tests", "cpp", "row_tiles_check.cpp")
    lib = os.path.join(ROOT, "repulsor_b200", "csrc", "host", "tree_builder.cpp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "repulsor_b200", "csrc"), src, lib, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
