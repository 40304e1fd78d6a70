"""Supernodal Cholesky of the H1 preconditioner (repulsor_b200/csrc/host/supernodal_chol.hpp):
tests/cpp/supernodal_check.cpp runs the symbolic analysis, the per-supernode numeric code
(the arithmetic the GPU factorization performs, here on host threads) and the conversion to
the row and column forms on seeded random sparse positive definite matrices with random
orderings and supernode width caps 1, 2, 3, 8 and 256, and checks L L^T = P A P^T to 1e-12
relative and the layout of both forms (CPU only)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_supernodal_factor_reproduces_the_matrix(tmp_path):
    exe = str(tmp_path / "supernodal_check")
    host = os.path.join(ROOT, "repulsor_b200", "csrc", "host")
    srcs = [os.path.join(ROOT, "tests", "cpp", "supernodal_check.cpp")] + [
        os.path.join(host, f) for f in ("supernodal_chol.cpp", "sparse_cholesky.cpp", "tree_builder.cpp")]
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "repulsor_b200", "csrc")] + srcs + ["-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
