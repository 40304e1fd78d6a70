"""Makes tests/golden/reference_meshes.npz from the meshes HenrikSchumacher/Repulsor ships
(its Meshes/ directory): the inputs of the reference's own example programs, used by the
parity tests as reference-held inputs (the reference ships no expected outputs).

  twospheres_*           Meshes/TwoSpheres.hpp, the arrays of Example/main.cpp: two unit
                         spheres (162 vertices, 320 triangles each) 0.0078 apart, one the
                         mesh, the other the obstacle (vertex_coordinates / simplices and
                         obstacle_vertex_coordinates / obstacle_simplices, parsed as data)
  torus2400_*            Meshes/TorusMesh_00002400T.txt  (1,200 vertices, 2,400 triangles)
  torus38400_*           Meshes/TorusMesh_00038400T.txt  (19,200 vertices, 38,400 triangles)
  sphere40560_*          Meshes/Sphere_00040560T.txt     (20,282 vertices, 40,560 triangles)

The .txt meshes are read with repulsor_b200.read_mesh_file, the reader of the reference's
format that SimplicialMesh_Factory.Make_FromFile uses. Run from the repository root:
    python tests/golden/make_reference_meshes.py /path/to/Repulsor
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from repulsor_b200.meshio import read_mesh_file  # noqa: E402

TXT = {"torus2400": "TorusMesh_00002400T.txt", "torus38400": "TorusMesh_00038400T.txt",
       "sphere40560": "Sphere_00040560T.txt"}


def parse_cpp_array(src, name, cols, dtype):
    """The initializer list of `<type> name [..][..] = { {..}, ... };` as an array."""
    m = re.search(r"\b" + re.escape(name) + r"\s*\[[^\]]*\]\s*\[[^\]]*\]\s*=\s*\{(.*?)\};", src, re.S)
    if not m:
        raise ValueError(f"array {name} not found")
    nums = re.findall(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?", m.group(1))
    return np.array(nums, dtype=dtype).reshape(-1, cols)


def two_spheres(meshes_dir):
    src = open(os.path.join(meshes_dir, "TwoSpheres.hpp")).read()
    out = {
        "twospheres_V": parse_cpp_array(src, "vertex_coordinates", 3, np.float64),
        "twospheres_S": parse_cpp_array(src, "simplices", 3, np.int64).astype(np.int32),
        "twospheres_obstacle_V": parse_cpp_array(src, "obstacle_vertex_coordinates", 3, np.float64),
        "twospheres_obstacle_S": parse_cpp_array(src, "obstacle_simplices", 3, np.int64).astype(np.int32),
    }
    counts = {k: int(v) for k, v in re.findall(r"constexpr Int (\w+_count)\s*=\s*(\d+);", src)}
    assert out["twospheres_V"].shape == (counts["vertex_count"], 3)
    assert out["twospheres_S"].shape == (counts["simplex_count"], 3)
    assert out["twospheres_obstacle_V"].shape == (counts["obstacle_vertex_count"], 3)
    assert out["twospheres_obstacle_S"].shape == (counts["obstacle_simplex_count"], 3)
    return out


def load_all(reference_root):
    meshes_dir = os.path.join(reference_root, "Meshes")
    out = two_spheres(meshes_dir)
    for key, name in TXT.items():
        dom, amb, V, S = read_mesh_file(os.path.join(meshes_dir, name))
        assert dom == 2 and amb == 3
        out[f"{key}_V"], out[f"{key}_S"] = V, S
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    np.savez_compressed(os.path.join(HERE, "reference_meshes.npz"), **load_all(root))


if __name__ == "__main__":
    main()
