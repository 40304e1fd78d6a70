"""Repulsor's mesh text format (SimplicialMesh_Factory::Make_FromFile and
SimplicialMesh::WriteToFile, src/SimplicialMesh/SimplicialMesh_Factory.hpp:160-246 and
src/SimplicialMesh.hpp:780-818).

A file holds four "name value" lines -- domain dimension, ambient dimension, vertex
count, simplex count (the reader skips the names, so "dom_dim" and "domain_dimension"
both work) -- then the vertex coordinates row by row and the simplices row by row, all
separated by white space. The writer prints the coordinates in scientific notation with
digits10 + 1 = 16 digits after the point (17 significant digits, enough to read every
double back exactly), upper case, tab-separated, as the reference does.
"""
from __future__ import annotations

import numpy as np


def read_mesh_file(path):
    """(dom_dim, amb_dim, V, S): V (vertex_count, amb_dim) float64, S (simplex_count,
    dom_dim + 1) int32. Raises ValueError when the file is truncated or malformed."""
    with open(path) as f:
        tok = f.read().split()
    if len(tok) < 8:
        raise ValueError(f"{path}: header of four 'name value' lines expected")
    try:
        dom, amb, nv, ns = (int(tok[1]), int(tok[3]), int(tok[5]), int(tok[7]))
    except ValueError as e:
        raise ValueError(f"{path}: malformed header") from e
    if dom < 0 or amb < 1 or nv < 0 or ns < 0:
        raise ValueError(f"{path}: invalid dimensions or counts")
    nvals, nidx = nv * amb, ns * (dom + 1)
    body = tok[8:]
    if len(body) < nvals + nidx:
        raise ValueError(f"{path}: {len(body)} values, {nvals + nidx} expected")
    V = np.array(body[:nvals], dtype=np.float64).reshape(nv, amb)
    S = np.array(body[nvals:nvals + nidx], dtype=np.int64).reshape(ns, dom + 1)
    if ns and (S.min() < 0 or S.max() >= nv):
        raise ValueError(f"{path}: simplex vertex index out of range")
    return dom, amb, V, S.astype(np.int32)


def write_mesh_file(path, V, S):
    """Writes V (n_v, amb) and S (n_s, dom + 1) in the reference's text format."""
    V = np.asarray(V, dtype=np.float64)
    S = np.asarray(S)
    with open(path, "w") as f:
        f.write(f"domain_dimension\t{S.shape[1] - 1}\n")
        f.write(f"ambient_dimension\t{V.shape[1]}\n")
        f.write(f"vertex_count\t{V.shape[0]}\n")
        f.write(f"simplex_count\t{S.shape[0]}\n")
        for row in V:
            f.write("".join(f"{x:.16E}\t" for x in row) + "\n")
        for row in S:
            f.write("".join(f"{int(i)}\t" for i in row) + "\n")
