"""The C++ facade (include/otmap_b200.hpp) compiles with and without Eigen, and its
host-side mesh calls (grid mesh, OFF write/read, prune_empty_faces) give what the
reference's Surface_mesh code gives. No GPU needed."""

import os
import subprocess

import numpy as np
import pytest

import facade_build


def test_facade_builds_without_eigen_and_runs_host_calls(tmp_path):
    exe = facade_build.build(str(tmp_path))
    r = subprocess.run([exe, "mesh", str(tmp_path)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    res = facade_build.results(str(tmp_path))
    from otmap_b200 import otmap as ot

    g = ot.Mesh.grid(8)
    g.xy[10] = (0.3, 0.2)
    g.write(str(tmp_path / "py.off"))
    assert (tmp_path / "py.off").read_bytes() == (tmp_path / "grid8.off").read_bytes()
    d = np.ones(64)
    d[::3] = 0
    p = ot.prune_empty_faces(g, d)
    p.write(str(tmp_path / "py_pruned.off"))
    assert (tmp_path / "py_pruned.off").read_bytes() == (tmp_path / "grid8_pruned.off").read_bytes()
    assert res["pruned_vertices"] == p.n_vertices and res["pruned_faces"] == p.n_faces

    from oracle import ref

    if ref.available():
        st, ix = g.face_start, g.face_vertices
        xy, s2, i2 = ref.prune_empty_faces(g.xy, st, ix, d)
        ref.write_off(tmp_path / "ref_pruned.off", xy, s2, i2)
        assert (tmp_path / "ref_pruned.off").read_bytes() == (tmp_path / "grid8_pruned.off").read_bytes()


def test_facade_builds_with_eigen(tmp_path):
    from oracle.build import reference_root

    root = reference_root()
    eigen = os.path.join(root, "extern") if root else ""
    if not root or not os.path.exists(os.path.join(eigen, "Eigen", "Core")):
        pytest.skip("no Eigen headers here")
    exe = facade_build.build(str(tmp_path), eigen_include=eigen)
    r = subprocess.run([exe, "mesh", str(tmp_path)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
