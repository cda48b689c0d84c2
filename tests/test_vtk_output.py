"""htf_write_vtk against the reference's own box.vtk (Mesh::SaveVTK,
Mesh.cpp:292-351): the same mesh and displacements give the same bytes, so
post-processing written for the reference's output reads this library's."""
import os

import numpy as np
import pytest

import hfls_b200 as hb

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASE = "ref_ker_dirichlet_3"


def _mesh(points, elements, partition):
    ns = int(partition.max()) + 1
    return hb.Mesh(points, elements, partition, np.zeros(ns), np.ones(ns), np.full(ns, 0.3),
                   np.zeros(0), np.zeros(0), np.zeros(3))


def _displacements(text, n):
    lines = text.split("\n")
    k = lines.index("LOOKUP_TABLE my_table")
    return np.array([[float(v) for v in l.split()] for l in lines[k + 1:k + 1 + n]]).ravel()


def test_bytes_match_the_reference_box_vtk(tmp_path):
    g = np.load(os.path.join(GOLDEN, CASE + ".npz"))
    ref = open(os.path.join(GOLDEN, CASE + "_box.vtk"), "rb").read()
    pts = g["points"]
    u = _displacements(ref.decode(), len(pts))
    # the fixture's field is the golden solution printed with "%f"
    assert np.abs(u - g["u"]).max() <= 5e-7
    m = _mesh(pts, g["elements"], g["partition"])
    out = tmp_path / "box.vtk"
    hb.write_vtk(str(out), m, u)                          # material ids by the reference's rule
    assert out.read_bytes() == ref
    hb.write_vtk(str(out), m, u, material=g["material"])  # the reference's own ids, same file
    assert out.read_bytes() == ref


def test_reference_material_rule():
    # remainder(p, 2) with the quotient rounded to nearest even (Mesh.cpp:280-281)
    g = np.load(os.path.join(GOLDEN, "ref_ker_implicit_3x2x1_4.npz"))
    p = g["partition"]
    # even p -> 0; odd p -> +1 when p // 2 is even, -1 when it is odd (p = 3 here)
    assert np.array_equal(g["material"], (p % 2) * np.where((p // 2) % 2 == 0, 1, -1))
    assert -1 in g["material"]


def test_generated_mesh_round_trip(tmp_path):
    spec = hb.mesh_spec(clusters=(2, 1, 1), subs=(2, 2, 1), elems=(3, 2, 2), jitter=0.1, seed=4)
    m = hb.generate_mesh(spec)
    u = np.random.default_rng(0).normal(size=3 * m.n_nodes) * 1e-2
    out = tmp_path / "u.vtk"
    hb.write_vtk(str(out), m, u)
    lines = out.read_text().split("\n")
    assert lines[5] == f"POINTS {m.n_nodes} float"
    xyz = np.array([[float(v) for v in l.split()] for l in lines[6:6 + m.n_nodes]])
    assert np.abs(xyz - m.coords).max() <= 5e-7
    k = lines.index(f"CELLS {len(m.elem_sub)} {9 * len(m.elem_sub)}")
    cells = np.array([[int(v) for v in l.split()] for l in lines[k + 1:k + 1 + len(m.elem_sub)]])
    assert np.all(cells[:, 0] == 8) and np.array_equal(cells[:, 1:], m.elems)
    assert np.abs(_displacements(out.read_text(), m.n_nodes) - u).max() <= 5e-7
    k = lines.index("LOOKUP_TABLE decomposition")
    assert np.array_equal(np.array(lines[k + 1:k + 1 + len(m.elem_sub)], dtype=int), m.elem_sub)


def test_errors(tmp_path):
    spec = hb.mesh_spec(subs=(1, 1, 1), elems=(1, 1, 1))
    m = hb.generate_mesh(spec)
    with pytest.raises(hb.HTFError) as e:
        hb.write_vtk(str(tmp_path / "no_such_dir" / "box.vtk"), m, np.zeros(3 * m.n_nodes))
    assert e.value.code == -10
    bad = hb.Mesh(m.coords, m.elems + m.n_nodes, m.elem_sub, m.sub_cluster, m.sub_E, m.sub_nu, m.dirichlet,
                  m.corner, m.body_force)
    with pytest.raises(hb.HTFError) as e:
        hb.write_vtk(str(tmp_path / "box.vtk"), bad, np.zeros(3 * m.n_nodes))
    assert e.value.code == -1
    with pytest.raises(hb.HTFError):
        hb.write_vtk(str(tmp_path / "box.vtk"), m, np.zeros(5))
