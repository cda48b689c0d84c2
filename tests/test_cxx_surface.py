"""The reference's C++ class surface (Driver, Cluster, Solver, Mesh, Vector)
over the C ABI: a main in the shape of the reference's htfeti.cpp
(tests/cxx/htfeti_main.cpp) compiles against include/hfls/ and links
libhtfeti_b200.so; on the GPU it solves the reference's own mesh and writes
the reference's box.vtk, whose displacements match the reference's run of
the same case (golden ref_ker_dirichlet_3, eps 1e-10) within 1e-8 and whose
other sections are byte-identical to the reference's file."""
import os
import subprocess

import numpy as np
import pytest

from tests.golden_util import GOLDEN_DIR, load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "hfls_b200")


def build_main(tmp_path):
    exe = str(tmp_path / "htfeti_main")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include", "hfls"), "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cxx", "htfeti_main.cpp"), "-o", exe, "-L" + LIBDIR, "-lhtfeti_b200",
           "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_reference_shaped_main_compiles_and_links(tmp_path):
    exe = build_main(tmp_path)
    assert os.path.exists(exe)


def vtk_sections(path):
    with open(path) as f:
        lines = f.read().split("\n")
    k = next(i for i, l in enumerate(lines) if l.startswith("LOOKUP_TABLE my_table"))
    n = int(next(l for l in lines if l.startswith("POINTS")).split()[1])
    u = np.array([list(map(float, l.split())) for l in lines[k + 1:k + 1 + n]]).ravel()
    return lines[:k + 1], u, lines[k + 1 + n:]


@pytest.mark.gpu
def test_reference_shaped_main_solves_the_reference_case(tmp_path):
    exe = build_main(tmp_path)
    g, args = load(os.path.join(GOLDEN_DIR, "ref_ker_dirichlet_3.npz"))
    out = tmp_path / "data"
    out.mkdir()
    argv = [exe, f"path2data={out}", "eps_iter=1e-10", "max_iter=1000"] + [f"{k}={v}" for k, v in args.items()]
    r = subprocess.run(argv, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "----------------- done" in r.stdout
    head, u, tail = vtk_sections(out / "box.vtk")
    assert np.linalg.norm(u - g["u_tight"]) / np.linalg.norm(g["u_tight"]) < 1e-8
    rhead, _, rtail = vtk_sections(os.path.join(GOLDEN_DIR, "ref_ker_dirichlet_3_box.vtk"))
    assert head == rhead and tail == rtail
