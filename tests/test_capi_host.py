"""Host logic of the C ABI (no GPU): exported symbols, the mesh generator
against the reference's own meshes, the dual layout and the fix DOFs against
the oracle."""
import ast
import os
import re

import numpy as np
import pytest

import hfls_b200 as hb
from oracle.htfeti_oracle import HTFETI, Options, MeshArrays
from tests.golden_util import golden_paths, load, mesh_from_golden, options_from_args

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "htfeti.h")).read()
    declared = set(re.findall(r"\b(htf_[a-z_]+)\s*\(", hdr))
    assert len(declared) >= 15
    for name in sorted(declared):
        assert hasattr(hb.lib, name), name


def _spec_for_golden(args):
    g = {k: int(args.get(k, d)) for k, d in (("Nx", 2), ("Ny", 2), ("Nz", 2), ("nx", 5), ("ny", 5), ("nz", 5))}
    bc = hb.HTF_BC_CLAMP_X0 if args.get("clamp") == "true" else hb.HTF_BC_ROLLERS
    ratio = float(args.get("ratio_mat", "1"))
    return hb.mesh_spec(subs=(g["Nx"], g["Ny"], g["Nz"]), elems=(g["nx"], g["ny"], g["nz"]), bc=bc,
                        material=hb.HTF_MAT_CHECKER, E=float(args["young_modulus"]), E_hi=ratio,
                        body_force=(0, 0, 98.10 * 2.0))


@pytest.mark.parametrize("path", golden_paths(), ids=lambda p: os.path.basename(p)[:-4])
def test_generator_matches_reference_mesh(path):
    """Mesh::createMesh (Mesh.cpp:69-289): points bit-exact, connectivity,
    partition, materials, Dirichlet and corner DOFs identical."""
    g, args = load(path)
    m = hb.generate_mesh(_spec_for_golden(args))
    assert np.array_equal(m.coords, g["points"])
    assert np.array_equal(m.elems, g["elements"])
    assert np.array_equal(m.elem_sub, g["partition"])
    assert np.array_equal(m.dirichlet, g["dirichlet"])
    assert np.array_equal(m.corner, g["corner"])
    ref = mesh_from_golden(g, args)
    assert np.array_equal(m.sub_E, ref.sub_E)


def _oracle_mesh(m):
    return MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64),
                      m.sub_cluster.astype(np.int64), m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64),
                      m.corner.astype(np.int64), m.body_force)


CASES = [
    dict(clusters=(1, 1, 1), subs=(2, 2, 2), elems=(3, 3, 3), bc=hb.HTF_BC_ROLLERS, typeBc="ker"),
    dict(clusters=(2, 1, 1), subs=(2, 2, 1), elems=(2, 3, 2), bc=hb.HTF_BC_CLAMP_X0, typeBc="cor"),
    dict(clusters=(1, 2, 2), subs=(2, 1, 2), elems=(3, 2, 2), bc=hb.HTF_BC_CLAMP_X0, typeBc="ker", jitter=0.1),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['clusters']}x{c['subs']}x{c['elems']}-{c['typeBc']}")
def test_dual_layout_and_fix_dofs_match_oracle(case):
    case = dict(case)
    typeBc = case.pop("typeBc")
    spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, seed=3, **case)
    m = hb.generate_mesh(spec)
    s = hb.Solver({"typeBc": typeBc})
    s.set_mesh(m)
    rs, rd, sg, w = s.dual_layout()
    h = HTFETI(_oracle_mesh(m), Options(typeBc=typeBc, fix_rule="boundary", kerGc="analytic"))
    assert len(w) == h.n_lam
    assert np.array_equal(w, h.weight)
    for r, row in enumerate(h.bf_rows):
        for k, (d, gdof, sign) in enumerate(row):
            assert (rs[r, k], rd[r, k], sg[r, k]) == (d, gdof, sign)
        if len(row) == 1:
            assert rs[r, 1] == -1
    fix = s.fix_dofs()
    for d in range(m.n_sub):
        assert np.array_equal(fix[d], h.l2g[d][h.fix[d]])


def test_generator_jitter_is_interior_and_bounded():
    spec = hb.mesh_spec(subs=(2, 1, 1), elems=(4, 3, 3), jitter=0.1, seed=11)
    m = hb.generate_mesh(spec)
    m0 = hb.generate_mesh(hb.mesh_spec(subs=(2, 1, 1), elems=(4, 3, 3)))
    d = np.abs(m.coords - m0.coords)
    h = np.array([1 / 8, 1 / 3, 1 / 3])
    assert np.all(d <= 0.1 * h + 1e-15)
    on_boundary = np.any((m0.coords < 1e-12) | (m0.coords > 1 - 1e-12), axis=1)
    assert np.all(d[on_boundary] == 0)
    assert np.all(d[~on_boundary] > 0)
    m2 = hb.generate_mesh(spec)
    assert np.array_equal(m.coords, m2.coords)


def test_options_and_errors():
    with pytest.raises(hb.HTFError) as e:
        hb.Solver({"preconditioner": "bogus"})
    assert e.value.code == -1
    s = hb.Solver({"typeBc": "all", "eps_iter": "1e-8", "vtkWithinIter": "false"})
    with pytest.raises(hb.HTFError) as e:
        s.setup()
    assert e.value.code == -7


def _broken(mesh, **changes):
    a = dict(coords=mesh.coords, elems=mesh.elems, elem_sub=mesh.elem_sub, sub_cluster=mesh.sub_cluster,
             sub_E=mesh.sub_E, sub_nu=mesh.sub_nu, dirichlet=mesh.dirichlet, corner=mesh.corner,
             body_force=mesh.body_force)
    a.update(changes)
    return hb.Mesh(**a)


@pytest.mark.parametrize("what, change", [
    ("element node id out of range", lambda m: dict(elems=np.where(np.arange(m.elems.size).reshape(m.elems.shape) == 5,
                                                                   m.n_nodes, m.elems))),
    ("elem_sub out of range", lambda m: dict(elem_sub=np.where(np.arange(len(m.elem_sub)) == 0, m.n_sub,
                                                               m.elem_sub))),
    ("subdomain without elements", lambda m: dict(sub_cluster=np.append(m.sub_cluster, 0),
                                                  sub_E=np.append(m.sub_E, 1.0), sub_nu=np.append(m.sub_nu, 0.3))),
    ("negative cluster id", lambda m: dict(sub_cluster=np.where(np.arange(m.n_sub) == 1, -1, m.sub_cluster))),
    ("Dirichlet DOF out of range", lambda m: dict(dirichlet=np.append(m.dirichlet, 3 * m.n_nodes))),
    ("no dual rows", lambda m: dict(elem_sub=np.zeros_like(m.elem_sub), sub_cluster=m.sub_cluster[:1],
                                    sub_E=m.sub_E[:1], sub_nu=m.sub_nu[:1], dirichlet=m.dirichlet[:0],
                                    corner=m.corner[:0])),
])
def test_malformed_meshes_are_rejected_before_any_device_work(what, change):
    """The host problem build checks the mesh arrays and returns HTF_EINVAL
    with a message (the reference reads past its arrays or exits instead);
    it runs before any device call, so these need no GPU."""
    m = hb.generate_mesh(hb.mesh_spec(subs=(2, 2, 1), elems=(2, 2, 2)))
    s = hb.Solver({"typeBc": "cor"})
    s.set_mesh(_broken(m, **change(m)))
    with pytest.raises(hb.HTFError) as e:
        s.setup()
    assert e.value.code == -1 and what in str(e.value)


C_CALLER = r"""
#include <stdio.h>
#include <stdlib.h>
#include "htfeti.h"

int main(int argc, char **argv) {
    htf_mesh_spec s = {{1, 1, 1}, {2, 2, 2}, {2, 2, 2}, {NULL, NULL, NULL}, 0.0, 7u, HTF_BC_CLAMP_X0,
                       HTF_MAT_CONST, 2.1e5, 1.0, 0.3, {0.0, 0.0, -1.0}};
    int nn, ne, ns, nc, nd, ncr;
    if (htf_mesh_sizes(&s, &nn, &ne, &ns, &nc, &nd, &ncr) != HTF_OK) return 1;
    double *xyz = malloc(sizeof(double) * 3 * nn), *u = calloc(3 * nn, sizeof(double));
    int *el = malloc(sizeof(int) * 8 * ne), *part = malloc(sizeof(int) * ne);
    if (htf_mesh_fill(&s, xyz, el, part, NULL, NULL, NULL, NULL, NULL) != HTF_OK) return 2;
    if (htf_write_vtk(argv[1], nn, xyz, ne, el, part, NULL, u) != HTF_OK) return 3;
    htf_ctx *ctx = NULL;
    if (htf_create("typeBc=cor;preconditioner=bogus", &ctx) != HTF_EINVAL || ctx) return 4;
    if (htf_create("typeBc=cor;eps_iter=1e-8", &ctx) != HTF_OK) return 5;
    if (htf_setup(ctx) != HTF_ESTATE) return 6;
    printf("%d %d %d %s\n", nn, ne, ns, htf_last_error(ctx));
    htf_destroy(ctx);
    free(xyz); free(u); free(el); free(part);
    return 0;
}
"""


def test_header_and_library_from_plain_c(tmp_path):
    """The boundary as a C caller (cgo, JNI or any FFI) sees it: htfeti.h
    compiles as C99 and the library links and runs from C, with no C++ or
    torch types in the signatures (host entry points only: no GPU here)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    lib_dir = os.path.join(ROOT, "hfls_b200")
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L" + lib_dir, "-lhtfeti_b200", "-Wl,-rpath," + lib_dir], check=True, capture_output=True)
    out = subprocess.run([str(exe), str(tmp_path / "box.vtk")], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    nn, ne, ns, msg = out.stdout.split(" ", 3)
    assert (int(nn), int(ne), int(ns)) == (125, 64, 8)
    assert "before htf_set_mesh" in msg
    assert (tmp_path / "box.vtk").read_text().startswith("# vtk DataFile Version 3.0\n")


def test_factor_wave_option_is_checked():
    """factor_wave_gb (factor panels held a wave of subdomains at a time) is
    parsed at htf_create: a negative size is refused with HTF_EINVAL."""
    with pytest.raises(hb.HTFError) as e:
        hb.Solver({"factor_wave_gb": "-1"})
    assert e.value.code == hb.HTF_EINVAL
    hb.Solver({"factor_wave_gb": "2.5", "precision": "mixed"}).close()


def test_oversize_admission_option_is_checked():
    """admit_oversize (the server admits a request that does not fit its
    budget alone with factor waves) is 0 or 1; anything else is refused with
    HTF_EINVAL by the option parser, before the server touches a device."""
    for bad in ("2", "yes", ""):
        with pytest.raises(hb.HTFError) as e:
            hb.Server({"admit_oversize": bad})
        assert e.value.code == hb.HTF_EINVAL
        with pytest.raises(hb.HTFError) as e:
            hb.Solver({"admit_oversize": bad})
        assert e.value.code == hb.HTF_EINVAL
    hb.Solver({"admit_oversize": "1", "precision": "mixed"}).close()


def _random_case(seed):
    """A seeded small mesh: 1-2 clusters and 1-3 subdomains per axis, uneven
    slab widths of 1-3 elements, either boundary condition, either Bc type."""
    rng = np.random.default_rng(seed)
    clusters = tuple(int(x) for x in rng.integers(1, 3, size=3))
    subs = tuple(int(x) for x in rng.integers(1, 4, size=3))
    if np.prod(clusters) * np.prod(subs) < 2:
        subs = (2,) + subs[1:]
    widths = [rng.integers(1, 4, size=clusters[a] * subs[a]) for a in range(3)]
    bc = int(rng.integers(0, 2))
    typeBc = ("cor", "ker")[int(rng.integers(0, 2))]
    return dict(clusters=clusters, subs=subs, elems=(2, 2, 2), widths=widths, bc=bc,
                jitter=float(rng.choice([0.0, 0.1]))), typeBc


@pytest.mark.parametrize("seed", range(12))
def test_random_meshes_layout_and_fix_dofs_match_oracle(seed):
    """Bf rows, signs, weights and fix DOFs of the host front-end are the
    oracle's, entry for entry, on twelve seeded meshes of uneven slab widths
    (corner and kernel Bc, clamped face and rollers)."""
    case, typeBc = _random_case(seed)
    spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, seed=seed, **case)
    m = hb.generate_mesh(spec)
    s = hb.Solver({"typeBc": typeBc})
    s.set_mesh(m)
    rs, rd, sg, w = s.dual_layout()
    h = HTFETI(_oracle_mesh(m), Options(typeBc=typeBc, fix_rule="boundary", kerGc="analytic"))
    assert len(w) == h.n_lam
    assert np.array_equal(w, h.weight)
    want = np.full((h.n_lam, 2), -1)
    for r, row in enumerate(h.bf_rows):
        for k, (d, gdof, sign) in enumerate(row):
            assert (rd[r, k], sg[r, k]) == (gdof, sign)
            want[r, k] = d
    assert np.array_equal(rs, want)
    fix = s.fix_dofs()
    for d in range(m.n_sub):
        assert np.array_equal(fix[d], h.l2g[d][h.fix[d]])
