"""htf_dump: the set-up problem's matrices as the reference's MatrixMarket
dump files (Matrix::printToFile, Matrix.cpp:556-632), read back with
scipy.io.mmread and compared with the oracle's: K_i, rhs_i, Bf_i, R_i, S_i
(explicit Dirichlet) and GfTGf, for every subdomain."""
import os

import numpy as np
import pytest
import scipy.io

import hfls_b200 as hb
from oracle.htfeti_oracle import HTFETI, MeshArrays, Options

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_dump_matches_oracle_matrices(tmp_path):
    spec = hb.mesh_spec(clusters=(2, 1, 1), subs=(2, 1, 2), elems=(3, 2, 3), jitter=0.1, seed=4,
                        material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e2)
    m = hb.generate_mesh(spec)
    s = hb.Solver({"typeBc": "cor", "preconditioner": "Dirichlet_explicit", "print_matrices": "4"})
    s.set_mesh(m)
    s.setup()
    s.dump(str(tmp_path), 4)
    o = HTFETI(MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64),
                          m.sub_cluster.astype(np.int64), m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64),
                          m.corner.astype(np.int64), m.body_force),
               Options(typeBc="cor", fix_rule="boundary", kerGc="analytic"))
    read = lambda name, d: scipy.io.mmread(os.path.join(tmp_path, f"dump_{name}_{d}.txt"))
    with open(os.path.join(tmp_path, "dump_K_0.txt")) as f:
        assert f.readline().startswith("%%MatrixMarket matrix coordinate real symmetric")
    for d in range(m.n_sub):
        assert rel(read("K", d).toarray(), o.K[d]) < 1e-13
        assert rel(read("rhs", d).toarray()[:, 0], o.f[d][:, 0]) < 1e-13
        Bf = read("Bf", d).toarray()
        ref = np.zeros_like(Bf)
        ref[o.bf_l2g[d][o.bf_rowloc[d]], o.bf_col[d]] = o.bf_val[d]
        assert np.array_equal(Bf, ref)
        assert rel(read("R", d).toarray(), o.R[d]) < 1e-13
        assert rel(read("S", d).toarray(), o.S[d]) < 1e-11
    assert rel(scipy.io.mmread(os.path.join(tmp_path, "dump_GfTGf_0.txt")).toarray(), o.GfTGf) < 1e-12


def test_dump_needs_the_option_at_setup(tmp_path):
    s = hb.Solver({"typeBc": "cor"})
    s.set_mesh(hb.generate_mesh(hb.mesh_spec(subs=(2, 1, 1), elems=(2, 2, 2))))
    s.setup()
    with pytest.raises(hb.HTFError) as e:
        s.dump(str(tmp_path), 2)
    assert e.value.code == hb.HTF_ESTATE


@pytest.mark.parametrize("typeBc", ["cor", "ker"])
def test_kernel_and_fix_dofs_on_device_are_the_host_ones(tmp_path, typeBc):
    """A set-up computes the kernel bases R_i and the fix DOFs on the GPU
    (kernel_fix.cu); the layout inspection without a set-up computes them on
    the host.  Both are bit-identical, and R_i equals the oracle's
    (Data.cpp:61-109 + Matrix.cpp:2450-2472) bit for bit."""
    w = [np.array(v, np.int32) for v in ([3, 5, 2, 4], [4, 2, 3, 5], [2, 4, 5, 3])]
    spec = hb.mesh_spec(clusters=(2, 2, 1), subs=(2, 2, 4), widths=w, jitter=0.1, seed=6,
                        material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3)
    m = hb.generate_mesh(spec)
    host = hb.Solver({"typeBc": typeBc})
    host.set_mesh(m)
    fix_host = host.fix_dofs()
    host.close()
    dev = hb.Solver({"typeBc": typeBc, "print_matrices": "3"})
    dev.set_mesh(m)
    dev.setup()
    assert np.array_equal(dev.fix_dofs(), fix_host)
    dev.dump(str(tmp_path), 3)
    dev.close()
    o = HTFETI(MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64),
                          m.sub_cluster.astype(np.int64), m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64),
                          m.corner.astype(np.int64), m.body_force),
               Options(typeBc=typeBc, fix_rule="boundary", kerGc="analytic"))
    for d in range(m.n_sub):
        R = scipy.io.mmread(os.path.join(tmp_path, f"dump_R_{d}.txt")).toarray()
        assert np.array_equal(R, o.R[d])
        assert np.array_equal(np.sort(fix_host[d] if fix_host.ndim == 2 else fix_host[6 * d:6 * d + 6]),
                              np.sort(o.l2g[d][o.fix[d]]))


@pytest.mark.parametrize("case", ["cor-uneven", "ker-clamp", "cor-cube"])
def test_front_end_on_device_is_the_host_one(tmp_path, case):
    """A set-up builds l2g, the Bf rows and weights and the b sets on the GPU
    (frontend.cu); the layout inspection without a set-up builds them on the
    host (problem.cpp).  Rows, signs, weights, fix DOFs and the Bf / Bc / K_i
    dumps (l2g, b sets and permutations) are identical, bit for bit."""
    if case == "cor-uneven":
        w = [np.array(v, np.int32) for v in ([3, 5, 2, 4], [4, 2, 3, 5], [2, 4, 5, 3])]
        spec = hb.mesh_spec(clusters=(2, 2, 1), subs=(2, 2, 4), widths=w, jitter=0.1, seed=6,
                            material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3)
        typeBc = "cor"
    elif case == "ker-clamp":
        spec = hb.mesh_spec(clusters=(1, 2, 1), subs=(3, 2, 2), elems=(3, 3, 3), jitter=0.1, seed=2,
                            bc=hb.HTF_BC_CLAMP_X0)
        typeBc = "ker"
    else:
        spec = hb.mesh_spec(clusters=(2, 2, 2), subs=(2, 2, 2), elems=(4, 4, 4), jitter=0.1, seed=1)
        typeBc = "cor"
    m = hb.generate_mesh(spec)
    out = {}
    for where in ("host", "device"):
        s = hb.Solver({"typeBc": typeBc, "print_matrices": "2"})
        s.set_mesh(m)
        if where == "device":
            s.setup()
        out[where] = s.dual_layout() + (s.fix_dofs(),)
        if where == "device":
            s.dump(str(tmp_path), 2)
        s.close()
    for a, b in zip(out["host"], out["device"]):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    # the dumps of the device-built problem against the host layout: Bf_i rows / local columns
    rs, rd, sg, wt, _ = out["host"]
    for d in range(m.n_sub):
        Bf = scipy.io.mmread(os.path.join(tmp_path, f"dump_Bf_{d}.txt")).tocoo()
        rows = np.where(rs == d)
        assert Bf.nnz == len(rows[0])
        assert np.array_equal(np.sort(Bf.row), np.sort(rows[0]))
