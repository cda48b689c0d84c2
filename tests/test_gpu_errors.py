"""Failure paths of the C ABI, made from the inputs alone (nothing here can
fault or hang a GPU): every failure returns its negative code instead of
exiting the process as the reference does (Matrix.cpp:1174-1178,
1279-1283), and the same process then solves the next problem.

  * a subdomain with a negative Young's modulus makes its regularised K_i
    indefinite: htf_setup returns HTF_ENOTSPD and htf_status_sub names it;
  * max_iter below the iterations a solve needs: HTF_ENOCONV (plain FP64
    and batched mixed-precision forms);
  * a mesh with no Dirichlet DOFs leaves the whole body floating, so
    Gf^T Gf (Cluster.cpp:1227-1273) is singular: HTF_ENOTSPD from the outer
    coarse problem."""
import numpy as np
import pytest

import hfls_b200 as hb
from oracle.htfeti_oracle import HTFETI, MeshArrays, Options

pytestmark = pytest.mark.gpu

SPEC = dict(clusters=(2, 1, 1), subs=(2, 2, 2), elems=(3, 3, 3), jitter=0.1, seed=5,
            material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3)
OPTS = {"typeBc": "cor", "preconditioner": "Dirichlet_explicit", "device": "0"}


def solve_next_problem():
    """The process still solves a good problem, against the oracle."""
    m = hb.generate_mesh(hb.mesh_spec(**SPEC))
    s = hb.Solver(dict(OPTS, eps_iter="1e-10", max_iter="2000"))
    s.set_mesh(m)
    s.setup()
    u, st = s.pcpg()
    s.close()
    o = HTFETI(MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64),
                          m.sub_cluster.astype(np.int64), m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64),
                          m.corner.astype(np.int64), m.body_force),
               Options(typeBc="cor", fix_rule="boundary", kerGc="analytic"))
    ref = o.pcpg(eps_iter=1e-10, max_iter=2000)
    assert np.linalg.norm(u[0] - ref["u"]) / np.linalg.norm(ref["u"]) < 1e-8


@pytest.mark.parametrize("bad", [0, 5, 13])
def test_negative_modulus_gives_enotspd_with_the_subdomain(bad):
    m = hb.generate_mesh(hb.mesh_spec(**SPEC))
    m.sub_E[bad] = -m.sub_E[bad]
    s = hb.Solver(OPTS)
    s.set_mesh(m)
    with pytest.raises(hb.HTFError) as e:
        s.setup()
    assert e.value.code == hb.HTF_ENOTSPD
    assert s.status_sub() == bad
    assert f"subdomain {bad} " in str(e.value)
    s.close()
    solve_next_problem()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_max_iter_gives_enoconv(precision):
    m = hb.generate_mesh(hb.mesh_spec(**SPEC))
    s = hb.Solver(dict(OPTS, max_iter="3", precision=precision, batch="16", check_every="1"))
    s.set_mesh(m)
    s.setup()
    with pytest.raises(hb.HTFError) as e:
        s.pcpg()
    assert e.value.code == hb.HTF_ENOCONV
    s.close()
    solve_next_problem()


def test_unreachable_eps_stops_the_mixed_form_as_stagnated():
    """eps_iter = 1e-15 is below what an FP32 operator can carry the FP64
    residual to: the batched mixed form stops with HTF_ENOCONV once ten FP64
    residual replacements over at least 500 iterations have passed without
    the FP64 residual halving, long before max_iter."""
    m = hb.generate_mesh(hb.mesh_spec(**SPEC))
    s = hb.Solver(dict(OPTS, eps_iter="1e-15", max_iter="20000", precision="mixed", batch="16"))
    s.set_mesh(m)
    s.setup()
    with pytest.raises(hb.HTFError) as e:
        s.pcpg()
    assert e.value.code == hb.HTF_ENOCONV
    msg = str(e.value)
    assert "stagnated" in msg, msg
    it = int(msg.split(" to ")[1].split()[0])
    assert it < 5000, msg
    s.close()
    solve_next_problem()


def test_floating_body_gives_singular_gftgf():
    m = hb.generate_mesh(hb.mesh_spec(**SPEC))
    free = hb.Mesh(m.coords, m.elems, m.elem_sub, m.sub_cluster, m.sub_E, m.sub_nu,
                   np.zeros(0, np.int32), m.corner, m.body_force)
    s = hb.Solver(OPTS)
    s.set_mesh(free)
    with pytest.raises(hb.HTFError) as e:
        s.setup()
    assert e.value.code == hb.HTF_ENOTSPD
    assert "Gf^T Gf" in str(e.value)
    s.close()
    solve_next_problem()
