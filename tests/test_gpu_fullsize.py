"""The benchmark's cube at full size against the oracle (goldens written by
tests/golden/make_large_goldens.py: the oracle solves the same seeded mesh
on the host, iteration counts at eps 1e-8 and displacements at eps 1e-11).

  cube1:  2x2x2 clusters x 4x4x4 subdomains x 8^3 hex8 (823 875 DOFs), one
          N(0,1) traction load case, plain FP64 form: the residual history
          equal to the oracle's to 1e-9 over the first 20 iterations, the
          stopping iteration at eps 1e-8 within 4 % of the oracle's
          (same_stop; the oracle stops at 627 with its residual between 0.92
          and 1.18 x eps from iteration 620 to 635), displacements at eps
          1e-10 within 1e-8 of the oracle's;
  cube32: the same mesh, body force + 32 traction load cases: the batched
          mixed-precision form's displacements within 1e-7 of the oracle's
          for every load case, and the plain FP64 form's stopping iterations
          on four of them within 4 % of the oracle's (same_stop)."""
import numpy as np
import pytest

import hfls_b200 as hb
from tests.golden_util import golden_rel_err, oracle_golden, same_stop

pytestmark = pytest.mark.gpu

CUBE = dict(clusters=(2, 2, 2), subs=(4, 4, 4), elems=(8, 8, 8), jitter=0.1, seed=1, E=1e3, E_hi=1e6, nu=0.3,
            material=hb.HTF_MAT_LOGUNIFORM, bc=hb.HTF_BC_CLAMP_X0)
OPTS = {"typeBc": "cor", "preconditioner": "Dirichlet_explicit", "max_iter": "5000", "device": "0"}


def solver(spec, f, **opts):
    s = hb.Solver(dict(OPTS, **opts))
    s.set_mesh(hb.generate_mesh(spec))
    s.set_loads(f)
    s.setup()
    return s


def test_cube1_fp64_matches_oracle():
    g = oracle_golden("cube1")
    spec = hb.mesh_spec(body_force=(0.0, 0.0, 0.0), **CUBE)
    f = hb.traction(spec, seed=2, n_rhs=1)
    s = solver(spec, f, eps_iter="1e-8")
    _, st = s.pcpg()
    h = s.residual_history(0)
    s.close()
    ho = g["hist"][:, 0]
    # the same arithmetic up to round-off for the first iterations, the same plateau at the stop
    assert np.max(np.abs(h[:20] - ho[:20]) / ho[:20]) < 1e-9
    assert same_stop(st.iterations[0], int(g["iterations"][0]))
    s = solver(spec, f, eps_iter="1e-10")
    u, st = s.pcpg()
    s.close()
    assert u.shape[1] == int(g["n_dof"])
    assert golden_rel_err(g, u[0], 0) < 1e-8


def test_cube32_mixed_and_fp64_match_oracle():
    g = oracle_golden("cube32")
    spec = hb.mesh_spec(body_force=(0.0, 0.0, -1.0), **CUBE)
    f = hb.traction(spec, seed=3, n_rhs=32)
    s = solver(spec, f, eps_iter="1e-8", precision="mixed", batch="32")
    u, st = s.pcpg()
    s.close()
    err = [golden_rel_err(g, u[k], k) for k in range(32)]
    assert max(err) < 1e-7, err
    pick = [0, 11, 21, 31]
    s = hb.Solver(dict(OPTS, eps_iter="1e-8"))
    s.set_mesh(hb.generate_mesh(spec))
    s.setup()
    _, st = s.solve(f[pick])
    for i, k in enumerate(pick):
        assert same_stop(st.iterations[i], int(g["iterations"][k]))
