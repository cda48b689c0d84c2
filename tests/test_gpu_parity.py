"""GPU path against the oracle and the reference goldens (CUDA, sm_100a).

Tolerances (FP64 plain form): F apply 1e-8, projector and preconditioner 1e-11 relative, displacements 1e-8
relative at eps_iter 1e-10, PCPG iteration counts +-2."""
import numpy as np
import pytest

import hfls_b200 as hb
from oracle.htfeti_oracle import HTFETI, Options, MeshArrays
from tests.golden_util import golden_paths, load, mesh_from_golden, same_stop

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def oracle_mesh(m, f_nodal=None):
    return MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64),
                      m.sub_cluster.astype(np.int64), m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64),
                      m.corner.astype(np.int64), m.body_force, f_nodal)


def make(spec_kw, opts, f_nodal=None):
    m = hb.generate_mesh(hb.mesh_spec(**spec_kw))
    s = hb.Solver(opts)
    s.set_mesh(m)
    if f_nodal is not None:
        s.set_loads(f_nodal)
    s.setup()
    o = HTFETI(oracle_mesh(m, None if f_nodal is None else f_nodal.T.copy()),
               Options(typeBc=opts.get("typeBc", "cor"), preconditioner=opts.get("preconditioner", "Dirichlet_explicit"),
                       eps_iter=float(opts.get("eps_iter", 1e-8)), fix_rule="boundary", kerGc="analytic"))
    return m, s, o


SMALL = [
    (dict(subs=(2, 2, 2), elems=(3, 3, 3)), dict(typeBc="cor", preconditioner="Dirichlet_explicit")),
    (dict(subs=(2, 2, 2), elems=(3, 3, 3), jitter=0.1, seed=5), dict(typeBc="ker", preconditioner="lumped")),
    (dict(clusters=(2, 1, 1), subs=(2, 2, 2), elems=(3, 2, 3), jitter=0.1, seed=7,
          material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4), dict(typeBc="cor", preconditioner="Dirichlet_explicit")),
    (dict(clusters=(2, 1, 1), subs=(2, 2, 2), elems=(3, 3, 2), jitter=0.1, seed=8,
          material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3), dict(typeBc="cor", preconditioner="Dirichlet_implicit")),
]
IDS = ["cor-dirichlet", "ker-lumped-jitter", "2clusters-cor-logE", "2clusters-cor-implicit"]


@pytest.fixture(scope="module", params=list(range(len(SMALL))), ids=IDS)
def small(request):
    spec, opts = SMALL[request.param]
    return make(spec, opts)


def test_operators_match_oracle(small):
    m, s, o = small
    rng = np.random.default_rng(0)
    w = rng.standard_normal((2, o.n_lam))
    Fw = s.mult_Ff(w)
    for k in range(2):
        assert rel(Fw[k], o.mult_F(w[k])) < 1e-8      # round-off amplified by the coarse correction
        assert rel(s.projection(w[k:k + 1])[0], o.project(w[k])[0]) < 1e-12
        assert rel(s.preconditioning(w[k:k + 1])[0], o.precondition(w[k])) < 1e-11


def test_pcpg_matches_oracle(small):
    m, s, o = small
    u, st = s.pcpg()
    ref = o.pcpg()
    assert same_stop(st.iterations[0], ref["iterations"])
    assert rel(u[0], ref["u"]) < 1e-6          # both stop at eps_iter 1e-8


def test_pcpg_tight_tolerance_displacements():
    spec, opts = SMALL[2]
    m, s, o = make(spec, dict(opts, eps_iter="1e-10", max_iter="2000"))
    u, st = s.pcpg()
    ref = o.pcpg(eps_iter=1e-10, max_iter=2000)
    assert abs(st.iterations[0] - ref["iterations"]) <= 2
    assert rel(u[0], ref["u"]) < 1e-8


@pytest.mark.parametrize("path", golden_paths(), ids=lambda p: p.split("/")[-1][:-4])
def test_reference_golden_cases(path):
    """The reference's own meshes: iterations +-2 at eps 1e-8 and the
    displacement field of the reference's tight run within 1e-8."""
    g, args = load(path)
    ref_mesh = mesh_from_golden(g, args)
    m = hb.Mesh(ref_mesh.coords, ref_mesh.elems, ref_mesh.elem_sub, ref_mesh.sub_cluster, ref_mesh.sub_E,
                ref_mesh.sub_nu, ref_mesh.dirichlet_dofs, ref_mesh.corner_dofs, ref_mesh.body_force)
    pre = args["preconditioner"]
    s = hb.Solver({"typeBc": args["typeBc"], "preconditioner": pre, "eps_iter": "1e-8"})
    s.set_mesh(m)
    s.setup()
    u, st = s.pcpg()
    assert abs(st.iterations[0] - int(g["iterations"])) <= 2
    s2 = hb.Solver({"typeBc": args["typeBc"], "preconditioner": pre, "eps_iter": "1e-10", "max_iter": "1000"})
    s2.set_mesh(m)
    s2.setup()
    u2, st2 = s2.pcpg()
    assert st2.iterations[0] < 1000
    assert rel(u2[0], g["u_tight"]) < 1e-8


def test_multiple_load_cases():
    spec = dict(subs=(2, 2, 1), elems=(3, 3, 3), jitter=0.1, seed=2)
    f = hb.traction(hb.mesh_spec(**spec), seed=9, n_rhs=3)
    m, s, o = make(spec, dict(typeBc="cor", eps_iter="1e-10"), f_nodal=f)
    u, st = s.pcpg()
    for k in range(3):
        ref = o.pcpg(rhs_index=k, eps_iter=1e-10)
        assert abs(st.iterations[k] - ref["iterations"]) <= 2
        assert rel(u[k], ref["u"]) < 1e-8


def test_failed_setup_leaves_the_library_usable():
    """A setup that runs out of device memory (one subdomain of 60^3
    elements: a 3.7 TB dense factor) fails with HTF_ENOMEM and leaves no CUDA
    error behind: the next problem sets up and solves."""
    big = hb.Solver({"typeBc": "cor"})
    big.set_mesh(hb.generate_mesh(hb.mesh_spec(subs=(1, 1, 1), elems=(60, 60, 60))))
    with pytest.raises(hb.HTFError) as e:
        big.setup()
    assert e.value.code == hb.HTF_ENOMEM
    big.close()
    spec, opts = SMALL[0]
    m, s, o = make(spec, opts)
    u, st = s.pcpg()
    assert rel(u[0], o.pcpg()["u"]) < 1e-6


def test_implicit_preconditioner_keeps_no_s_blocks():
    """Dirichlet_implicit applies S_d through the resident factor's L_bb: the
    same operator as the explicit blocks (1e-11), without their device
    memory (at least the algorithmic bytes of the S_d triangles less)."""
    spec = dict(subs=(2, 2, 2), elems=(5, 5, 5), jitter=0.1, seed=9)
    m = hb.generate_mesh(hb.mesh_spec(**spec))
    out = {}
    for pre in ("Dirichlet_explicit", "Dirichlet_implicit"):
        s = hb.Solver({"typeBc": "cor", "preconditioner": pre})
        s.set_mesh(m)
        s.setup()
        rng = np.random.default_rng(3)
        w = rng.standard_normal((1, s.n_lambda()))
        out[pre] = (s.preconditioning(w)[0], s.profile(reps=2))
        s.close()
    (me, pe), (mi, pi) = out["Dirichlet_explicit"], out["Dirichlet_implicit"]
    assert rel(mi, me) < 1e-11
    assert pe.device_bytes - pi.device_bytes >= 0.99 * pe.symv_S_bytes


def test_residual_history_is_the_stopping_record():
    """htf_residual_history: hist[0] = 1, one value per iteration, the last
    one below eps and all earlier ones not (the reference's criterion,
    Cluster.cpp:1422-1426), equal to the solve's final_rel."""
    spec, opts = SMALL[2]
    m, s, o = make(spec, opts)
    u, st = s.pcpg()
    h = s.residual_history(0)
    assert len(h) == st.iterations[0] + 1 and h[0] == 1.0
    assert h[-1] < 1e-8 and np.all(h[:-1] >= 1e-8)
    assert h[-1] == st.final_rel[0]
    ref = o.pcpg()
    # the same arithmetic up to round-off: equal for the first iterations (the
    # histories drift apart later, as those of any two FP64 implementations do)
    assert np.max(np.abs(h[:12] - ref["hist"][:12]) / ref["hist"][:12]) < 1e-8
