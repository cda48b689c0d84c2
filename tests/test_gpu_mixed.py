"""Batched mixed-precision form on the GPU: F_i / S_i stored as scaled FP16
hi + lo pairs (4 bytes per entry, 22 significant bits) and applied on the
tensor cores (tcgen05 kind::f16, three products per K step, FP32
accumulation in TMEM) for a batch of load cases; coarse problems, projector,
residual replacement and displacements in FP64.

Tolerances: the tensor-core F apply against the FP64 oracle 1e-5 relative
(FP32-level storage, about 1e-6 after the coarse-correction cancellation), the
preconditioner 1e-6, the batched FP64 projector 1e-12; the displacements of
the mixed solve against the FP64 oracle 1e-7 relative (the bound for the
mixed form)."""
import numpy as np
import pytest

import hfls_b200 as hb
from oracle.htfeti_oracle import HTFETI, MeshArrays, Options

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def oracle_mesh(m, f=None):
    return MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64), m.sub_cluster.astype(np.int64),
                      m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64), m.corner.astype(np.int64), m.body_force, f)


SPEC = dict(clusters=(2, 1, 1), subs=(2, 2, 2), elems=(3, 3, 3), jitter=0.1, seed=7,
            material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3, body_force=(0.0, 0.0, -1.0))


@pytest.mark.parametrize("batch", [16, 32])
def test_tensor_core_operators(batch):
    m = hb.generate_mesh(hb.mesh_spec(**SPEC))
    s = hb.Solver({"typeBc": "cor", "precision": "mixed", "batch": str(batch)})
    s.set_mesh(m)
    s.setup()
    o = HTFETI(oracle_mesh(m), Options(typeBc="cor", fix_rule="boundary", kerGc="analytic"))
    rng = np.random.default_rng(1)
    w = rng.standard_normal((5, o.n_lam))
    Fw = s.mult_Ff(w)
    Mw = s.preconditioning(w)
    Pw = s.projection(w)
    for k in range(5):
        assert rel(Fw[k], o.mult_F(w[k])) < 1e-5
        assert rel(Mw[k], o.precondition(w[k])) < 1e-6
        assert rel(Pw[k], o.project(w[k])[0]) < 1e-12
    assert np.array_equal(s.mult_Ff(w), Fw)          # a fixed linear operator: bitwise repeatable


def test_mixed_batched_solve_matches_fp64_oracle():
    spec = hb.mesh_spec(**SPEC)
    m = hb.generate_mesh(spec)
    f = hb.traction(spec, seed=5, n_rhs=6)
    s = hb.Solver({"typeBc": "cor", "precision": "mixed", "batch": "16", "eps_iter": "1e-8", "max_iter": "3000"})
    s.set_mesh(m)
    s.setup()
    u, st = s.solve(f)
    o = HTFETI(oracle_mesh(m, f.T.copy()), Options(typeBc="cor", fix_rule="boundary", kerGc="analytic"))
    for k in range(6):
        ref = o.pcpg(rhs_index=k, eps_iter=1e-11, max_iter=3000)
        fp64 = o.pcpg(rhs_index=k, eps_iter=1e-8, max_iter=3000)
        assert rel(u[k], ref["u"]) < 1e-7, k
        # FP32 operators cost iterations, but boundedly
        assert 0 < st.iterations[k] <= 1.5 * fp64["iterations"], k


def test_mixed_same_result_alone_and_in_a_batch():
    """A load case solved alone and inside a batch of others gives the same
    displacements within the mixed-form tolerance."""
    spec = hb.mesh_spec(**SPEC)
    m = hb.generate_mesh(spec)
    f = hb.traction(spec, seed=9, n_rhs=4)
    s = hb.Solver({"typeBc": "cor", "precision": "mixed", "batch": "16", "eps_iter": "1e-8"})
    s.set_mesh(m)
    s.setup()
    u_all, st_all = s.solve(f)
    u_one, st_one = s.solve(f[2:3])
    assert rel(u_one[0], u_all[2]) < 1e-7
    # columns of the batch do not interact: the same iterations alone and in the mix
    assert st_one.iterations[0] == st_all.iterations[2]
