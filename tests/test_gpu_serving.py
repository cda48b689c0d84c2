"""Continuous-batching server (htf_server_*) on the GPU: requests of different
meshes and load-case counts, admitted by device footprint, iterating together
with one tensor-core launch for all their F (and S) products.

Tolerances: every served displacement field within 1e-7 relative of the FP64
oracle (the mixed form's bound) and of the same request solved alone; the
same request alone and in a mix gives the same iterations."""
import numpy as np
import pytest

import hfls_b200 as hb
from oracle.htfeti_oracle import HTFETI, MeshArrays, Options

pytestmark = pytest.mark.gpu

OPTS = {"typeBc": "cor", "eps_iter": "1e-8", "max_iter": "3000", "batch": "16"}


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def oracle_mesh(m, f=None):
    return MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64), m.sub_cluster.astype(np.int64),
                      m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64), m.corner.astype(np.int64), m.body_force, f)


REQS = [
    (dict(clusters=(1, 1, 1), subs=(2, 2, 2), elems=(3, 3, 3), jitter=0.1, seed=3,
          material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3), 2),
    (dict(clusters=(2, 1, 1), subs=(2, 2, 2), elems=(3, 2, 3), jitter=0.1, seed=4,
          material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, nu=0.25), 1),
    (dict(clusters=(1, 1, 1), subs=(3, 2, 2), widths=([3, 4, 2], [3, 3], [4, 2]), jitter=0.1, seed=5,
          material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e2), 3),
    (dict(clusters=(1, 2, 1), subs=(2, 2, 2), elems=(4, 4, 4), jitter=0.05, seed=6,
          material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, nu=0.35), 4),
]


def spec_and_loads(i):
    kw, nrhs = REQS[i]
    spec = hb.mesh_spec(**kw)
    return spec, hb.traction(spec, seed=100 + i, n_rhs=nrhs)


def alone(i):
    spec, f = spec_and_loads(i)
    s = hb.Solver(dict(OPTS, precision="mixed"))
    s.set_mesh(hb.generate_mesh(spec))
    s.setup()
    u, st = s.solve(f)
    return u, st


def test_served_mix_matches_alone_and_oracle():
    srv = hb.Server(OPTS, max_live=8)
    tickets = []
    for i in range(len(REQS)):
        spec, f = spec_and_loads(i)
        tickets.append(srv.submit(spec, f))
    out = [srv.wait(t) for t in tickets]
    srv.close()
    for i, (u, info) in enumerate(out):
        assert info.status == hb.HTF_REQ_DONE and info.rc == 0
        assert info.t_submit_ms <= info.t_admit_ms <= info.t_start_ms <= info.t_done_ms
        ua, sta = alone(i)
        assert rel(u, ua) < 1e-7, i
        assert info.iterations_max == max(sta.iterations[:REQS[i][1]]), i
    # one request against the FP64 oracle
    spec, f = spec_and_loads(0)
    m = hb.generate_mesh(spec)
    o = HTFETI(oracle_mesh(m, f.T.copy()), Options(typeBc="cor", fix_rule="boundary", kerGc="analytic"))
    for k in range(REQS[0][1]):
        ref = o.pcpg(rhs_index=k, eps_iter=1e-11, max_iter=3000)
        assert rel(out[0][0][k], ref["u"]) < 1e-7


def test_same_result_alone_and_in_a_mix():
    srv = hb.Server(OPTS)
    spec, f = spec_and_loads(3)
    u_alone, i_alone = srv.wait(srv.submit(spec, f))
    others = [srv.submit(*spec_and_loads(i)) for i in range(3)]
    t = srv.submit(spec, f)
    u_mix, i_mix = srv.wait(t)
    for o in others:
        srv.wait(o)
    srv.close()
    assert rel(u_mix, u_alone) < 1e-7
    assert i_mix.iterations_max == i_alone.iterations_max


def test_admission_by_budget_and_oversize_request():
    spec, f = spec_and_loads(3)
    one = hb.Server(OPTS)
    u0, info0 = one.wait(one.submit(spec, f))
    one.close()
    assert 0.5 * info0.bytes < info0.bytes_estimate < 3.0 * info0.bytes
    # room for one admission estimate but not for a set-up request plus another
    # estimate: requests run one after another
    srv = hb.Server(OPTS, hbm_budget_bytes=info0.bytes_estimate + 0.5 * info0.bytes)
    t = [srv.submit(spec, f) for _ in range(3)]
    infos = [srv.wait(x)[1] for x in t]
    for a, b in zip(infos, infos[1:]):
        assert b.t_admit_ms >= a.t_done_ms - 1e-6
    # a request far above the budget fails cleanly, the server keeps serving
    big = hb.mesh_spec(clusters=(2, 2, 2), subs=(4, 4, 4), elems=(8, 8, 8))
    tb = srv.submit(big, n_rhs=1)
    with pytest.raises(hb.HTFError) as e:
        srv.wait(tb)
    assert e.value.code == hb.HTF_ENOMEM
    u1, _ = srv.wait(srv.submit(spec, f))
    srv.close()
    assert rel(u1, u0) < 1e-12


def test_largest_request_of_a_mix_against_tight_fp64():
    """The largest request of a served mix (4x3x3 clusters of 2x2x2
    subdomains of 5^3 hex8, E contrast 1e4, 4 load cases) against the plain
    FP64 form solved to eps 1e-11: within the mixed form's 1e-7 bound (the
    served form stops at eps_iter x mixed_eps_factor = 1e-9)."""
    big = dict(clusters=(4, 3, 3), subs=(2, 2, 2), elems=(5, 5, 5), jitter=0.1, seed=11,
               material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, nu=0.3)
    spec = hb.mesh_spec(**big)
    f = hb.traction(spec, seed=77, n_rhs=4)
    srv = hb.Server(OPTS, max_live=8)
    small = [srv.submit(*spec_and_loads(i)) for i in range(2)]
    t = srv.submit(spec, f)
    u, info = srv.wait(t)
    for x in small:
        srv.wait(x)
    srv.close()
    s = hb.Solver(dict(OPTS, precision="fp64", eps_iter="1e-11", max_iter="6000"))
    s.set_mesh(hb.generate_mesh(spec))
    s.setup()
    u64, _ = s.solve(f)
    s.close()
    for k in range(4):
        assert rel(u[k], u64[k]) < 1e-7, k


# 8 subdomains of 6^3 hex8: factor panels of ~4.3 MB each, the larger part of
# the request's device footprint
WAVE_SPEC = dict(clusters=(1, 1, 1), subs=(2, 2, 2), elems=(6, 6, 6), jitter=0.1, seed=21,
                 material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3, nu=0.3)


def test_factor_waves_same_as_resident_factors():
    """factor_wave_gb = 6 MB holds one subdomain's panels at a time: the set-up
    factorises wave by wave and the start solve and the reconstruction
    assemble and factorise every wave again.  Each subdomain's arithmetic is
    the one of the resident-factor solve, so iterations and displacements
    agree (to rounding, 1e-13)."""
    spec = hb.mesh_spec(**WAVE_SPEC)
    f = hb.traction(spec, seed=31, n_rhs=3)
    out = []
    for extra in ({}, {"factor_wave_gb": "0.006"}):
        s = hb.Solver(dict(OPTS, precision="mixed", **extra))
        s.set_mesh(hb.generate_mesh(spec))
        s.setup()
        out.append(s.solve(f))
        s.close()
    (u0, st0), (u1, st1) = out
    assert list(st1.iterations[:3]) == list(st0.iterations[:3])
    assert rel(u1, u0) < 1e-13


def test_server_holds_factor_panels_in_waves_when_they_do_not_fit():
    """Factor waves in the server.  Forced (factor_wave_gb = 20 MB, one
    subdomain of 8^3 hex8 per wave): smaller estimate and device bytes, the
    displacements of the resident-factor run.  Chosen by admission: a budget
    just above the forced run's estimate, below the resident-factor estimate,
    refuses the request (HTF_ENOMEM) by default and, with admit_oversize=1,
    admits it with its panels held a wave at a time."""
    spec = hb.mesh_spec(**dict(WAVE_SPEC, elems=(8, 8, 8)))
    f = hb.traction(spec, seed=31, n_rhs=2)
    one = hb.Server(OPTS)
    u0, info0 = one.wait(one.submit(spec, f))
    one.close()
    forced = hb.Server(dict(OPTS, factor_wave_gb="0.02"))
    u1, info1 = forced.wait(forced.submit(spec, f))
    forced.close()
    assert info1.bytes < info0.bytes and info1.bytes_estimate < info0.bytes_estimate
    assert info1.iterations_max == info0.iterations_max
    assert rel(u1, u0) < 1e-13
    budget = 1.05 * info1.bytes_estimate
    assert budget < info0.bytes_estimate
    refuse = hb.Server(OPTS, hbm_budget_bytes=budget)
    with pytest.raises(hb.HTFError) as e:
        refuse.wait(refuse.submit(spec, f))
    refuse.close()
    assert e.value.code == hb.HTF_ENOMEM
    srv = hb.Server(dict(OPTS, admit_oversize="1"), hbm_budget_bytes=budget)
    u2, info2 = srv.wait(srv.submit(spec, f))
    srv.close()
    assert info2.rc == 0 and info2.status == hb.HTF_REQ_DONE
    assert info2.bytes_estimate <= budget
    assert info2.iterations_max == info0.iterations_max
    assert rel(u2, u0) < 1e-13
    print("resident / forced waves / admitted in waves: estimate MB %.1f %.1f %.1f, device MB %.1f %.1f %.1f" % (
        info0.bytes_estimate / 1e6, info1.bytes_estimate / 1e6, info2.bytes_estimate / 1e6,
        info0.bytes / 1e6, info1.bytes / 1e6, info2.bytes / 1e6))


def test_s_kept_as_tensor_core_slabs_only():
    """S_fp64=0 with factor waves: S_i is snapshotted into one wave's FP64
    scratch, made into its tensor-core slabs and dropped; the FP64 residual
    replacements apply it through the tensor-core product too.  The
    displacements stay within the mixed form's 1e-7 of the resident run, the
    iteration counts within a few check intervals."""
    spec = hb.mesh_spec(**WAVE_SPEC)
    f = hb.traction(spec, seed=31, n_rhs=3)
    out = []
    for extra in ({}, {"factor_wave_gb": "0.006", "S_fp64": "0"}):
        s = hb.Solver(dict(OPTS, precision="mixed", **extra))
        s.set_mesh(hb.generate_mesh(spec))
        s.setup()
        out.append(s.solve(f))
        s.close()
    (u0, st0), (u1, st1) = out
    for k in range(3):
        assert abs(int(st1.iterations[k]) - int(st0.iterations[k])) <= 16 + 0.02 * st0.iterations[k], k
        assert rel(u1[k], u0[k]) < 1e-7, k
