"""The oracle against outputs of the reference itself (tests/golden/*.npz,
generated by tests/golden/make_goldens.py from oracle/_ref/hfls_ref)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.htfeti_oracle import HTFETI, hex8_element
from tests.golden_util import golden_paths, load, mesh_from_golden, options_from_args, REF_BODY_FORCE

PATHS = golden_paths()
IDS = [p.split("/")[-1][:-4] for p in PATHS]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module", params=PATHS, ids=IDS)
def case(request):
    g, args = load(request.param)
    h = HTFETI(mesh_from_golden(g, args), options_from_args(args))
    return g, args, h


def test_dual_layout_bit_exact(case):
    """l2g maps, Bf rows / columns / signs and multiplicity weights equal the
    reference's (Data.cpp:111-144, Cluster.cpp:832-959)."""
    g, _, h = case
    for d in range(int(g["nsub"])):
        assert np.array_equal(h.l2g[d], g[f"l2g_{d}"])
        assert np.array_equal(h.bf_l2g[d], g[f"bf_rows_{d}"])
        iptr, jcol, val = g[f"bf_iptr_{d}"], g[f"bf_jcol_{d}"], g[f"bf_val_{d}"]
        rows = np.repeat(np.arange(len(iptr) - 1), np.diff(iptr))
        ref = sorted(zip(rows.tolist(), jcol.tolist(), val.tolist()))
        mine = sorted(zip(h.bf_rowloc[d].tolist(), h.bf_col[d].tolist(), h.bf_val[d].tolist()))
        assert ref == mine
    assert np.array_equal(h.weight, g["weight"])


def test_element_matrices(case):
    """Data::stf_mtrx_solid45: bit-exact with the reference's gradient; the
    standard J^{-T} gradient agrees on the axis-aligned element and differs on
    the distorted one, where the reference's K_e does not annihilate rotations."""
    g, _, _ = case
    for v in range(2):
        K, f = hex8_element(g["elem_coords"][v][None], 2.1e5, 0.3, REF_BODY_FORCE, "reference")
        assert np.array_equal(K[0], g["elem_K"][v])
        assert np.array_equal(f[0], g["elem_f"][v])
    Ks, _ = hex8_element(g["elem_coords"][0][None], 2.1e5, 0.3, REF_BODY_FORCE, "standard")
    assert rel(Ks[0], g["elem_K"][0]) < 1e-14
    Kd, _ = hex8_element(g["elem_coords"][1][None], 2.1e5, 0.3, REF_BODY_FORCE, "standard")
    assert rel(Kd[0], g["elem_K"][1]) > 1e-3


def test_projected_operators(case):
    """P F P w and P M P w (Cluster.cpp:1043-1188, 1314-1329) are invariant
    under the choice of generalised inverse and kernel basis."""
    g, _, h = case
    Pw = h.project(g["w"])[0]
    assert rel(Pw, g["Pw"]) < 1e-12
    assert rel(h.project(h.mult_F(Pw))[0], g["PFPw"]) < 1e-10
    assert rel(h.project(h.precondition(Pw))[0], g["PMPw"]) < 1e-12


def test_pcpg_iterations_and_displacements(case):
    g, _, h = case
    s = h.pcpg()
    assert abs(s["iterations"] - int(g["iterations"])) <= 2
    tight = h.pcpg(eps_iter=1e-10, max_iter=1000)
    assert tight["iterations"] < 1000
    assert rel(tight["u"], g["u_tight"]) < 1e-8


def test_fix_rule_and_kernel_basis_do_not_change_u(case):
    """Fix DOFs restricted to the Bf column set (the GPU path's rule) and the
    analytic ker(Gc) give the same displacements and iterations."""
    g, args, h = case
    a = h.pcpg(eps_iter=1e-10, max_iter=1000)
    h2 = HTFETI(mesh_from_golden(g, args),
                options_from_args(args, fix_rule="boundary", kerGc="analytic"))
    b = h2.pcpg(eps_iter=1e-10, max_iter=1000)
    assert rel(b["u"], a["u"]) < 1e-9
    assert abs(a["iterations"] - b["iterations"]) <= 2


def _direct(h):
    m = h.m
    n = 3 * len(m.coords)
    rows, cols, vals = [], [], []
    f = np.zeros(n)
    for d in range(m.n_sub):
        l2g = h.l2g[d]
        r, c = np.meshgrid(l2g, l2g, indexing="ij")
        rows.append(r.ravel()); cols.append(c.ravel()); vals.append(h.K[d].ravel())
        np.add.at(f, l2g, h.f[d][:, 0])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    free = np.setdiff1d(np.arange(n), m.dirichlet_dofs)
    u = np.zeros(n)
    u[free] = spla.spsolve(A[free][:, free].tocsc(), f[free])
    return u


@pytest.mark.parametrize("typeBc", ["cor", "ker"])
def test_multi_cluster_matches_direct_solve(typeBc):
    """Two clusters (the reference handles one): u equals a direct global
    solve of the assembled problem."""
    g, args = load([p for p in PATHS if "clamp_5" in p][0])
    clusters = np.array([0, 0, 0, 0, 1, 1, 1, 1])
    args = dict(args, typeBc=typeBc)
    h = HTFETI(mesh_from_golden(g, args, clusters), options_from_args(args))
    s = h.pcpg(eps_iter=1e-10, max_iter=1000)
    assert h.Gf.shape[1] == 12
    assert rel(s["u"], _direct(h)) < 1e-8


def test_uneven_slabs_match_direct_solve():
    """Subdomains of different sizes in two clusters with a 1e3 material
    contrast (the shape of the 4 096-subdomain configuration at a size the
    oracle solves in a second): u equals a direct global solve."""
    import hfls_b200 as hb
    from oracle.htfeti_oracle import MeshArrays, Options
    spec = hb.mesh_spec(clusters=(2, 1, 1), subs=(2, 2, 1), widths=([2, 4, 3, 1], [3, 1], [2]), jitter=0.1,
                        seed=5, material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3)
    m = hb.generate_mesh(spec)
    ma = MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64), m.sub_cluster.astype(np.int64),
                    m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64), m.corner.astype(np.int64), m.body_force)
    h = HTFETI(ma, Options(typeBc="cor", fix_rule="boundary", kerGc="analytic"))
    sizes = [len(h.l2g[d]) for d in range(m.n_sub)]
    assert min(sizes) < max(sizes) / 2                      # really uneven
    s = h.pcpg(eps_iter=1e-11, max_iter=3000)
    assert rel(s["u"], _direct(h)) < 1e-8
