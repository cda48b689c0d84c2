"""Generate the full-size oracle goldens of the benchmark meshes.

The oracle (oracle/htfeti_oracle.py, memory-lean form ``HTFETIExplicit``)
solves, on the host, the two configurations the benchmark measures:

  cube1:    2x2x2 clusters x 4x4x4 subdomains x 8^3 hex8 (512 subdomains,
            823 875 DOFs), jitter 0.1h (seed 1), E logU[1e3, 1e6], nu 0.3,
            u = 0 on x = 0, one seeded N(0,1) nodal traction on x = 1 (seed 2),
            no body force, corner Bc, Dirichlet preconditioner;
  cube32:   the same mesh with body force (0, 0, -1) and 32 seeded N(0,1)
            tractions (seed 3), the multi-load-case form.

For every load case it records the PCPG iteration at which the reference's
criterion sqrt(g'Pz) < eps sqrt(g0'Pz0) (Cluster.cpp:1422-1426) first holds
at eps 1e-8, and the displacement field of a run continued to eps 1e-11.
A golden stores the iteration counts, the relative residual history around
eps 1e-8, and the displacements at 20 000 (cube1) / 4 096 (cube32) seeded
DOFs plus their projections on 8 seeded N(0,1) vectors over all DOFs
(tests regenerate the vectors from the seed), so a 1e-8 comparison needs no
multi-megabyte fixture.

The mesh comes from the library's host mesh generator (htf_mesh_fill); the
oracle's element, layout and kernel code is independent of the library.

Run from the repository root (about 30-60 min per case on 8 cores):
    python tests/golden/make_large_goldens.py cube1
    python tests/golden/make_large_goldens.py cube32
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUTDIR = os.path.join(ROOT, "tests", "golden")

CUBE = dict(clusters=(2, 2, 2), subs=(4, 4, 4), elems=(8, 8, 8), jitter=0.1, seed=1, E=1e3, E_hi=1e6, nu=0.3)
CASES = {
    "cube1": dict(spec=dict(CUBE, body_force=(0.0, 0.0, 0.0)), traction_seed=2, n_rhs=1, n_sample=20000),
    "cube32": dict(spec=dict(CUBE, body_force=(0.0, 0.0, -1.0)), traction_seed=3, n_rhs=32, n_sample=4096),
}
SAMPLE_SEED = 12345
PROJ_SEED = 777
N_PROJ = 8
EPS_RECORD, EPS_STOP = 1e-8, 1e-11


def sample_dofs(n_dof, n_sample):
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(n_dof, size=n_sample, replace=False))


def projection_vectors(n_dof):
    return np.random.default_rng(PROJ_SEED).standard_normal((N_PROJ, n_dof))


def make(name):
    import hfls_b200 as hb
    from oracle.htfeti_oracle import HTFETIExplicit, MeshArrays, Options
    c = CASES[name]
    spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, bc=hb.HTF_BC_CLAMP_X0, **c["spec"])
    m = hb.generate_mesh(spec)
    f = hb.traction(spec, seed=c["traction_seed"], n_rhs=c["n_rhs"])
    mesh = MeshArrays(m.coords, m.elems.astype(np.int64), m.elem_sub.astype(np.int64),
                      m.sub_cluster.astype(np.int64), m.sub_E, m.sub_nu, m.dirichlet.astype(np.int64),
                      m.corner.astype(np.int64), m.body_force, f.T.copy())
    t0 = time.time()
    o = HTFETIExplicit(mesh, Options(typeBc="cor", preconditioner="Dirichlet_explicit", fix_rule="boundary",
                                     kerGc="analytic"))
    print(f"{name}: setup {time.time() - t0:.0f} s, n_lambda {o.n_lam}", flush=True)
    def progress(it, rel, active):
        print(f"  it {it}: max rel {rel[active].max() if active.any() else 0:.3e}, active {active.sum()}",
              flush=True)

    t0 = time.time()
    r = o.pcpg_block(eps_record=EPS_RECORD, eps_stop=EPS_STOP, max_iter=20000, progress=progress)
    print(f"{name}: pcpg {time.time() - t0:.0f} s, iterations at 1e-8 {r['it_record']}, "
          f"at 1e-11 {r['it_stop']}", flush=True)
    u = r["u"]                                          # n_dof x n_rhs
    idx = sample_dofs(u.shape[0], c["n_sample"])
    P = projection_vectors(u.shape[0])
    np.savez_compressed(
        os.path.join(OUTDIR, f"oracle_{name}.npz"),
        iterations=r["it_record"], iterations_tight=r["it_stop"], eps_record=EPS_RECORD, eps_stop=EPS_STOP,
        n_dof=u.shape[0], sample_idx=idx, u_sample=u[idx].T.copy(), u_proj=(P @ u).T.copy(),
        u_norm=np.linalg.norm(u, axis=0), norm_gPz0=r["norm_gPz0"],
        hist=r["hist"][:int(r["it_record"].max()) + 12],
        n_lambda=o.n_lam)


if __name__ == "__main__":
    for n in sys.argv[1:] or list(CASES):
        make(n)
