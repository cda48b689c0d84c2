"""FP64 CPU restatement of the reference's HTFETI hot path (ostravaTokyo/hfls).

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it.  The product path (``hfls_b200``) never calls it and fails loudly
when its CUDA library is missing.

Parity pin: the element matrices, the dual layout (``Bf`` rows, weights) and
the projected operators ``P F P w`` / ``P M P w`` as well as the displacement
field and iteration count are checked against outputs of the reference itself
(``oracle/_ref/hfls_ref``, compiled from the reference sources by
``oracle/ref_build/Makefile``); the committed fixtures live in
``tests/golden/`` together with the script that generated them.

Every function cites the reference file:line it restates.  Two deliberate,
documented deviations exist and are selectable:

* ``gradient="standard"`` (default) builds the hex8 strain operator with
  J^{-T}; the reference (Data.cpp:449-454) applies the cofactor matrix of J
  transposed, which equals J^{-T} only when J is symmetric (axis-aligned
  box elements, i.e. the reference's own meshes).  ``gradient="reference"``
  reproduces the reference's arithmetic exactly.
* ``fix_rule="reference"`` picks the 6 fix DOFs by the full-pivot elimination
  of Matrix::getNullPivots (Matrix.cpp:835-884) over all rows of R_i;
  ``fix_rule="boundary"`` applies the same elimination to the rows of R_i at
  the Bf column set only (the GPU path's rule).  Both make K_reg^{-1} a
  generalised inverse of K_i, so u and the projected operator are identical.
"""
from __future__ import annotations

import dataclasses
import numpy as np
import scipy.linalg as sla

# ---------------------------------------------------------------------------
# a1  hex8 element stiffness and body force  (Data.cpp:297-490)
# ---------------------------------------------------------------------------
_PT = 0.577350269189626          # Data.cpp:344 (the reference's literal)
# Gauss point i: r = gp[i], s = gp[i+8], t = gp[i+16]   (Data.cpp:363-386)
_GR = [-_PT, -_PT, -_PT, -_PT, _PT, _PT, _PT, _PT]
_GS = [-_PT, -_PT, _PT, _PT, -_PT, -_PT, _PT, _PT]
_GT = [-_PT, _PT, -_PT, _PT, -_PT, _PT, -_PT, _PT]


def _shape(r, s, t):
    """Trilinear shape functions and derivatives, Data.cpp:396-430 (same
    expression order so the values are bit-identical)."""
    dNr = [0.125 * -(1. - s) * (1. - t), 0.125 * (1. - s) * (1. - t),
           0.125 * (1. + s) * (1. - t), 0.125 * -(1. + s) * (1. - t),
           0.125 * -(1. - s) * (1. + t), 0.125 * (1. - s) * (1. + t),
           0.125 * (1. + s) * (1. + t), 0.125 * -(1. + s) * (1. + t)]
    dNs = [0.125 * -(1. - r) * (1. - t), 0.125 * -(1. + r) * (1. - t),
           0.125 * (1. + r) * (1. - t), 0.125 * (1. - r) * (1. - t),
           0.125 * -(1. - r) * (1. + t), 0.125 * -(1. + r) * (1. + t),
           0.125 * (1. + r) * (1. + t), 0.125 * (1. - r) * (1. + t)]
    dNt = [0.125 * -(1. - r) * (1. - s), 0.125 * -(1. + r) * (1. - s),
           0.125 * -(1. + r) * (1. + s), 0.125 * -(1. - r) * (1. + s),
           0.125 * (1. - r) * (1. - s), 0.125 * (1. + r) * (1. - s),
           0.125 * (1. + r) * (1. + s), 0.125 * (1. - r) * (1. + s)]
    N = [0.125 * (1. - r) * (1. - s) * (1. - t), 0.125 * (r + 1.) * (1. - s) * (1. - t),
         0.125 * (r + 1.) * (s + 1.) * (1. - t), 0.125 * (1. - r) * (s + 1.) * (1. - t),
         0.125 * (1. - r) * (1. - s) * (t + 1.), 0.125 * (r + 1.) * (1. - s) * (t + 1.),
         0.125 * (r + 1.) * (s + 1.) * (t + 1.), 0.125 * (1. - r) * (s + 1.) * (t + 1.)]
    return dNr, dNs, dNt, N


def hex8_element(X, E, nu, body_force=(0.0, 0.0, 0.0), gradient="standard"):
    """Element stiffness K_e (ne,24,24) and load f_e (ne,24).

    Restates Data::stf_mtrx_solid45 (Data.cpp:297-490) vectorised over
    elements, with the reference's accumulation order.  DOF order inside an
    element is [u_x of nodes 0-7, u_y 0-7, u_z 0-7] (Data.cpp:42-44);
    ``K_e[e, I, J]`` is the reference's val_K[I + 24 J].
    ``body_force`` is rho*a per unit volume (the reference hard-codes
    rho=2, a=(0,0,98.1), Data.cpp:315-318).
    """
    X = np.asarray(X, dtype=np.float64)
    ne = X.shape[0]
    E = np.broadcast_to(np.asarray(E, dtype=np.float64), (ne,))
    mu = np.broadcast_to(np.asarray(nu, dtype=np.float64), (ne,))
    x, y, z = X[:, :, 0], X[:, :, 1], X[:, :, 2]
    const1 = E / ((1. + mu) * (1. - 2. * mu))          # Data.cpp:341
    mu2 = 1. - mu
    mu3 = 0.5 - mu
    C = np.zeros((ne, 6, 6))                           # C[:, I, K] = C[I + 6K]
    C[:, 0, 0] = mu2 * const1; C[:, 0, 1] = mu * const1; C[:, 0, 2] = mu * const1
    C[:, 1, 0] = mu * const1; C[:, 1, 1] = mu2 * const1; C[:, 1, 2] = mu * const1
    C[:, 2, 0] = mu * const1; C[:, 2, 1] = mu * const1; C[:, 2, 2] = mu2 * const1
    C[:, 3, 3] = mu3 * const1; C[:, 4, 4] = mu3 * const1; C[:, 5, 5] = mu3 * const1
    Ke = np.zeros((ne, 24, 24))
    fe = np.zeros((ne, 24))
    bf = [float(b) for b in body_force]
    for g in range(8):
        dNr, dNs, dNt, N = _shape(_GR[g], _GS[g], _GT[g])
        J = [np.zeros(ne) for _ in range(9)]
        for j in range(8):                              # Data.cpp:437-447
            J[0] = J[0] + dNr[j] * x[:, j]; J[1] = J[1] + dNs[j] * x[:, j]; J[2] = J[2] + dNt[j] * x[:, j]
            J[3] = J[3] + dNr[j] * y[:, j]; J[4] = J[4] + dNs[j] * y[:, j]; J[5] = J[5] + dNt[j] * y[:, j]
            J[6] = J[6] + dNr[j] * z[:, j]; J[7] = J[7] + dNs[j] * z[:, j]; J[8] = J[8] + dNt[j] * z[:, j]
        A = J                                           # Data.cpp:276-294
        det = (+A[0] * (A[4] * A[8] - A[5] * A[7])
               - A[3] * (A[1] * A[8] - A[7] * A[2])
               + A[6] * (A[1] * A[5] - A[4] * A[2]))
        inv = 1. / det
        iA = [(A[4] * A[8] - A[5] * A[7]) * inv, -(A[3] * A[8] - A[6] * A[5]) * inv,
              (A[3] * A[7] - A[6] * A[4]) * inv, -(A[1] * A[8] - A[7] * A[2]) * inv,
              (A[0] * A[8] - A[6] * A[2]) * inv, -(A[0] * A[7] - A[1] * A[6]) * inv,
              (A[1] * A[5] - A[2] * A[4]) * inv, -(A[0] * A[5] - A[2] * A[3]) * inv,
              (A[0] * A[4] - A[1] * A[3]) * inv]
        if gradient == "reference":                     # Data.cpp:452-454 verbatim
            cx, cy, cz = (iA[0], iA[3], iA[6]), (iA[1], iA[4], iA[7]), (iA[2], iA[5], iA[8])
        elif gradient == "standard":                    # dN/dx = J^{-T} dN/dr
            cx, cy, cz = (iA[0], iA[1], iA[2]), (iA[3], iA[4], iA[5]), (iA[6], iA[7], iA[8])
        else:
            raise ValueError(gradient)
        Gt = np.zeros((ne, 6, 24))                      # Gt[:, K, J] = Gt[24K + J]
        for j in range(8):                              # Data.cpp:451-464
            dx = cx[0] * dNr[j] + cx[1] * dNs[j] + cx[2] * dNt[j]
            dy = cy[0] * dNr[j] + cy[1] * dNs[j] + cy[2] * dNt[j]
            dz = cz[0] * dNr[j] + cz[1] * dNs[j] + cz[2] * dNt[j]
            Gt[:, 0, j] = dx; Gt[:, 1, j + 8] = dy; Gt[:, 2, j + 16] = dz
            Gt[:, 3, j] = dy; Gt[:, 3, j + 8] = dx
            Gt[:, 4, j + 8] = dz; Gt[:, 4, j + 16] = dy
            Gt[:, 5, j] = dz; Gt[:, 5, j + 16] = dx
        CG = np.zeros((ne, 6, 24))                      # Data.cpp:468-475
        for K in range(6):
            CG = CG + C[:, :, K, None] * Gt[:, K, None, :]
        dj = det[:, None, None]
        for K in range(6):                              # Data.cpp:476-482
            Ke = Ke + (Gt[:, K, :, None] * CG[:, K, None, :]) * dj
        for j in range(8):                              # Data.cpp:484-488
            fe[:, j] = fe[:, j] + (bf[0] * N[j]) * det
            fe[:, j + 8] = fe[:, j + 8] + (bf[1] * N[j]) * det
            fe[:, j + 16] = fe[:, j + 16] + (bf[2] * N[j]) * det
    return Ke, fe


def element_dofs(elems):
    """ieq of every element: [3n+0 for nodes 0-7, 3n+1 ..., 3n+2 ...]
    (Data.cpp:42-44)."""
    elems = np.asarray(elems, dtype=np.int64)
    return np.concatenate([3 * elems + 0, 3 * elems + 1, 3 * elems + 2], axis=1)


# ---------------------------------------------------------------------------
# a4/a5  kernel, Gram-Schmidt and fix DOFs
# ---------------------------------------------------------------------------
def _dot_seq(a, b):
    """Left-to-right sum like Matrix::dot (Matrix.cpp:1583-1590)."""
    if a.size == 0:
        return 0.0
    return float(np.cumsum(a * b)[-1])


def gram_schmidt(R):
    """Matrix::GramSchmidtOrtho, Matrix.cpp:2450-2472 (classical GS,
    column by column, sequential dot products)."""
    R = np.array(R, dtype=np.float64, order="F")
    n, m = R.shape
    for j in range(m):
        w = R[:, j].copy()
        coef = [_dot_seq(w, R[:, i]) for i in range(j)]
        for i in range(j):
            w = w - R[:, i] * coef[i]
        nrm = np.sqrt(_dot_seq(w, w))
        R[:, j] = w / nrm
    return R


def rigid_body_modes(node_xyz):
    """Analytic kernel of a floating elasticity subdomain, column order of
    Data::create_analytic_ker_K (Data.cpp:61-109): translations x,y,z, then
    (-y,x,0), (-z,0,x), (0,-z,y).  Rows follow the local DOF order 3*node+c
    with nodes in the order given.  Not normalised here."""
    P = np.asarray(node_xyz, dtype=np.float64)
    nn = P.shape[0]
    R = np.zeros((3 * nn, 6))
    x, y, z = P[:, 0], P[:, 1], P[:, 2]
    R[0::3, 0] = 1; R[1::3, 1] = 1; R[2::3, 2] = 1
    R[0::3, 3] = -y; R[1::3, 3] = x
    R[0::3, 4] = -z; R[2::3, 4] = x
    R[1::3, 5] = -z; R[2::3, 5] = y
    return R


def null_pivots(R):
    """Matrix::getNullPivots (Matrix.cpp:835-884): full-pivot elimination on
    the dense column-major n x m matrix R; returns the m sorted row indices.
    ``max_element`` with ``fabs(a) <= fabs(b)`` keeps the LAST maximum in
    column-major order (Matrix.cpp:75-76, 852)."""
    R = np.asarray(R, dtype=np.float64)
    n, m = R.shape
    N = np.array(R, order="F", copy=True)
    piv = np.arange(n)
    for j in range(m):
        sub = N[:, : m - j].ravel(order="F")
        a = np.abs(sub)
        mx = a.max()
        I = int(np.flatnonzero(a == mx)[-1])
        col, row = divmod(I, n)
        last = n - 1 - j
        tmp = N[last, : m - j].copy()
        N[last, : m - j] = N[row, : m - j]
        N[row, : m - j] = tmp
        piv[row], piv[last] = piv[last], piv[row]
        if m - 1 - j != col:
            tmp = N[:, m - 1 - j].copy()
            N[:, m - 1 - j] = N[:, col]
            N[:, col] = tmp
        p = N[last, m - 1 - j]
        for J in range(m - j - 1):
            N[: n - j, J] = N[: n - j, J] - N[: n - j, m - 1 - j] * N[last, J] / p
    return np.sort(piv[n - 1 - np.arange(m)])


def bc_rank_full(A):
    """Matrix::test_of_Bc_constraints (Matrix.cpp:1538-1571): singular values
    of A A^T, a ratio below 1e-4 between consecutive ones means defect."""
    s = np.linalg.svd(A @ A.T, compute_uv=False)
    for i in range(len(s) - 1):
        if abs(s[i + 1] / s[i]) < 1e-4:
            return False
    return True


# ---------------------------------------------------------------------------
# problem container
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class MeshArrays:
    coords: np.ndarray          # (n_nodes, 3)
    elems: np.ndarray           # (n_elem, 8) global node ids, Mesh.cpp:250-257 order
    elem_sub: np.ndarray        # (n_elem,) subdomain of each element
    sub_cluster: np.ndarray     # (n_sub,) cluster of each subdomain
    sub_E: np.ndarray           # (n_sub,) Young's modulus per subdomain
    sub_nu: np.ndarray          # (n_sub,) Poisson ratio per subdomain
    dirichlet_dofs: np.ndarray  # fixed DOFs (3*node + c), reference order
    corner_dofs: np.ndarray     # DOFs eligible for corner (typeBc="cor") gluing
    body_force: np.ndarray      # (3,) rho*a per unit volume
    f_nodal: np.ndarray | None = None   # (3*n_nodes, n_rhs) extra nodal forces

    @property
    def n_sub(self):
        return int(len(self.sub_cluster))


@dataclasses.dataclass
class Options:
    typeBc: str = "cor"                     # "cor" | "ker"   (Cluster.cpp:737-747)
    preconditioner: str = "Dirichlet_explicit"  # | "Dirichlet_implicit" | "lumped" | "none"
    eps_iter: float = 1e-8
    max_iter: int = 500
    gradient: str = "standard"
    fix_rule: str = "reference"             # | "boundary"
    kerGc: str = "numerical"                # | "analytic"


class HTFETI:
    """Setup + PCPG of hybrid total FETI, generalised from the reference's
    single cluster (Cluster.cpp:21-385) to several clusters: Bf glues every
    interface, Bc glues subdomains of the same cluster only, each cluster has
    its own coarse matrix Ac, Gf has 6 columns per cluster."""

    def __init__(self, mesh: MeshArrays, opt: Options = Options(), fix_dofs=None):
        self.m = mesh
        self.opt = opt
        self._fix_override = fix_dofs
        self._assemble()
        self._dual_layout()
        self._kernels()
        self._cluster_constraints()
        self._local_operators()
        self._coarse()
        self._outer_coarse()

    # -- a2/a3 assembly (Data.cpp:25-54, 111-273) -------------------------
    def _assemble(self):
        m = self.m
        X = m.coords[m.elems]                               # (ne, 8, 3)
        Ee = m.sub_E[m.elem_sub]
        nue = m.sub_nu[m.elem_sub]
        Ke, fe = hex8_element(X, Ee, nue, m.body_force, self.opt.gradient)
        ieq = element_dofs(m.elems)
        ns = m.n_sub
        self.l2g, self.K, self.f = [], [], []
        iu, ju = np.triu_indices(24)
        nrhs = 1 if m.f_nodal is None else m.f_nodal.shape[1]
        owner = np.full(3 * len(m.coords), -1, dtype=np.int64)
        for d in range(ns):
            el = np.flatnonzero(m.elem_sub == d)
            l2g = np.unique(ieq[el])
            g2l = {int(g): i for i, g in enumerate(l2g)}
            n = len(l2g)
            U = np.zeros((n, n))
            f = np.zeros(n)
            loc = np.searchsorted(l2g, ieq[el])
            for k, e in enumerate(el):                     # Data.cpp:231-259
                li = loc[k]
                a, b = li[iu], li[ju]
                r, c = np.minimum(a, b), np.maximum(a, b)
                U[r, c] += Ke[e][iu, ju]
                np.add.at(f, li, fe[e])
            Kd = U + U.T - np.diag(np.diag(U))
            self.l2g.append(l2g)
            self.K.append(Kd)
            F = np.repeat(f[:, None], nrhs, axis=1)
            unowned = owner[l2g] < 0
            owner[l2g[unowned]] = d
            self.f.append(F)
        if m.f_nodal is not None:                        # nodal loads go to the lowest subdomain
            for d in range(ns):
                mine = owner[self.l2g[d]] == d
                self.f[d][mine] += m.f_nodal[self.l2g[d][mine]]
        self.nrhs = nrhs

    # -- a7 interfaces, Bf, weights (Cluster.cpp:682-769, 832-959) --------
    def _dual_layout(self):
        m = self.m
        ns = m.n_sub
        dof_all = np.concatenate(self.l2g)
        sub_all = np.concatenate([np.full(len(l), d) for d, l in enumerate(self.l2g)])
        order = np.lexsort((sub_all, dof_all))
        dof_s, sub_s = dof_all[order], sub_all[order]
        starts = np.flatnonzero(np.r_[True, dof_s[1:] != dof_s[:-1]])
        ends = np.r_[starts[1:], len(dof_s)]
        self.iface = [dict() for _ in range(ns)]    # data.interface[d]: dof -> sorted other subs
        for s0, e0 in zip(starts, ends):
            if e0 - s0 < 2:
                continue
            subs = sub_s[s0:e0]
            g = int(dof_s[s0])
            for d in subs:
                self.iface[int(d)][g] = [int(k) for k in subs if k != d]
        dirset = set(int(v) for v in m.dirichlet_dofs)
        rows = []        # each row: list of (sub, global dof, sign)
        weight = []
        for d in range(ns):                           # Cluster.cpp:846-903
            for g in sorted(self.iface[d]):
                if g in dirset:
                    continue
                neigh = self.iface[d][g]
                for k in neigh:
                    if k > d:
                        rows.append([(d, g, 1.0), (k, g, -1.0)])
                        weight.append(1.0 / (float(len(neigh)) + 1))
        for d in range(ns):                           # Cluster.cpp:906-924
            l2g = self.l2g[d]
            for g in m.dirichlet_dofs:
                g = int(g)
                i = np.searchsorted(l2g, g)
                if i < len(l2g) and l2g[i] == g:
                    rows.append([(d, g, 1.0)])
                    weight.append(1.0)
        self.bf_rows = rows
        self.n_lam = len(rows)
        self.weight = np.array(weight)
        # per-subdomain compressed Bf (Cluster.cpp:931-959)
        self.bf_l2g, self.bf_rowloc, self.bf_col, self.bf_val = [], [], [], []
        ent = [[] for _ in range(ns)]
        for r, row in enumerate(rows):
            for (d, g, s) in row:
                ent[d].append((r, int(np.searchsorted(self.l2g[d], g)), s))
        self.bset = []
        for d in range(ns):
            e = np.array(ent[d], dtype=np.float64).reshape(-1, 3)
            rr = e[:, 0].astype(np.int64)
            l2g_r = np.unique(rr)
            self.bf_l2g.append(l2g_r)
            self.bf_rowloc.append(np.searchsorted(l2g_r, rr))
            self.bf_col.append(e[:, 1].astype(np.int64))
            self.bf_val.append(e[:, 2])
            self.bset.append(np.unique(e[:, 1].astype(np.int64)))   # j_col_cmpr, Cluster.cpp:756-765

    # -- a4/a5 kernel and regularisation ----------------------------------
    def _kernels(self):
        m = self.m
        self.R, self.fix = [], []
        for d in range(m.n_sub):
            nodes = self.l2g[d][0::3] // 3
            R = gram_schmidt(rigid_body_modes(m.coords[nodes]))
            self.R.append(R)
            if self._fix_override is not None:
                fix = np.asarray(self._fix_override[d], dtype=np.int64)
            elif self.opt.fix_rule == "reference":
                fix = null_pivots(R)
            elif self.opt.fix_rule == "boundary":
                b = self.bset[d]
                fix = np.sort(b[null_pivots(R[b])])
            else:
                raise ValueError(self.opt.fix_rule)
            self.fix.append(fix)

    # -- a7 Bc per cluster (Cluster.cpp:772-821, 832-928) ------------------
    def _cluster_constraints(self):
        m = self.m
        ns = m.n_sub
        clusters = np.unique(m.sub_cluster)
        self.clusters = [np.flatnonzero(m.sub_cluster == c) for c in clusters]
        self.bc = [[] for _ in range(ns)]      # list of (row in cluster, local col, value)
        self.nlam_c = []
        corner = set(int(v) for v in m.corner_dofs)
        for subs in self.clusters:
            cnt = 0
            sset = set(int(s) for s in subs)
            if self.opt.typeBc == "cor":
                for d in subs:
                    d = int(d)
                    for g in sorted(self.iface[d]):
                        if g not in corner:
                            continue
                        for k in self.iface[d][g]:
                            if k > d and k in sset:
                                self.bc[d].append((cnt, int(np.searchsorted(self.l2g[d], g)), 1.0))
                                self.bc[k].append((cnt, int(np.searchsorted(self.l2g[k], g)), -1.0))
                                cnt += 1
                                break
            elif self.opt.typeBc == "ker":
                for ii, i in enumerate(subs):
                    i = int(i)
                    for j in subs[ii + 1:]:
                        j = int(j)
                        com = np.intersect1d(self.l2g[i], self.l2g[j])
                        if len(com) == 0:
                            continue
                        li = np.searchsorted(self.l2g[i], com)
                        lj = np.searchsorted(self.l2g[j], com)
                        A = self.R[i][li].T                 # 6 x ncom
                        if not bc_rank_full(A):
                            continue
                        for k in range(A.shape[0]):
                            for l in range(A.shape[1]):
                                self.bc[i].append((cnt, int(li[l]), A[k, l]))
                                self.bc[j].append((cnt, int(lj[l]), -A[k, l]))
                            cnt += 1
            else:
                raise ValueError(self.opt.typeBc)
            self.nlam_c.append(cnt)

    def _bc_dense(self, d):
        """Bc_d as a dense (c_d x n_d) matrix over its compressed rows plus
        the cluster row ids (l2g_i_coo)."""
        e = self.bc[d]
        rows = np.unique([r for r, _, _ in e]).astype(np.int64) if e else np.zeros(0, np.int64)
        B = np.zeros((len(rows), len(self.l2g[d])))
        for r, c, v in e:
            B[np.searchsorted(rows, r), c] += v
        return B, rows

    # -- a8/a9 local operators --------------------------------------------
    def _local_operators(self):
        ns = self.m.n_sub
        self.Kreg_cho, self.KplusBcT, self.Bc, self.bc_l2g = [], [], [], []
        self.Fc, self.Gc, self.S = [], [], []
        for d in range(ns):
            K = self.K[d]
            Kreg = K.copy()
            Kreg[self.fix[d], self.fix[d]] *= 2.0           # Matrix.cpp:1029-1057
            cho = sla.cho_factor(Kreg, lower=True)
            self.Kreg_cho.append(cho)
            B, rows = self._bc_dense(d)
            self.Bc.append(B); self.bc_l2g.append(rows)
            KpB = sla.cho_solve(cho, B.T) if B.shape[0] else np.zeros((K.shape[0], 0))
            self.KplusBcT.append(KpB)
            self.Fc.append(B @ KpB)
            self.Gc.append(-(B @ self.R[d]))
            b = self.bset[d]
            r = np.setdiff1d(np.arange(K.shape[0]), b)
            if self.opt.preconditioner in ("Dirichlet_explicit", "Dirichlet_implicit"):
                Krr = K[np.ix_(r, r)]
                Krs = K[np.ix_(r, b)]
                S = K[np.ix_(b, b)] - Krs.T @ sla.cho_solve(sla.cho_factor(Krr, lower=True), Krs)
                self.S.append(S)                              # Matrix.cpp:1708-1871
            else:
                self.S.append(None)

    def kplus_solve(self, d, x):
        return sla.cho_solve(self.Kreg_cho[d], x)

    def fhat(self, d):
        """(K_reg^{-1})_bb for subdomain d."""
        b = self.bset[d]
        n = self.K[d].shape[0]
        E = np.zeros((n, len(b)))
        E[b, np.arange(len(b))] = 1.0
        return self.kplus_solve(d, E)[b]

    # -- a10 cluster coarse problem (Cluster.cpp:215-324, 500-678) ---------
    def _coarse(self):
        self.H, self.Ac_lu, self.rbm_off = [], [], []
        self.ngc = []
        for ci, subs in enumerate(self.clusters):
            nc = self.nlam_c[ci]
            nsc = len(subs)
            Fc = np.zeros((nc, nc))
            Gc = np.zeros((nc, 6 * nsc))
            for k, d in enumerate(subs):
                rows = self.bc_l2g[d]
                Fc[np.ix_(rows, rows)] += self.Fc[d]
                Gc[rows, 6 * k:6 * k + 6] += self.Gc[d]
            GtG = Gc.T @ Gc
            if self.opt.kerGc == "numerical":
                w, V = np.linalg.eigh(GtG)
                tol = 1e-8 * max(w.max(), 1e-300)
                H = V[:, w < tol]
            else:
                H = self._analytic_kerGc(subs)
            if H.shape[1] != 6:
                raise RuntimeError(f"cluster {ci}: ker(GcTGc) has dimension {H.shape[1]}, expected 6")
            self.H.append(H)
            nr = 6 * nsc
            n = nc + nr + 6
            Ac = np.zeros((n, n))                         # Cluster.cpp:582-678 (extended form)
            Ac[:nc, :nc] = Fc
            Ac[:nc, nc:nc + nr] = Gc
            Ac[nc:nc + nr, :nc] = Gc.T
            Ac[nc:nc + nr, nc + nr:] = H
            Ac[nc + nr:, nc:nc + nr] = H.T
            self.Ac_lu.append(sla.lu_factor(Ac))
            self.ngc.append(n)

    def _analytic_kerGc(self, subs):
        """ker(Gc) spanned by the cluster's rigid modes written in the
        subdomain kernel bases: alpha_d = R_d^T r|_d (R_d orthonormal)."""
        cols = []
        for d in subs:
            nodes = self.l2g[d][0::3] // 3
            r = rigid_body_modes(self.m.coords[nodes])
            cols.append(self.R[d].T @ r)
        H = np.vstack(cols)
        Q, _ = np.linalg.qr(H)
        return Q

    # -- a11 outer coarse space (Cluster.cpp:1227-1273, 1332-1352) ---------
    def _outer_coarse(self):
        ns = self.m.n_sub
        nclu = len(self.clusters)
        self.Rf = [None] * ns
        self.Gf = np.zeros((self.n_lam, 6 * nclu))
        for ci, subs in enumerate(self.clusters):
            for k, d in enumerate(subs):
                Hd = self.H[ci][6 * k:6 * k + 6]
                self.Rf[d] = self.R[d] @ Hd
                Gd = self._bf_mult_rows(d, self.Rf[d])       # Bf_d Rf_d
                self.Gf[self.bf_l2g[d], 6 * ci:6 * ci + 6] += Gd
        self.GfTGf = self.Gf.T @ self.Gf
        L = np.linalg.cholesky(self.GfTGf)
        Li = sla.solve_triangular(L, np.eye(L.shape[0]), lower=True)
        self.invGfTGf = Li.T @ Li

    # -- Bf products (Cluster.cpp:1193-1224) --------------------------------
    def _bf_mult_rows(self, d, Y):
        out = np.zeros((len(self.bf_l2g[d]),) + Y.shape[1:])
        np.add.at(out, self.bf_rowloc[d], self.bf_val[d].reshape((-1,) + (1,) * (Y.ndim - 1)) * Y[self.bf_col[d]])
        return out

    def mult_Bf(self, xs):
        lam = np.zeros((self.n_lam,) + xs[0].shape[1:])
        for d in range(self.m.n_sub):
            lam[self.bf_l2g[d]] += self._bf_mult_rows(d, xs[d])
        return lam

    def mult_BfT(self, lam):
        xs = []
        for d in range(self.m.n_sub):
            x = np.zeros((len(self.l2g[d]),) + lam.shape[1:])
            loc = lam[self.bf_l2g[d]][self.bf_rowloc[d]]
            np.add.at(x, self.bf_col[d], self.bf_val[d].reshape((-1,) + (1,) * (lam.ndim - 1)) * loc)
            xs.append(x)
        return xs

    # -- a13 K_HT^+ (Cluster.cpp:967-1040) -----------------------------------
    def mult_Kplus(self, xs):
        out = [None] * self.m.n_sub
        for ci, subs in enumerate(self.clusters):
            nc = self.nlam_c[ci]
            gc = np.zeros((self.ngc[ci],) + xs[subs[0]].shape[1:])
            for k, d in enumerate(subs):
                gc[self.bc_l2g[d]] += self.KplusBcT[d].T @ xs[d]
                gc[nc + 6 * k:nc + 6 * k + 6] = -(self.R[d].T @ xs[d])
            sol = sla.lu_solve(self.Ac_lu[ci], gc)
            for k, d in enumerate(subs):
                lamc = sol[self.bc_l2g[d]]
                alpha = sol[nc + 6 * k:nc + 6 * k + 6]
                out[d] = self.kplus_solve(d, xs[d]) - self.KplusBcT[d] @ lamc + self.R[d] @ alpha
        return out

    # -- a12 F apply (Cluster.cpp:1114-1188) ---------------------------------
    def mult_F(self, w):
        return self.mult_Bf(self.mult_Kplus(self.mult_BfT(w)))

    # -- a14 preconditioner (Cluster.cpp:1043-1112, 1356-1360) ---------------
    def precondition(self, w):
        wt = w * self.weight.reshape((-1,) + (1,) * (w.ndim - 1))
        if self.opt.preconditioner == "none":
            return wt * self.weight.reshape((-1,) + (1,) * (w.ndim - 1))
        xs = self.mult_BfT(wt)
        ys = []
        for d in range(self.m.n_sub):
            if self.opt.preconditioner.startswith("Dirichlet"):
                b = self.bset[d]
                y = np.zeros_like(xs[d])
                y[b] = self.S[d] @ xs[d][b]
            else:                                      # lumped: K x
                y = self.K[d] @ xs[d]
            ys.append(y)
        z = self.mult_Bf(ys)
        return z * self.weight.reshape((-1,) + (1,) * (w.ndim - 1))

    # -- a15 projector (Cluster.cpp:1314-1329) -------------------------------
    def project(self, x):
        a = self.invGfTGf @ (self.Gf.T @ x)
        return x - self.Gf @ a, -a

    # -- a16 PCPG (Cluster.cpp:1363-1458) -------------------------------------
    def pcpg(self, rhs_index=0, eps_iter=None, max_iter=None):
        eps = self.opt.eps_iter if eps_iter is None else eps_iter
        maxit = self.opt.max_iter if max_iter is None else max_iter
        f = [fd[:, rhs_index] for fd in self.f]
        x = self.mult_Kplus(f)
        d_rhs = self.mult_Bf(x)
        e = np.zeros(self.Gf.shape[1])                  # mult_RfT, Cluster.cpp:1296-1312
        for ci, subs in enumerate(self.clusters):
            for d in subs:
                e[6 * ci:6 * ci + 6] += self.Rf[d].T @ f[d]
        lam = self.Gf @ (self.invGfTGf @ e)
        g = self.mult_F(lam) - d_rhs
        Pg, alpha = self.project(g)
        z = self.precondition(Pg)
        Pz, _ = self.project(z)
        gPz = float(g @ Pz)
        norm_gPz0 = np.sqrt(gPz)
        w = Pz
        hist = []
        it = 0
        for it in range(maxit):
            hist.append(np.sqrt(gPz) / norm_gPz0)
            if np.sqrt(gPz) < eps * norm_gPz0:
                break
            Fw = self.mult_F(w)
            wFw = float(w @ Fw)
            rho = -gPz / wFw
            lam = lam + rho * w
            g = g + rho * Fw
            Pg, alpha = self.project(g)
            z = self.precondition(Pg)
            Pz, _ = self.project(z)
            gPz_prev = gPz
            gPz = float(g @ Pz)
            gamma = gPz / gPz_prev
            w = Pz + gamma * w
        else:
            it = maxit
        # Cluster::printVTK (Cluster.cpp:1648-1678)
        bt = self.mult_BfT(lam)
        ys = [f[d] - bt[d] for d in range(self.m.n_sub)]
        xs = self.mult_Kplus(ys)
        u_loc = []
        for ci, subs in enumerate(self.clusters):
            for d in subs:
                xs[d] = xs[d] - self.Rf[d] @ alpha[6 * ci:6 * ci + 6]
        u_loc = xs
        u = np.zeros(3 * len(self.m.coords))
        for d in range(self.m.n_sub):                  # last writer wins
            u[self.l2g[d]] = u_loc[d]
        return dict(u=u, u_loc=u_loc, lam=lam, alpha=alpha, iterations=it,
                    hist=np.array(hist), norm_gPz0=norm_gPz0)

    # -- checks ---------------------------------------------------------------
    def primal_residual(self, sol, rhs_index=0):
        """max_d ||K_d u_d - f_d + Bf_d^T lam|| / ||f||."""
        bt = self.mult_BfT(sol["lam"])
        num = 0.0
        den = 0.0
        for d in range(self.m.n_sub):
            r = self.K[d] @ sol["u_loc"][d] - self.f[d][:, rhs_index] + bt[d]
            num += float(r @ r)
            den += float(self.f[d][:, rhs_index] @ self.f[d][:, rhs_index])
        return np.sqrt(num / den)


# ---------------------------------------------------------------------------
# memory-lean form for the large configurations
# ---------------------------------------------------------------------------
class HTFETIExplicit(HTFETI):
    """The same algorithm with the dual operator applied through the
    explicit local blocks F_i = (K_reg,i^{-1})_bb instead of a K_reg^{-1}
    solve per subdomain (the two are equal in exact arithmetic; the
    reference's mult_Ff, Cluster.cpp:1114-1188, only ever reads K_HT^+ w at
    the Bf columns).  K_i is kept sparse and no factor is kept: the two full
    K_reg^{-1} solves of a solve (start, Cluster.cpp:1385-1392, and the
    displacements, Cluster.cpp:1648-1678) refactor subdomain by subdomain.
    This keeps a 512-subdomain cube of 8^3 elements in about 10 GB of host
    memory, so the oracle solves the benchmark meshes at full size.

    ``pcpg_block`` runs Cluster::pcpg's recurrences (Cluster.cpp:1363-1458)
    for all load cases at once, one set of scalars per column; a column stops
    when it meets its tolerance, and the iteration at which it first met a
    looser one is recorded, so one run gives the reference's iteration count
    at eps_iter and a tightly converged displacement field."""

    def _assemble(self):
        import scipy.sparse as sp
        super()._assemble()
        self.K = [sp.csr_matrix(K) for K in self.K]

    def _assemble_one(self, d):
        return self.K[d].toarray()

    def _local_operators(self):
        ns = self.m.n_sub
        self.Fhat, self.KplusBcT, self.Bc, self.bc_l2g = [], [], [], []
        self.Fc, self.Gc, self.S, self.Rb, self.KpBb = [], [], [], [], []
        for d in range(ns):
            K = self._assemble_one(d)
            Kreg = K.copy()
            Kreg[self.fix[d], self.fix[d]] *= 2.0           # Matrix.cpp:1029-1057
            cho = sla.cho_factor(Kreg, lower=True)
            B, rows = self._bc_dense(d)
            self.Bc.append(B); self.bc_l2g.append(rows)
            KpB = sla.cho_solve(cho, B.T) if B.shape[0] else np.zeros((K.shape[0], 0))
            self.KplusBcT.append(KpB)
            self.Fc.append(B @ KpB)
            self.Gc.append(-(B @ self.R[d]))
            b = self.bset[d]
            E = np.zeros((K.shape[0], len(b)))
            E[b, np.arange(len(b))] = 1.0
            Fh = sla.cho_solve(cho, E)[b]
            self.Fhat.append(0.5 * (Fh + Fh.T))
            self.Rb.append(np.ascontiguousarray(self.R[d][b]))
            self.KpBb.append(np.ascontiguousarray(KpB[b]))
            r = np.setdiff1d(np.arange(K.shape[0]), b)
            if self.opt.preconditioner in ("Dirichlet_explicit", "Dirichlet_implicit"):
                Krr = K[np.ix_(r, r)]
                Krs = K[np.ix_(r, b)]
                self.S.append(K[np.ix_(b, b)] - Krs.T @ sla.cho_solve(sla.cho_factor(Krr, lower=True), Krs))
            else:
                self.S.append(None)
            del K, Kreg, cho, E

    def kplus_solve(self, d, x):
        K = self._assemble_one(d)
        K[self.fix[d], self.fix[d]] *= 2.0
        return sla.cho_solve(sla.cho_factor(K, lower=True, overwrite_a=True), x)

    def fhat(self, d):
        return self.Fhat[d]

    def _gather_b(self, lam):
        """x_b of every subdomain: Bf_i^T lam restricted to the Bf columns."""
        out = []
        for d in range(self.m.n_sub):
            b = self.bset[d]
            loc = lam[self.bf_l2g[d]][self.bf_rowloc[d]]
            xb = np.zeros((len(b),) + lam.shape[1:])
            np.add.at(xb, np.searchsorted(b, self.bf_col[d]),
                      self.bf_val[d].reshape((-1,) + (1,) * (lam.ndim - 1)) * loc)
            out.append(xb)
        return out

    def _scatter_b(self, ys, like):
        lam = np.zeros_like(like)
        for d in range(self.m.n_sub):
            b = self.bset[d]
            y = ys[d][np.searchsorted(b, self.bf_col[d])]
            contrib = np.zeros((len(self.bf_l2g[d]),) + like.shape[1:])
            np.add.at(contrib, self.bf_rowloc[d], self.bf_val[d].reshape((-1,) + (1,) * (like.ndim - 1)) * y)
            lam[self.bf_l2g[d]] += contrib
        return lam

    def mult_F(self, w):
        """Bf K_HT^+ Bf^T w with K_reg^{-1} read at the Bf columns only
        (Cluster.cpp:1114-1188: K_reg^{-1} x, the cluster coarse solve and
        the correction -KplusBcT lam_c + R alpha)."""
        xb = self._gather_b(w)
        ys = [None] * self.m.n_sub
        for ci, subs in enumerate(self.clusters):
            nc = self.nlam_c[ci]
            gc = np.zeros((self.ngc[ci],) + w.shape[1:])
            for k, d in enumerate(subs):
                gc[self.bc_l2g[d]] += self.KpBb[d].T @ xb[d]
                gc[nc + 6 * k:nc + 6 * k + 6] = -(self.Rb[d].T @ xb[d])
            sol = sla.lu_solve(self.Ac_lu[ci], gc)
            for k, d in enumerate(subs):
                ys[d] = (self.Fhat[d] @ xb[d] - self.KpBb[d] @ sol[self.bc_l2g[d]]
                         + self.Rb[d] @ sol[nc + 6 * k:nc + 6 * k + 6])
        return self._scatter_b(ys, w)

    def precondition(self, w):
        if self.opt.preconditioner in ("none", "lumped"):
            return super().precondition(w)
        wt = w * self.weight.reshape((-1,) + (1,) * (w.ndim - 1))
        xb = self._gather_b(wt)
        z = self._scatter_b([self.S[d] @ xb[d] for d in range(self.m.n_sub)], w)
        return z * self.weight.reshape((-1,) + (1,) * (w.ndim - 1))

    def pcpg_block(self, eps_record=1e-8, eps_stop=1e-11, max_iter=20000, progress=None):
        """Cluster::pcpg (Cluster.cpp:1363-1458) for every load case at once.
        Returns u (3 n_nodes x nrhs), the iteration at which each column first
        met eps_record, the iteration at which it met eps_stop, and the
        relative residual sqrt(g'Pz)/sqrt(g0'Pz0) per iteration and column
        (NaN once a column has stopped)."""
        nr = self.nrhs
        f = [fd for fd in self.f]                          # n_d x nrhs
        x = self.mult_Kplus(f)
        d_rhs = self.mult_Bf(x)
        e = np.zeros((self.Gf.shape[1], nr))
        for ci, subs in enumerate(self.clusters):
            for d in subs:
                e[6 * ci:6 * ci + 6] += self.Rf[d].T @ f[d]
        lam = self.Gf @ (self.invGfTGf @ e)
        g = self.mult_F(lam) - d_rhs
        Pg, alpha = self.project(g)
        z = self.precondition(Pg)
        Pz, _ = self.project(z)
        gPz = np.einsum("ij,ij->j", g, Pz)
        norm0 = np.sqrt(gPz)
        w = Pz.copy()
        it_rec = np.full(nr, -1)
        it_stop = np.full(nr, -1)
        alpha_stop = np.zeros((self.Gf.shape[1], nr))
        lam_stop = np.zeros_like(lam)
        active = np.ones(nr, bool)
        hist = []
        for it in range(max_iter + 1):
            rel = np.sqrt(np.maximum(gPz, 0.0)) / norm0
            hist.append(np.where(active, rel, np.nan))
            newly = active & (rel < eps_record) & (it_rec < 0)
            it_rec[newly] = it
            done = active & (rel < eps_stop)
            if it == max_iter:
                done = active.copy()
            it_stop[done] = it
            alpha_stop[:, done] = alpha[:, done]
            lam_stop[:, done] = lam[:, done]
            active &= ~done
            if progress is not None and it % 50 == 0:
                progress(it, rel, active)
            if not active.any():
                break
            Fw = self.mult_F(w)
            wFw = np.einsum("ij,ij->j", w, Fw)
            rho = np.where(active, -gPz / np.where(active, wFw, 1.0), 0.0)
            lam = lam + rho * w
            g = g + rho * Fw
            Pg, alpha = self.project(g)
            z = self.precondition(Pg)
            Pz, _ = self.project(z)
            gPz_prev = gPz
            gPz = np.einsum("ij,ij->j", g, Pz)
            gamma = np.where(active, gPz / np.where(active, gPz_prev, 1.0), 0.0)
            w = np.where(active, Pz + gamma * w, w)
        bt = self.mult_BfT(lam_stop)
        ys = [f[d] - bt[d] for d in range(self.m.n_sub)]
        xs = self.mult_Kplus(ys)
        for ci, subs in enumerate(self.clusters):
            for d in subs:
                xs[d] = xs[d] - self.Rf[d] @ alpha_stop[6 * ci:6 * ci + 6]
        u = np.zeros((3 * len(self.m.coords), nr))
        for d in range(self.m.n_sub):                      # last writer wins
            u[self.l2g[d]] = xs[d]
        return dict(u=u, it_record=it_rec, it_stop=it_stop, norm_gPz0=norm0, hist=np.array(hist))
