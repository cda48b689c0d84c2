"""hfls_b200 - B200-native HTFETI solve path with the reference's surface.

Python view of the C ABI in include/htfeti.h (ctypes over the in-tree
libhtfeti_b200.so).  There is no fallback: importing raises if the library is
missing, and GPU entry points return HTF_ENODEV errors without a device.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhtfeti_b200.so")
if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python hfls_b200/build.py`")
lib = ctypes.CDLL(LIB_PATH)

HTF_BC_ROLLERS, HTF_BC_CLAMP_X0 = 0, 1
HTF_MAT_CONST, HTF_MAT_CHECKER, HTF_MAT_LOGUNIFORM = 0, 1, 2
ERRORS = {0: "HTF_OK", -1: "HTF_EINVAL", -2: "HTF_ENOMEM", -3: "HTF_ECUDA", -4: "HTF_ENOTSPD",
          -5: "HTF_EBREAKDOWN", -6: "HTF_ENOCONV", -7: "HTF_ESTATE", -8: "HTF_ETIMEDOUT", -9: "HTF_ENODEV",
          -10: "HTF_EIO"}
for _c, _n in ERRORS.items():
    globals()[_n] = _c


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class MeshSpec(ctypes.Structure):
    _fields_ = [("clusters", ctypes.c_int * 3), ("subs", ctypes.c_int * 3), ("elems", ctypes.c_int * 3),
                ("widths", _ip * 3), ("jitter", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("bc", ctypes.c_int), ("material", ctypes.c_int), ("E", ctypes.c_double),
                ("E_hi", ctypes.c_double), ("nu", ctypes.c_double), ("body_force", ctypes.c_double * 3)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int * 64), ("norm_gPz0", ctypes.c_double * 64),
                ("final_rel", ctypes.c_double * 64), ("setup_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("fapply_ms", ctypes.c_double),
                ("fapply_bytes", ctypes.c_double), ("n_lambda", ctypes.c_int), ("n_sub", ctypes.c_int),
                ("n_clusters", ctypes.c_int), ("n_rhs", ctypes.c_int), ("status_sub", ctypes.c_int),
                ("kernel_launches", ctypes.c_longlong)]


class ProfileInfo(ctypes.Structure):
    _fields_ = [("symv_F_ms", ctypes.c_double), ("symv_F_bytes", ctypes.c_double),
                ("symv_S_ms", ctypes.c_double), ("symv_S_bytes", ctypes.c_double),
                ("fapply_ms", ctypes.c_double), ("fapply_bytes", ctypes.c_double),
                ("iteration_ms", ctypes.c_double), ("kernels_per_iteration", ctypes.c_int),
                ("batch_width", ctypes.c_int), ("tc_F_ms", ctypes.c_double), ("tc_F_bytes", ctypes.c_double),
                ("batch_iteration_ms", ctypes.c_double), ("kernels_per_batch_iteration", ctypes.c_int),
                ("setup_phase_ms", ctypes.c_double * 8), ("symv_unit_tiles", ctypes.c_int * 5),
                ("symv_tuned", ctypes.c_int), ("device_bytes", ctypes.c_double),
                ("kernel_detection_ms", ctypes.c_double), ("frontend_ms", ctypes.c_double)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("rc", ctypes.c_int), ("n_rhs", ctypes.c_int),
                ("iterations_max", ctypes.c_int), ("t_submit_ms", ctypes.c_double), ("t_admit_ms", ctypes.c_double),
                ("t_start_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double), ("setup_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("bytes", ctypes.c_double), ("bytes_estimate", ctypes.c_double)]


HTF_REQ_QUEUED, HTF_REQ_SETUP, HTF_REQ_RUNNING, HTF_REQ_DONE, HTF_REQ_FAILED = range(5)

_SIGS = {
    "htf_mesh_sizes": [ctypes.POINTER(MeshSpec)] + [_ip] * 6,
    "htf_mesh_fill": [ctypes.POINTER(MeshSpec), _dp, _ip, _ip, _ip, _dp, _dp, _ip, _ip],
    "htf_mesh_traction": [ctypes.POINTER(MeshSpec), ctypes.c_uint64, ctypes.c_int, ctypes.c_double, _dp],
    "htf_write_vtk": [ctypes.c_char_p, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip, _dp],
    "htf_create": [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)],
    "htf_destroy": [ctypes.c_void_p],
    "htf_set_mesh": [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, ctypes.c_int, _ip, _dp, _dp,
                     ctypes.c_int, _ip, ctypes.c_int, _ip, _dp],
    "htf_set_loads": [ctypes.c_void_p, ctypes.c_int, _dp],
    "htf_setup": [ctypes.c_void_p],
    "htf_pcpg": [ctypes.c_void_p, _dp, ctypes.POINTER(Stats)],
    "htf_solve": [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.POINTER(Stats)],
    "htf_profile": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ProfileInfo)],
    "htf_mult_Ff": [ctypes.c_void_p, _dp, _dp, ctypes.c_int],
    "htf_projection": [ctypes.c_void_p, _dp, _dp, ctypes.c_int],
    "htf_preconditioning": [ctypes.c_void_p, _dp, _dp, ctypes.c_int],
    "htf_dual_sizes": [ctypes.c_void_p, _ip, _ip, _ip],
    "htf_dual_layout": [ctypes.c_void_p, _ip, _ip, _dp, _dp],
    "htf_fix_dofs": [ctypes.c_void_p, _ip],
    "htf_dump": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int],
    "htf_residual_history": [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int],
    "htf_projection_noalloc": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "htf_server_create": [ctypes.c_char_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "htf_server_destroy": [ctypes.c_void_p],
    "htf_server_submit": [ctypes.c_void_p, ctypes.POINTER(MeshSpec), ctypes.c_int, _dp, _dp,
                          ctypes.POINTER(ctypes.c_longlong)],
    "htf_server_wait": [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.POINTER(RequestInfo)],
    "htf_server_info": [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(RequestInfo)],
}
HTF_NOALLOC_SCRATCH_DOUBLES = 1048576
for _name, _args in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = ctypes.c_int
lib.htf_status_sub.argtypes = [ctypes.c_void_p]
lib.htf_status_sub.restype = ctypes.c_int
lib.htf_last_error.argtypes = [ctypes.c_void_p]
lib.htf_last_error.restype = ctypes.c_char_p
lib.htf_server_error.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
lib.htf_server_error.restype = ctypes.c_char_p


class HTFError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class Mesh:
    """Arrays of one mesh (the reference's Mesh public fields, Mesh.hpp:72-84)."""

    def __init__(self, coords, elems, elem_sub, sub_cluster, sub_E, sub_nu, dirichlet, corner, body_force):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        self.elems = np.ascontiguousarray(elems, dtype=np.int32).reshape(-1, 8)
        self.elem_sub = np.ascontiguousarray(elem_sub, dtype=np.int32)
        self.sub_cluster = np.ascontiguousarray(sub_cluster, dtype=np.int32)
        self.sub_E = np.ascontiguousarray(sub_E, dtype=np.float64)
        self.sub_nu = np.ascontiguousarray(sub_nu, dtype=np.float64)
        self.dirichlet = np.ascontiguousarray(dirichlet, dtype=np.int32)
        self.corner = np.ascontiguousarray(corner, dtype=np.int32)
        self.body_force = np.ascontiguousarray(body_force, dtype=np.float64)

    @property
    def n_nodes(self):
        return len(self.coords)

    @property
    def n_sub(self):
        return len(self.sub_cluster)


def mesh_spec(clusters=(1, 1, 1), subs=(2, 2, 2), elems=(5, 5, 5), widths=None, jitter=0.0, seed=0,
              bc=HTF_BC_CLAMP_X0, material=HTF_MAT_CONST, E=2.1e5, E_hi=1.0, nu=0.3, body_force=(0, 0, -1)):
    s = MeshSpec()
    for a in range(3):
        s.clusters[a], s.subs[a], s.elems[a] = clusters[a], subs[a], elems[a]
    keep = []
    if widths is not None:
        for a in range(3):
            w = np.ascontiguousarray(widths[a], dtype=np.int32)
            keep.append(w)
            s.widths[a] = _i(w)
    s._keep = keep
    s.jitter, s.seed, s.bc, s.material = jitter, seed, bc, material
    s.E, s.E_hi, s.nu = E, E_hi, nu
    for a in range(3):
        s.body_force[a] = body_force[a]
    return s


def generate_mesh(spec):
    """Mesh::createMesh generalised (htf_mesh_sizes + htf_mesh_fill)."""
    n = [ctypes.c_int() for _ in range(6)]
    rc = lib.htf_mesh_sizes(ctypes.byref(spec), *[ctypes.byref(v) for v in n])
    if rc:
        raise HTFError(rc, "htf_mesh_sizes")
    nn, ne, ns, nc, nd, ncr = [v.value for v in n]
    coords = np.zeros((nn, 3)); elems = np.zeros((ne, 8), np.int32); es = np.zeros(ne, np.int32)
    scl = np.zeros(ns, np.int32); sE = np.zeros(ns); snu = np.zeros(ns)
    dirs = np.zeros(nd, np.int32); corner = np.zeros(ncr, np.int32)
    rc = lib.htf_mesh_fill(ctypes.byref(spec), _d(coords), _i(elems), _i(es), _i(scl), _d(sE), _d(snu),
                           _i(dirs), _i(corner))
    if rc:
        raise HTFError(rc, "htf_mesh_fill")
    return Mesh(coords, elems, es, scl, sE, snu, dirs, corner, np.array(spec.body_force[:]))


def traction(spec, seed, n_rhs, scale=1.0):
    """Seeded N(0,1) nodal forces on x=1, shape (n_rhs, 3*n_nodes)."""
    n = [ctypes.c_int() for _ in range(6)]
    lib.htf_mesh_sizes(ctypes.byref(spec), *[ctypes.byref(v) for v in n])
    f = np.zeros((n_rhs, 3 * n[0].value))
    rc = lib.htf_mesh_traction(ctypes.byref(spec), seed, n_rhs, scale, _d(f))
    if rc:
        raise HTFError(rc, "htf_mesh_traction")
    return f


def write_vtk(path, mesh, u, material=None):
    """Mesh::SaveVTK (Mesh.cpp:292-351): the displacement field u (one load
    case, 3*n_nodes) written as the reference's box.vtk.  material: one id
    per element; None applies the reference's rule, remainder(subdomain, 2)."""
    u = np.ascontiguousarray(u, dtype=np.float64).ravel()
    if u.size != 3 * mesh.n_nodes:
        raise HTFError(-1, f"htf_write_vtk: u has {u.size} values, expected {3 * mesh.n_nodes}")
    mat = None if material is None else np.ascontiguousarray(material, dtype=np.int32)
    if mat is not None and mat.size != len(mesh.elem_sub):
        raise HTFError(-1, "htf_write_vtk: one material id per element expected")
    rc = lib.htf_write_vtk(os.fsencode(path), mesh.n_nodes, _d(mesh.coords), len(mesh.elem_sub), _i(mesh.elems),
                           _i(mesh.elem_sub), None if mat is None else _i(mat), _d(u))
    if rc:
        raise HTFError(rc, f"htf_write_vtk({path})")


class Solver:
    """One HTFETI problem: Driver/Cluster surface over the C ABI.

    options: dict with the reference's keys (eps_iter, max_iter,
    preconditioner, typeBc, ...) plus precision=fp64|mixed.
    """

    def __init__(self, options=None):
        opts = ";".join(f"{k}={v}" for k, v in (options or {}).items())
        h = ctypes.c_void_p()
        rc = lib.htf_create(opts.encode(), ctypes.byref(h))
        if rc:
            raise HTFError(rc, f"htf_create({opts})")
        self._h = h
        self.mesh = None

    def _check(self, rc, what):
        if rc:
            raise HTFError(rc, f"{what}: {lib.htf_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            lib.htf_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_mesh(self, m):
        self.mesh = m
        self._check(lib.htf_set_mesh(self._h, m.n_nodes, _d(m.coords), len(m.elems), _i(m.elems), _i(m.elem_sub),
                                     m.n_sub, _i(m.sub_cluster), _d(m.sub_E), _d(m.sub_nu), len(m.dirichlet),
                                     _i(m.dirichlet), len(m.corner), _i(m.corner), _d(m.body_force)),
                    "htf_set_mesh")

    def status_sub(self):
        """Subdomain of the last HTF_ENOTSPD set-up failure, or -1."""
        return lib.htf_status_sub(self._h)

    def set_loads(self, f_nodal):
        f = np.ascontiguousarray(np.atleast_2d(f_nodal), dtype=np.float64)
        self.nrhs = f.shape[0]
        self._check(lib.htf_set_loads(self._h, f.shape[0], _d(f)), "htf_set_loads")

    def setup(self):
        self._check(lib.htf_setup(self._h), "htf_setup")

    def pcpg(self):
        nrhs = getattr(self, "nrhs", 1)
        u = np.zeros((nrhs, 3 * self.mesh.n_nodes))
        st = Stats()
        self._check(lib.htf_pcpg(self._h, _d(u), ctypes.byref(st)), "htf_pcpg")
        return u, st

    def solve(self, f_nodal=None, u=None, nrhs=None):
        """New load cases against the resident factors (htf_solve).  f_nodal
        (n_rhs, 3*n_nodes) is added to the body force; None = body force only."""
        if f_nodal is None:
            nrhs = nrhs or 1
            fp = None
        else:
            f_nodal = np.ascontiguousarray(np.atleast_2d(f_nodal), dtype=np.float64)
            nrhs = f_nodal.shape[0]
            fp = _d(f_nodal)
        if u is None:
            u = np.zeros((nrhs, 3 * self.mesh.n_nodes))
        st = Stats()
        self._check(lib.htf_solve(self._h, nrhs, fp, _d(u), ctypes.byref(st)), "htf_solve")
        return u, st

    def profile(self, reps=20):
        info = ProfileInfo()
        self._check(lib.htf_profile(self._h, reps, ctypes.byref(info)), "htf_profile")
        return info

    def n_lambda(self):
        n = ctypes.c_int()
        self._check(lib.htf_dual_sizes(self._h, ctypes.byref(n), None, None), "htf_dual_sizes")
        return n.value

    def dual_layout(self):
        nl = self.n_lambda()
        rs = np.zeros(2 * nl, np.int32); rd = np.zeros(2 * nl, np.int32)
        sg = np.zeros(2 * nl); w = np.zeros(nl)
        self._check(lib.htf_dual_layout(self._h, _i(rs), _i(rd), _d(sg), _d(w)), "htf_dual_layout")
        return rs.reshape(-1, 2), rd.reshape(-1, 2), sg.reshape(-1, 2), w

    def residual_history(self, rhs=0):
        """Relative residual per PCPG iteration of load case rhs of the last plain solve."""
        n = lib.htf_residual_history(self._h, rhs, None, 0)
        if n < 0:
            self._check(n, "htf_residual_history")
        h = np.zeros(n)
        self._check(min(0, lib.htf_residual_history(self._h, rhs, _d(h), n)), "htf_residual_history")
        return h

    def dump(self, folder, level):
        """MatrixMarket files of the problem (htf_dump) in folder."""
        self._check(lib.htf_dump(self._h, os.fsencode(folder), int(level)), "htf_dump")

    def fix_dofs(self):
        ns = self.mesh.n_sub
        out = np.zeros(6 * ns, np.int32)
        self._check(lib.htf_fix_dofs(self._h, _i(out)), "htf_fix_dofs")
        return out.reshape(ns, 6)

    def _op(self, fn, x, name):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        y = np.zeros_like(x)
        self._check(fn(self._h, _d(x), _d(y), x.shape[0]), name)
        return y

    def projection_noalloc(self, x_dev_ptr, px_dev_ptr, stream_ptr=0):
        """htf_projection_noalloc on device pointers (ints); enqueued on the
        given CUDA stream, returns without waiting."""
        self._check(lib.htf_projection_noalloc(self._h, ctypes.c_void_p(x_dev_ptr), ctypes.c_void_p(px_dev_ptr),
                                               ctypes.c_void_p(stream_ptr)), "htf_projection_noalloc")

    def mult_Ff(self, w):
        return self._op(lib.htf_mult_Ff, w, "htf_mult_Ff")

    def projection(self, x):
        return self._op(lib.htf_projection, x, "htf_projection")

    def preconditioning(self, x):
        return self._op(lib.htf_preconditioning, x, "htf_preconditioning")


class Server:
    """Continuous-batching solve server (htf_server_*): requests of different
    meshes and load cases are admitted by device footprint and advance
    together in the batched mixed-precision form.

    submit() copies the loads and returns a ticket; the displacements land in
    an array owned by this object, returned by wait(ticket)."""

    def __init__(self, options=None, hbm_budget_bytes=0.0, max_live=8):
        opts = ";".join(f"{k}={v}" for k, v in (options or {}).items())
        h = ctypes.c_void_p()
        rc = lib.htf_server_create(opts.encode(), float(hbm_budget_bytes), int(max_live), ctypes.byref(h))
        if rc:
            raise HTFError(rc, "htf_server_create")
        self._h = h
        self._out = {}

    def submit(self, spec, f_nodal=None, n_rhs=None):
        if f_nodal is not None:
            f = np.ascontiguousarray(np.atleast_2d(f_nodal), dtype=np.float64)
            n_rhs = f.shape[0]
        else:
            f, n_rhs = None, n_rhs or 1
        n = [ctypes.c_int() for _ in range(6)]
        lib.htf_mesh_sizes(ctypes.byref(spec), *[ctypes.byref(v) for v in n])
        u = np.zeros((n_rhs, 3 * n[0].value))
        t = ctypes.c_longlong()
        rc = lib.htf_server_submit(self._h, ctypes.byref(spec), n_rhs, _d(f) if f is not None else None, _d(u),
                                   ctypes.byref(t))
        if rc:
            raise HTFError(rc, "htf_server_submit: " + lib.htf_server_error(self._h, 0).decode())
        self._out[t.value] = (u, spec)          # keep u (written by the server) and the spec alive
        return t.value

    def info(self, ticket):
        i = RequestInfo()
        rc = lib.htf_server_info(self._h, ticket, ctypes.byref(i))
        if rc:
            raise HTFError(rc, "htf_server_info")
        return i

    def wait(self, ticket, timeout_ms=-1.0):
        """Displacements (n_rhs, 3*n_nodes) and the RequestInfo; raises on a failed request."""
        i = RequestInfo()
        rc = lib.htf_server_wait(self._h, ticket, float(timeout_ms), ctypes.byref(i))
        if rc:
            raise HTFError(rc, "request %d: %s" % (ticket, lib.htf_server_error(self._h, ticket).decode()))
        return self._out[ticket][0], i

    def close(self):
        """Lets every submitted request finish, then stops the server."""
        if getattr(self, "_h", None):
            lib.htf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
