"""Generate the golden fixtures that pin the oracle to the reference.

Builds the reference from its sources (oracle/ref_build/Makefile ->
oracle/_ref/hfls_ref), runs it on the cases below and stores, per case, the
reference's mesh, dual layout (Bf, weights), projected-operator probes,
element matrices, iteration count and displacement field (read from the
box.vtk the reference writes) in tests/golden/<case>.npz, and one case's box.vtk
verbatim (tests/golden/<case>_box.vtk).

Young's modulus is scaled to ~1e-3 so the displacements printed with "%f"
by Mesh::SaveVTK (Mesh.cpp:346-349) keep about 12 significant digits; the
problem is linear in 1/E, so the oracle is run with the same modulus.

Run from the repository root:  python tests/golden/make_goldens.py
"""
import os
import re
import subprocess
import sys
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "hfls_ref")
OUTDIR = os.path.join(ROOT, "tests", "golden")

CASES = {
    # name: harness arguments
    "ref_ker_dirichlet_3": dict(nx=3, ny=3, nz=3, typeBc="ker", preconditioner="Dirichlet_explicit",
                                young_modulus="1e-3", ratio_mat="1"),
    "ref_cor_lumped_contrast_3": dict(nx=3, ny=3, nz=3, typeBc="cor", preconditioner="lumped",
                                      young_modulus="1e-3", ratio_mat="100"),
    "ref_cor_dirichlet_clamp_5": dict(nx=5, ny=5, nz=5, typeBc="cor", preconditioner="Dirichlet_explicit",
                                      young_modulus="2.1e-3", ratio_mat="1", clamp="true"),
    "ref_ker_implicit_3x2x1_4": dict(Nx=3, Ny=2, Nz=1, nx=4, ny=4, nz=4, typeBc="ker",
                                     preconditioner="Dirichlet_implicit", young_modulus="1e-3",
                                     ratio_mat="10"),
}


def read_blocks(path):
    out = {}
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    while i < len(lines):
        ln = lines[i].strip()
        i += 1
        if not ln:
            continue
        name, *rest = ln.split()
        if len(rest) != 1:
            continue
        if name in ("nsub", "nlam", "nlam_c"):
            out[name] = int(rest[0])
            continue
        n = int(rest[0])
        vals = lines[i:i + n]
        i += n
        arr = np.array([float(v) for v in vals]) if n else np.zeros(0)
        out.setdefault(name, []).append(arr)
    return out


def read_vtk_displacements(path, npoints):
    with open(path) as f:
        txt = f.read().split("\n")
    k = next(i for i, l in enumerate(txt) if l.startswith("LOOKUP_TABLE my_table"))
    rows = [list(map(float, l.split())) for l in txt[k + 1:k + 1 + npoints]]
    return np.array(rows).ravel()


def run_tight(name, args):
    """Second run at eps_iter=1e-10: its u pins the displacement field."""
    work = os.path.join(ROOT, "oracle", "_ref", "runs", name + "_tight")
    os.makedirs(work, exist_ok=True)
    a = dict(args, eps_iter="1e-10", max_iter="1000")
    argv = [REF_BIN, f"out={work}"] + [f"{k}={v}" for k, v in a.items()]
    p = subprocess.run(argv, capture_output=True, text=True, check=True)
    its = [int(m.group(1)) for m in re.finditer(r"^\s*(\d+)\t([0-9.e+-]+)\s*$", p.stdout, re.M)]
    npts = len(read_blocks(os.path.join(work, "mesh.txt"))["points"][0]) // 3
    return read_vtk_displacements(os.path.join(work, "box.vtk"), npts), its[-1] - 1


def run_case(name, args):
    work = os.path.join(ROOT, "oracle", "_ref", "runs", name)
    os.makedirs(work, exist_ok=True)
    argv = [REF_BIN, f"out={work}"] + [f"{k}={v}" for k, v in args.items()]
    p = subprocess.run(argv, capture_output=True, text=True, check=True)
    log = p.stdout
    its = [int(m.group(1)) for m in re.finditer(r"^\s*(\d+)\t([0-9.e+-]+)\s*$", log, re.M)]
    hist = [float(m.group(2)) for m in re.finditer(r"^\s*(\d+)\t([0-9.e+-]+)\s*$", log, re.M)]
    mesh = read_blocks(os.path.join(work, "mesh.txt"))
    lay = read_blocks(os.path.join(work, "layout.txt"))
    probe = read_blocks(os.path.join(work, "probe.txt"))
    elem = read_blocks(os.path.join(work, "elem.txt"))
    pts = mesh["points"][0].reshape(-1, 3)
    u = read_vtk_displacements(os.path.join(work, "box.vtk"), len(pts))
    nsub = len(lay["l2g"])
    rec = dict(
        args=np.array(repr(args)),
        points=pts,
        elements=mesh["elements"][0].astype(np.int64).reshape(-1, 8),
        partition=mesh["partition"][0].astype(np.int64),
        material=mesh["material"][0].astype(np.int64),
        dirichlet=mesh["dirichlet"][0].astype(np.int64),
        corner=mesh["corner"][0].astype(np.int64),
        weight=lay["weight"][0],
        w=probe["w"][0], Pw=probe["Pw"][0], PFPw=probe["PFPw"][0], PMPw=probe["PMPw"][0],
        elem_coords=np.stack([c.reshape(8, 3) for c in elem["coords"]]),
        elem_K=np.stack([k.reshape(24, 24).T for k in elem["Ke_colmajor"]]),
        elem_f=np.stack(elem["fe"]),
        iterations=np.array(its[-1] - 1),      # printed index is it+1 at the stopping check
        hist=np.array(hist),
        u=u,
    )
    for d in range(nsub):
        rec[f"l2g_{d}"] = lay["l2g"][d].astype(np.int64)
        rec[f"bf_rows_{d}"] = lay["bf_rows"][d].astype(np.int64)
        rec[f"bf_iptr_{d}"] = lay["bf_iptr"][d].astype(np.int64)
        rec[f"bf_jcol_{d}"] = lay["bf_jcol"][d].astype(np.int64)
        rec[f"bf_val_{d}"] = lay["bf_val"][d]
    rec["nsub"] = np.array(nsub)
    rec["u_tight"], it_tight = run_tight(name, args)
    rec["iterations_tight"] = np.array(it_tight)
    np.savez_compressed(os.path.join(OUTDIR, name + ".npz"), **rec)
    print(f"{name}: nsub={nsub} iterations={its[-1] - 1} nlam={len(rec['weight'])}")


VTK_CASE = "ref_ker_dirichlet_3"


def write_vtk_fixture():
    """The reference's own box.vtk (Mesh::SaveVTK) of VTK_CASE, kept verbatim
    as tests/golden/<case>_box.vtk: the byte-for-byte target of htf_write_vtk."""
    work = os.path.join(ROOT, "oracle", "_ref", "runs", VTK_CASE + "_vtk")
    os.makedirs(work, exist_ok=True)
    argv = [REF_BIN, f"out={work}"] + [f"{k}={v}" for k, v in CASES[VTK_CASE].items()]
    subprocess.run(argv, capture_output=True, text=True, check=True)
    with open(os.path.join(work, "box.vtk"), "rb") as f:
        data = f.read()
    with open(os.path.join(OUTDIR, VTK_CASE + "_box.vtk"), "wb") as f:
        f.write(data)
    print(f"{VTK_CASE}_box.vtk: {len(data)} bytes")


def main():
    if not os.path.exists(REF_BIN):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle", "ref_build"),
                        "REF=" + os.environ.get("HFLS_REFERENCE", "/root/reference")], check=True)
    for name, args in CASES.items():
        run_case(name, args)
    write_vtk_fixture()


if __name__ == "__main__":
    sys.exit(main())
