"""HTFETI solve benchmark.

Headline workload (one step = one PCPG solve, g0 -> convergence at 1e-8, with
the factors and F_i / S_i resident on the device), the largest configuration
that fits one GPU:
  the uneven cube: 16 subdomain slabs per axis whose element counts are drawn
  from {4..12} (seed 0), grouped into 2x2x2 clusters of 8x8x8 subdomains
  (4096 subdomains of 375-6591 DOFs, 5.47 M DOFs), interior nodes jittered by
  U(-0.1h, 0.1h), E_i log-uniform in [1, 1e4] per subdomain, nu 0.3, u = 0 on
  x = 0, body force (0, 0, -1), corner gluing inside clusters, Dirichlet
  preconditioner, F_i / S_i dense FP64 (packed triangular tiles).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Beside it in the same JSON line:
  cube512   the regular cube (2x2x2 clusters x 4x4x4 subdomains x 8^3 hex8,
            E logU[1e3, 1e6], N(0,1) traction on x = 1) in FP64, with its
            iteration count against the oracle golden;
  mixed     the same cube with body force and 32 seeded traction load cases
            solved as one batch in mixed precision (F_i / S_i FP32 on the
            tensor cores, FP64 residual replacement), the displacement error
            of every load case against the oracle golden;
  serving   a prefix of the seeded serving stream through htf_server against
            the plain FP64 per-request path;
  cpu_baseline  the reference (oracle/_ref/hfls_ref, built from the reference
            sources, one core) solving its own CPU configuration in full -
            2x2x2 subdomains x 5^3 hex8 - with the GPU's time on the same
            configuration beside it.

Under torchrun (N > 1) every rank solves its own replica on its own GPU (the
solve has no cross-GPU exchange here), timing is the max over ranks.
--impl reference reports that the reference cannot solve the headline
workload (it has one cluster) and times it on its own configuration instead.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "HTFETI solve s & F-apply GB/s at 1e-8 rel res; mixed vs FP64 GPU; p99 latency"
OPTS = {"typeBc": "cor", "preconditioner": "Dirichlet_explicit", "eps_iter": "1e-8", "max_iter": "5000"}

UNEVEN_WORKLOAD = ("HTFETI uneven cube: 16 slabs/axis of {4..12} hex8 (seed 0), 2x2x2 clusters x 8x8x8 subdomains "
                   "(4096 subdomains, 375-6591 DOFs each), jitter 0.1h, E logU[1,1e4], nu 0.3, clamp x=0, body force "
                   "(0,0,-1), corner Bc, Dirichlet preconditioner, F_i/S_i dense FP64, eps 1e-8")
CUBE_WORKLOAD = ("HTFETI cube: 2x2x2 clusters x 4x4x4 subdomains x 8^3 hex8 (512 subdomains, 823875 DOFs), "
                 "jitter 0.1h, E logU[1e3,1e6], nu 0.3, clamp x=0, N(0,1) traction x=1, corner Bc, "
                 "Dirichlet preconditioner, F_i dense FP64, eps 1e-8")
CUBE = dict(clusters=(2, 2, 2), subs=(4, 4, 4), elems=(8, 8, 8), jitter=0.1, seed=1,
            E=1e3, E_hi=1e6, nu=0.3, body_force=(0.0, 0.0, 0.0))
SMALL_WORKLOAD = ("the reference's CPU configuration: 2x2x2 subdomains x 5^3 hex8 on the unit cube (one cluster), "
                  "E 2.1e5, nu 0.3, u = 0 on x = 0, body force, interior nodes jittered by 0.1h, "
                  "Bc of kernel type, Dirichlet preconditioner, eps 1e-8")
MIXED_RHS = 32
MIXED_WORKLOAD = ("cube512 mesh, body force (0,0,-1) + 32 seeded N(0,1) tractions on x=1, solved as one batch of 32: "
                  "F_i/S_i as scaled FP16 hi+lo slabs, tcgen05 kind::f16 products (A_hi X_hi + A_hi X_lo + A_lo X_hi), "
                  "FP64 coarse/projector/residual replacement, eps 1e-8")
SERVE_REQUESTS = 12          # requests of the seeded stream that one bench run serves
SERVE_RATE = 1.0             # Poisson arrivals per second
SERVE_WORKLOAD = ("seeded Poisson stream (rate %.1f/s): cube meshes of c^3 clusters, (c s)^3 subdomains of e^3 hex8, "
                  "c in 1..4, s in 2..5, e in 4..10, 1..16 load cases (body force + N(0,1) traction on x=1), "
                  "E logU[1,1e4] per subdomain, nu U[0.2,0.4] per request, clamp x=0, jitter 0.1h, eps 1e-8; "
                  "served by htf_server (mixed precision, batch 16) vs the plain FP64 per-request path "
                  "(set up and solve one request after another, FIFO on the same arrivals)" % SERVE_RATE)
PROFILE_UNEVEN = os.path.join(ROOT, "profiles", "k_symv_fp64_uneven.md")
PROFILE_CUBE = os.path.join(ROOT, "profiles", "k_symv_fp64_cfg1.md")


def uneven_widths(n=16, seed=0, lo=4, hi=12):
    rng = np.random.default_rng(seed)
    return [rng.integers(lo, hi + 1, n).astype(np.int32) for _ in range(3)]


def uneven_spec(hb, clusters=(2, 2, 2), subs=(8, 8, 8), widths=None):
    w = widths if widths is not None else uneven_widths(clusters[0] * subs[0])
    return hb.mesh_spec(clusters=clusters, subs=subs, widths=w, jitter=0.1, seed=0,
                        material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, nu=0.3, bc=hb.HTF_BC_CLAMP_X0,
                        body_force=(0.0, 0.0, -1.0))


# reduced meshes of the same constructions, for ncu captures only
REDUCED = {"uneven-small": dict(clusters=(1, 1, 1), subs=(4, 4, 4)),     # 64 subdomains: FP64 tiles ~0.3 GB > L2
           "small": dict(clusters=(1, 1, 1), subs=(2, 4, 4)),            # cube: F_i tiles 120 MB
           "mid": dict(clusters=(2, 1, 1), subs=(2, 4, 4))}              # cube: F_i tiles 240 MB


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU under torchrun (RANK / WORLD_SIZE / LOCAL_RANK from
    the environment); every rank solves its own replica of the workload, and
    the process group only carries the barriers and the max over ranks."""
    if n_gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, 0, None
    import datetime
    import torch
    import torch.distributed as dist
    rank, world, local = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"]), int(os.environ["LOCAL_RANK"])
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, world, local, dist


def max_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_seconds_per_solve(max_ms_per_solve, world):
    """World replicas each finish one solve per step within the slowest
    rank's time: the job's seconds per solve."""
    return max_ms_per_solve / 1e3 / world


def barrier(dist):
    if dist is not None:
        dist.barrier()


def traffic_from_profile(path, key="traffic_bytes_per_launch_scaled"):
    if not os.path.exists(path):
        return None
    m = re.search(r"^%s:\s*([0-9.eE+]+)" % key, open(path).read(), re.M)
    return float(m.group(1)) if m else None


# ---------------------------------------------------------------------------
# reference CPU solver on its own configuration
# ---------------------------------------------------------------------------
REF_SMALL = dict(Nx=2, Ny=2, Nz=2, nx=5, ny=5, nz=5, young_modulus="2.1e5", poissons_ratio="0.3", clamp="true",
                 jitter_seed=1, typeBc="ker", preconditioner="Dirichlet_explicit", eps_iter="1e-8", max_iter=500)


def ref_binary():
    return os.path.join(ROOT, "oracle", "_ref", "hfls_ref")


def ref_run_small():
    """One run of the reference on REF_SMALL: its own timed intervals (wall
    seconds of Cluster::initialization's setup and Cluster::pcpg,
    Cluster.cpp:24-379, 1364-1451), the process wall time and the PCPG
    iteration count it prints."""
    with tempfile.TemporaryDirectory() as td:
        args = [ref_binary(), f"out={td}", "dumps=false"] + [f"{k}={v}" for k, v in REF_SMALL.items()]
        t0 = time.perf_counter()
        r = subprocess.run(args, capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS="1",
                                                                           OPENBLAS_NUM_THREADS="1"))
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError("reference run failed: " + r.stderr[-400:])
        t = {}
        for ln in open(os.path.join(td, "timing.txt")):
            k, v = ln.split()
            t[k] = float(v)
    its = [int(m.group(1)) for m in re.finditer(r"^\s*(\d+)\s+[0-9.eE+-]+\s*$", r.stdout, re.M)]
    return dict(setup_s=t["setup_s"], pcpg_s=t["pcpg_s"], total_s=t["total_s"], wall_s=wall,
                iterations=max(its) if its else None)


def ref_small_measure(steps, warmup):
    for _ in range(warmup):
        ref_run_small()
    runs = [ref_run_small() for _ in range(steps)]
    return {k: statistics.mean(r[k] for r in runs) for k in ("setup_s", "pcpg_s", "total_s", "wall_s")} | \
        {"iterations": runs[-1]["iterations"], "runs": len(runs)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    why = ("the reference solves one cluster only (one Cluster object, Driver.cpp:29; Mesh::createMesh builds one "
           "cluster) and cannot solve the 8-cluster 4096-subdomain workload; its single-cluster form of that mesh "
           "needs a coarse problem of ~10^5 unknowns that takes hours on one core. Measured instead on its own CPU "
           "configuration (reference_small), which bench.py's GPU line also solves (cpu_baseline)")
    line = {"impl": "reference", "unavailable": why}
    if os.path.exists(ref_binary()):
        m = ref_small_measure(args.steps, args.warmup)
        line["reference_small"] = {"workload": SMALL_WORKLOAD, "unit": "s", "cores": 1, "kind": "reference",
                                   "pcpg_s_per_solve": m["pcpg_s"], "setup_s": m["setup_s"],
                                   "setup_and_solve_s": m["total_s"], "process_wall_s": m["wall_s"],
                                   "iterations": m["iterations"], "runs": m["runs"]}
    print(json.dumps(line))
    return 0


def cpu_baseline_small(hb, local, steps=5, warmup=1):
    """The reference on its own configuration, measured in full, and the GPU
    on the same configuration (same mesh construction and options)."""
    if not os.path.exists(ref_binary()):
        return None
    ref = ref_small_measure(steps, warmup)
    spec = hb.mesh_spec(subs=(2, 2, 2), elems=(5, 5, 5), jitter=0.1, seed=1, E=2.1e5, nu=0.3,
                        bc=hb.HTF_BC_CLAMP_X0, body_force=(0.0, 0.0, -1.0))
    mesh = hb.generate_mesh(spec)
    opts = dict(OPTS, typeBc="ker", device=str(local))
    t0 = time.perf_counter()
    s = hb.Solver(opts)
    s.set_mesh(mesh)
    s.setup()
    setup_wall = time.perf_counter() - t0
    u = np.zeros((1, 3 * mesh.n_nodes))
    for _ in range(3):
        s.solve(None, u=u)
    ms, e2e, its = [], [], []
    for _ in range(20):
        t = time.perf_counter()
        _, st = s.solve(None, u=u)
        e2e.append(time.perf_counter() - t)
        ms.append(st.solve_ms)
        its.append(st.iterations[0])
    s.close()
    gpu = statistics.mean(ms) / 1e3
    return {"value": ref["pcpg_s"], "unit": "s", "cores": 1, "kind": "reference",
            "sample": ("not a sample: the reference (oracle/_ref/hfls_ref, built -O2 from the reference sources, "
                       "PARDISO stand-in = skyline Cholesky, 1 thread) solving its own CPU configuration in full, "
                       "mean of %d runs; value = its Cluster::pcpg interval (Cluster.cpp:1364-1451) in wall seconds"
                       % ref["runs"]),
            "workload": SMALL_WORKLOAD, "same_config": True,
            "reference": {"pcpg_s": ref["pcpg_s"], "setup_s": ref["setup_s"], "setup_and_solve_s": ref["total_s"],
                          "iterations": ref["iterations"]},
            "gpu_same_config": {"pcpg_s": gpu, "e2e_solve_s": statistics.mean(e2e), "setup_wall_s": setup_wall,
                                "iterations": int(statistics.median(its)),
                                "speedup_pcpg": ref["pcpg_s"] / gpu,
                                "speedup_setup_and_solve": ref["total_s"] / (setup_wall + statistics.mean(e2e))}}


# ---------------------------------------------------------------------------
def oracle_golden(name):
    p = os.path.join(ROOT, "tests", "golden", f"oracle_{name}.npz")
    return np.load(p) if os.path.exists(p) else None


def golden_rel_err(g, u, k):
    """Relative displacement error of load case k against an oracle golden:
    the larger of the error on the golden's seeded DOF sample and on its
    seeded projections of the whole field."""
    idx = g["sample_idx"]
    e1 = np.linalg.norm(u[idx] - g["u_sample"][k]) / np.linalg.norm(g["u_sample"][k])
    P = np.random.default_rng(777).standard_normal((g["u_proj"].shape[1], u.size))
    e2 = np.linalg.norm(P @ u - g["u_proj"][k]) / np.linalg.norm(g["u_proj"][k])
    return float(max(e1, e2))


def run_cube(hb, local, dist, steps):
    """The regular 512-subdomain cube in FP64: seconds per solve, F apply
    bandwidth and the iteration count against the oracle golden."""
    spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, bc=hb.HTF_BC_CLAMP_X0, **CUBE)
    mesh = hb.generate_mesh(spec)
    f = hb.traction(spec, seed=2, n_rhs=1)
    s = hb.Solver(dict(OPTS, device=str(local)))
    s.set_mesh(mesh)
    s.set_loads(f)
    t0 = time.perf_counter()
    s.setup()
    setup_wall = time.perf_counter() - t0
    u = np.zeros((1, 3 * mesh.n_nodes))
    for _ in range(3):
        s.solve(f, u=u)
    barrier(dist)
    ms, e2e, its = [], [], []
    for _ in range(steps):
        t = time.perf_counter()
        _, st = s.solve(f, u=u)
        e2e.append(time.perf_counter() - t)
        ms.append(st.solve_ms)
        its.append(st.iterations[0])
    prof = s.profile(reps=20)
    s.close()
    peak, peak_kind = peaks()
    g = oracle_golden("cube1")
    achieved = prof.symv_F_bytes / (prof.symv_F_ms * 1e-3) / 1e9
    return {"workload": CUBE_WORKLOAD, "solve_s": max_over_ranks(dist, statistics.mean(ms)) / 1e3,
            "e2e_s": max_over_ranks(dist, statistics.mean(e2e)), "setup_s": setup_wall,
            "iterations": int(statistics.median(its)),
            "iterations_oracle": int(g["iterations"][0]) if g is not None else None,
            "fapply_gbs": prof.fapply_bytes / (prof.fapply_ms * 1e-3) / 1e9, "fapply_ms": prof.fapply_ms,
            "iteration_ms": prof.iteration_ms,
            "symv_F": {"kernel": "k_symv_units<double>", "ms": prof.symv_F_ms, "bytes": prof.symv_F_bytes,
                       "gbs": achieved, "frac": achieved / peak, "peak_kind": peak_kind,
                       "traffic": traffic_from_profile(PROFILE_CUBE)}}


def run_mixed(hb, local, dist, reduced=None):
    """Batched mixed-precision solve of MIXED_RHS load cases vs the FP64 form
    on four of them (time per load case); displacement error of every load
    case against the oracle golden (full size) or an FP64 solve at eps 1e-10
    (reduced meshes).  Times are CUDA-event solve times, max over ranks."""
    spec_kw = dict(CUBE, body_force=(0.0, 0.0, -1.0), **(reduced or {}))
    spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, bc=hb.HTF_BC_CLAMP_X0, **spec_kw)
    mesh = hb.generate_mesh(spec)
    f = hb.traction(spec, seed=3, n_rhs=MIXED_RHS)
    pick = [0, MIXED_RHS // 3, 2 * MIXED_RHS // 3, MIXED_RHS - 1]
    s = hb.Solver(dict(OPTS, device=str(local), precision="mixed", batch="32"))
    s.set_mesh(mesh)
    s.setup()
    u = np.zeros((MIXED_RHS, 3 * mesh.n_nodes))
    s.solve(f, u=u)                                     # warm-up (graph capture, caches)
    barrier(dist)
    t = time.perf_counter()
    _, st = s.solve(f, u=u)
    wall = time.perf_counter() - t
    mixed_ms = max_over_ranks(dist, st.solve_ms)
    wall = max_over_ranks(dist, wall)
    its = list(st.iterations[:MIXED_RHS])
    prof = s.profile(reps=10)
    s.close()
    s64 = hb.Solver(dict(OPTS, device=str(local)))
    s64.set_mesh(mesh)
    s64.setup()
    u64, st64 = s64.solve(f[pick])
    fp64_ms = max_over_ranks(dist, st64.solve_ms) / len(pick)
    its64 = list(st64.iterations[:len(pick)])
    s64.close()
    g = oracle_golden("cube32") if reduced is None else None
    if g is not None:
        err = [golden_rel_err(g, u[k], k) for k in range(MIXED_RHS)]
        err64 = [golden_rel_err(g, u64[i], k) for i, k in enumerate(pick)]
        against = "oracle golden (tests/golden/oracle_cube32.npz, eps 1e-11), every load case"
        its_oracle = [int(x) for x in g["iterations"]]
    else:
        sref = hb.Solver(dict(OPTS, device=str(local), eps_iter="1e-10", max_iter="10000"))
        sref.set_mesh(mesh)
        sref.setup()
        uref, _ = sref.solve(f[pick])
        sref.close()
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        err = [rel(u[k], uref[i]) for i, k in enumerate(pick)]
        err64 = [rel(u64[i], uref[i]) for i in range(len(pick))]
        against = "FP64 GPU solve at eps 1e-10 of load cases %s" % pick
        its_oracle = None
    peak, peak_kind = peaks()
    tc_gbs = prof.tc_F_bytes / (prof.tc_F_ms * 1e-3) / 1e9
    return {
        "workload": MIXED_WORKLOAD, "load_cases": MIXED_RHS, "batch": 32,
        "solve_s_per_load_case": mixed_ms / 1e3 / MIXED_RHS,
        "fp64_solve_s_per_load_case": fp64_ms / 1e3,
        "speedup_vs_fp64": fp64_ms / (mixed_ms / MIXED_RHS),
        "e2e_s_per_load_case": wall / MIXED_RHS,
        "iterations_median": int(statistics.median(its)), "iterations_max": int(max(its)),
        "fp64_iterations": its64, "oracle_iterations_fp64": its_oracle,
        "u_rel_err_max": max(err), "fp64_u_rel_err_max": max(err64), "u_err_against": against,
        "batch_iteration_ms": prof.batch_iteration_ms,
        "tc_F": {"kernel": "k_tc_gemm<32> (F_i FP16-pair slabs x 32 load cases)", "ms": prof.tc_F_ms,
                 "bytes": prof.tc_F_bytes, "gbs": tc_gbs, "frac": tc_gbs / peak, "peak_kind": peak_kind},
    }


def serve_stream(hb, n, seed=4):
    """The first n requests of the seeded serving stream: (arrival s, spec, load cases, seed)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(n):
        t += float(rng.exponential(1.0 / SERVE_RATE))
        c, s, e = int(rng.integers(1, 5)), int(rng.integers(2, 6)), int(rng.integers(4, 11))
        k, nu = int(rng.integers(1, 17)), float(rng.uniform(0.2, 0.4))
        spec = hb.mesh_spec(clusters=(c, c, c), subs=(s, s, s), elems=(e, e, e), jitter=0.1, seed=1000 + i,
                            material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e4, nu=nu, bc=hb.HTF_BC_CLAMP_X0,
                            body_force=(0.0, 0.0, -1.0))
        out.append((t, spec, k, 2000 + i, (c, s, e)))
    return out


def pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_serving(hb, local, n_req, fp64_requests=None):
    """Continuous-batching server on a bounded prefix of the serving stream,
    then the plain FP64 per-request path on the first fp64_requests served
    requests (all by default), FIFO on their own arrival times."""
    import torch
    free, _ = torch.cuda.mem_get_info(local)
    budget = 0.85 * free
    stream = serve_stream(hb, n_req)
    loads = [hb.traction(spec, seed=fseed, n_rhs=k) for (_, spec, k, fseed, _) in stream]
    opts = dict(OPTS, device=str(local), precision="mixed", batch="16", max_iter="12000")
    srv = hb.Server(opts, hbm_budget_bytes=budget, max_live=8)
    tickets = []
    t0 = time.perf_counter()
    for (ta, spec, k, _, _), f in zip(stream, loads):
        dt = t0 + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        try:
            tickets.append(srv.submit(spec, f, n_rhs=k))
        except hb.HTFError as e:
            tickets.append(e)
    served = []
    for i, t in enumerate(tickets):
        if isinstance(t, hb.HTFError):
            served.append((i, None, None, None, t.code, str(t)[:200]))
            continue
        try:
            u, info = srv.wait(t)
            served.append((i, u.copy(), info.t_submit_ms, info.t_done_ms, info.iterations_max,
                           dict(queue_ms=round(info.t_admit_ms - info.t_submit_ms, 1),
                                setup_ms=round(info.t_start_ms - info.t_admit_ms, 1),
                                run_ms=round(info.t_done_ms - info.t_start_ms, 1),
                                iterations=info.iterations_max, gb=round(info.bytes / 1e9, 2),
                                gb_estimate=round(info.bytes_estimate / 1e9, 2))))
        except hb.HTFError as e:
            served.append((i, None, None, None, e.code, str(e)[:200]))
    srv.close()
    ok = [x for x in served if x[1] is not None]
    lat = [x[3] - x[2] for x in ok]
    cases = sum(stream[x[0]][2] for x in ok)
    makespan = (max(x[3] for x in ok) - min(x[2] for x in ok)) / 1e3 if ok else None
    # plain FP64 per-request path: service time of each served request, FIFO on the same arrivals
    service, err = [], 0.0
    ok64 = ok if fp64_requests is None else ok[:fp64_requests]
    for (i, u, *_) in ok64:
        ta, spec, k, _, _ = stream[i]
        t = time.perf_counter()
        s = hb.Solver(dict(OPTS, device=str(local), max_iter="5000"))
        s.set_mesh(hb.generate_mesh(spec))
        s.setup()
        u64, _ = s.solve(loads[i])
        s.close()
        service.append(time.perf_counter() - t)
        err = max(err, max(float(np.linalg.norm(u[j] - u64[j]) / np.linalg.norm(u64[j])) for j in range(k)))
    # the served displacements against tight FP64 solves (eps 1e-10) of the three
    # smallest served requests: the mixed form's bound is 1e-7 against a converged u
    tight_err, tight_req = 0.0, []
    for (i, u, *_) in sorted(ok, key=lambda x: int(np.prod(stream[x[0]][4])))[:3]:      # c s e: elements^(1/3)
        spec, k = stream[i][1], stream[i][2]
        s = hb.Solver(dict(OPTS, device=str(local), eps_iter="1e-10", max_iter="20000"))
        try:
            s.set_mesh(hb.generate_mesh(spec))
            s.setup()
            ut, _ = s.solve(loads[i])
        except hb.HTFError:
            continue
        finally:
            s.close()
        tight_req.append(i)
        tight_err = max(tight_err, max(float(np.linalg.norm(u[j] - ut[j]) / np.linalg.norm(ut[j])) for j in range(k)))
    fin, lat64 = 0.0, []
    for (i, *_), sv in zip(ok64, service):
        ta = stream[i][0]
        fin = max(fin, ta) + sv
        lat64.append(1e3 * (fin - ta))
    first = stream[ok64[0][0]][0] if ok64 else 0.0
    cases64 = sum(stream[x[0]][2] for x in ok64)
    return {
        "workload": SERVE_WORKLOAD, "requests": n_req, "served": len(ok),
        "rejected_oversize": sum(1 for x in served if x[1] is None and x[4] == hb.HTF_ENOMEM),
        "failed_other": sum(1 for x in served if x[1] is None and x[4] != hb.HTF_ENOMEM),
        "load_cases": cases, "budget_gb": budget / 1e9,
        "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "mean_ms": float(np.mean(lat)) if lat else None,
        "solves_per_s": cases / makespan if makespan else None,
        "requests_per_s": len(ok) / makespan if makespan else None,
        "fp64_per_request": {"requests": len(ok64), "p50_ms": pct(lat64, 50), "p99_ms": pct(lat64, 99),
                             "solves_per_s": cases64 / (fin - first) if ok64 else None,
                             "service_s": [round(x, 3) for x in service]},
        "u_rel_err_max_vs_fp64": err,
        "u_rel_err_vs_fp64_note": "both stop at eps 1e-8 (the served form at 1e-8 x mixed_eps_factor 0.1): the "
                                  "difference includes the FP64 solve's own distance from convergence",
        "u_rel_err_max_vs_tight_fp64": tight_err if tight_req else None,
        "tight_fp64_requests": tight_req,
        "sizes": [dict(c=x[4][0], s=x[4][1], e=x[4][2], load_cases=x[2]) for x in stream],
        "per_request": [dict(request=x[0], **x[5]) for x in ok],
        "errors": [x[5] for x in served if x[1] is None],
    }


def soft(fn, *args, dist=None):
    """Run one of the measurements beside the headline; on one process an
    exception there is reported in its field instead of losing the headline
    line.  Under several ranks it propagates, so that no rank leaves the
    others waiting in a collective that it skips."""
    if dist is not None:
        return fn(*args)
    try:
        return fn(*args)
    except Exception as e:          # noqa: BLE001  (any failure of a side measurement)
        return {"error": f"{type(e).__name__}: {e}"[:400]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision multi-load-case measurement")
    ap.add_argument("--mixed-only", action="store_true",
                    help="only the mixed-precision measurement on the 512-subdomain cube (for launch lists)")
    ap.add_argument("--no-cube", action="store_true", help="skip the 512-subdomain cube measurement")
    ap.add_argument("--serve-requests", type=int, default=SERVE_REQUESTS,
                    help="requests of the seeded serving stream to serve (0 skips the serving measurement)")
    ap.add_argument("--serve-only", action="store_true",
                    help="only the serving measurement (its own JSON line); the plain FP64 comparison runs on the "
                         "first --serve-fp64 served requests")
    ap.add_argument("--serve-fp64", type=int, default=None)
    ap.add_argument("--setup-only", action="store_true",
                    help="set up the headline mesh once, print its set-up phases and exit (for launch lists)")
    ap.add_argument("--workload", default="full", choices=["full"] + sorted(REDUCED),
                    help="reduced meshes of the same constructions, for ncu captures only: uneven-small is one "
                         "cluster of the uneven cube; small / mid are one / two clusters of 2x4x4 cube subdomains "
                         "and run the cube in place of the uneven headline (the mixed form runs at the same size)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local, dist = dist_setup(args.gpus)
    import hfls_b200 as hb
    if args.mixed_only:
        out = run_mixed(hb, local, dist, None)
        if rank == 0:
            print(json.dumps({"mixed": out}))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    if args.setup_only:
        s = hb.Solver(dict(OPTS, device=str(local)))
        s.set_mesh(hb.generate_mesh(uneven_spec(hb)))
        t = time.perf_counter()
        s.setup()
        wall = time.perf_counter() - t
        prof = s.profile(reps=1)
        s.close()
        if rank == 0:
            print(json.dumps({"workload": UNEVEN_WORKLOAD, "setup_s": wall,
                              "setup_phase_ms": [round(x, 1) for x in prof.setup_phase_ms],
                              "frontend_ms": round(prof.frontend_ms, 1),
                              "kernel_detection_ms": round(prof.kernel_detection_ms, 1)}))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    if args.serve_only:
        out = run_serving(hb, local, args.serve_requests, args.serve_fp64)
        if rank == 0:
            print(json.dumps({"serving": out}))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    reduced = REDUCED.get(args.workload)
    if args.workload in ("small", "mid"):
        spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, bc=hb.HTF_BC_CLAMP_X0, **dict(CUBE, **reduced))
        workload = CUBE_WORKLOAD + " (reduced: %s)" % args.workload
        f = hb.traction(spec, seed=2, n_rhs=1)
    else:
        spec = uneven_spec(hb, **(reduced or {}))
        workload = UNEVEN_WORKLOAD + ("" if reduced is None else " (reduced: %s)" % args.workload)
        f = None
    mesh = hb.generate_mesh(spec)
    if f is None:
        # the load case is the body force; htf_solve still takes the (zero) extra nodal load from
        # host memory, as a caller solving a new load case does
        f = np.zeros((1, 3 * mesh.n_nodes))
        s_loads = False
    else:
        s_loads = True
    s = hb.Solver(dict(OPTS, device=str(local)))
    s.set_mesh(mesh)
    if s_loads:
        s.set_loads(f)
    t0 = time.perf_counter()
    s.setup()
    setup_wall = time.perf_counter() - t0
    u = np.zeros((1, 3 * mesh.n_nodes))
    for _ in range(args.warmup):
        _, st = s.solve(f, u=u)
    barrier(dist)
    solve_ms, e2e_s, launches, iters = [], [], 0, []
    with ClockSampler(local) as clk:
        barrier(dist)
        for _ in range(args.steps):
            t = time.perf_counter()
            _, st = s.solve(f, u=u)          # host buffers in and out
            e2e_s.append(time.perf_counter() - t)
            solve_ms.append(st.solve_ms)
            launches += st.kernel_launches
            iters.append(st.iterations[0])
        barrier(dist)
    ms = max_over_ranks(dist, statistics.mean(solve_ms))
    e2e = max_over_ranks(dist, statistics.mean(e2e_s))
    prof = s.profile(reps=10)
    n_lambda = st.n_lambda
    s.close()
    full = args.workload == "full"
    cube = None if (args.no_cube or not full) else soft(run_cube, hb, local, dist, min(args.steps, 5), dist=dist)
    mixed = None if args.no_mixed else soft(run_mixed, hb, local, dist, None if full else REDUCED.get(
        args.workload if args.workload in ("small", "mid") else "mid"), dist=dist)
    serving = None
    if args.serve_requests > 0 and full:
        barrier(dist)
        serving = soft(run_serving, hb, local, args.serve_requests, dist=dist)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    cpu = None if args.no_cpu_baseline else soft(cpu_baseline_small, hb, local)
    peak, peak_kind = peaks()
    achieved = prof.symv_F_bytes / (prof.symv_F_ms * 1e-3) / 1e9
    ndof = 3 * mesh.n_nodes
    line = {
        "metric": METRIC, "value": whole_job_seconds_per_solve(ms, world), "unit": "s", "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload, "n_sub": mesh.n_sub, "n_dof": ndof, "n_lambda": n_lambda,
                   "iterations": int(statistics.median(iters)), "setup_s": setup_wall,
                   "setup_device_ms": st.setup_ms,
                   "setup_phase_ms": {k: round(v, 1) for k, v in zip(
                       ["problem_build", "device_context", "layout_upload", "assembly_factor_FS", "load_maps",
                        "cluster_coarse", "outer_coarse", "symv_tuning_fp32_slabs"], prof.setup_phase_ms)},
                   "kernel_detection_ms": round(prof.kernel_detection_ms, 1),
                   "frontend_ms": round(prof.frontend_ms, 1),
                   "symv_unit_tiles": list(prof.symv_unit_tiles), "symv_tuned": int(prof.symv_tuned),
                   "l2": "inputs larger than L2 (F_i and S_i tiles: %.2f GB per PCPG iteration)"
                         % ((prof.symv_F_bytes + prof.symv_S_bytes) / 1e9),
                   "parallelism": f"replicas x{world}",
                   "value": "seconds per solve of the whole job: the slowest rank's time per solve / ranks"},
        "fapply_gbs": prof.fapply_bytes / (prof.fapply_ms * 1e-3) / 1e9,
        "fapply_ms": prof.fapply_ms, "iteration_ms": prof.iteration_ms,
        "e2e": {"value": whole_job_seconds_per_solve(e2e * 1e3, world), "unit": "s",
                "h2d_bytes_per_step": 8 * ndof, "d2h_bytes_per_step": 8 * ndof,
                "note": "htf_solve with host buffers: the nodal load vector in (zero on the body-force headline, "
                        "whose load the library assembles from the mesh) and the displacement field out"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "k_symv_units<double> (F_i packed tiles)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic_from_profile(PROFILE_UNEVEN) if full else None,
                     "peak_kind": peak_kind, "bytes_per_launch": prof.symv_F_bytes,
                     "launch_ms": prof.symv_F_ms},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "cube512": cube,
        "mixed": mixed,
        "serving": serving,
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
