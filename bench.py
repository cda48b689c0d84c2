"""HTFETI solve benchmark (plain FP64 form at scale).

Workload (one step = one PCPG solve, g0 -> convergence at 1e-8, with the
factors and F_i / S_i resident on the device):
  2x2x2 clusters x 4x4x4 subdomains x 8x8x8 trilinear hex8 elements on the
  unit cube, interior nodes jittered by U(-0.1h, 0.1h), E_i log-uniform in
  [1e3, 1e6] per subdomain, nu = 0.3, u = 0 on x = 0, seeded N(0,1) nodal
  traction on x = 1, corner gluing inside clusters, Dirichlet preconditioner,
  F_i stored dense FP64 (packed triangular tiles).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Alongside it (same mesh, body force (0, 0, -1), 32 seeded N(0,1) traction
load cases): the batched mixed-precision form (F_i / S_i FP32 on the tensor
cores, FP64 residual replacement) against the FP64 form on the same load
cases, with the displacement error against an FP64 solve at eps 1e-10
("mixed" in the JSON line; --no-mixed skips it).

Under torchrun (N > 1) every rank solves its own replica of the workload on
its own GPU (the solve has no cross-GPU exchange on one node here), timing
is the max over ranks.  --impl reference times the reference CPU solver
(oracle/_ref/hfls_ref, built from the reference sources) on a bounded
sample and scales it to the same metric.
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
WORKLOAD = ("HTFETI cube: 2x2x2 clusters x 4x4x4 subdomains x 8^3 hex8 (512 subdomains, 1.12M local DOFs), "
            "jitter 0.1h, E logU[1e3,1e6], nu 0.3, clamp x=0, N(0,1) traction x=1, corner Bc, "
            "Dirichlet preconditioner, F_i dense FP64, eps 1e-8")
SPEC = dict(clusters=(2, 2, 2), subs=(4, 4, 4), elems=(8, 8, 8), jitter=0.1, seed=1,
            E=1e3, E_hi=1e6, nu=0.3, body_force=(0.0, 0.0, 0.0))
WORKLOAD_ITERATIONS = 638   # PCPG iterations of the workload at 1e-8 (measured by the GPU arm)
OPTS = {"typeBc": "cor", "preconditioner": "Dirichlet_explicit", "eps_iter": "1e-8", "max_iter": "5000"}
REF_SAMPLE = dict(Nx=2, Ny=1, Nz=1, nx=8, ny=8, nz=8)     # subdomains of the workload's size, one cluster
MIXED_RHS = 32
MIXED_WORKLOAD = ("same cube, body force (0,0,-1) + 32 seeded N(0,1) tractions on x=1, solved as one batch of 32: "
                  "F_i/S_i FP32 slabs, 3xTF32 tcgen05 products, FP64 coarse/projector/residual replacement, eps 1e-8")
SERVE_REQUESTS = 12          # requests of the seeded stream that one bench run serves
SERVE_RATE = 1.0             # Poisson arrivals per second
SERVE_WORKLOAD = ("seeded Poisson stream (rate %.1f/s): cube meshes of c^3 clusters, (c s)^3 subdomains of e^3 hex8, "
                  "c in 1..4, s in 2..5, e in 4..10, 1..16 load cases (body force + N(0,1) traction on x=1), "
                  "E logU[1,1e4] per subdomain, nu U[0.2,0.4] per request, clamp x=0, jitter 0.1h, eps 1e-8; "
                  "served by htf_server (mixed precision, batch 16) vs the plain FP64 per-request path "
                  "(set up and solve one request after another, FIFO on the same arrivals)" % SERVE_RATE)


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
                 "--format=csv,noheader,nounits", "-lms", "100"],
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


# ---------------------------------------------------------------------------
# reference CPU solver on a bounded sample
# ---------------------------------------------------------------------------
def ref_binary():
    return os.path.join(ROOT, "oracle", "_ref", "hfls_ref")


def ref_iteration_seconds(iters_a=1, iters_b=101):
    """Wall seconds per PCPG iteration of the reference on REF_SAMPLE
    (difference of two runs that differ only in max_iter)."""
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for it in (iters_a, iters_b):
            args = [ref_binary(), f"out={td}/r{it}", "typeBc=cor", "preconditioner=Dirichlet_explicit",
                    "clamp=true", "young_modulus=1e3", "ratio_mat=1", "eps_iter=1e-30", f"max_iter={it}"]
            args += [f"{k}={v}" for k, v in REF_SAMPLE.items()]
            t0 = time.perf_counter()
            r = subprocess.run(args, capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS="1"))
            out[it] = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError("reference run failed: " + r.stderr[-400:])
    nsub = REF_SAMPLE["Nx"] * REF_SAMPLE["Ny"] * REF_SAMPLE["Nz"]
    per_iter = (out[iters_b] - out[iters_a]) / (iters_b - iters_a)
    return per_iter, nsub, out


def cpu_baseline(iterations, n_sub_cfg):
    if not os.path.exists(ref_binary()):
        return None
    per_iter, nsub, runs = ref_iteration_seconds()
    value = per_iter / nsub * n_sub_cfg * iterations
    return {"value": value, "unit": "s", "cores": 1, "kind": "reference",
            "sample": (f"reference (oracle/_ref/hfls_ref, PARDISO stand-in = skyline Cholesky) on one cluster of "
                       f"{nsub} subdomains of 8^3 hex8: {per_iter:.4f} s per PCPG iteration from runs of "
                       f"{runs[1]:.1f}s (1 it) and {runs[101]:.1f}s (101 it); scaled to {n_sub_cfg} subdomains x "
                       f"{iterations} iterations")}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not os.path.exists(ref_binary()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/hfls_ref was not built"}))
        return 0
    # the reference cannot run the multi-cluster workload; it times PCPG iterations on
    # subdomains of the workload's size and scales by the workload's iteration count,
    # which the FP64 GPU solve of the same problem measures (checked by the GPU arm).
    iterations = WORKLOAD_ITERATIONS
    for _ in range(args.warmup):
        ref_iteration_seconds()
    vals = []
    for _ in range(args.steps):
        per_iter, nsub, _ = ref_iteration_seconds()
        vals.append(per_iter / nsub * 512 * iterations)
    v = statistics.mean(vals)
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "iterations_scaled_to": iterations},
            "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "reference",
                             "sample": f"{REF_SAMPLE} one cluster, per-iteration time scaled to 512 subdomains"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
REDUCED = {"small": dict(clusters=(1, 1, 1), subs=(2, 4, 4)),     # F_i tiles 120 MB, FP32 slabs 100 MB
           "mid": dict(clusters=(2, 1, 1), subs=(2, 4, 4))}       # F_i tiles 240 MB, FP32 slabs 200 MB


def run_mixed(hb, local, dist, reduced=None):
    """Batched mixed-precision solve of MIXED_RHS load cases vs the FP64 form
    on four of them (time per load case; displacement error against FP64 at
    eps 1e-10).  Times are CUDA-event solve times, max over ranks."""
    spec_kw = dict(SPEC, body_force=(0.0, 0.0, -1.0), **(reduced or {}))
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
    del s
    s64 = hb.Solver(dict(OPTS, device=str(local)))
    s64.set_mesh(mesh)
    s64.setup()
    u64, st64 = s64.solve(f[pick])
    fp64_ms = max_over_ranks(dist, st64.solve_ms) / len(pick)
    its64 = list(st64.iterations[:len(pick)])
    del s64
    sref = hb.Solver(dict(OPTS, device=str(local), eps_iter="1e-10", max_iter="10000"))
    sref.set_mesh(mesh)
    sref.setup()
    uref, _ = sref.solve(f[pick])
    del sref
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    peak, peak_kind = peaks()
    tc_gbs = prof.tc_F_bytes / (prof.tc_F_ms * 1e-3) / 1e9
    return {
        "workload": MIXED_WORKLOAD, "load_cases": MIXED_RHS, "batch": 32,
        "solve_s_per_load_case": mixed_ms / 1e3 / MIXED_RHS,
        "fp64_solve_s_per_load_case": fp64_ms / 1e3,
        "speedup_vs_fp64": fp64_ms / (mixed_ms / MIXED_RHS),
        "e2e_s_per_load_case": wall / MIXED_RHS,
        "iterations_median": int(statistics.median(its)), "iterations_max": int(max(its)),
        "fp64_iterations": its64,
        "u_rel_err_max": max(rel(u[k], uref[i]) for i, k in enumerate(pick)),
        "fp64_u_rel_err_max": max(rel(u64[i], uref[i]) for i in range(len(pick))),
        "u_err_reference": "FP64 GPU solve at eps 1e-10 of load cases %s" % pick,
        "batch_iteration_ms": prof.batch_iteration_ms,
        "tc_F": {"kernel": "k_tc_gemm<32> (F_i FP32 slabs x 32 load cases)", "ms": prof.tc_F_ms,
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


def run_serving(hb, local, n_req):
    """Continuous-batching server on a bounded prefix of the serving stream,
    then the plain FP64 per-request path on the same requests."""
    import torch
    free, _ = torch.cuda.mem_get_info(local)
    budget = 0.85 * free
    stream = serve_stream(hb, n_req)
    loads = []
    for (_, spec, k, fseed, dims) in stream:
        c, s, e = dims
        lower = 8.0 * 9.0 * ((c * s) * (e + 1) ** 2) ** 3      # dense factors alone
        loads.append(hb.traction(spec, seed=fseed, n_rhs=k) if lower <= budget else None)
    opts = dict(OPTS, device=str(local), precision="mixed", batch="16", max_iter="3000")
    srv = hb.Server(opts, hbm_budget_bytes=budget, max_live=8)
    tickets = []
    t0 = time.perf_counter()
    for (ta, spec, k, _, _), f in zip(stream, loads):
        dt = t0 + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        tickets.append(srv.submit(spec, f, n_rhs=k))
    served = []
    for i, t in enumerate(tickets):
        try:
            u, info = srv.wait(t)
            served.append((i, u.copy(), info.t_submit_ms, info.t_done_ms, info.iterations_max,
                           dict(queue_ms=round(info.t_admit_ms - info.t_submit_ms, 1),
                                setup_ms=round(info.t_start_ms - info.t_admit_ms, 1),
                                run_ms=round(info.t_done_ms - info.t_start_ms, 1),
                                iterations=info.iterations_max, gb=round(info.bytes / 1e9, 2))))
        except hb.HTFError as e:
            served.append((i, None, None, None, e.code, str(e)[:200]))
    srv.close()
    ok = [x for x in served if x[1] is not None]
    lat = [x[3] - x[2] for x in ok]
    cases = sum(stream[x[0]][2] for x in ok)
    makespan = (max(x[3] for x in ok) - min(x[2] for x in ok)) / 1e3 if ok else None
    # plain FP64 per-request path: service time of each served request, FIFO on the same arrivals
    service, err = [], 0.0
    for (i, u, *_) in ok:
        ta, spec, k, _, _ = stream[i]
        t = time.perf_counter()
        s = hb.Solver(dict(OPTS, device=str(local), max_iter="5000"))
        s.set_mesh(hb.generate_mesh(spec))
        s.setup()
        u64, _ = s.solve(loads[i])
        del s
        service.append(time.perf_counter() - t)
        err = max(err, max(float(np.linalg.norm(u[j] - u64[j]) / np.linalg.norm(u64[j])) for j in range(k)))
    fin, lat64 = 0.0, []
    for (i, *_), sv in zip(ok, service):
        ta = stream[i][0]
        fin = max(fin, ta) + sv
        lat64.append(1e3 * (fin - ta))
    first = stream[ok[0][0]][0] if ok else 0.0
    return {
        "workload": SERVE_WORKLOAD, "requests": n_req, "served": len(ok),
        "rejected_oversize": sum(1 for x in served if x[1] is None and x[4] == hb.HTF_ENOMEM),
        "failed_other": sum(1 for x in served if x[1] is None and x[4] != hb.HTF_ENOMEM),
        "load_cases": cases, "budget_gb": budget / 1e9,
        "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "mean_ms": float(np.mean(lat)) if lat else None,
        "solves_per_s": cases / makespan if makespan else None,
        "requests_per_s": len(ok) / makespan if makespan else None,
        "fp64_per_request": {"p50_ms": pct(lat64, 50), "p99_ms": pct(lat64, 99),
                             "solves_per_s": cases / (fin - first) if ok else None,
                             "service_s": [round(x, 3) for x in service]},
        "u_rel_err_max_vs_fp64": err,
        "sizes": [dict(c=x[4][0], s=x[4][1], e=x[4][2], load_cases=x[2]) for x in stream],
        "per_request": [dict(request=x[0], **x[5]) for x in ok],
        "errors": [x[5] for x in served if x[1] is None],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision multi-load-case measurement")
    ap.add_argument("--serve-requests", type=int, default=SERVE_REQUESTS,
                    help="requests of the seeded serving stream to serve (0 skips the serving measurement)")
    ap.add_argument("--workload", default="full", choices=["full", "small", "mid"],
                    help="small: one cluster of 2x4x4 subdomains of 8^3 (F_i + S_i 0.24 GB > L2); mid: two such "
                         "clusters; reduced cases for ncu captures only (the mixed form runs at the same size)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local, dist = dist_setup(args.gpus)
    import hfls_b200 as hb
    spec_kw = dict(SPEC)
    if args.workload != "full":
        spec_kw.update(REDUCED[args.workload])
    spec = hb.mesh_spec(material=hb.HTF_MAT_LOGUNIFORM, bc=hb.HTF_BC_CLAMP_X0, **spec_kw)
    mesh = hb.generate_mesh(spec)
    f = hb.traction(spec, seed=2, n_rhs=1)
    s = hb.Solver(dict(OPTS, device=str(local)))
    s.set_mesh(mesh)
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
    prof = s.profile(reps=20)
    del s
    # every rank solves its mixed-precision replica too (collective max inside)
    mixed = None if args.no_mixed else run_mixed(hb, local, dist, REDUCED.get(args.workload))
    serving = None
    if args.serve_requests > 0 and args.workload == "full":
        barrier(dist)
        serving = run_serving(hb, local, args.serve_requests)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    peak, peak_kind = peaks()
    achieved = prof.symv_F_bytes / (prof.symv_F_ms * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "k_symv_fp64_cfg1.md")
    if os.path.exists(tf) and args.workload == "full":
        m = re.search(r"^traffic_bytes_per_launch_scaled:\s*([0-9.eE+]+)", open(tf).read(), re.M)
        traffic = float(m.group(1)) if m else None
    iterations = int(statistics.median(iters))
    cpu = None if args.no_cpu_baseline else cpu_baseline(iterations, mesh.n_sub)
    ndof = 3 * mesh.n_nodes
    line = {
        "metric": METRIC, "value": whole_job_seconds_per_solve(ms, world), "unit": "s", "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_sub": mesh.n_sub, "n_lambda": st.n_lambda,
                   "iterations": iterations, "iterations_expected": WORKLOAD_ITERATIONS, "setup_s": setup_wall, "setup_device_ms": st.setup_ms,
                   "l2": "inputs larger than L2 (F_i and S_i tiles: %.2f GB per PCPG iteration)"
                         % ((prof.symv_F_bytes + prof.symv_S_bytes) / 1e9),
                   "parallelism": f"replicas x{world}",
                   "value": "seconds per solve of the whole job: the slowest rank's time per solve / ranks"},
        "fapply_gbs": prof.fapply_bytes / (prof.fapply_ms * 1e-3) / 1e9,
        "fapply_ms": prof.fapply_ms, "iteration_ms": prof.iteration_ms,
        "e2e": {"value": whole_job_seconds_per_solve(e2e * 1e3, world), "unit": "s",
                "h2d_bytes_per_step": 8 * ndof, "d2h_bytes_per_step": 8 * ndof},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "k_symv<double> (F_i packed tiles)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "bytes_per_launch": prof.symv_F_bytes,
                     "launch_ms": prof.symv_F_ms},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "mixed": mixed,
        "serving": serving,
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
