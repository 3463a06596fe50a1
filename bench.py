"""
Benchmark of the matrix-free Newton-Krylov hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload plain]

Workload "plain" (default): one step = one complete FP64 Newton-Krylov solve of the plain problem --
100 x 100 structured Q4 on the unit square (10,000 elements), neo-Hookean E = 1, nu = 0.3, left edge
clamped, dead traction of total (0.1, 0) on the right edge (~10 % stretch), 3 load steps, Newton
tol 1e-10, Jacobi-PCG with the reference's forcing term and 500-iteration cap.  value = solves/s over
all ranks (each rank solves its own copy: replicas, weak scaling), with p50/p99 solve latency.

Beside it, in the same JSON line:
  roofline      the dominant kernel, the FP64 stored-moduli tangent product (kernel (b)), timed with CUDA
                events on its launch stream at the tangent-product microbench size (structured Q4,
                1600 x 1600 = 2.56M elements; inputs 2.2 GB >> L2), achieved = algorithmic bytes / time
  cpu_baseline  the oracle (CPU restatement of the reference, tangent "qp" = the reference's CPU
                default) timed on this host on one solve of the same problem
  e2e           the same solves through the public API with the problem dictionary in pinned host
                memory: host->device copies, mesh packing, solve, and the read-back of u inside the
                timed region

--impl reference times the reference algorithm's CPU implementation (the oracle) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "differentiable-fea_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import torch  # noqa: E402

METRIC = "solves/s + p50/p99 latency, batched vs plain, at <=1e-8 rel err; A(v) HBM %"
PLAIN = dict(element_type="quad4", nx=100, ny=100, width=1.0, height=1.0, E=1.0, nu=0.3, load=(0.1, 0.0),
             n_load_steps=3, tol=1e-10)
MATVEC_N = 1600


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------------------------------------
# distributed plumbing (one process per GPU; replicas)
# ------------------------------------------------------------------------------------------------
def dist_init(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, world, local


def dist_max(value, world, device):
    if world == 1:
        return value
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------------------------------------
# workloads
# ------------------------------------------------------------------------------------------------
def plain_problem(device):
    from difffea_b200.problem import build_rectangle_problem
    c = PLAIN
    return build_rectangle_problem(c["element_type"], c["nx"], c["ny"], c["width"], c["height"], E=c["E"],
                                   nu=c["nu"], load=c["load"], device=device)


def plain_solve(params, theta, ws=None):
    from difffea_b200.newton_krylov import newton_krylov_solve
    return newton_krylov_solve(params, theta, PLAIN["n_load_steps"], PLAIN["tol"], verbose=False, workspace=ws)


def matvec_roofline(device, reps=20):
    """
    Time kernel (b) (FP64 stored moduli) at 2.56M Q4 elements with CUDA events on its launch stream.
    v and y live in one allocation, as the PCG's Krylov vectors do, so the L2 window covers both.
    Algorithmic bytes per product: n_el*n_q*16*8 (moduli) + n_el*n_q*nen*2*8 (gradients) + n_el*nen*4
    (connectivity) + 3*2N*8 (v read, y written, mask).
    """
    import ctypes
    from difffea_b200 import _lib
    from difffea_b200.cuda_mesh import ptr, stream_handle
    from difffea_b200.operators import make_tangent_operator
    from difffea_b200.problem import build_rectangle_problem
    n = MATVEC_N
    p = build_rectangle_problem("quad4", n, n, float(n), float(n), E=1.0, nu=0.3, device=device)
    g = torch.Generator().manual_seed(0)
    N2 = p["f"].shape[0]
    u = (((torch.rand(N2, dtype=torch.float64, generator=g) * 2 - 1) * 0.05).to(device)) * p["m"]
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=device)
    A = make_tangent_operator("cuda", u, th, p)
    pad = (N2 + 3) // 4 * 4
    buf = torch.empty(2 * pad, dtype=torch.float64, device=device)
    v, y = buf[:N2], buf[pad:pad + N2]
    v.copy_(torch.randn(N2, dtype=torch.float64, generator=g).to(device))
    n_el, nen, nq = p["conn"].shape[0], 4, 4
    alg_bytes = n_el * nq * 16 * 8 + n_el * nq * nen * 2 * 8 + n_el * nen * 4 + 3 * N2 * 8

    def product():
        _lib.call("dfea_tangent_apply", A.mesh.view_ref, ptr(A.C), _lib.DFEA_F64, ptr(v), ptr(y), _lib.DFEA_F64,
                  stream_handle())
    for _ in range(3):
        product()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s)
    for _ in range(reps):
        product()
    t1.record(s)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / reps
    y_ref = A(v)
    ok = bool(torch.equal(y_ref, y))
    del A, p, buf
    torch.cuda.empty_cache()
    return dict(n_el=n_el, bytes=alg_bytes, ms=ms, gbs=alg_bytes / (ms * 1e-3) / 1e9, same_as_op=ok)


def cpu_oracle_solve(params_cpu, theta_cpu):
    import oracle
    torch.set_num_threads(os.cpu_count() or 1)
    P = oracle.as_problem(params_cpu)
    t = time.perf_counter()
    u, info = oracle.newton_krylov_solve(P, theta_cpu, PLAIN["n_load_steps"], PLAIN["tol"], tangent="qp")
    return time.perf_counter() - t, u, info


# ------------------------------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from difffea_b200.problem import build_rectangle_problem
    c = PLAIN
    p = build_rectangle_problem(c["element_type"], c["nx"], c["ny"], c["width"], c["height"], E=c["E"], nu=c["nu"],
                                load=c["load"])
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64)
    budget_s, times, spent = 240.0, [], 0.0
    for i in range(args.warmup + args.steps):
        dt, _, _ = cpu_oracle_solve(p, th)
        spent += dt
        if i >= args.warmup:
            times.append(dt)
        if spent > budget_s and len(times) >= 1:
            break
    v = len(times) / sum(times)
    cores = os.cpu_count()
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "plain: 100x100 Q4 neo-Hookean, 3 load steps, Newton tol 1e-10, Jacobi-PCG",
                       "parallelism": "host CPU"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{len(times)} complete solves (oracle restatement, tangent qp)"},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    from difffea_b200 import _lib
    from difffea_b200.problem import to_device
    from difffea_b200.workspace import NewtonWorkspace
    rank, world, local = dist_init("nccl")
    dev = torch.device("cuda", torch.cuda.current_device())
    p = plain_problem(dev)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=dev)
    ws = NewtonWorkspace(p)
    for _ in range(max(3, args.warmup)):
        u, info = plain_solve(p, th, ws)
    torch.cuda.synchronize()

    lat = []
    lib = _lib.load()
    with ClockSampler(local) as clocks:
        dist_barrier(world)
        torch.cuda.synchronize()
        n0 = lib.dfea_launch_count()
        s = torch.cuda.current_stream()
        e_start = torch.cuda.Event(enable_timing=True)
        e_start.record(s)
        ev = []
        for _ in range(args.steps):
            u, info = plain_solve(p, th, ws)
            e = torch.cuda.Event(enable_timing=True)
            e.record(s)
            ev.append(e)
        torch.cuda.synchronize()
        launches = lib.dfea_launch_count() - n0
        dist_barrier(world)
    prev = e_start
    for e in ev:
        lat.append(prev.elapsed_time(e))
        prev = e
    total_ms = dist_max(sum(lat), world, dev)
    value = world * args.steps / (total_ms * 1e-3)

    # end to end through the public API: host (pinned) dictionary -> device -> solve -> host u
    from difffea_b200.newton_krylov import newton_krylov_solve
    host = {k: (v.cpu().pin_memory() if torch.is_tensor(v) else v) for k, v in p.items()}
    th_h = th.cpu().pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in host.values() if torch.is_tensor(v)) + th_h.numel() * 8
    d2h = p["f"].numel() * 8
    e2e_steps = max(1, min(args.steps, 5))
    dist_barrier(world)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(e2e_steps):
        pd = to_device(host, dev)
        u_e, _ = newton_krylov_solve(pd, th_h.to(dev, non_blocking=True), PLAIN["n_load_steps"], PLAIN["tol"],
                                     verbose=False)
        u_host = u_e.cpu()
    torch.cuda.synchronize()
    e2e_s = dist_max(time.perf_counter() - t, world, dev)
    e2e = world * e2e_steps / e2e_s

    roof = matvec_roofline(dev) if rank == 0 else None
    out = None
    if rank == 0:
        hbm, kind = peaks()
        cpu_dt, u_ref, info_ref = cpu_oracle_solve({k: (v.cpu() if torch.is_tensor(v) else v) for k, v in p.items()},
                                                   th.cpu())
        err = float((u.cpu() - u_ref).abs().max() / u_ref.abs().max())
        lat_sorted = sorted(lat)
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": "plain: 100x100 Q4 (10,000 el) neo-Hookean E=1 nu=0.3, left clamped, right "
                                      "traction (0.1, 0), 3 load steps, Newton tol 1e-10, Jacobi-PCG (EW forcing, cap 500)",
                          "parallelism": f"replicas x{world}", "l2": "roofline leg inputs 2.2 GB > 126 MB L2"},
               "latency_ms": {"p50": lat_sorted[len(lat) // 2], "p99": lat_sorted[min(len(lat) - 1, int(0.99 * len(lat)))]},
               "accuracy": {"rel_err_vs_oracle": err, "newton": info["total_newton"], "cg": info["total_cg"],
                            "newton_oracle": info_ref["total_newton"], "cg_oracle": info_ref["total_cg"]},
               "roofline": {"bound": "hbm", "achieved": roof["gbs"], "peak": hbm, "unit": "GB/s",
                            "frac": roof["gbs"] / hbm, "traffic": None, "peak_kind": kind,
                            "kernel": "k_apply<4,4,double> (A(v), FP64 stored moduli)",
                            "workload": f"structured Q4 {MATVEC_N}x{MATVEC_N} = {roof['n_el']} elements",
                            "alg_bytes_per_launch": roof["bytes"], "ms_per_product": roof["ms"]},
               "cpu_baseline": {"value": 1.0 / cpu_dt, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": "1 complete solve of the same problem (oracle, tangent qp)"},
               "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
               "gpu_launches": int(launches),
               "clocks": clocks.summary()}
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="plain", choices=("plain",))
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    return run_reference(args) if args.impl == "reference" else run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
