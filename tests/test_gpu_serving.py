"""
Serving form: continuous batching of device-resident solves.  Every result is the same alone and in the
mix, the mixed-precision results meet 1e-8 against FP64, and admission respects the HBM budget.
"""
import pytest
import torch

from difffea_b200.serving import Request, ServingEngine, hbm_estimate, run_plain
from golden_utils import rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _requests():
    specs = [("quad4", 16, 1.0, 0.3, 0.03), ("quad9", 24, 0.7, 0.25, 0.02), ("quad4", 40, 1.8, 0.42, 0.05),
             ("quad9", 16, 0.5, 0.35, 0.01), ("quad4", 64, 1.2, 0.3, 0.04), ("quad9", 32, 1.5, 0.44, 0.05),
             ("quad4", 28, 0.9, 0.21, 0.015), ("quad9", 20, 1.1, 0.33, 0.035)]
    return [Request(i, et, nx, E, nu, ld, arrival=0.002 * i) for i, (et, nx, E, nu, ld) in enumerate(specs)]


def test_results_are_the_same_alone_and_in_the_mix():
    reqs = _requests()
    eng = ServingEngine(n_slots=4, device=DEV)
    alone = run_plain(reqs, DEV, precision="fp32", max_blocks=eng.max_blocks)
    mixed = eng.run(reqs)
    for a, b in zip(alone, mixed):
        assert b.error == "" and b.converged and a.converged
        assert torch.equal(a.u, b.u)                   # deterministic: bit for bit
        assert (a.newton, a.cg) == (b.newton, b.cg)


def test_mixed_precision_serving_meets_1e8_against_fp64():
    reqs = _requests()
    plain = run_plain(reqs, DEV, precision="fp64")
    mixed = ServingEngine(n_slots=8, device=DEV).run(reqs)
    for p, m in zip(plain, mixed):
        assert p.converged and m.converged
        assert rel(m.u, p.u) <= 1e-8


def test_hbm_budget_admission():
    reqs = _requests()[:4]
    biggest = max(hbm_estimate(r) for r in reqs)
    eng = ServingEngine(n_slots=4, hbm_budget=biggest, device=DEV)
    res = eng.run(reqs)
    assert all(r.converged for r in res)
    assert eng.peak_in_flight == 1 and eng.peak_in_use <= biggest
    small = ServingEngine(n_slots=2, hbm_budget=1000, device=DEV).run(reqs[:1])
    assert "MemoryError" in small[0].error


def test_batched_engine_gives_the_slot_results_bit_for_bit():
    reqs = _requests()
    slots = ServingEngine(n_slots=4, device=DEV).run(reqs)
    eng = ServingEngine(n_slots=4, device=DEV, batched=True)
    batched = eng.run(reqs)
    assert eng.batch.peak_batch >= 2                       # solves really advanced together
    for a, b in zip(slots, batched):
        assert b.error == "" and b.converged
        assert torch.equal(a.u, b.u) and (a.newton, a.cg) == (b.newton, b.cg)


def test_faulty_requests_in_the_mix_are_reported_and_leave_the_others_unchanged():
    """A request whose load inverts elements at every attempt (a traction of 4,000 E: NaN residuals, rejected
    line searches, two cut-backs allowed) and malformed requests run inside a mix; they are reported, every
    other result is bit for bit the one of the clean mix."""
    reqs = _requests()
    clean = ServingEngine(n_slots=4, device=DEV, max_cutbacks=2).run(reqs)
    inverting = Request(100, "quad4", 32, 0.5, 0.3, 2000.0, arrival=0.003)
    malformed = [Request(101, "quad5", 16, 1.0, 0.3, 0.02, arrival=0.004),
                 Request(102, "quad4", 0, 1.0, 0.3, 0.02, arrival=0.005),
                 Request(103, "quad9", 16, float("nan"), 0.3, 0.02, arrival=0.006),
                 Request(104, "quad4", 16, 1.0, 0.5, 0.02, arrival=0.007)]
    mix = reqs[:3] + [inverting] + malformed + reqs[3:]
    res = {r.rid: r for r in ServingEngine(n_slots=4, device=DEV, max_cutbacks=2).run(mix)}
    for a in clean:
        b = res[a.rid]
        assert a.converged and b.converged and b.error == ""
        assert torch.equal(a.u, b.u) and (a.newton, a.cg) == (b.newton, b.cg)
    bad = res[100]
    assert not bad.converged and bad.error.startswith("NotConverged") and bad.load_factor < 1.0
    for m in malformed:
        assert res[m.rid].error.startswith("ValueError"), res[m.rid].error


@pytest.mark.parametrize("et,nx,preconditioner", [("quad4", 32, "jacobi"), ("quad9", 24, "jacobi"),
                                                  ("quad4", 256, "multigrid"), ("quad9", 128, "multigrid")])
def test_hbm_estimate_bounds_the_memory_a_request_allocates(et, nx, preconditioner):
    """The admission estimate covers what a request really allocates on the device (torch's peak counter)."""
    from difffea_b200.serving import solve_request
    req = Request(7, et, nx, 1.0, 0.3, 0.03)
    torch.cuda.synchronize()
    base = torch.cuda.memory_allocated(DEV)
    torch.cuda.reset_peak_memory_stats(DEV)
    u, info = solve_request(req, DEV, preconditioner=preconditioner, pcg_form="gather", max_blocks=64)
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated(DEV) - base
    est = hbm_estimate(req, "fp32", preconditioner)
    print(f"\n{et} nx={nx} {preconditioner}: peak {peak / 2**20:.1f} MiB, estimate {est / 2**20:.1f} MiB")
    assert info["converged"] and peak <= est


def test_pooled_meshes_give_the_fresh_results_bit_for_bit():
    """Requests on meshes the engine has served before reuse the kept mesh and workspace (new load and
    material only; with graph-driven multigrid, also the graphs an earlier request captured); every result
    equals the one of an engine that builds each request from scratch."""
    specs = [("quad4", 32, 1.0, 0.3, 0.03), ("quad9", 24, 0.7, 0.25, 0.02), ("quad4", 128, 1.8, 0.42, 0.05),
             ("quad4", 32, 0.6, 0.4, 0.011), ("quad9", 24, 1.9, 0.21, 0.045), ("quad4", 128, 0.9, 0.33, 0.02),
             ("quad4", 32, 1.3, 0.35, 0.04), ("quad9", 64, 1.1, 0.3, 0.03), ("quad9", 64, 0.8, 0.27, 0.015)]
    reqs = [Request(i, et, nx, E, nu, ld) for i, (et, nx, E, nu, ld) in enumerate(specs)]
    fresh = ServingEngine(n_slots=1, device=DEV, pool_bytes=0).run(reqs)
    eng = ServingEngine(n_slots=1, device=DEV, pool_bytes=None, mg_graphs=True)
    pooled = eng.run(reqs)
    assert eng.pool.hits >= 4                               # the repeated meshes were served from the pool
    for a, b in zip(fresh, pooled):
        assert a.converged and b.converged and b.error == ""
        assert torch.equal(a.u, b.u) and (a.newton, a.cg) == (b.newton, b.cg)
    again = eng.run(reqs)                                   # every mesh pooled now, several slots
    for a, b in zip(fresh, again):
        assert torch.equal(a.u, b.u)


def test_host_built_requests_match_the_device_built_ones():
    """source="host" (each problem built on the host, pinned, copied inside the slot) gives the results of the
    same host dictionaries passed in, bit for bit, and those of problems built on the device to 1e-8 (host and
    device geometry differ in the last bits)."""
    from difffea_b200.serving import request_problem, request_stream
    reqs = request_stream(12, seed=5)
    eng = ServingEngine(n_slots=4, device=DEV, precision="fp32")
    host = eng.run(reqs, source="host")
    given = {r.rid: {k: (v.pin_memory() if torch.is_tensor(v) else v) for k, v in request_problem(r, "cpu").items()}
             for r in reqs}
    passed = eng.run(reqs, host_params=given)
    built_on_device = eng.run(reqs)
    for a, b, c in zip(host, passed, built_on_device):
        assert a.converged and b.converged and c.converged
        assert torch.equal(a.u, b.u), a.rid
        assert rel(a.u, c.u) < 1e-8, a.rid


@pytest.mark.parametrize("et,nx", [("quad4", 16), ("quad9", 12), ("quad4", 100), ("quad9", 64)])
def test_device_request_problem_matches_the_builder(et, nx):
    """A request built on the GPU by the library (dfea_build_rectangle) has build_rectangle_problem's keys, mesh,
    supports and material exactly, and its geometry and load to rounding; its solution agrees to 1e-9."""
    from difffea_b200.problem import build_rectangle_problem
    from difffea_b200.serving import reference_request_problem, request_problem, solve_request
    req = Request(0, et, nx, 1.3, 0.31, 0.04)
    p = request_problem(req, DEV, build_on_device=True)
    q = build_rectangle_problem(et, req.nx, req.ny, 4.0, 1.0, E=req.E, nu=req.nu, load=(req.load, 0.0), device=DEV,
                                build_on_device=True)
    assert list(p) == list(q)
    for k in ("conn", "fixed", "m", "u_D", "mat_p", "mat_scalable", "GP", "GW"):
        assert torch.equal(p[k], q[k]), k
    for k in ("nodes", "dN_dX", "w_detJ", "f"):
        assert p[k].shape == q[k].shape and rel(p[k], q[k]) < 1e-13, k
    u, info = solve_request(req, DEV, preconditioner="auto")
    u_ref, info_ref = solve_request(req, DEV, preconditioner="auto", host_params=reference_request_problem(req))
    assert info["converged"] and info_ref["converged"] and rel(u, u_ref) < 1e-9
