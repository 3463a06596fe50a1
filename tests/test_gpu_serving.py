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
