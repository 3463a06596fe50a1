"""
Host logic of the serving path and of the benchmark's multi-process plumbing, on the CPU: the seeded
request stream, Poisson arrivals, HBM estimates and admission, percentiles, sharding of the stream
over replicas, and a world-size-2 ``gloo`` run of the rank helpers (barrier, max over ranks).
"""
import math
import os
import socket
import threading

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from difffea_b200.serving import (MULTIGRID_MIN_NODES, Request, ServingEngine, hbm_estimate, percentile,
                                  preconditioner_for, request_problem, request_stream, shard_requests, with_arrivals)


def test_request_stream_is_seeded_and_follows_its_distributions():
    a, b = request_stream(2000, seed=0), request_stream(2000, seed=0)
    assert [(r.element_type, r.nx, r.E, r.nu, r.load) for r in a] == [(r.element_type, r.nx, r.E, r.nu, r.load)
                                                                      for r in b]
    assert request_stream(50, seed=1)[0] != a[0]
    nx = np.array([r.nx for r in a])
    assert nx.min() >= 16 and nx.max() <= 512 and np.all(nx % 4 == 0)
    assert 0.4 < np.mean([r.element_type == "quad4" for r in a]) < 0.6
    E = np.array([r.E for r in a])
    assert E.min() >= 0.5 and E.max() <= 2.0 and abs(np.mean(np.log(E))) < 0.05       # log-uniform, centred on 1
    assert all(0.2 <= r.nu <= 0.45 and 0.01 <= r.load <= 0.05 for r in a)
    assert [r.rid for r in a] == list(range(2000))
    assert all(r.arrival == 0.0 for r in a)


def test_poisson_arrivals_have_the_asked_rate():
    reqs = with_arrivals(request_stream(2000, seed=0), rate=40.0, seed=3)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 40.0) < 0.1 / 40.0
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1                                     # exponential: CV 1
    s = request_stream(200, seed=0, rate=10.0)
    assert s[-1].arrival > 0 and all(x.arrival < y.arrival for x, y in zip(s, s[1:]))


def test_request_geometry_and_problem_dictionary():
    r = Request(7, "quad9", 64, 1.3, 0.3, 0.02)
    assert (r.ny, r.n_elements, r.n_nodes) == (16, 1024, 129 * 33)
    p = request_problem(r, "cpu")
    assert p["conn"].shape == (1024, 9) and p["nodes"].shape == (r.n_nodes, 2)
    x = p["nodes"][:, 0]
    assert float(x.min()) == 0.0 and float(x.max()) == 4.0
    assert float(p["f"][0::2].sum()) == pytest.approx(0.02 * 1.0, rel=1e-12)   # traction x edge length 1
    assert float(p["f"][1::2].abs().sum()) == 0.0


def test_hbm_estimate_grows_with_size_and_precision():
    small, large = Request(0, "quad4", 16, 1, 0.3, 0.02), Request(1, "quad4", 512, 1, 0.3, 0.02)
    q9 = Request(2, "quad9", 512, 1, 0.3, 0.02)
    assert hbm_estimate(small) < hbm_estimate(large) < hbm_estimate(q9)
    assert hbm_estimate(large, "fp32") < hbm_estimate(large, "fp64")
    assert hbm_estimate(q9) < 2 ** 30                      # the largest request of the stream fits easily


def test_auto_preconditioner_threshold_and_its_memory():
    small, large = Request(0, "quad4", 64, 1, 0.3, 0.02), Request(1, "quad9", 512, 1, 0.3, 0.02)
    assert small.n_nodes < MULTIGRID_MIN_NODES <= large.n_nodes
    assert preconditioner_for(small) == "jacobi" and preconditioner_for(large) == "multigrid"
    assert preconditioner_for(large, "jacobi") == "jacobi" and preconditioner_for(small, "multigrid") == "multigrid"
    assert hbm_estimate(large, "fp32", "auto") > hbm_estimate(large, "fp32", "jacobi")
    assert hbm_estimate(small, "fp32", "auto") == hbm_estimate(small, "fp32", "jacobi")
    assert hbm_estimate(large, "fp32", "auto") < 2 ** 30
    served = [preconditioner_for(r) for r in request_stream(400, seed=0)]
    assert 0.7 < served.count("multigrid") / len(served) < 0.95        # most of the stream is large


def test_percentile_is_nearest_rank():
    v = list(range(1, 101))
    assert percentile(v, 50) == 50 and percentile(v, 99) == 99 and percentile(v, 100) == 100
    assert percentile([3.0], 99) == 3.0
    assert math.isnan(percentile([], 50))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_partition_the_stream(world):
    reqs = request_stream(101, seed=0)
    shards = [shard_requests(reqs, k, world) for k in range(world)]
    ids = sorted(r.rid for s in shards for r in s)
    assert ids == list(range(101))
    assert max(len(s) for s in shards) - min(len(s) for s in shards) <= 1


def test_admission_waits_for_budget_and_rejects_oversized():
    eng = ServingEngine.__new__(ServingEngine)             # admission logic only: no device needed
    eng.hbm_budget = 100
    eng._cv = threading.Condition()
    eng._in_use = eng._in_flight = eng.peak_in_use = eng.peak_in_flight = 0
    with pytest.raises(MemoryError):
        eng._reserve(101)
    eng._reserve(60)
    order = []

    def second():
        eng._reserve(60)                                   # must wait until the first 60 are released
        order.append("second admitted")

    t = threading.Thread(target=second)
    t.start()
    t.join(0.2)
    assert t.is_alive() and not order
    order.append("first released")
    eng._release(60)
    t.join(5)
    assert order == ["first released", "second admitted"]
    assert eng.peak_in_use == 60 and eng.peak_in_flight == 1
    eng._release(60)
    assert eng._in_use == 0


# ------------------------------------------------------------------------------------------------
# two gloo ranks: the benchmark's rank helpers and its stream windows
# ------------------------------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, w, _ = bench.dist_init("gloo")
    assert (r, w) == (rank, world)
    bench.dist_barrier(w)
    m = bench.dist_max(float(10 * rank + 1), w, torch.device("cpu"))
    timed, warm = bench.full_windows(r, w, steps=2, warmup=3)
    warm_s, timed_s = bench.sample_windows(r, w, steps=2, warmup=3)
    import torch.distributed as dist
    ids, sample_ids = [None] * w, [None] * w
    dist.all_gather_object(ids, [q.rid for q in timed])
    dist.all_gather_object(sample_ids, [q.rid for q in warm_s + timed_s])
    out[rank] = (m, ids, len(warm), sample_ids, max(q.nx for q in timed_s), bench.serve_config(2))
    dist.destroy_process_group()


def test_two_rank_bench_helpers_over_gloo():
    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    for rank in range(world):
        m, ids, n_warm, sample_ids, max_nx, config = out[rank]
        assert m == 11.0                                      # max over ranks of (1, 11)
        assert set(ids[0]).isdisjoint(ids[1])                 # each replica serves its own requests
        assert all(i % world == 0 for i in ids[0]) and all(i % world == 1 for i in ids[1])
        assert len(ids[0]) == len(ids[1]) == 2 * 32
        assert n_warm > 0
        # the like-for-like sample: disjoint per replica, 4 requests per step, small requests only
        assert set(sample_ids[0]).isdisjoint(sample_ids[1])
        assert len(sample_ids[0]) == len(sample_ids[1]) == (3 + 2) * 4
        assert max_nx <= 64
        assert config == out[0][5]                            # both arms and all ranks print one config


@pytest.mark.parametrize("et,nx", [("quad4", 16), ("quad9", 12), ("quad4", 100), ("quad9", 64), ("quad4", 4)])
def test_host_request_problem_matches_the_builder(et, nx):
    """A request built on the host by the library (dfea_build_rectangle_host) has build_rectangle_problem's keys,
    connectivity, supports and material exactly, and its coordinates, geometry and load to rounding."""
    from difffea_b200.problem import build_rectangle_problem
    req = Request(0, et, nx, 1.3, 0.31, 0.04)
    p = request_problem(req, "cpu")
    q = build_rectangle_problem(et, req.nx, req.ny, 4.0, 1.0, E=req.E, nu=req.nu, load=(req.load, 0.0))
    assert list(p) == list(q)
    for k in ("conn", "fixed", "m", "u_D", "mat_p", "mat_scalable", "GP", "GW"):
        assert torch.equal(p[k], q[k]), k
    for k in ("nodes", "dN_dX", "w_detJ", "f"):
        assert p[k].shape == q[k].shape, k
        assert float((p[k] - q[k]).abs().max()) <= 1e-13 * float(q[k].abs().max()), k


@pytest.mark.parametrize("et,nx", [("quad4", 24), ("quad9", 20)])
def test_library_built_requests_are_recognised_as_structured_grids(et, nx):
    """The multigrid hierarchy needs the mesher's numbering: the library-built connectivity is recognised as the
    nx x ny grid, with every node at its grid position."""
    from difffea_b200.multigrid import structured_grid
    req = Request(0, et, nx, 1.0, 0.3, 0.02)
    p = request_problem(req, "cpu")
    g = structured_grid(p["conn"], p["nodes"].shape[0])
    assert g is not None and (g["ncx"], g["ncy"]) == (req.nx, req.ny)
    span = 2 if et == "quad9" else 1
    x = p["nodes"][:, 0] * (span * req.nx / 4.0)
    y = p["nodes"][:, 1] * (span * req.ny / 1.0)
    assert torch.equal(torch.round(x).to(torch.int32), g["node_ij"][:, 0])
    assert torch.equal(torch.round(y).to(torch.int32), g["node_ij"][:, 1])
