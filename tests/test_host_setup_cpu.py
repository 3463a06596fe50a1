"""Host-side set-up (meshes, loads, geometry, API validation) against the reference's golden arrays."""
import math

import pytest
import torch

import oracle
from difffea_b200 import newton_krylov, operators
from difffea_b200.elements import element_names
from difffea_b200.problem import build_problem, build_quarter_plate_problem, default_spec
from golden_utils import load, params_from, rel


@pytest.mark.parametrize("et", element_names())
@pytest.mark.parametrize("h,tag", [(0.5, "unit"), (0.25, "theta")])
def test_problem_builder_matches_reference(et, h, tag):
    d = load(f"operator_{et}_h{h}_{tag}")
    spec = default_spec("rectangle", et, h)
    spec.update(load_value=(60.0, 0.0), E=2600.0, nu=0.3)
    p = build_problem(spec)
    for k in ("nodes", "conn", "f", "m", "u_D", "mat_p"):
        assert torch.equal(p[k].double(), torch.as_tensor(d[k]).double()), k
    assert torch.equal(p["fixed"], torch.as_tensor(d["fixed"]))
    assert rel(p["dN_dX"], d["dN_dX"]) < 1e-13
    assert rel(p["w_detJ"], d["w_detJ"]) < 1e-14


def test_quarter_plate_mesh_is_valid():
    p = build_quarter_plate_problem("quad9", n_theta=16, n_radial=12)
    W, R = 10.0, 1.0
    area = float(p["w_detJ"].sum())
    assert abs(area - (W * W - math.pi * R * R / 4)) < 1e-5 * W * W
    assert float(p["w_detJ"].min()) > 0
    X = p["nodes"]
    fx = p["fixed"].reshape(-1, 2)
    assert torch.equal(fx[:, 0], X[:, 0] <= 1e-8) and torch.equal(fx[:, 1], X[:, 1] <= 1e-8)
    f = p["f"].reshape(-1, 2)
    assert abs(float(f[:, 0].sum()) - 0.1 * W) < 1e-12 and float(f[:, 1].abs().max()) == 0.0
    assert bool((f[:, 0] != 0).le(X[:, 0] >= W - 1e-8).all())


def test_unknown_and_reference_only_variants_are_rejected():
    u = torch.zeros(4, dtype=torch.float64)
    with pytest.raises(ValueError):
        operators.make_tangent_operator("nope", u, u, {})
    for kind in ("jvp", "linearize", "qp", "qp_ew"):
        with pytest.raises(ValueError):
            operators.make_tangent_operator(kind, u, u, {})
    with pytest.raises(ValueError):
        operators.make_preconditioner("ilu", u, u, {})
    with pytest.raises(RuntimeError):
        operators.make_tangent_operator("auto", u, u, {})      # CPU tensor: no CPU path in this package


def test_solver_refuses_cpu_problems():
    spec = default_spec("rectangle", "quad4", 0.5)
    p = build_problem(spec)
    with pytest.raises(RuntimeError):
        newton_krylov.newton_krylov_solve(p, torch.ones(p["conn"].shape[0], dtype=torch.float64), verbose=False)


def test_step_by_step_pcg_matches_oracle_on_closures():
    """The closure-driven PCG (used for arbitrary operators) follows the reference recurrences."""
    d = load("operator_quad4_h0.25_theta")
    P = oracle.as_problem(params_from(d))
    u, th = torch.as_tensor(d["u"]), torch.as_tensor(d["theta"])
    A = oracle.make_operator("qp_ew", u, th, P)
    dg = oracle.jacobi_diagonal(u, th, P)
    b = P["m"] * torch.as_tensor(d["v"])
    for rtol, it in ((1e-8, 500), (1e-3, 500), (1e-12, 7)):
        x1, k1 = newton_krylov.pcg(A, b, lambda r: r / dg, rtol, it)
        x2, k2 = oracle.pcg(A, b, lambda r: r / dg, rtol, it)
        assert k1 == k2 and torch.equal(x1, x2)
    x, k = newton_krylov.pcg(A, torch.zeros_like(b), lambda r: r / dg)
    assert k == 0 and float(x.abs().max()) == 0.0


@pytest.mark.parametrize("name", ["operator_quad4_h0.5_unit", "operator_quad4_h0.25_theta", "operator_quad4_h0.1_theta",
                                  "operator_quad9_h0.5_unit", "operator_quad9_h0.25_theta"])
def test_library_rectangle_builder_matches_reference(name):
    """The library's rectangle builder (dfea_build_rectangle_host, which writes the serving requests' problems)
    reproduces the reference's own problem arrays for its rectangle cantilever: the mesh, supports and
    prescribed values exactly, geometry and load to rounding."""
    import ctypes
    from difffea_b200 import _lib, serving
    from difffea_b200.cuda_mesh import ptr
    d = load(name)
    et = "quad9" if "quad9" in name else "quad4"
    h = float(name.split("_h")[1].split("_")[0])
    spec = _lib.RectSpec.from_buffer_copy(serving._rect_template(et))
    spec.nx, spec.ny, spec.width, spec.height = round(2.0 / h), round(1.0 / h), 2.0, 1.0
    spec.load_x, spec.load_y = 60.0, 0.0
    N, n_el, nen, nq = d["nodes"].shape[0], d["conn"].shape[0], d["conn"].shape[1], d["w_detJ"].shape[1]
    f64 = dict(dtype=torch.float64)
    a = dict(nodes=torch.empty(N, 2, **f64), conn=torch.empty(n_el, nen, dtype=torch.int64),
             dN_dX=torch.empty(n_el, nq, nen, 2, **f64), w_detJ=torch.empty(n_el, nq, **f64),
             f=torch.empty(2 * N, **f64), m=torch.empty(2 * N, **f64), fixed=torch.empty(2 * N, dtype=torch.bool),
             u_D=torch.empty(2 * N, **f64))
    assert _lib.load().dfea_build_rectangle_host(ctypes.byref(spec), *(ptr(a[k]) for k in serving._RECT_ARGS)) == 0
    for k in ("conn", "m", "u_D"):
        assert torch.equal(a[k].double(), torch.as_tensor(d[k]).double()), k
    assert torch.equal(a["fixed"], torch.as_tensor(d["fixed"]))
    assert rel(a["nodes"], d["nodes"]) < 1e-15
    assert rel(a["dN_dX"], d["dN_dX"]) < 1e-13 and rel(a["w_detJ"], d["w_detJ"]) < 1e-13
    assert rel(a["f"], d["f"]) < 1e-13
