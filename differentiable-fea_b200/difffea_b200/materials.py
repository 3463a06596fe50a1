"""
Material data of the CUDA path: compressible neo-Hookean in plane strain.

    psi(F) = mu/2 (I1 - 3 - 2 ln J) + lambda/2 (ln J)^2,   I1 = |F|^2 + 1,   J = det F

(the reference's materials.py:209-217 with the embedding F3 = [[F, 0], [0, 1]]).  The parameter
vector is p = [mu, lambda]; the design field theta multiplies both (materials.py:308-312, 383-390), so
the element force is linear in theta_e -- which is what the sensitivity kernel uses.  The kernels
evaluate P and d2psi/dF2 in closed form; the other materials of the reference library are not built
on the device.
"""
import torch

MATERIALS = ("neo_hookean",)
NEO_HOOKEAN_DEFAULTS = {"mu": 1000.0, "lmbda": 1500.0}


def lame_parameters(E, nu):
    """(mu, lambda) from Young's modulus and Poisson's ratio (plane strain / 3D relations)."""
    return E / (2.0 * (1.0 + nu)), E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))


def material_vector(name="neo_hookean", values=None, dtype=torch.float64):
    """(p (2,), scalable mask (2,) bool) for the neo-Hookean material; ``values`` overrides by name."""
    if name not in MATERIALS:
        raise ValueError(f"Material '{name}' is not built on the device; choose one of {list(MATERIALS)}.")
    vals = dict(NEO_HOOKEAN_DEFAULTS)
    if values:
        unknown = set(values) - set(vals)
        if unknown:
            raise ValueError(f"Unknown parameters {sorted(unknown)} for '{name}'; valid: {list(vals)}")
        vals.update({k: float(v) for k, v in values.items()})
    return (torch.tensor([vals["mu"], vals["lmbda"]], dtype=dtype), torch.ones(2, dtype=torch.bool))


def material_of(params):
    """(name, p0, scalable) of a problem dictionary; legacy mu0/lmbda0 dictionaries are neo-Hookean."""
    if "material" in params:
        return params["material"], params["mat_p"], params["mat_scalable"]
    dev = params["nodes"].device
    p = torch.tensor([params["mu0"], params["lmbda0"]], dtype=params["nodes"].dtype, device=dev)
    return "neo_hookean", p, torch.ones(2, dtype=torch.bool, device=dev)


def neo_hookean_parameters(params):
    """(mu0, lambda0) as Python floats; raises for any other material or a non-scalable parameter."""
    name, p0, scalable = material_of(params)
    if name != "neo_hookean":
        raise ValueError(f"the CUDA path implements the neo-Hookean material only, got '{name}'")
    if not bool(torch.as_tensor(scalable).all()):
        raise ValueError("the CUDA path needs theta to scale both mu and lambda")
    p0 = torch.as_tensor(p0).detach().to("cpu", torch.float64)
    return float(p0[0]), float(p0[1])


def element_material_parameters(theta, params):
    """(n_el, 2) table p_e = p0 * theta_e on the scalable entries."""
    _, p0, scalable = material_of(params)
    p0 = torch.as_tensor(p0, dtype=theta.dtype, device=theta.device)
    scalable = torch.as_tensor(scalable, device=theta.device)
    factor = torch.where(scalable[None, :], theta[:, None], torch.ones_like(theta)[:, None])
    return p0[None, :] * factor
