"""
Material library of the CUDA path (the reference's materials.py API).

    material_names(), get_material(name)                 materials.py:189-196
    material_vector(name, values=None)                   materials.py:208-222
    material_of(params), element_material_parameters()   materials.py:225-246
    device_material(params) -> _lib.Material             the C ABI's dfea_material

The five hyperelastic energies of the reference (materials.py:65-161), each a function of the plane-strain
embedding F3 = [[F, 0], [0, 1]]:

    neo_hookean       mu/2 (I1 - 3 - 2 lnJ) + lambda/2 lnJ^2                          p = (mu, lmbda)
    mooney_rivlin     c10 (J^-2/3 I1 - 3) + c01 (J^-4/3 I2 - 3) + kappa/2 lnJ^2         p = (c10, c01, kappa)
    saint_venant      lambda/2 (tr E)^2 + mu tr(E^2),  E = (C - I)/2                    p = (mu, lmbda)
    demiray           mu/(2 gamma) (exp(gamma (I1 - 3)) - 1) - mu lnJ + lambda/2 lnJ^2 p = (mu, gamma, lmbda)
    fiber_reinforced  neo-Hookean + sum_i k1/(2 k2) (exp(k2 <E_i>^2) - 1),
                      E_i = d I1 + (1 - 3d) I4_i - 1, I4_i = a_i . C a_i,
                      a = (cos beta, +-sin beta)                  p = (mu, lmbda, k1, k2, beta_deg, d, second_family)

The kernels evaluate neo-Hookean in closed form and differentiate the other energies on the device
(forward mode, first and second derivatives).  The design field theta multiplies the scalable parameters
of each element (materials.py:239-246).
"""
import torch

from difffea_b200 import _lib

MATERIAL_LIBRARY = {
    "neo_hookean": dict(label="Neo-Hookean (isotropic rubber)", param_names=["mu", "lmbda"],
                        defaults=[1000.0, 1500.0], scalable=["mu", "lmbda"], fibrous=False),
    "mooney_rivlin": dict(label="Mooney-Rivlin (isotropic rubber, two invariants)",
                          param_names=["c10", "c01", "kappa"], defaults=[400.0, 100.0, 1500.0],
                          scalable=["c10", "c01", "kappa"], fibrous=False),
    "saint_venant": dict(label="Saint Venant-Kirchhoff (linear in Green strain)", param_names=["mu", "lmbda"],
                         defaults=[1000.0, 1500.0], scalable=["mu", "lmbda"], fibrous=False),
    "demiray": dict(label="Demiray (exponential, strain-stiffening tissue)", param_names=["mu", "gamma", "lmbda"],
                    defaults=[500.0, 3.0, 1500.0], scalable=["mu", "lmbda"], fibrous=False),
    "fiber_reinforced": dict(label="Fibre-reinforced (HGO: matrix + two fibre families)",
                             param_names=["mu", "lmbda", "k1", "k2", "beta_deg", "d", "second_family"],
                             defaults=[400.0, 1200.0, 1500.0, 4.0, 30.0, 0.0, 1.0],
                             scalable=["mu", "lmbda", "k1"], fibrous=True),
}
for _name, _m in MATERIAL_LIBRARY.items():
    _m["model"] = _lib.DFEA_MAT[_name]
MATERIALS = tuple(MATERIAL_LIBRARY)
NEO_HOOKEAN_DEFAULTS = dict(zip(MATERIAL_LIBRARY["neo_hookean"]["param_names"],
                                MATERIAL_LIBRARY["neo_hookean"]["defaults"]))


def lame_parameters(E, nu):
    """(mu, lambda) from Young's modulus and Poisson's ratio (plane strain / 3D relations)."""
    return E / (2.0 * (1.0 + nu)), E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))


def material_names():
    return list(MATERIAL_LIBRARY)


def get_material(name):
    """The library entry: label, param_names, defaults, scalable, fibrous and the device model id."""
    if name not in MATERIAL_LIBRARY:
        raise ValueError(f"Unknown material '{name}'. Choose one of {material_names()}.")
    return MATERIAL_LIBRARY[name]


def material_vector(name="neo_hookean", values=None, dtype=torch.float64):
    """(p (n_p,), scalable mask (n_p,) bool) of a material; ``values`` overrides the defaults by name."""
    mat = get_material(name)
    vals = dict(zip(mat["param_names"], mat["defaults"]))
    if values:
        unknown = set(values) - set(vals)
        if unknown:
            raise ValueError(f"Unknown parameters {sorted(unknown)} for '{name}'; valid: {mat['param_names']}")
        vals.update({k: float(v) for k, v in values.items()})
    p = torch.tensor([vals[n] for n in mat["param_names"]], dtype=dtype)
    mask = torch.tensor([n in mat["scalable"] for n in mat["param_names"]], dtype=torch.bool)
    return p, mask


def material_of(params):
    """(name, p0, scalable) of a problem dictionary; legacy mu0/lmbda0 dictionaries are neo-Hookean."""
    if "material" in params:
        return params["material"], params["mat_p"], params["mat_scalable"]
    dev = params["nodes"].device
    p = torch.tensor([params["mu0"], params["lmbda0"]], dtype=params["nodes"].dtype, device=dev)
    return "neo_hookean", p, torch.ones(2, dtype=torch.bool, device=dev)


def device_material(params):
    """The problem's material as the C ABI's ``dfea_material`` (host struct)."""
    name, p0, scalable = material_of(params)
    mat = get_material(name)
    p0 = torch.as_tensor(p0).detach().to("cpu", torch.float64).reshape(-1)
    scalable = torch.as_tensor(scalable).detach().to("cpu").reshape(-1).bool()
    n = len(mat["param_names"])
    if p0.numel() != n or scalable.numel() != n:
        raise ValueError(f"'{name}' has {n} parameters; got mat_p of {p0.numel()} and mat_scalable of "
                         f"{scalable.numel()} entries")
    out = _lib.Material()
    out.model = mat["model"]
    out.scalable = sum(1 << k for k in range(n) if bool(scalable[k]))
    for k in range(n):
        out.p[k] = float(p0[k])
    return out


def neo_hookean_parameters(params):
    """(mu0, lambda0) as Python floats; raises for any other material or a non-scalable parameter."""
    name, p0, scalable = material_of(params)
    if name != "neo_hookean":
        raise ValueError(f"expected the neo-Hookean material, got '{name}'")
    if not bool(torch.as_tensor(scalable).all()):
        raise ValueError("expected theta to scale both mu and lambda")
    p0 = torch.as_tensor(p0).detach().to("cpu", torch.float64)
    return float(p0[0]), float(p0[1])


def element_material_parameters(theta, params):
    """(n_el, n_p) table p_e = p0 * theta_e on the scalable entries."""
    _, p0, scalable = material_of(params)
    p0 = torch.as_tensor(p0, dtype=theta.dtype, device=theta.device)
    scalable = torch.as_tensor(scalable, device=theta.device)
    factor = torch.where(scalable[None, :], theta[:, None], torch.ones_like(theta)[:, None])
    return p0[None, :] * factor
