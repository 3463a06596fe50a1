"""Helpers shared by the tests: golden fixtures, problem dictionaries from them, error measures."""
import os

import numpy as np
import torch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TYPES = {(4, 4): "quad4", (9, 9): "quad9", (3, 1): "tri3", (6, 6): "tri6", (8, 9): "quad8"}


def golden_names(prefix=""):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith(prefix))


def load(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as d:
        return {k: d[k] for k in d.files}


def params_from(d, device="cpu"):
    """A problem dictionary (reference keys) built from a golden fixture's arrays."""
    t = lambda k, dt=torch.float64: torch.as_tensor(d[k]).to(dtype=dt, device=device)  # noqa: E731
    conn = t("conn", torch.int64)
    dN = t("dN_dX")
    scalable = (t("mat_scalable", torch.bool) if "mat_scalable" in d
                else torch.ones(d["mat_p"].size, dtype=torch.bool, device=device))
    return {"nodes": t("nodes"), "conn": conn, "dN_dX": dN, "w_detJ": t("w_detJ"), "f": t("f"), "m": t("m"),
            "fixed": t("fixed", torch.bool), "u_D": t("u_D"), "mat_p": t("mat_p"), "mat_scalable": scalable,
            "material": str(d["material"]) if "material" in d else "neo_hookean",
            "element_type": TYPES[(conn.shape[1], dN.shape[1])]}


def rel(a, b):
    a = torch.as_tensor(a, dtype=torch.float64).cpu()
    b = torch.as_tensor(b, dtype=torch.float64).cpu()
    den = float(b.abs().max())
    return float((a - b).abs().max()) / (den if den > 0 else 1.0)
