"""Host side of the material library: parameter vectors and masks, and their encoding as ``dfea_material``."""
import pytest
import torch

from difffea_b200 import _lib
from difffea_b200.materials import (MATERIAL_LIBRARY, device_material, element_material_parameters, get_material,
                                    material_names, material_vector)


def test_library_matches_the_reference_names_and_defaults():
    assert material_names() == ["neo_hookean", "mooney_rivlin", "saint_venant", "demiray", "fiber_reinforced"]
    assert get_material("demiray")["param_names"] == ["mu", "gamma", "lmbda"]
    p, mask = material_vector("fiber_reinforced", {"k1": 2000.0, "beta_deg": 45.0})
    assert p.tolist() == [400.0, 1200.0, 2000.0, 4.0, 45.0, 0.0, 1.0]
    assert mask.tolist() == [True, True, True, False, False, False, False]
    with pytest.raises(ValueError):
        material_vector("fiber_reinforced", {"k3": 1.0})
    with pytest.raises(ValueError):
        get_material("ogden")


@pytest.mark.parametrize("name", list(MATERIAL_LIBRARY))
def test_device_material_encoding(name):
    p, mask = material_vector(name)
    mat = device_material({"material": name, "mat_p": p, "mat_scalable": mask})
    assert mat.model == _lib.DFEA_MAT[name]
    assert mat.scalable == sum(1 << k for k, s in enumerate(mask.tolist()) if s)
    assert list(mat.p)[:p.numel()] == p.tolist() and all(x == 0.0 for x in list(mat.p)[p.numel():])


def test_device_material_rejects_mismatched_vectors():
    with pytest.raises(ValueError):
        device_material({"material": "demiray", "mat_p": torch.ones(2), "mat_scalable": torch.ones(2, dtype=torch.bool)})


def test_element_parameters_scale_only_the_scalable_entries():
    p, mask = material_vector("demiray")
    th = torch.tensor([1.0, 2.0], dtype=torch.float64)
    pe = element_material_parameters(th, {"material": "demiray", "mat_p": p, "mat_scalable": mask})
    assert pe[1].tolist() == [1000.0, 3.0, 3000.0]
