"""The C-ABI library loads and exports every declared symbol; host-side entry points work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from difffea_b200 import _lib
from difffea_b200.cuda_mesh import colour_elements
from difffea_b200.mesh import create_rectangle_mesh

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "difffea_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dfea_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.exported_symbols())     # the binding declares exactly the header


def test_version_and_element_table():
    lib = _lib.load()
    assert lib.dfea_version() >= 10000
    for nen, nq in ((4, 4), (9, 9), (3, 1), (6, 6), (8, 9)):
        assert lib.dfea_element_supported(nen, nq) == 1
    assert lib.dfea_element_supported(4, 9) == 0


def _valid_colouring(conn, colour):
    conn = np.asarray(conn)
    for c in np.unique(colour):
        nodes = conn[colour == c].reshape(-1)
        assert len(np.unique(nodes)) == len(nodes), f"colour {c} shares a node"


@pytest.mark.parametrize("et,expected", [("quad4", 4), ("quad8", 4), ("quad9", 4), ("tri3", None), ("tri6", None)])
def test_greedy_colouring(et, expected):
    _, conn = create_rectangle_mesh(et, 3.0, 2.0, 13, 7)
    colour, nc = colour_elements(conn)
    _valid_colouring(conn, colour)
    assert colour.min() == 0 and colour.max() == nc - 1
    if expected:
        assert nc == expected
    else:
        assert nc <= 8


def test_colouring_rejects_bad_node_ids():
    lib = _lib.load()
    conn = np.array([[0, 1, 2, 7]], dtype=np.int64)
    col = np.zeros(1, dtype=np.int32)
    nc = ctypes.c_int32(0)
    rc = lib.dfea_colour_elements(conn.ctypes.data_as(ctypes.c_void_p), 1, 4, 5, col.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.byref(nc))
    assert rc == 1 and "outside" in _lib.last_error()


def test_pcg_work_size_query_is_host_only():
    view = _lib.MeshView()
    view.n_nodes, view.n_colours = 1000, 4
    n64 = _lib.load().dfea_pcg_work_bytes(ctypes.byref(view), _lib.DFEA_F64)
    n32 = _lib.load().dfea_pcg_work_bytes(ctypes.byref(view), _lib.DFEA_F32)
    assert n64 > n32 > 3 * 2 * 1000 * 4


def test_compute_entry_points_validate_before_touching_the_gpu():
    view = _lib.MeshView()            # all zero: invalid
    rc = _lib.load().dfea_tangent_apply(ctypes.byref(view), None, 0, None, None, 0, None)
    assert rc != 0


def test_ctypes_mirrors_match_the_library_struct_layouts():
    """Every struct the binding mirrors has the size the library was compiled with (a host query)."""
    lib = _lib.load()
    mirrors = {"dfea_material": _lib.Material, "dfea_mesh_view": _lib.MeshView, "dfea_mg_grid": _lib.MgGrid,
               "dfea_mg_level": _lib.MgLevel, "dfea_mg": _lib.Mg, "dfea_newton": _lib.Newton,
               "dfea_newton_record": _lib.NewtonRecord, "dfea_newton_info": _lib.NewtonInfo,
               "dfea_rect_spec": _lib.RectSpec}
    for name, cls in mirrors.items():
        assert lib.dfea_struct_size(name.encode()) == ctypes.sizeof(cls), name
    assert lib.dfea_struct_size(b"no_such_struct") == -1


def test_newton_driver_validates_before_touching_the_gpu():
    lib = _lib.load()
    info = _lib.NewtonInfo()
    assert lib.dfea_newton_solve(None, 1, 1e-8, 25, 8, 500, ctypes.byref(info), None, 0, None) == 1
    nw = _lib.Newton()                 # no mesh, no buffers
    assert lib.dfea_newton_solve(ctypes.byref(nw), 1, 1e-8, 25, 8, 500, ctypes.byref(info), None, 0, None) == 1


def test_rectangle_builder_rejects_bad_specs():
    """dfea_build_rectangle_host (the host builder of the serving requests' problems) refuses element types other
    than Q4 / Q9, empty rectangles and NULL outputs with an error code and a message, writing nothing."""
    from difffea_b200.serving import Request, _rect_arrays
    lib = _lib.load()
    invalid = int(re.search(r"#define DFEA_ERR_INVALID (\d+)", open(HEADER).read()).group(1))
    spec, a = _rect_arrays(Request(0, "quad4", 8, 1.0, 0.3, 0.02))
    ptrs = [ctypes.c_void_p(a[k].data_ptr()) for k in ("nodes", "conn", "dN_dX", "w_detJ", "f", "m", "fixed", "u_D")]
    assert lib.dfea_build_rectangle_host(ctypes.byref(spec), *ptrs) == _lib.DFEA_OK
    for field, value in (("nen", 8), ("nx", 0), ("ny", -1), ("width", 0.0)):
        bad = _lib.RectSpec.from_buffer_copy(spec)
        setattr(bad, field, value)
        assert lib.dfea_build_rectangle_host(ctypes.byref(bad), *ptrs) == invalid, field
        assert b"rectangle" in lib.dfea_last_error(), field
    assert lib.dfea_build_rectangle_host(ctypes.byref(spec), *ptrs[:-1], ctypes.c_void_p(0)) == invalid
    assert lib.dfea_build_rectangle_host(None, *ptrs) == invalid
