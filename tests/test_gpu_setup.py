"""Boundary set-up on the device (GPU only): ``pxb_label_polygons`` must give the host
labelling's cells, in the same raster order, for every layout."""
import numpy as np
import pytest
import torch

from bc_specs import BC_SPECS, ROE_BC_SPECS, grid_coords

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def same_manager(params, X, Y):
    from pyexner_b200 import BoundaryManager

    h = BoundaryManager(params, X, Y, setup="host")
    d = BoundaryManager(params, X, Y, setup="device")
    assert np.array_equal(h.boundary_mask, d.boundary_mask)
    assert len(h.handlers) == len(d.handlers)
    for a, b in zip(h.handlers, d.handlers):
        assert a["kind"] == b["kind"]
        for x, y in zip(a["cells"] + a["donors"], b["cells"] + b["donors"]):
            assert np.array_equal(x, y)
    return h


@pytest.mark.parametrize("name", sorted(BC_SPECS))
@pytest.mark.parametrize("shape", [(11, 14), (97, 203)])
def test_device_labels_match_host(name, shape):
    ny, nx = shape
    X, Y = grid_coords(ny, nx)
    same_manager(dict(flux_scheme="Roe Exner", boundaries=BC_SPECS[name](ny, nx)), X, Y)


def test_device_labels_roe_layouts():
    X, Y = grid_coords(40, 33)
    for name in ROE_BC_SPECS:
        same_manager(dict(flux_scheme="Roe", boundaries=ROE_BC_SPECS[name](40, 33)), X, Y)


def test_device_labels_on_file_coordinates():
    """The Berthon case's mesh (file coordinates + dh/2, edges through cell centres)."""
    from pyexner_b200.cases import berthon_case

    for dh in (0.1, 0.025):
        x, y, fields, params = berthon_case(dh)
        X, Y = np.meshgrid(x + dh / 2, y - dh / 2, indexing="xy")
        h = same_manager(params, X, Y)
        assert all(len(hd["cells"][0]) > 0 for hd in h.handlers)


def test_device_labels_large_ring():
    from pyexner_b200.boundaries import index_coords, ring_boundaries

    n = 2050
    X, Y = index_coords(n, n)
    spec = ring_boundaries(n, n, ["Transmissive", "TransmissiveBed"], ["Transmissive", "TransmissiveBed"],
                           ["Reflective"], ["Reflective"])
    h = same_manager(dict(flux_scheme="Roe Exner", boundaries=spec), X, Y)
    assert h.boundary_mask.sum() == 4 * n - 4
