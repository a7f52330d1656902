"""The YAML / NetCDF front end and the output-window loop."""
import os

import numpy as np
import pytest
import torch
import yaml

from pyexner_b200 import io as pio
from pyexner_b200.integrators import IntegratorConfig, _run_time_loop


class _FakeBundle:
    """Records the (time, dt) of every step the loop takes; dt follows a script."""

    def __init__(self, dts):
        self.dts = list(dts)
        self.k = 0
        self.calls = []

    def mask_fn(self, state, *a):
        return None

    def init_fn(self, state, mask, cfg):
        return state

    def compute_dt_fn(self, state, cfl, mask, cfg):
        d = self.dts[min(self.k, len(self.dts) - 1)]
        self.k += 1
        return d

    def step_fn(self, state, time, dt, mask, cfg, avg=None):
        self.calls.append((round(time, 12), round(dt, 12)))
        return state


def _reference_loop(dts, end_time, out_freq, tol=5e-7):
    """src/PyExner/integrators/forwardeuler.py:32-117 restated on plain floats."""
    it = iter(dts + [dts[-1]] * 1000)
    calls, time, dt = [], 0.0, 0.0
    while time < end_time - tol:
        while True:
            target = min((int(time / out_freq) + 1) * out_freq, end_time)
            if not (time + dt < target - tol):
                break
            dt = next(it)
            calls.append((round(time, 12), round(dt, 12)))
            time += dt
        dt = next(it)
        target = min((int(time / out_freq) + 1) * out_freq, end_time)
        if time + dt >= target - tol:
            calls.append((round(time, 12), round(target - time, 12)))
        calls.append((round(time, 12), round(dt, 12)))
        time += dt
    return calls


@pytest.mark.parametrize("dts,end,freq", [([0.03, 0.031, 0.029, 0.05, 0.02], 0.3, 0.1),
                                          ([0.07], 1.0, 0.25), ([0.1, 0.2, 0.05], 0.45, 1.0)])
def test_output_window_loop_matches_forward_euler(monkeypatch, dts, end, freq):
    import pyexner_b200.integrators as I

    monkeypatch.setattr(I, "check_state", lambda *a: None)
    b = _FakeBundle(dts)
    cfg = IntegratorConfig(cfl=0.5, end_time=end, out_freq=freq, solver_config=type("C", (), {"mpi_handler": None})(),
                           solver_bundle=b)
    _run_time_loop(object(), cfg, None, None, None, ssprk2=False)
    assert b.calls == _reference_loop(dts, end, freq)


def test_dambreak_case_files(tmp_path):
    params = _dambreak_case(tmp_path, "fp64")
    with open(tmp_path / "input.yaml") as f:
        assert yaml.safe_load(f)["boundaries"].keys() == params["boundaries"].keys()
    io = pio.NetCDFStateIO(str(tmp_path / "input.nc"))
    assert io.generate_mesh().local_shape == (41, 41)


def test_netcdf_roundtrip(tmp_path):
    x = np.arange(-1.0, 1.0 + 1e-9, 0.1)
    y = np.arange(-0.5, 0.5 + 1e-9, 0.1)
    rng = np.random.default_rng(0)
    fields = {k: rng.random((len(y), len(x))) for k in ("h", "hu", "hv", "z", "z_b", "n")}
    p = tmp_path / "in.nc"
    pio.write_input(str(p), x, y, fields)
    io = pio.NetCDFStateIO(str(p))
    mesh = io.generate_mesh()
    assert mesh.local_shape == (len(y), len(x))
    assert mesh.dh == 0.1
    assert np.allclose(mesh.local_X[0], x + 0.05)
    from pyexner_b200.state import RoeExnerState

    st = io.read_state(RoeExnerState, mesh, {"erosion": {"grass_factor": 0.01}}, dtype=torch.float64, device="cpu")
    assert np.array_equal(st.h.numpy(), fields["h"].astype(np.float32).astype(np.float64))
    assert np.all(st.G.numpy() == 0.01)


def _dambreak_case(tmp_path, precision):
    dh = 0.1
    x = np.round(np.arange(-2.0, 2.0 + dh / 2, dh), 6)
    y = x.copy()
    X, Y = np.meshgrid(x, y, indexing="xy")
    h = np.where(X**2 + Y**2 <= 0.5**2, 1.0, 0.2)
    fields = dict(h=h, hu=np.zeros_like(h), hv=np.zeros_like(h), z=np.ones_like(h), z_b=np.ones_like(h),
                  n=np.zeros_like(h))
    pio.write_input(str(tmp_path / "input.nc"), x, y, fields)
    lo, hi = x[0] + dh / 2, x[-1] + dh / 2
    ylo, yhi = y[0] - dh / 2, y[-1] - dh / 2

    def rect(x0, x1, y0, y1):
        x0, x1, y0, y1 = (float(v) for v in (x0, x1, y0, y1))
        return [[x0, y0], [x1, y0], [x1, y1], [x0, y1]]

    e = 0.5 * dh
    bnd = {
        "outlet1": {"type": "Reflective", "polygon": rect(lo - e, lo + e, ylo - e, yhi + e), "values": [0, 0, 0, 0],
                    "normal": [-1.0, 0.0]},
        "outlet2": {"type": "Reflective", "polygon": rect(hi - e, hi + e, ylo - e, yhi + e), "values": [0, 0, 0, 0],
                    "normal": [1.0, 0.0]},
        "outlet3": {"type": "Reflective", "polygon": rect(lo - e, hi + e, ylo - e, ylo + e), "values": [0, 0, 0, 0],
                    "normal": [0.0, -1.0]},
        "outlet4": {"type": "Reflective", "polygon": rect(lo - e, hi + e, yhi - e, yhi + e), "values": [0, 0, 0, 0],
                    "normal": [0.0, 1.0]},
    }
    params = dict(end_time=0.12, out_freq=0.05, cfl=0.5, flux_scheme="Roe Exner", integrator="Forward Euler",
                  parNx=1, parNy=1, input_file="input.nc", output_file="output.nc",
                  erosion={"grass_factor": 0.01}, boundaries=bnd, precision=precision)
    with open(tmp_path / "input.yaml", "w") as f:
        yaml.safe_dump(params, f)
    return params


@pytest.mark.gpu
def test_run_driver_dambreak_matches_oracle(tmp_path):
    """run_driver on a reference-format input (YAML + NetCDF3) against the oracle running the
    same Forward-Euler output windows; output frames land in the NetCDF file."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from scipy.io import netcdf_file

    from oracle import boundaries as OB
    from oracle import roe_exner as ORE
    from pyexner_b200 import build, run_driver

    build.build()
    params = _dambreak_case(tmp_path, "fp64")
    state, (X, Y) = run_driver(str(tmp_path / "input.yaml"))
    got = state.to_numpy()

    io = pio.NetCDFStateIO(str(tmp_path / "input.nc"))
    mesh = io.generate_mesh()
    with netcdf_file(str(tmp_path / "input.nc"), "r", mmap=False) as f:
        st = {k: np.array(f.variables[k][:], dtype=np.float32).astype(np.float64)
              for k in ("h", "hu", "hv", "z", "z_b", "n")}
    st["G"] = 0.01 * np.ones_like(st["h"])
    st["n_b"] = np.zeros_like(st["h"])
    st["seds"] = np.zeros((1, 1))
    bcs = OB.Boundaries("Roe Exner", params["boundaries"], mesh.local_X, mesh.local_Y)
    mask = OB.roe_exner_mask(st["z"].copy(), bcs.boundary_mask)
    st = ORE.init(st, mask, bcs, False)
    frames = [st]
    time, dt, tol = 0.0, 0.0, 5e-7
    end, freq = params["end_time"], params["out_freq"]
    while time < end - tol:
        while time + dt < min((int(time / freq) + 1) * freq, end) - tol:
            dt = float(ORE.compute_dt(st, 0.5, mesh.dh, mask[0]))
            st = ORE.stage(st, dt, mesh.dh, mask, bcs, False)
            time += dt
        dt = float(ORE.compute_dt(st, 0.5, mesh.dh, mask[0]))
        target = min((int(time / freq) + 1) * freq, end)
        if time + dt >= target - tol:
            frames.append(ORE.stage(st, target - time, mesh.dh, mask, bcs, False))
        st = ORE.stage(st, dt, mesh.dh, mask, bcs, False)
        time += dt
    for k in ("h", "hu", "hv", "z_b", "G"):
        scale = max(np.max(np.abs(st[k])), 1e-300)
        assert np.max(np.abs(got[k] - st[k])) / scale <= 1e-10, k
    with netcdf_file(str(tmp_path / "output.nc"), "r", mmap=False) as f:
        out_h = np.array(f.variables["h"][:])
    assert out_h.shape[0] == len(frames)
    for k, fr in enumerate(frames):
        ref = np.where(mask[0], np.nan, fr["h"]).astype(np.float32)
        assert np.allclose(out_h[k], ref, rtol=1e-6, atol=1e-7, equal_nan=True), k
