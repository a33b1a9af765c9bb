"""Callback schedules, evolve's firing plan and the HDF5 layout, on the CPU.

The schedules and evolve's firing/progress steps are checked against what the
reference's own ``callbacks.py`` / ``integrators.evolve`` produced on the same
cases (``tests/golden/reference_aux.npz``, made by ``make_golden.py``); the
HDF5 writers against the reference's key layout (src/hit3d/schema.py:30-57)
through the in-memory ``h5py`` stand-in ``h5stub``."""

import contextlib
import io
import os
import sys

import numpy as np
import pytest
import torch

from conftest import REPO

AUX = os.path.join(REPO, "tests", "golden", "reference_aux.npz")


@pytest.fixture(scope="module")
def aux():
    return dict(np.load(AUX))


@pytest.fixture
def h5(monkeypatch):
    import h5stub
    monkeypatch.setitem(sys.modules, "h5py", h5stub)
    return h5stub


def _cases(aux, prefix):
    return sorted({k.split("/")[0] for k in aux if k.startswith(prefix)})


def test_time_schedules_match_reference(h3, aux, h5, tmp_path):
    for c in _cases(aux, "sched"):
        every_time, warm, dt, t0, n = aux[f"{c}/case"]
        n = int(n)
        fw = h3.FieldWriter(str(tmp_path / "s.h5"), every_time=every_time, warmup_time=None if warm < 0 else warm)
        cb = h3.Callback(lambda s: None, every_time=every_time)
        got_fw = [k for k in range(n + 1) if fw.is_due(k, t0 + k * dt, dt)]
        got_cb = [k for k in range(n + 1) if cb.is_due(k, t0 + k * dt, dt)]
        assert got_fw == aux[f"{c}/fieldwriter"].tolist(), c
        assert got_cb == aux[f"{c}/callback"].tolist(), c


def test_evolve_firing_and_progress_steps_match_reference(h3, aux):
    """evolve with a trivial RHS on CPU tensors: which steps fire the
    callbacks and which print a progress line."""
    grid = type("G", (), {"Nx": 8, "Ny": 8, "Nz": 8, "Lx": 1.0, "Ly": 1.0, "Lz": 1.0})()

    def rhs(u, p, t):
        return torch.zeros_like(u)

    for c in _cases(aux, "evolve"):
        nsteps, dt, every, every_time, progress = aux[f"{c}/case"]
        nsteps, every = int(nsteps), int(every)
        progress = True if progress == -1.0 else (False if progress == 0 else int(progress))
        seen = {"cb": [], "diag": []}
        cb = (h3.Callback(lambda s: seen["cb"].append(s.step), every_time=every_time) if every_time > 0
              else h3.Callback(lambda s: seen["cb"].append(s.step), every=every))
        diag = h3.Diagnostic(lambda s: (seen["diag"].append(s.step), 0.0)[1], every=every)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            h3.evolve(rhs, torch.zeros(3, 8, 8, 5, dtype=torch.complex128), h3.NSParams(nu=0.05), grid, float(dt),
                      nsteps, callbacks=(cb, diag), progress=progress)
        printed = [int(line.split()[1].split("/")[0]) for line in buf.getvalue().splitlines() if line.strip()]
        assert seen["cb"] == aux[f"{c}/callback_steps"].tolist(), c
        assert seen["diag"] == aux[f"{c}/diagnostic_steps"].tolist(), c
        assert printed == aux[f"{c}/progress_steps"].tolist(), c
        assert len(diag.values) == len(seen["diag"]) and len(diag.times) == len(seen["diag"])


def test_progress_line_tokens(h3):
    """The progress line carries the fields the reference's test reads."""
    grid = type("G", (), {})()
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        h3.evolve(lambda u, p, t: torch.zeros_like(u), torch.zeros(3, 4, 4, 3, dtype=torch.complex64),
                  h3.NSParams(nu=0.0), grid, 1e-3, 10, progress=5)
    out = buf.getvalue()
    assert out.count("\n") == 2
    assert "step 10/10 (100%)" in out and "t = " in out and "eta " in out


def _state(h3, step, t, u, grid=None):
    grid = grid or type("G", (), {"Nx": 4, "Ny": 4, "Nz": 4, "Lx": 6.0, "Ly": 6.5, "Lz": 7.0})()
    return h3.State(u_hat=u, t=t, step=step, params=h3.NSParams(nu=0.05), grid=grid)


def test_fieldwriter_and_series_layout(h3, h5, tmp_path):
    """Keys and values of the reference layout: grid/*, step_<8 digits>/{t,
    u_hat}, series/<name>/{t, <key>} for dict values and series/<name>/
    {t, values} for scalars."""
    path = str(tmp_path / "run" / "snap.h5")
    fw = h3.FieldWriter(path, every=2)
    us = [torch.full((3, 4, 4, 3), float(k), dtype=torch.complex64) for k in range(3)]
    for k, u in enumerate(us):
        fw.fire(_state(h3, 2 * k, 0.1 * k, u))
    fw.finalize()
    d = h3.Diagnostic(lambda s: {"E": torch.tensor(1.0 + s.step), "eps": 2.0 * s.step}, path=path, name="budget")
    e = h3.Diagnostic(lambda s: 3.0 * s.step, path=path, name="energy")
    for k in range(4):
        d.fire(_state(h3, k, 0.5 * k, us[0]))
        e.fire(_state(h3, k, 0.5 * k, us[0]))
    d.finalize()
    e.finalize()
    with h5.File(path, "r") as f:
        assert sorted(k for k in f if k.startswith("step_")) == ["step_00000000", "step_00000002",
                                                                    "step_00000004"]
        assert f["grid/Nx"][()] == 4 and f["grid/Lz"][()] == 7.0 and f["grid/nu"][()] == 0.05
        assert f["step_00000004/t"][()] == pytest.approx(0.2)
        np.testing.assert_array_equal(f["step_00000002/u_hat"][()], us[1].numpy())
        assert sorted(f["series"].keys()) == ["budget", "energy"]
        np.testing.assert_allclose(f["series/budget/t"][()], [0.0, 0.5, 1.0, 1.5])
        np.testing.assert_allclose(f["series/budget/E"][()], [1.0, 2.0, 3.0, 4.0])
        np.testing.assert_allclose(f["series/budget/eps"][()], [0.0, 2.0, 4.0, 6.0])
        np.testing.assert_allclose(f["series/energy/values"][()], [0.0, 3.0, 6.0, 9.0])
    with pytest.raises(ValueError):  # a series is saved once per file
        h3.save_series(path, "energy", e)


def test_fieldwriter_overwrite(h3, h5, tmp_path):
    path = str(tmp_path / "snap.h5")
    fw = h3.FieldWriter(path, every=1)
    fw.fire(_state(h3, 0, 0.0, torch.zeros(3, 4, 4, 3, dtype=torch.complex64)))
    fw.finalize()
    assert os.path.exists(path)
    h3.FieldWriter(path, overwrite=False)
    assert os.path.exists(path)
    h3.FieldWriter(path)
    assert not os.path.exists(path)


def test_diagnostic_file_needs_name(h3):
    with pytest.raises(ValueError):
        h3.Diagnostic(lambda s: 0.0, path="somewhere.h5")


def test_writers_need_h5py(h3, monkeypatch, tmp_path):
    monkeypatch.setitem(sys.modules, "h5py", None)  # import h5py -> ImportError
    with pytest.raises(ImportError):
        h3.FieldWriter(str(tmp_path / "x.h5"))
