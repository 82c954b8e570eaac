"""The C ABI: libanb.so loads and exports every function include/*.h declares (no GPU needed)."""
import ctypes as ct
import re
import types
from pathlib import Path

import numpy as np
import pytest

import anabasis_b200 as anb
import oracle

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(anb_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 25
    lib = anb.lib()
    for n in sorted(names):
        assert hasattr(lib, n), n
        assert n in anb.SIGNATURES, f"{n} has no ctypes signature"


def test_signatures_only_for_declared_symbols():
    assert set(anb.SIGNATURES) <= declared_functions()


def test_library_entry_points_without_gpu():
    lib = anb.lib()
    p = anb.Params()
    lib.anb_default_params(ct.byref(p))
    # reference defaults, main.cu:73-103
    assert (p.mu, p.u_relax, p.p_relax, p.n_nonorth_corr, p.vel_maxit, p.p_maxit) == (0.05, 0.7, 1.0, 2, 100, 4000)
    assert (p.vel_tol, p.p_tol, p.corr_tol, p.p_amg_rebuild_every) == (1e-10, 1e-10, 1e-12, 1)
    # invalid arguments are rejected before any device work
    assert lib.anb_create(None, None, None) == anb.ANB_ERR_INVALID
    assert lib.anb_set_state(None, None, None, None, None) == anb.ANB_ERR_INVALID
    assert lib.anb_launch_count() >= 0


def test_oracle_loads():
    assert oracle.lib() is not None


def test_get_state_refills_caller_arrays(monkeypatch):
    """Solver.get_state(out=...) hands the caller's arrays to anb_get_state (no GPU: the library call
    is replaced by a recorder) and rejects arrays of the wrong size."""
    seen = []

    class Recorder:
        def anb_get_state(self, h, u, v, w, p, phi):
            seen.append((u, phi))
            return 0

    monkeypatch.setattr(anb, "lib", lambda: Recorder())
    fake = types.SimpleNamespace(n_cells=5, n_faces=7, _h=None, _check=lambda rc: None)
    first = anb.Solver.get_state(fake)
    assert first["u"].shape == (5,) and first["phi"].shape == (7,)
    again = anb.Solver.get_state(fake, with_phi=False, out=first)
    assert again is first and again["phi"] is None
    assert seen[1][0].contents is not None and seen[1][1] is None
    with pytest.raises(ValueError):
        anb.Solver.get_state(fake, out=dict(u=np.zeros(4), v=np.zeros(5), w=np.zeros(5), p=np.zeros(5)))
