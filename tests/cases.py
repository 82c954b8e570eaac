"""Synthetic channel cases shared by the tests (shapes of the benchmark configurations, scaled down).

Channel box 2.5 x 0.41 x 0.41 with patch_0_0 walls, patch_1_0 inlet (x = 0), patch_2_0 outlet
(x = 2.5) and patch_3_0 obstacle; boundary conditions as the benchmark case: parabolic box inlet
H = 0.41, Umax = 0.45 along the inward average patch normal, outlet p fixed_value and U
zero_gradient, no-slip walls (reference cases/cylinder.case without its extra wall patch).
"""
from __future__ import annotations

import os
import tempfile
from pathlib import Path

import numpy as np

import anabasis_b200 as anb

BC_TEXT = """# channel benchmark boundary conditions
velocity patch_0_0 wall_noslip
velocity patch_1_0 parabolic_box_inlet 0.41 0.45 y z average_patch_normal
velocity patch_2_0 zero_gradient
pressure patch_0_0 zero_gradient
pressure patch_1_0 zero_gradient
pressure patch_2_0 fixed_value {pout}
"""
BC_OBSTACLE = "velocity patch_3_0 wall_noslip\npressure patch_3_0 zero_gradient\n"

_TMP = Path(tempfile.mkdtemp(prefix="anb_cases_"))


def channel(nx, ny, nz, jitter=0.0, seed=0, obstacle=False, tets=False, pout=0.0):
    """Returns (HostMesh, bc dict, polyMesh dir) for a channel case."""
    m = anb.HostMesh.channel(nx, ny, nz, jitter=jitter, seed=seed, obstacle=obstacle, tets=tets)
    d = _TMP / f"ch_{nx}_{ny}_{nz}_{jitter}_{seed}_{int(obstacle)}_{int(tets)}_{pout}"
    d.mkdir(parents=True, exist_ok=True)
    bcf = d / "case.bc"
    bcf.write_text(BC_TEXT.format(pout=pout) + (BC_OBSTACLE if obstacle else ""))
    bc = m.evaluate_bc(bcf)
    return m, bc, d


def initial_state(m, bc):
    """Mean inlet velocity everywhere, p = 0 (reference main.cu:3302-3322)."""
    t = m.topology()
    k = t["patch_names"].index("patch_1_0")
    sl = slice(int(t["patch_start"][k]), int(t["patch_start"][k] + t["patch_size"][k]))
    C = m.n_cells
    return (np.full(C, bc["u"][sl].mean()), np.full(C, bc["v"][sl].mean()), np.full(C, bc["w"][sl].mean()),
            np.zeros(C))


def random_state(m, seed=0):
    rng = np.random.default_rng(seed)
    C = m.n_cells
    u = 0.3 + 0.05 * rng.standard_normal(C)
    v = 0.05 * rng.standard_normal(C)
    w = 0.05 * rng.standard_normal(C)
    p = 0.01 * rng.standard_normal(C)
    return u, v, w, p


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)
