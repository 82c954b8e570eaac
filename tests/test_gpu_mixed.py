"""Mixed-precision SIMPLE (ANB_PRECISION_MIXED): FP32 matrices and FP32 BiCGSTAB / AMG-PCG inner
solves inside FP64 defect correction, FP64 face loops, residuals, flux update and forces.

The mixed method solves the same discrete equations up to the FP32 rounding of the matrix
coefficients (relative 6e-8), so its fields track the FP64 method closely and its converged
patch force must agree to 1e-6 relative (the precision bar of the mixed method)."""
import numpy as np
import pytest

import anabasis_b200 as anb
import oracle
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=2)


def _run(m, bc, state, precision, nsteps, tol_mass=-1.0, tol_vel=-1.0):
    s = anb.Solver(m, anb.default_params(precision=precision, **PRM))
    s.set_bc(bc)
    s.set_state(*state)
    _, st = s.iterate(nsteps, tol_mass, tol_vel)
    names = m.topology()["patch_names"]
    k = names.index("patch_3_0") if "patch_3_0" in names else 0
    return s.get_state(), s.patch_force(k, -1), len(st), st


def _scale(st):
    return max(np.abs(st[k]).max() for k in ("u", "v", "w"))


def test_mixed_tracks_fp64_step_by_step():
    m, bc, _ = channel(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True)
    init = initial_state(m, bc)
    a, fa, _, sa = _run(m, bc, init, 0, 20)
    b, fb, _, sb = _run(m, bc, init, 1, 20)
    us = _scale(a)
    for k in ("u", "v", "w"):
        assert np.abs(a[k] - b[k]).max() <= 1e-5 * us, k
    assert np.abs(a["p"] - b["p"]).max() <= 1e-5 * np.abs(a["p"]).max()
    for q in ("Fp", "Fv", "F"):
        assert np.abs(np.array(fa[q]) - np.array(fb[q])).max() <= 1e-5 * np.abs(fa["F"]).max(), q
    # every step's linear solves converged in both methods
    assert all(x["status"] == 0 for x in sa) and all(x["status"] == 0 for x in sb)


def test_mixed_against_oracle():
    m, bc, _ = channel(nx=12, ny=6, nz=6, jitter=0.15, seed=3, obstacle=False)
    init = initial_state(m, bc)
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    ref, _ = o.run(oracle.params(p_tol=1e-13, vel_tol=1e-13, **PRM), 8, *init)
    s = anb.Solver(m, anb.default_params(precision=1, p_tol=1e-13, vel_tol=1e-13, **PRM))
    s.set_bc(bc)
    s.set_state(*init)
    s.iterate(8)
    g = s.get_state()
    us = _scale(ref)
    for k in ("u", "v", "w"):
        assert np.abs(g[k] - ref[k]).max() <= 1e-5 * us, k
    assert np.abs(g["p"] - ref["p"]).max() <= 1e-5 * np.abs(ref["p"]).max()


def test_mixed_converged_force_within_1e6():
    """FP64 run to convergence (continuity 1e-9, velocity change 1e-9); the mixed run for the same
    number of steps: patch force and fields agree to 1e-6.  The mixed method cannot itself reach a
    1e-9 velocity change: the FP32 rounding of the re-assembled matrix coefficients leaves a
    step-to-step noise floor near 1e-8."""
    m, bc, _ = channel(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True)
    init = initial_state(m, bc)
    a, fa, da, _ = _run(m, bc, init, 0, 3000, 1e-9, 1e-9)
    assert da < 3000
    b, fb, db, sb = _run(m, bc, init, 1, da + 20)
    assert sb[-1]["mass_res"] < 1e-9
    F = np.array(fa["F"])
    assert np.abs(np.array(fb["F"]) - F).max() <= 1e-6 * np.abs(F).max()
    us = _scale(a)
    for k in ("u", "v", "w"):
        assert np.abs(a[k] - b[k]).max() <= 1e-6 * us, k


def test_fp64_only_entry_points_refuse_mixed_context():
    m, bc, _ = channel(nx=8, ny=4, nz=4)
    s = anb.Solver(m, anb.default_params(precision=1, **PRM))
    s.set_bc(bc)
    n = m.n_cells
    with pytest.raises(anb.AnbError, match="needs an FP64"):
        s.debug_pressure_solve(np.ones(n), np.zeros(n))
    with pytest.raises(anb.AnbError, match="needs an FP64"):
        s.scalar_elliptic_solve(np.ones(n), np.zeros(m.n_faces, np.int32), np.zeros(m.n_faces))
