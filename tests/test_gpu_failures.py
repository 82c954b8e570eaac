"""Failure behaviour, detected on the host without any GPU fault: an inner solve that hits its
iteration cap is a warning and the iteration goes on (the reference warns on HYPRE error 256 and
continues, main.cu:2660-2670); a non-finite continuity residual stops the run with
ANB_ERR_DIVERGED; misuse of the API returns an error and leaves the context usable."""
import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu
PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3)


def test_inner_iteration_cap_warns_and_continues():
    m, bc, _ = channel(nx=16, ny=6, nz=6, jitter=0.1, seed=1)
    s = anb.Solver(m, anb.default_params(p_maxit=1, **PRM))
    s.set_bc(bc)
    s.set_state(*initial_state(m, bc))
    rc, st = s.iterate(3)
    assert rc == anb.ANB_NOT_CONVERGED
    assert len(st) == 3 and all(x["status"] == anb.ANB_NOT_CONVERGED for x in st)
    assert all(np.isfinite(x["mass_res"]) for x in st)


def test_non_finite_state_is_reported_as_divergence():
    m, bc, _ = channel(nx=12, ny=6, nz=6)
    s = anb.Solver(m, anb.default_params(p_maxit=20, vel_maxit=20, **PRM))
    s.set_bc(bc)
    u, v, w, p = initial_state(m, bc)
    u = u.copy()
    u[5] = np.nan
    s.set_state(u, v, w, p)
    rc, st = s.iterate(5)
    assert rc == anb.ANB_ERR_DIVERGED and len(st) == 1
    assert "diverged" in anb.lib().anb_last_error(s._h).decode()
    # the context stays usable: a clean state runs again (the iteration caps of 20 used here may
    # leave the inner solves short of their tolerance, which is only a warning)
    s.set_state(*initial_state(m, bc))
    rc, st = s.iterate(2)
    assert rc in (anb.ANB_OK, anb.ANB_NOT_CONVERGED) and len(st) == 2
    assert np.isfinite(st[-1]["mass_res"]) and np.isfinite(st[-1]["du_rel"])
    g = s.get_state()
    assert all(np.isfinite(g[k]).all() for k in ("u", "v", "w", "p", "phi"))


def test_api_misuse_returns_errors():
    m, bc, _ = channel(nx=8, ny=4, nz=4)
    s = anb.Solver(m, anb.default_params(**PRM))
    with pytest.raises(anb.AnbError, match="boundary conditions not set"):
        s.iterate(1)
    s.set_bc(bc)
    with pytest.raises(anb.AnbError, match="state not set"):
        s.iterate(1)
    s.set_state(*initial_state(m, bc))
    assert s.patch_force(99)["valid"] == 0
    with pytest.raises(anb.AnbError, match="invalid patch index"):
        s.force_objective(99)
    rc, _ = s.iterate(1)
    assert rc == anb.ANB_OK
