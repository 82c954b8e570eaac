"""Steady sensitivities on the GPU: the steady residual R of the SIMPLE fixed point, its tangent
(J v) against central differences of R, its adjoint (J^T w) by the dot-product identity, Newton
convergence, and the adjoint gradient of the obstacle force against the tangent-linear model and
against central finite differences of converged solutions."""
import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=2, p_tol=1e-13, vel_tol=1e-13)


def _case(steps=400, **kw):
    geo = dict(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True)
    geo.update(kw)
    m, bc, _ = channel(**geo)
    s = anb.Solver(m, anb.default_params(**PRM))
    s.set_bc(bc)
    s.set_state(*initial_state(m, bc))
    s.iterate(steps, 1e-12, 1e-11)
    names = m.topology()["patch_names"]
    return m, bc, s, names.index("patch_1_0"), names.index("patch_3_0")


def _inlet_mask(m, k_in):
    t = m.topology()
    F = m.n_faces
    mask = np.zeros(F, bool)
    s0, n = int(t["patch_start"][k_in]), int(t["patch_size"][k_in])
    mask[s0:s0 + n] = True
    return mask


def _set_perturbed(s, m, bc, state, dX, dbc, dmu, h):
    C, F = m.n_cells, m.n_faces
    u, v, w, p = (state[k] + h * dX[i * C:(i + 1) * C] for i, k in enumerate("uvwp"))
    s.set_state(u, v, w, p)
    b = dict(bc)
    for i, k in enumerate("uvw"):
        b[k] = bc[k] + h * dbc[i * F:(i + 1) * F]
    s.set_bc(b)
    s.set_viscosity(PRM["mu"] + h * dmu)


def test_residual_vanishes_at_the_simple_fixed_point():
    m, bc, s, _, _ = _case()
    _, n_conv = s.steady_residual()
    s2 = anb.Solver(m, anb.default_params(**PRM))
    s2.set_bc(bc)
    s2.set_state(*initial_state(m, bc))
    s2.iterate(3)
    _, n_early = s2.steady_residual()
    assert n_conv[0] < 1e-7 * n_early[0] and n_conv[1] < 1e-7 * max(n_early[1], 1e-30) + 1e-15


def test_jvp_matches_central_differences():
    m, bc, s, k_in, _ = _case(steps=60)
    st = s.get_state(with_phi=False)
    C, F = m.n_cells, m.n_faces
    rng = np.random.default_rng(7)
    dX = rng.standard_normal(4 * C)
    dX[:3 * C] *= 0.01
    dX[3 * C:] *= 1e-4
    mask = np.tile(_inlet_mask(m, k_in), 3)
    dbc = np.where(mask, 0.01 * rng.standard_normal(3 * F), 0.0)
    dmu = 2e-4
    jv = s.debug_jvp(dX, dbc, dmu)
    h = 1e-4
    _set_perturbed(s, m, bc, st, dX, dbc, dmu, h)
    rp, _ = s.steady_residual()
    _set_perturbed(s, m, bc, st, dX, dbc, dmu, -h)
    rm, _ = s.steady_residual()
    fd = (rp - rm) / (2 * h)
    for blk in range(4):
        a, b = jv[blk * C:(blk + 1) * C], fd[blk * C:(blk + 1) * C]
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), blk


def test_vjp_dot_product_identity():
    m, bc, s, k_in, _ = _case(steps=60)
    C, F = m.n_cells, m.n_faces
    rng = np.random.default_rng(11)
    v = rng.standard_normal(4 * C)
    w = rng.standard_normal(4 * C)
    mask = np.tile(_inlet_mask(m, k_in), 3)
    dbc = np.where(mask, rng.standard_normal(3 * F), 0.0)
    dmu = 0.3
    jv = s.debug_jvp(v, dbc, dmu)
    jtw, gbc, gmu = s.debug_vjp(w)
    lhs = w @ jv
    rhs = jtw @ v + gbc @ dbc + gmu * dmu
    assert abs(lhs - rhs) <= 1e-11 * (np.abs(w) @ np.abs(jv))


def test_newton_converges_quadratically():
    m, bc, s, _, _ = _case(steps=80)
    r0 = s.steady_residual()[1]
    info = s.newton_solve(max_newton=8, tol=1e-13 * max(r0[0], 1.0))
    assert info["converged"] and info["steps"] <= 6
    assert s.steady_residual()[1][0] <= 1e-12


def _converged_force(s, k_obs, direction):
    info = s.newton_solve(max_newton=10, tol=1e-14)
    assert info["converged"]
    return s.force_objective(k_obs, direction)[0]


def test_adjoint_gradient_matches_tangent_linear_and_finite_differences():
    m, bc, s, k_in, k_obs = _case()
    direction = (1.0, 0.0, 0.0)
    J0 = _converged_force(s, k_obs, direction)
    base = s.get_state(with_phi=False)
    g, gmu, J, info = s.adjoint_force_grad(k_obs, direction)
    assert info["converged"] and J == pytest.approx(J0, rel=1e-12)
    F = m.n_faces
    mask = np.tile(_inlet_mask(m, k_in), 3)
    rng = np.random.default_rng(42)
    for trial in range(3):
        d = np.where(mask, rng.standard_normal(3 * F), 0.0)
        dmu = rng.standard_normal()
        nrm = np.sqrt(d @ d + dmu * dmu)
        d, dmu = d / nrm, dmu / nrm
        adj = g @ d + gmu * dmu
        tl, tinfo = s.tangent_linear(k_obs, direction, d, dmu)
        assert tinfo["converged"]
        assert tl == pytest.approx(adj, rel=1e-8, abs=1e-14)
        h = 1e-6
        Jpm = []
        for sg in (1.0, -1.0):
            s.set_state(base["u"], base["v"], base["w"], base["p"])
            b = dict(bc)
            for i, k in enumerate("uvw"):
                b[k] = bc[k] + sg * h * d[i * F:(i + 1) * F]
            s.set_bc(b)
            s.set_viscosity(PRM["mu"] + sg * h * dmu)
            Jpm.append(_converged_force(s, k_obs, direction))
        fd = (Jpm[0] - Jpm[1]) / (2 * h)
        assert fd == pytest.approx(adj, rel=1e-5), (trial, fd, adj)
        s.set_state(base["u"], base["v"], base["w"], base["p"])
        s.set_bc(bc)
        s.set_viscosity(PRM["mu"])


def test_torch_autograd_wrapper_matches_finite_differences():
    """SteadyForce (torch.autograd.Function): backward = the library adjoint; checked along two
    random directions against central differences of the forward (re-converged) objective."""
    import torch

    from anabasis_b200.autograd import SteadyForce, SteadyForceProblem

    m, bc, _ = channel(nx=16, ny=8, nz=8, jitter=0.1, seed=5, obstacle=True)
    s = anb.Solver(m, anb.default_params(**PRM))
    s.set_bc(bc)
    s.set_state(*initial_state(m, bc))
    t = m.topology()
    names = t["patch_names"]
    k_in = names.index("patch_1_0")
    faces = np.arange(int(t["patch_start"][k_in]), int(t["patch_start"][k_in] + t["patch_size"][k_in]))
    prob = SteadyForceProblem(solver=s, bc=bc, inlet_faces=faces, patch=names.index("patch_3_0"), simple_steps=300)
    inlet0 = torch.tensor(np.stack([bc[k][faces] for k in "uvw"]), dtype=torch.float64)
    mu0 = torch.tensor(PRM["mu"], dtype=torch.float64)
    x = inlet0.clone().requires_grad_(True)
    mu = mu0.clone().requires_grad_(True)
    J = SteadyForce.apply(x, mu, prob)
    J.backward()
    assert prob.last["adjoint"]["converged"] == 1
    rng = np.random.default_rng(3)
    h = 1e-6
    for _ in range(2):
        d = torch.tensor(rng.standard_normal(inlet0.shape))
        dm = float(rng.standard_normal()) * 1e-3
        ad = float((x.grad * d).sum() + mu.grad * dm)
        with torch.no_grad():
            Jp = SteadyForce.apply(inlet0 + h * d, mu0 + h * dm, prob)
            Jm = SteadyForce.apply(inlet0 - h * d, mu0 - h * dm, prob)
        fd = float(Jp - Jm) / (2 * h)
        assert fd == pytest.approx(ad, rel=1e-5)
