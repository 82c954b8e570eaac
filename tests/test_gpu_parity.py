"""B200 library vs the CPU oracle on the same seeded inputs (FP64 plain method).

Tolerances: single-stage kernels 1e-12 relative to the field's max magnitude (FMA contraction and
a different summation order are the only differences); full SIMPLE runs with inner solves
tightened to near round-off 1e-8 relative (the north-star parity bar).
"""
import numpy as np
import pytest

import anabasis_b200 as anb
import oracle
from tests.cases import channel, initial_state, random_state, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    dict(nx=12, ny=6, nz=6),
    dict(nx=16, ny=8, nz=8, jitter=0.15, seed=1),
    dict(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True),
    dict(nx=5, ny=3, nz=3, jitter=0.1, seed=4, tets=True),
]


def _pair(kw, **prm):
    m, bc, _ = channel(**kw)
    params = anb.default_params(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, **prm)
    s = anb.Solver(m, params)
    s.set_bc(bc)
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    return m, bc, s, o


@pytest.mark.parametrize("kw", CASES)
def test_gradient(kw):
    m, bc, s, o = _pair(kw)
    cc = o.geometry()["cc"].reshape(-1, 3)
    rng = np.random.default_rng(0)
    phi = np.sin(3 * cc[:, 0]) + cc[:, 1] ** 2 + 0.1 * rng.standard_normal(m.n_cells)
    for field in range(4):
        assert rel_err(s.debug_gradient(field, phi), o.gradient(field, phi)) < 1e-12


@pytest.mark.parametrize("kw", CASES)
def test_momentum_system(kw):
    m, bc, s, o = _pair(kw)
    u, v, w, p = random_state(m, 1)
    a = s.debug_momentum(u, v, w, p)
    b = o.momentum(1.0, 1e-3, 0.7, u, v, w, p)
    for k in ("diag", "a_pn", "a_np"):
        assert rel_err(a[k], b[k]) < 1e-12, k
    # rAU = V / aP: a random velocity field makes aP a difference of convective terms, so its
    # rounding error is bounded by the sum of |terms|, not by |aP|; compare per cell on that scale
    terms = np.abs(a["diag"]) + 4 * np.abs(a["a_pn"]).max()
    assert np.all(np.abs(a["rau"] - b["rau"]) <= 1e-13 * np.abs(b["rau"]) * terms / np.abs(b["diag"]) + 1e-300)
    C = m.n_cells
    for q in range(3):
        assert rel_err(a["rhs"][q * C:(q + 1) * C], b["rhs"][q * C:(q + 1) * C]) < 1e-11, q


@pytest.mark.parametrize("kw", CASES)
def test_pressure_system(kw):
    m, bc, s, o = _pair(kw)
    u, v, w, p = random_state(m, 2)
    rau = 1e-3 * (1 + 0.1 * np.random.default_rng(3).random(m.n_cells))
    a = s.debug_pressure(u, v, w, p, rau)
    b = o.pressure(1.0, u, v, w, p, rau)
    for k in ("diag", "a_pn", "phi_star"):
        assert rel_err(a[k], b[k]) < 1e-12, k
    assert np.abs(a["div_star"] - b["div_star"]).max() < 1e-12 * np.abs(b["phi_star"]).max()


@pytest.mark.parametrize("kw", CASES)
def test_nonorth_divergence(kw):
    """k_nonorth_rhs alone: the divergence of the explicit non-orthogonal flux for a random rAU and
    pressure-correction gradient, against the oracle's restatement of GSV1:1538-1593."""
    m, bc, s, o = _pair(kw)
    rng = np.random.default_rng(7)
    rau = 1e-3 * (1 + 0.1 * rng.random(m.n_cells))
    grad = rng.standard_normal((3, m.n_cells))
    phi_no, div_ref = o.nonorth(rau, grad)
    div = s.debug_nonorth(rau, grad)
    assert np.abs(div - div_ref).max() <= 1e-12 * max(np.abs(phi_no).max(), 1e-300)


@pytest.mark.parametrize("amg", [1, 0])
def test_pressure_solve(amg):
    m, bc, s, o = _pair(dict(nx=40, ny=20, nz=20, jitter=0.15, seed=5), p_use_amg=amg, p_tol=1e-30,
                        p_rel_tol=1e-12, p_maxit=5000)
    u, v, w, p = random_state(m, 4)
    rau = 1e-3 * np.ones(m.n_cells)
    s.debug_pressure(u, v, w, p, rau)
    b = np.random.default_rng(5).standard_normal(m.n_cells)
    x, its, res = s.debug_pressure_solve(b, np.zeros(m.n_cells))
    assert res <= 1e-12 * np.linalg.norm(b) * 1.0001
    assert its > 0
    if amg:
        assert its < 200


@pytest.mark.parametrize("kw,steps", [(CASES[0], 20), (CASES[2], 12), (CASES[3], 10)])
def test_simple_iterations(kw, steps):
    tight = dict(vel_tol=1e-15, p_tol=1e-15, vel_maxit=5000, p_maxit=20000)
    m, bc, s, o = _pair(kw, **tight)
    u0, v0, w0, p0 = initial_state(m, bc)
    s.set_state(u0, v0, w0, p0)
    rc, st = s.iterate(steps)
    g = s.get_state()
    prm = oracle.params(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, **tight)
    ref, rst = o.run(prm, steps, u0, v0, w0, p0)
    assert len(st) == len(rst) == steps
    for k in ("u", "v", "w", "p", "phi"):
        assert rel_err(g[k], ref[k]) < 1e-8, k
    for a, b in zip(st, rst):
        assert abs(a["du_rel"] - b["du"]) <= 1e-6 * b["du"] + 1e-14


def test_patch_force():
    m, bc, s, o = _pair(CASES[2])
    u, v, w, p = random_state(m, 7)
    s.set_state(u, v, w, p)
    k = m.topology()["patch_names"].index("patch_3_0")
    a = s.patch_force(k, -1)
    b = o.patch_force(k, -1, 1e-3, u, v, w, p)
    assert a["valid"] == 1 and a["n_faces"] == int(b[10])
    assert rel_err(np.array(a["Fp"] + a["Fv"] + a["F"] + [a["area"]]), b[:10]) < 1e-12
