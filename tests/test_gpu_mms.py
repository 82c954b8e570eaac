"""Scalar libraries on the GPU (anb_scalar_elliptic_solve / anb_scalar_transport_solve): the
reference's observed MMS convergence orders (tests/golden/mms_orders.json, made from the
reference's own libpoisson / libscalar assembly) reproduced by the CUDA path, per-cell parity with
the oracle, the reference's error behaviour, and the SIMPLE state surviving a scalar solve."""
import json
from pathlib import Path

import numpy as np
import pytest

import anabasis_b200 as anb
import oracle
from anabasis_b200 import scalar as S
from oracle import mms
from tests import mms_cases as M
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "mms_orders.json").read_text())


@pytest.mark.parametrize("label", [s[0] for s in M.SEQUENCES])
def test_gpu_mms_reproduces_reference_orders(label):
    seq = GOLDEN["sequences"][label]
    for prob in M.PROBLEMS:
        errs = []
        for lvl, n in enumerate(seq["sizes"]):
            m = M.unit_cube(n, jitter=seq["jitter"], seed=GOLDEN["seed"], tets=seq["tets"])
            geo = M.geometry(m)
            p = M.problem(prob, geo)
            phi, info = M.gpu_solve(anb.Solver(m), p)
            assert info["converged"] == 1, (label, prob, n, info)
            e = mms.error_norms(phi, p["exact"], geo["vol"])
            g = seq["problems"][prob]["levels"][lvl]
            for k in ("l1", "l2", "linf"):
                assert e[k] == pytest.approx(g[k], rel=1e-6), (label, prob, n, k)
            errs.append(e["l2"])
        for o, og in zip(M.orders(errs), seq["problems"][prob]["order_l2"]):
            assert o == pytest.approx(og, abs=1e-4), (label, prob)


@pytest.mark.parametrize("tets", [False, True])
def test_gpu_scalar_solution_matches_oracle(tets):
    m = M.unit_cube(5 if tets else 12, jitter=0.15, seed=11, tets=tets)
    geo = M.geometry(m)
    asm = mms.OracleAssembler(oracle.Oracle(m.topology()), m.topology())
    s = anb.Solver(m)
    for prob in M.PROBLEMS:
        p = M.problem(prob, geo)
        ref = M.oracle_solve(asm, p)
        phi, _ = M.gpu_solve(s, p)
        assert np.abs(phi - ref).max() <= 1e-9 * np.abs(ref).max(), prob


def test_gpu_scalar_api_mirror_and_errors():
    m = M.unit_cube(8)
    sm = S.ScalarMesh(m)
    bcs = S.ScalarBCSet([S.make_dirichlet_patch_bc(nm, lambda x, n: M.sin3(x)) for nm in sm.patch_names])
    src = 3.0 * M.PI ** 2 * M.sin3(sm.cc)
    opts = S.EllipticOptions(nNonOrthCorr=1)
    opts.hypre.absTol = 1e-12
    r = S.solve_poisson(sm, src, bcs, opts)
    assert r.iterations > 0 and r.finalRelResNorm < 1e-8
    assert mms.error_norms(r.phi, M.sin3(sm.cc), sm.vol)["l2"] < 2e-2
    neu = S.ScalarBCSet([S.make_neumann_constant_bc(nm, 0.0) for nm in sm.patch_names])
    with pytest.raises(anb.AnbError, match="Pure-Neumann scalar elliptic problem needs useReferenceCell=true"):
        S.solve_poisson(sm, src, neu, S.EllipticOptions())
    with pytest.raises(anb.AnbError, match="Invalid reference cell"):
        S.solve_poisson(sm, src, neu, S.EllipticOptions(useReferenceCell=True, referenceCell=m.n_cells))
    with pytest.raises(RuntimeError, match="Su must have size mesh.nCells"):
        S.solve_steady_scalar_transport(sm, S.ScalarTransportInputs(np.zeros(m.n_faces), np.ones(m.n_faces),
                                                                     np.zeros(3), np.zeros(m.n_cells)),
                                        bcs, S.ScalarTransportOptions())


def test_simple_state_survives_scalar_solve():
    """A scalar solve on a SIMPLE context leaves U, p untouched and the next steps identical."""
    m, bc, _ = channel(nx=16, ny=6, nz=6, jitter=0.1, seed=4, obstacle=False)
    u, v, w, p = initial_state(m, bc)
    prm = anb.default_params(mu=1e-3, u_relax=0.7, p_relax=0.3)
    a, b = anb.Solver(m, prm), anb.Solver(m, prm)
    for s in (a, b):
        s.set_bc(bc)
        s.set_state(u, v, w, p)
        s.iterate(2)
    before = a.get_state()
    geo = M.geometry(m)
    q = M.problem("poisson_dirichlet", geo)
    a.scalar_elliptic_solve(q["src"], q["bt"], q["bv"], nonorth_corr=2, abs_tol=1e-12)
    q = M.problem("transport_upwind_mixed", geo)
    M.gpu_solve(a, q)
    after = a.get_state()
    for k in ("u", "v", "w", "p", "phi"):
        assert np.array_equal(before[k], after[k]), k
    # a rebuilds its pressure AMG from the current matrix, b keeps refreshing the first one: the
    # preconditioners differ, so the fields agree to the inner-solver tolerance, not bitwise
    a.iterate(3)
    b.iterate(3)
    sa, sb = a.get_state(), b.get_state()
    uscale = max(np.abs(sb[k]).max() for k in ("u", "v", "w"))
    for k in ("u", "v", "w"):
        assert np.abs(sa[k] - sb[k]).max() <= 1e-6 * uscale, k
    assert np.abs(sa["p"] - sb["p"]).max() <= 1e-6 * np.abs(sb["p"]).max()
