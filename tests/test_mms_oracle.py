"""Scalar libraries on the CPU: the oracle's restatement (oracle.cpp orc_scalar_*) against the
reference's own libpoisson / libscalar host functions (oracle/_ref/libscalarref.so), the oracle's
MMS error norms against the committed reference orders (tests/golden/mms_orders.json), and the
host-side BC mirror of anabasis_b200.scalar."""
import json
import tempfile
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

import oracle
from anabasis_b200 import scalar as S
from oracle import mms
from tests import mms_cases as M
from tests import refshim

needs_ref = pytest.mark.skipif(not refshim.scalar_available(), reason="reference scalar shim not built")
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "mms_orders.json").read_text())


def _mesh(kind):
    if kind == "hex":
        return M.unit_cube(6, jitter=0.15, seed=7)
    return M.unit_cube(3, jitter=0.1, seed=7, tets=True)


@needs_ref
@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("prob", M.PROBLEMS)
def test_scalar_assembly_matches_reference(kind, prob):
    m = _mesh(kind)
    d = Path(tempfile.mkdtemp())
    m.write(d)
    geo = M.geometry(m)
    p = M.problem(prob, geo)
    if p["transport"]:  # also exercise ZeroGradient on the outlet
        s = geo["start"][geo["names"].index(M.OUTLET)]
        p["bt"][s:s + geo["size"][geo["names"].index(M.OUTLET)]] = 2
    ref = refshim.RefScalar(d)
    asm = mms.OracleAssembler(oracle.Oracle(m.topology()), m.topology())
    rng = np.random.default_rng(5)
    phi = p["exact"] + 0.05 * rng.standard_normal(m.n_cells)
    ga = asm.gradient(p["transport"], p["bt"], p["bv"], phi)
    gr = ref.gradient(p["transport"], p["bt"], p["bv"], phi)
    assert np.abs(ga - gr).max() <= 1e-13 * np.abs(gr).max()
    args = (p["transport"], p.get("upwind", False), p["nonorth"], p["gamma"], p["src"], p.get("sp"), p.get("flux"),
            p["bt"], p["bv"], gr, p.get("ref_cell", -1), p.get("ref_value", 0.0))
    Aa, ba = asm.system(*args)
    Ar, br = ref.system(*args)
    assert abs(Aa - Ar).max() <= 1e-14 * abs(Ar).max()
    assert np.abs(ba - br).max() <= 1e-14 * np.abs(br).max()


@needs_ref
def test_reference_patterns_agree():
    m = _mesh("tet")
    d = Path(tempfile.mkdtemp())
    m.write(d)
    ref = refshim.RefScalar(d)
    ro, co = ref.transport_pattern()
    assert np.array_equal(ro, ref.row_off) and np.array_equal(co, ref.cols)


@pytest.mark.parametrize("label", [s[0] for s in M.SEQUENCES])
def test_oracle_mms_norms_match_reference_orders(label):
    """Oracle error norms on the two coarser meshes equal the reference's (golden) ones."""
    seq = GOLDEN["sequences"][label]
    for prob in M.PROBLEMS:
        for lvl, n in enumerate(seq["sizes"][:2]):
            m = M.unit_cube(n, jitter=seq["jitter"], seed=GOLDEN["seed"], tets=seq["tets"])
            geo = M.geometry(m)
            p = M.problem(prob, geo)
            phi = M.oracle_solve(mms.OracleAssembler(oracle.Oracle(m.topology()), m.topology()), p)
            e = mms.error_norms(phi, p["exact"], geo["vol"])
            g = seq["problems"][prob]["levels"][lvl]
            for k in ("l1", "l2", "linf"):
                assert e[k] == pytest.approx(g[k], rel=1e-9), (label, prob, n, k)


def test_golden_orders_are_the_expected_discretisation_orders():
    """Second order for the Laplacians and central convection on hex meshes, first order upwind."""
    hexo = GOLDEN["sequences"]["hex"]["problems"]
    for prob in ("poisson_dirichlet", "poisson_neumann", "poisson_mixed", "transport_central"):
        assert hexo[prob]["order_l2"][-1] == pytest.approx(2.0, abs=0.05)
    assert 0.7 < hexo["transport_upwind_mixed"]["order_l2"][-1] < 1.1


def _fake_mesh():
    names = ["walls", "inlet", "outlet"]
    return SimpleNamespace(patch_names=names, patch_start=np.array([4, 6, 7]), patch_size=np.array([2, 1, 1]),
                           n_faces=8, xf=np.arange(24, dtype=float).reshape(8, 3), nf=np.ones((8, 3)))


def test_boundary_face_data_mirror():
    m = _fake_mesh()
    bcs = S.ScalarBCSet([S.make_dirichlet_constant_bc("walls", 2.0), S.make_neumann_constant_bc("inlet", -1.0),
                         S.make_dirichlet_patch_bc("outlet", lambda x, n: x[:, 0])])
    t, v = S.build_boundary_face_data(m, bcs)
    assert list(t[4:]) == [0, 0, 1, 0] and list(v[4:]) == [2.0, 2.0, -1.0, 21.0]
    with pytest.raises(RuntimeError, match="No BC supplied for patch 'outlet'"):
        S.build_boundary_face_data(m, S.ScalarBCSet(bcs.patches[:2]))
    with pytest.raises(RuntimeError, match="No scalar BC provided for patch 'outlet'"):
        S.build_boundary_face_data(m, S.ScalarBCSet(bcs.patches[:2]), "libscalar")
    with pytest.raises(RuntimeError, match="BC evaluator missing for patch 'walls'"):
        S.build_boundary_face_data(m, S.ScalarBCSet([S.ScalarPatchBC("walls")] + bcs.patches[1:]))
    zg = S.ScalarBCSet([S.make_zero_gradient_patch_bc("walls")] + bcs.patches[1:])
    t, v = S.build_boundary_face_data(m, zg, "libscalar")
    assert list(t[4:6]) == [2, 2] and list(v[4:6]) == [0.0, 0.0]
