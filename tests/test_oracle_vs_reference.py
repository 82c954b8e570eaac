"""The CPU oracle (oracle/oracle.cpp) against the reference's own host functions, compiled from the
reference tree: the LSQ gradient twin (main.cu:601-618), Rhie-Chow flux (644-716), continuity
(718-728), non-orthogonal flux (744-789), flux correction (791-829), patch force (2828-2933) and
the VTU writer (975-983).  Also the committed golden vectors (tests/golden/), which carry the
same pins to machines without the reference tree."""
from pathlib import Path

import numpy as np
import pytest

import anabasis_b200 as anb
import oracle
from tests import refshim
from tests.cases import BC_OBSTACLE, BC_TEXT, random_state, rel_err

needs_ref = pytest.mark.skipif(not refshim.available(), reason="reference shim not built")
GOLDEN = Path(__file__).resolve().parent / "golden"


def _case(tmp_path, kw, pout=0.25):
    m = anb.HostMesh.channel(**kw)
    m.write(tmp_path)
    f = tmp_path / "c.bc"
    f.write_text(BC_TEXT.format(pout=pout) + (BC_OBSTACLE if kw.get("obstacle") else ""))
    m = anb.HostMesh.read(tmp_path)
    bc = m.evaluate_bc(f)
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    return m, bc, o


CASES = [dict(nx=10, ny=5, nz=5, jitter=0.15, seed=11), dict(nx=24, ny=8, nz=6, jitter=0.15, seed=2, obstacle=True),
         dict(nx=4, ny=3, nz=3, jitter=0.1, seed=5, tets=True)]


@needs_ref
@pytest.mark.parametrize("kw", CASES)
def test_oracle_kernels_match_reference_twins(tmp_path, kw):
    m, bc, o = _case(tmp_path, kw)
    ref = refshim.RefMesh(tmp_path)
    rng = np.random.default_rng(1)
    u, v, w, p = random_state(m, 3)
    rau = 1e-3 * (1 + 0.2 * rng.random(m.n_cells))
    # LSQ gradient with every field's BC set
    for field, key in enumerate("uvwp"):
        g = o.gradient(field, p)
        gr = ref.gradient(bc["type_" + key], bc[key], p)
        assert rel_err(g, gr) < 1e-14
    gp = o.gradient(3, p)
    # Rhie-Chow predicted flux and continuity
    mine = o.pressure(1.0, u, v, w, p, rau)
    rc = ref.rhie_chow(u, v, w, p, gp, rau, bc, 1.0)
    assert rel_err(mine["phi_star"], rc) < 1e-14
    div = ref.continuity(rc)
    assert np.abs(mine["div_star"] - div).max() <= 1e-14 * np.abs(rc).max()
    # a SIMPLE step of the oracle ends with a corrected flux; recompute it with the reference's
    # non-orthogonal and correction twins from the oracle's fields and compare
    # non-orthogonal flux/divergence and the corrected flux for a p' field (pout = 0.25 also
    # exercises the reference's use of pFaceBC as the boundary value of p', GSV1:1653)
    pc = 1e-2 * rng.standard_normal(m.n_cells)
    gpc = o.gradient(3, pc)
    phi_no, div_no = ref.nonorth(rau, bc["type_p"], gpc)
    a_no, a_div = o.nonorth(rau, gpc)
    assert rel_err(a_no, phi_no) < 1e-14
    assert np.abs(a_div - div_no).max() <= 1e-14 * np.abs(phi_no).max()
    phi = ref.flux_correct(rau, bc["type_p"], bc["p"], rc, pc, gpc)
    assert rel_err(o.flux_correct(rau, rc, pc, gpc), phi) < 1e-14


@needs_ref
def test_oracle_force_matches_reference(tmp_path):
    kw = CASES[1]
    m, bc, o = _case(tmp_path, kw)
    ref = refshim.RefMesh(tmp_path)
    u, v, w, p = random_state(m, 9)
    k = m.topology()["patch_names"].index("patch_3_0")
    a = o.patch_force(k, -1, 1e-3, u, v, w, p)
    b = ref.patch_force(k, u, v, w, p, 1.0, 1e-3, -1)
    assert np.array_equal(a, b)


@needs_ref
def test_vtu_byte_identical(tmp_path):
    kw = CASES[1]
    m, bc, o = _case(tmp_path, kw)
    u, v, w, p = random_state(m, 5)
    m.write_vtu(tmp_path / "mine.vtu", u, v, w, p)
    refshim.RefMesh(tmp_path).write_vtu(tmp_path / "ref.vtu", u, v, w, p)
    assert (tmp_path / "mine.vtu").read_bytes() == (tmp_path / "ref.vtu").read_bytes()


def test_golden_vectors():
    """Oracle against vectors produced by the reference's own code (tests/golden/make_golden.py)."""
    z = np.load(GOLDEN / "channel_6x4x4_j15.npz")
    m = anb.HostMesh.channel(6, 4, 4, jitter=0.15, seed=21)
    t = m.topology()
    o = oracle.Oracle(t)
    g = o.geometry()
    for k in ("cc", "vol", "xf", "nf", "sf", "af"):
        assert np.array_equal(g[k], z[k]), k
    bc = {k: z["bc_" + k] for k in ("type_u", "type_v", "type_w", "type_p", "u", "v", "w", "p")}
    o.set_bc(bc)
    for field, key in enumerate("uvwp"):
        assert rel_err(o.gradient(field, z["phi"]), z["grad_" + key]) < 1e-14
    mine = o.pressure(1.0, z["u"], z["v"], z["w"], z["p"], z["rau"])
    assert rel_err(mine["phi_star"], z["phi_star"]) < 1e-14
    assert np.abs(mine["div_star"] - z["div_star"]).max() <= 1e-14 * np.abs(z["phi_star"]).max()
    f = o.patch_force(0, -1, 1e-3, z["u"], z["v"], z["w"], z["p"])
    assert rel_err(f, z["force_patch0"]) < 1e-14
