"""End-to-end parity with the reference program itself.

oracle/_ref/gsv1_ref is the reference's generic_simple_v1 compiled from its own sources (see
oracle/build_ref.sh) with single-rank MPI and HYPRE stand-ins whose solves are Jacobi-CG /
BiCGSTAB on the host.  Both it and this repository's drop-in program run the same case file on the
same polyMesh with inner tolerances tightened to 1e-15 (so the fixed point does not depend on the
linear solver); the final VTU fields, the summary files and the patch forces must agree to 1e-8
relative.  The reference binary needs a GPU (its face loops are CUDA kernels).
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, rel_err

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
REF_BIN = ROOT / "oracle" / "_ref" / "gsv1_ref"

CASE = """polyMeshDir {mesh}
outPrefix {out}
rho 1.0
mu 0.001
Umean 0.45
pipeD 0.1
nsteps {nsteps}
printEvery 1
writeVtu 1
writeEvery 0
nVelNonOrthCorr 0
nNonOrthCorr 2
uRelax 0.7
pRelax 0.3
corrTol 1e-10
tolMass 0
tolVel 0
velMaxit 5000
velTol 1e-15
velRelTol 0
pUseAmg 1
pMaxit 20000
pTol 1e-15
pRelTol 0
forceEnable 1
forcePatch {force}
forceNormalSign -1
velocity patch_0_0 wall_noslip
velocity patch_1_0 parabolic_box_inlet 0.41 0.45 y z average_patch_normal
velocity patch_2_0 zero_gradient
pressure patch_0_0 zero_gradient
pressure patch_1_0 zero_gradient
pressure patch_2_0 fixed_value 0.0
{extra}"""


def read_vtu_fields(path: Path) -> dict:
    text = path.read_text()
    out = {}
    for name, ncomp in (("U", 3), ("p", 1)):
        m = re.search(r'Name="%s" NumberOfComponents="%d" format="ascii">(.*?)</DataArray>' % (name, ncomp), text,
                      re.S)
        assert m, name
        out[name] = np.array(m.group(1).split(), dtype=np.float64).reshape(-1, ncomp)
    return out


def read_summary(path: Path) -> dict:
    d = {}
    for line in path.read_text().splitlines():
        k, _, v = line.partition(" ")
        try:
            d[k] = float(v)
        except ValueError:
            d[k] = v
    return d


@pytest.mark.skipif(not REF_BIN.exists(), reason="reference program not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("kw,steps", [(dict(nx=12, ny=6, nz=6), 15),
                                      (dict(nx=24, ny=10, nz=10, jitter=0.15, seed=3, obstacle=True), 10)])
def test_against_reference_program(tmp_path, kw, steps):
    m, bc, d = channel(**kw)
    mesh_dir = tmp_path / "constant" / "polyMesh"
    m.write(mesh_dir)
    obstacle = kw.get("obstacle", False)
    extra = "velocity patch_3_0 wall_noslip\npressure patch_3_0 zero_gradient\n" if obstacle else ""
    force = "patch_3_0" if obstacle else "patch_0_0"
    runs = {}
    for tag, exe in (("ref", REF_BIN), ("anb", anb.APP_PATH)):
        case = tmp_path / f"{tag}.case"
        case.write_text(CASE.format(mesh=mesh_dir, out=tmp_path / tag, nsteps=steps, force=force, extra=extra))
        r = subprocess.run([str(exe), "-case-config", str(case)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
        runs[tag] = dict(vtu=read_vtu_fields(tmp_path / f"{tag}_final.vtu"),
                         summary=read_summary(tmp_path / f"{tag}_summary.txt"), stdout=r.stdout)
    a, b = runs["anb"], runs["ref"]
    assert a["summary"]["steps"] == b["summary"]["steps"] == steps
    assert rel_err(a["vtu"]["U"], b["vtu"]["U"]) < 1e-8
    assert rel_err(a["vtu"]["p"], b["vtu"]["p"]) < 1e-8
    # force components relative to the largest one (a symmetric channel has zero net side force,
    # whose value is pure cancellation noise)
    fkeys = [f"{f}Force_{x}" for f in ("pressure", "viscous", "total") for x in "xyz"]
    fscale = max(abs(b["summary"][k]) for k in fkeys)
    for k in fkeys:
        assert abs(a["summary"][k] - b["summary"][k]) <= 1e-8 * fscale, k
    for k in ("maxAbsU", "maxAbsV", "maxAbsW", "maxAbsP", "patchForceArea"):
        assert abs(a["summary"][k] - b["summary"][k]) <= 1e-8 * abs(b["summary"][k]), k
    # the iteration lines carry the same monitors (massRes is at round-off with these tolerances)
    du_a = [float(x) for x in re.findall(r"duRel = ([0-9.e+-]+)", a["stdout"])]
    du_b = [float(x) for x in re.findall(r"duRel = ([0-9.e+-]+)", b["stdout"])]
    assert len(du_a) == len(du_b) == steps
    assert np.allclose(du_a, du_b, rtol=1e-3)
