"""The drop-in manufactured-solution programs (anabasis_poisson_mms, ..._neumann, ..._mixed,
anabasis_scalar_mms; app_mms.cpp): the reference programs' command-line errors on the CPU, and on
the GPU their printed error norms against the reference's own (tests/golden/mms_orders.json, hex
8^3 level) with the reference programs' default options."""
import json
import re
import subprocess
from pathlib import Path

import pytest

import anabasis_b200 as anb
from tests import mms_cases as M

LIB = Path(anb.__file__).resolve().parent / "_lib"
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "mms_orders.json").read_text())


def _run(name, *args):
    return subprocess.run([str(LIB / name), *map(str, args)], capture_output=True, text=True, timeout=300)


@pytest.mark.parametrize("name", ["anabasis_poisson_mms", "anabasis_poisson_mms_neumann", "anabasis_poisson_mms_mixed",
                                  "anabasis_scalar_mms"])
def test_unknown_option_and_missing_value(name):
    r = _run(name, "-no-such-option")
    assert r.returncode == 1 and "Unknown option: -no-such-option" in r.stderr
    r = _run(name, "-tol")
    assert r.returncode == 1 and "Missing value after -tol" in r.stderr


def test_mixed_program_requires_dirichlet_patches():
    r = _run("anabasis_poisson_mms_mixed")
    assert r.returncode == 1 and "You must provide -dirichlet-patches patchA[,patchB,...]" in r.stderr


def _l2(out):
    return float(re.search(r"L2 error\s*:\s*(\S+)", out).group(1))


@pytest.mark.gpu
@pytest.mark.parametrize("name,prob,extra", [
    ("anabasis_poisson_mms", "poisson_dirichlet", []),
    ("anabasis_poisson_mms_neumann", "poisson_neumann", []),
    ("anabasis_poisson_mms_mixed", "poisson_mixed", ["-dirichlet-patches", M.INLET]),
    ("anabasis_scalar_mms", "transport_central", []),
    ("anabasis_scalar_mms", "transport_upwind_mixed",
     ["-convection-scheme", "upwind", "-diffusion-scheme", "nonorth", "-nNonOrthCorr", 2, "-bc-mode", "mixed",
      "-dirichlet-patches", f"{M.INLET},{M.WALLS}"]),
])
def test_program_reproduces_reference_norms(tmp_path, name, prob, extra):
    m = M.unit_cube(8)
    m.write(tmp_path)
    r = _run(name, "-polyMeshDir", tmp_path, "-tol", 1e-13, *extra)
    assert r.returncode == 0, r.stderr
    assert "summary ===" in r.stdout
    ref = GOLDEN["sequences"]["hex"]["problems"][prob]["levels"][0]["l2"]
    assert _l2(r.stdout) == pytest.approx(ref, rel=1e-6)
