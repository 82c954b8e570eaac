"""Host-side AMG set-up (no GPU): compiles tests/native/amg_setup_check.cpp against
anabasis_b200/csrc/amg_setup.cpp and runs it.  The check rebuilds each coarse operator through the
Galerkin gather lists, validates every index of the patterns, aggregates and gather lists, and
compares the SELL-32 and CSR storage forms of the same coarse levels."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("amg") / "amg_setup_check"
    src = ROOT / "anabasis_b200" / "csrc"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{src}", str(ROOT / "tests" / "native" / "amg_setup_check.cpp"),
                    str(src / "amg_setup.cpp"), "-o", str(exe)], check=True)
    return exe


@pytest.mark.parametrize("dims", [(40, 40, 20, 1000), (64, 48, 20, 4000), (33, 17, 9, 520)])
def test_sell_and_csr_coarse_levels_agree(checker, dims):
    r = subprocess.run([str(checker), *map(str, dims)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
