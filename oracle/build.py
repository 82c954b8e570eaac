"""Builds the oracle (TEST INFRASTRUCTURE ONLY).

  liboracle.so      oracle.cpp, the CPU restatement of the reference's SIMPLE iteration, and
                    channel.cpp, the synthetic channel case (mesh and boundary values)
  _ref/libgsv1ref.so the reference's own host code compiled from /root/reference where it lies
                     (only when that tree exists; see build_ref.sh for the recipe)
  _ref/libscalarref.so the reference's libpoisson / libscalar host assembly, same recipe

Usage: python -m oracle.build
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REFERENCE = Path("/root/reference")


def build_oracle(force: bool = False) -> Path:
    out = HERE / "liboracle.so"
    srcs = [HERE / "oracle.cpp", HERE / "channel.cpp"]
    newest = max(p.stat().st_mtime for p in srcs + [HERE / "oracle.h"])
    if force or not out.exists() or out.stat().st_mtime < newest:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-o", str(out),
               *map(str, srcs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stderr)
    return out


def build_ref(force: bool = False) -> Path | None:
    """Compiles the reference's host code (needs /root/reference; the GPU box uses the prebuilt .so)."""
    out = HERE / "_ref" / "libgsv1ref.so"
    if not REFERENCE.exists():
        return out if out.exists() else None
    script = HERE / "build_ref.sh"
    deps = [script, HERE / "ref_shim.cu", HERE / "ref_scalar_shim.cu", HERE / "ref_transport_shim.cu",
            *sorted((HERE / "ref_stubs").iterdir())]
    outs = [out, HERE / "_ref" / "libscalarref.so"]
    newest = max(d.stat().st_mtime for d in deps)
    if force or any(not o.exists() or o.stat().st_mtime < newest for o in outs):
        r = subprocess.run(["bash", str(script)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference build failed:\n" + r.stdout + r.stderr)
    return out


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
