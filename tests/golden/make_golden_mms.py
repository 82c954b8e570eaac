"""Generates tests/golden/mms_orders.json: the reference's observed MMS error norms and orders.

Runs only where the reference tree is mounted: every system is assembled by the reference's own
libpoisson / libscalar host functions (oracle/_ref/libscalarref.so, built by oracle/build_ref.sh)
inside the reference's outer loop (solve_scalar_elliptic / solve_steady_scalar_transport, restated
in oracle/mms.py), with linear solves to 1e-14 relative standing in for HYPRE.  Problems and mesh
sequences are tests/mms_cases.py (unit cubes; jittered meshes use seed 3).

    python tests/golden/make_golden_mms.py
"""
import json
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import mms  # noqa: E402
from tests import mms_cases as M  # noqa: E402
from tests import refshim  # noqa: E402

SEED = 3


def main():
    out = {"seed": SEED, "sequences": {}}
    for label, sizes, jitter, tets in M.SEQUENCES:
        seq = {"sizes": list(sizes), "jitter": jitter, "tets": tets, "problems": {}}
        for prob in M.PROBLEMS:
            rows = []
            for n in sizes:
                m = M.unit_cube(n, jitter=jitter, seed=SEED, tets=tets)
                d = Path(tempfile.mkdtemp())
                m.write(d)
                geo = M.geometry(m)
                p = M.problem(prob, geo)
                phi = M.oracle_solve(refshim.RefScalar(d), p)
                e = mms.error_norms(phi, p["exact"], geo["vol"])
                e["cells"] = m.n_cells
                rows.append(e)
            seq["problems"][prob] = {"levels": rows, "order_l2": M.orders([r["l2"] for r in rows]),
                                     "order_l1": M.orders([r["l1"] for r in rows])}
            print(label, prob, ["%.4e" % r["l2"] for r in rows], seq["problems"][prob]["order_l2"], flush=True)
        out["sequences"][label] = seq
    path = Path(__file__).resolve().parent / "mms_orders.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
