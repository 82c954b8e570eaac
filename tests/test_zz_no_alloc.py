"""The allocation-free force integral (anb_patch_force_nalloc) against anb_patch_force.

anb_patch_force_nalloc serves callers that cannot allocate device memory when they need the
force: an application that has handed the whole GPU to its own memory pool, code that runs while
another component records a CUDA graph, a plugin with a fixed memory budget.  It keeps its scratch
in a static device array, so its result must equal the allocating entry point's, call after call
(the array keeps the previous call's contents).  This file is collected last, so a run that stops
at the first failure has already run every other test; it also passes on its own in a fresh
process.
"""
import ctypes as ct

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, random_state

pytestmark = pytest.mark.gpu


def _force(fn, s, patch, sign):
    r = anb.ForceReport()
    rc = fn(s._h, patch, sign, ct.byref(r))
    assert rc == anb.ANB_OK, anb.lib().anb_last_error(s._h)
    return np.array(list(r.Fp) + list(r.Fv) + list(r.F) + [r.area, r.n_faces, r.min_wall_distance,
                                                           r.max_wall_distance, r.max_ut, r.max_shear_mag]), r.valid


def test_patch_force_without_allocation():
    m, bc, _ = channel(24, 10, 10, jitter=0.15, seed=2, obstacle=True)
    s = anb.Solver(m, anb.default_params(rho=1.0, mu=1e-3))
    s.set_bc(bc)
    names = m.topology()["patch_names"]
    lib = anb.lib()
    for seed, name in ((3, "patch_3_0"), (4, "patch_0_0")):   # obstacle (1 block) and walls (4 blocks)
        s.set_state(*random_state(m, seed))
        k = names.index(name)
        ref, valid = _force(lib.anb_patch_force, s, k, -1)
        assert valid == 1 and ref[10] > 0
        fscale = np.abs(ref[:9]).max()
        for _ in range(2):  # two calls in a row: the shared scratch must not leak between calls
            got, valid2 = _force(lib.anb_patch_force_nalloc, s, k, -1)
            assert valid2 == 1
            # force sums: the same terms added in a different order (1e-12 of the largest component)
            assert np.all(np.abs(got[:9] - ref[:9]) <= 1e-12 * fscale), (name, got[:9] - ref[:9])
            # area and face count: sums; wall distances and maxima: order-independent
            assert np.all(np.abs(got[9:] - ref[9:]) <= 1e-12 * np.abs(ref[9:])), (name, got[9:] - ref[9:])
    # an unknown patch is reported as not valid, like anb_patch_force
    _, valid3 = _force(lib.anb_patch_force_nalloc, s, 99, -1)
    assert valid3 == 0
