"""The allocation-free force integral (anb_patch_force_nalloc) against anb_patch_force.

anb_patch_force_nalloc serves callers that cannot allocate device memory when they need the
force: an application that has handed the whole GPU to its own memory pool, code that runs while
another component records a CUDA graph, a plugin with a fixed memory budget.  It keeps its scratch
in a static device array, so its result must equal the allocating entry point's, call after call
(the array keeps the previous call's contents), and the device's free memory must not move across
its calls.  This file is collected last, so a run that stops at the first failure has already run
every other test; it also passes on its own in a fresh process.
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


def _free_bytes(device=0):
    import torch

    return torch.cuda.mem_get_info(device)[0]


def test_patch_force_without_allocation():
    m, bc, _ = channel(24, 10, 10, jitter=0.15, seed=2, obstacle=True)
    s = anb.Solver(m, anb.default_params(rho=1.0, mu=1e-3))
    s.set_bc(bc)
    names = m.topology()["patch_names"]
    lib = anb.lib()
    _free_bytes()  # the first query sets up the caller's runtime state; measure after it
    for seed, name in ((3, "patch_3_0"), (4, "patch_0_0")):   # obstacle (1 block) and walls (4 blocks)
        s.set_state(*random_state(m, seed))
        k = names.index(name)
        ref, valid = _force(lib.anb_patch_force, s, k, -1)
        assert valid == 1 and ref[10] > 0
        fscale = np.abs(ref[:9]).max()
        free0 = _free_bytes()
        for _ in range(2):  # two calls in a row: the shared scratch must not leak between calls
            got, valid2 = _force(lib.anb_patch_force_nalloc, s, k, -1)
            assert valid2 == 1
            # force sums: the same terms added in a different order (1e-12 of the largest component)
            assert np.all(np.abs(got[:9] - ref[:9]) <= 1e-12 * fscale), (name, got[:9] - ref[:9])
            # area and face count: sums; wall distances and maxima: order-independent
            assert np.all(np.abs(got[9:] - ref[9:]) <= 1e-12 * np.abs(ref[9:])), (name, got[9:] - ref[9:])
        assert _free_bytes() == free0, "device memory changed across allocation-free calls"
    # an unknown patch is reported as not valid, like anb_patch_force
    _, valid3 = _force(lib.anb_patch_force_nalloc, s, 99, -1)
    assert valid3 == 0


def test_patch_force_without_allocation_limit():
    # 600 x 220 x 1 cells: the wall patch has 265,200 faces, above the 262,144 the static scratch covers
    m, bc, _ = channel(600, 220, 1)
    s = anb.Solver(m, anb.default_params(rho=1.0, mu=1e-3))
    s.set_bc(bc)
    s.set_state(*random_state(m, 5))
    k = m.topology()["patch_names"].index("patch_0_0")
    assert int(m.topology()["patch_size"][k]) > 262144
    r = anb.ForceReport()
    rc = anb.lib().anb_patch_force_nalloc(s._h, k, -1, ct.byref(r))
    assert rc == anb.ANB_ERR_INVALID
    assert b"262144" in anb.lib().anb_last_error(s._h)
    # the allocating entry point has no such limit
    ref, valid = _force(anb.lib().anb_patch_force, s, k, -1)
    assert valid == 1 and int(ref[10]) == int(m.topology()["patch_size"][k])
    # the context is still usable for a patch within the limit
    k2 = m.topology()["patch_names"].index("patch_1_0")
    ref2, _ = _force(anb.lib().anb_patch_force, s, k2, -1)
    got2, valid2 = _force(anb.lib().anb_patch_force_nalloc, s, k2, -1)
    assert valid2 == 1
    assert np.all(np.abs(got2[:9] - ref2[:9]) <= 1e-12 * np.abs(ref2[:9]).max())
