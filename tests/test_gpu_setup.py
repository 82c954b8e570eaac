"""Mesh set-up on the device: geometry, LSQ moments and slot-ordered face records.

anb_create builds the cell and face geometry (main.cu:591-597), the least-squares moment inverse
(main.cu:1169-1224) and the slot-ordered face records on the GPU.  The geometry must equal the host
restatement bit for bit, which the CPU tests pin to the reference's own read_openfoam_polymesh; the
whole solver state after a few SIMPLE steps must equal that of a context whose set-up ran on the
host (ANB_HOST_SETUP=1), which covers the moments and the slot records.
"""
import ctypes as ct
import os

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

MESHES = [
    dict(nx=6, ny=4, nz=4),
    dict(nx=16, ny=8, nz=8, jitter=0.15, seed=1),
    dict(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True),
    dict(nx=5, ny=3, nz=3, jitter=0.1, seed=4, tets=True),
]


def _geometry(s, m):
    C, F = m.n_cells, m.n_faces
    g = dict(cc=np.zeros(3 * C), vol=np.zeros(C), xf=np.zeros(3 * F), nf=np.zeros(3 * F), af=np.zeros(F))
    mx = np.zeros(1)
    d = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))  # noqa: E731
    assert anb.lib().anb_get_geometry(s._h, d(g["cc"]), d(g["vol"]), d(g["xf"]), d(g["nf"]), d(g["af"]), d(mx)) == 0
    g["max_nonorth"] = float(mx[0])
    return g


@pytest.mark.parametrize("kw", MESHES)
def test_device_geometry_bit_identical(kw):
    m, bc, _ = channel(**kw)
    host = m.geometry()
    s = anb.Solver(m, anb.default_params(rho=1.0, mu=1e-3))
    dev = _geometry(s, m)
    for k in ("cc", "vol", "xf", "nf", "af"):
        assert np.array_equal(dev[k], np.asarray(host[k]).reshape(-1)), k
    assert dev["max_nonorth"] == host["max_nonorth"]
    t = np.zeros(10)
    assert anb.lib().anb_setup_times(s._h, t.ctypes.data_as(ct.POINTER(ct.c_double))) == 0
    assert np.all(t >= 0) and t[:4].sum() > 0


@pytest.mark.parametrize("kw", MESHES[1:])
def test_device_setup_matches_host_setup(kw):
    m, bc, _ = channel(**kw)
    out = []
    for host in (False, True):
        if host:
            os.environ["ANB_HOST_SETUP"] = "1"
        try:
            s = anb.Solver(m, anb.default_params(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3))
        finally:
            os.environ.pop("ANB_HOST_SETUP", None)
        s.set_bc(bc)
        s.set_state(*initial_state(m, bc))
        s.iterate(3)
        out.append(s.get_state())
        u = np.random.default_rng(0).standard_normal(m.n_cells)
        out[-1]["grad"] = s.debug_gradient(0, u)
    for k in ("u", "v", "w", "p", "phi", "grad"):
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("kw", MESHES[1:])
def test_face_parallel_flux_form_matches_row_form(kw):
    # the corrected face flux computed once per face (ANB_FLUX_FORM=face) against the row form,
    # which evaluates each internal face from both of its cells
    m, bc, _ = channel(**kw)
    out = []
    for form in ("row", "face"):
        os.environ["ANB_FLUX_FORM"] = form
        try:
            s = anb.Solver(m, anb.default_params(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3))
            s.set_bc(bc)
            s.set_state(*initial_state(m, bc))
            s.iterate(4)
            out.append(s.get_state())
        finally:
            os.environ.pop("ANB_FLUX_FORM", None)
    for k in ("u", "v", "w", "p", "phi"):
        scale = max(np.abs(out[0][k]).max(), 1e-300)
        assert np.abs(out[0][k] - out[1][k]).max() <= 1e-13 * scale, k
