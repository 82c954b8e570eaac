"""Appended raw-binary VTU (anb_write_vtu_binary) against the reference-format ASCII VTU.

The binary file must carry the same arrays as the ASCII one (which is byte-identical to the
reference's writer, main.cu:975-983): the same connectivity, offsets, types, faces and face
offsets exactly, and the exact doubles where the ASCII text holds them rounded to %.15g.
"""
import re
import subprocess

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, random_state


def read_ascii(path):
    text = path.read_text()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?(?: NumberOfComponents="(\d)")? format="ascii">'
                         r'(.*?)</DataArray>', text, re.S):
        typ, name, _, body = m.groups()
        dt = np.float64 if typ == "Float64" else np.int64
        out[name or "points"] = np.array(body.split(), dtype=dt)
    return out


def read_appended(path):
    raw = path.read_bytes()
    head_end = raw.index(b"<AppendedData encoding=\"raw\">")
    head = raw[:head_end].decode()
    base = raw.index(b"_", head_end) + 1
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?(?: NumberOfComponents="(\d)")? '
                         r'format="appended" offset="(\d+)"/>', head):
        typ, name, _, off = m.groups()
        off = base + int(off)
        nbytes = int(np.frombuffer(raw[off:off + 8], np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[typ]
        out[name or "points"] = np.frombuffer(raw[off + 8:off + 8 + nbytes], dt)
    assert raw.rstrip().endswith(b"</VTKFile>")
    return out


@pytest.mark.parametrize("kw", [dict(nx=6, ny=4, nz=3), dict(nx=8, ny=5, nz=4, jitter=0.15, seed=1, obstacle=False),
                                dict(nx=4, ny=3, nz=2, jitter=0.1, seed=2, tets=True)])
def test_binary_vtu_matches_ascii(tmp_path, kw):
    m, bc, _ = channel(**kw)
    u, v, w, p = random_state(m, 3)
    dc = np.random.default_rng(4).standard_normal(m.n_cells)
    m.write_vtu(tmp_path / "a.vtu", u, v, w, p, dc)
    m.write_vtu(tmp_path / "b.vtu", u, v, w, p, dc, binary=True)
    a, b = read_ascii(tmp_path / "a.vtu"), read_appended(tmp_path / "b.vtu")
    for k in ("connectivity", "offsets", "faces", "faceoffsets"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(b["types"], np.full(m.n_cells, 42, np.uint8))
    assert np.array_equal(b["U"], np.stack([u, v, w], 1).reshape(-1))
    assert np.array_equal(b["p"], p) and np.array_equal(b["divCorr"], dc)
    assert np.array_equal(b["umag"], np.sqrt(u * u + v * v + w * w))
    for k in ("points", "U", "p", "umag", "cell_volume", "divCorr"):
        assert np.allclose(a[k], b[k], rtol=1e-14, atol=1e-300), k


@pytest.mark.gpu
def test_drop_in_program_binary_option(tmp_path):
    m, bc, d = channel(8, 4, 4)
    mesh_dir = tmp_path / "constant" / "polyMesh"
    m.write(mesh_dir)
    case = tmp_path / "c.case"
    case.write_text(f"polyMeshDir {mesh_dir}\noutPrefix {tmp_path / 'run'}\nnsteps 2\nwriteVtu 1\n"
                    f"anbVtuFormat binary\nbcConfig {d / 'case.bc'}\n")
    r = subprocess.run([str(anb.APP_PATH), "-case-config", str(case)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    b = read_appended(tmp_path / "run_final.vtu")
    assert b["cell_volume"].shape == (m.n_cells,)
    assert np.isfinite(b["p"]).all() and b["U"].shape == (3 * m.n_cells,)
