"""polyMesh reader, geometry and synthetic meshes against the reference's own reader
(read_openfoam_polymesh, main.cu:532-599, compiled from the reference tree)."""
import os

import numpy as np
import pytest

import anabasis_b200 as anb
from tests import refshim

needs_ref = pytest.mark.skipif(not refshim.available(), reason="reference shim not built")

MESHES = [
    dict(nx=6, ny=4, nz=4),
    dict(nx=8, ny=5, nz=4, jitter=0.15, seed=7),
    dict(nx=24, ny=10, nz=4, jitter=0.15, seed=1, obstacle=True),
    dict(nx=4, ny=3, nz=3, jitter=0.1, seed=2, tets=True),
]


def test_benchmark_mesh_counts():
    # configuration 1 of the benchmark table: 40x20x20 hexes
    m = anb.HostMesh.channel(40, 20, 20)
    assert (m.n_cells, m.n_internal, m.n_faces - m.n_internal) == (16000, 46000, 4000)
    # configuration 2: 200x70x70 with the obstacle block removed, +-15 % jitter, seed 0
    m = anb.HostMesh.channel(200, 70, 70, jitter=0.15, seed=0, obstacle=True)
    assert (m.n_cells, m.n_internal, m.n_faces - m.n_internal) == (970480, 2876926, 69028)
    t = m.topology()
    assert t["patch_names"] == ["patch_0_0", "patch_1_0", "patch_2_0", "patch_3_0"]


def test_tet_split_counts():
    m = anb.HostMesh.channel(4, 3, 3, tets=True)
    assert m.n_cells == 6 * 36
    # each hex gives 6 internal triangles, each interior quad 2 shared triangles
    interior_quads = 3 * 3 * 3 + 4 * 2 * 3 + 4 * 3 * 2
    assert m.n_internal == 6 * 36 + 2 * interior_quads
    g = m.geometry()
    assert np.isclose(g["vol"].sum(), 2.5 * 0.41 * 0.41, rtol=1e-12)


@pytest.mark.parametrize("kw", MESHES)
def test_roundtrip_and_closed_cells(tmp_path, kw):
    m = anb.HostMesh.channel(**kw)
    m.write(tmp_path)
    r = anb.HostMesh.read(tmp_path)
    a, b = m.topology(), r.topology()
    for k in ("points", "face_offsets", "face_points", "owner", "neighbour", "patch_start", "patch_size"):
        assert np.array_equal(a[k], b[k]), k
    g = r.geometry()
    assert np.all(g["vol"] > 0)
    # closed cells: the outward area vectors of each cell sum to zero
    C = r.n_cells
    s = np.zeros((C, 3))
    sf = g["sf"].reshape(-1, 3)
    np.add.at(s, b["owner"], sf)
    np.add.at(s, b["neighbour"], -sf[: r.n_internal])
    assert np.abs(s).max() < 1e-12 * np.abs(sf).max()
    # the cells tile the box when faces are planar (with jitter, the reference's tet decomposition
    # fans a non-planar shared quad from opposite vertices in its two cells, main.cu:592, so the
    # volumes overlap slightly)
    box = 2.5 * 0.41 * 0.41
    if not kw.get("obstacle") and not kw.get("jitter"):
        assert np.isclose(g["vol"].sum(), box, rtol=1e-12)


@needs_ref
@pytest.mark.parametrize("kw", MESHES)
def test_geometry_bit_identical_to_reference(tmp_path, kw):
    m = anb.HostMesh.channel(**kw)
    m.write(tmp_path)
    mine = anb.HostMesh.read(tmp_path).geometry()
    ref = refshim.RefMesh(tmp_path).geometry()
    for k in ("cc", "vol", "xf", "nf", "sf", "af"):
        assert np.array_equal(mine[k], ref[k]), k
    assert mine["max_nonorth"] == ref["max_nonorth"]


def _write_file(d, name, text):
    os.makedirs(d, exist_ok=True)
    (d / name).write_text(text)


@needs_ref
def test_comments_and_headers_like_reference(tmp_path):
    m = anb.HostMesh.channel(3, 2, 2)
    m.write(tmp_path)
    # add block and line comments in awkward places
    pts = (tmp_path / "points").read_text()
    pts = pts.replace("(\n(", "( // list opens\n/* a block\n comment */(", 1)
    (tmp_path / "points").write_text(pts)
    mine = anb.HostMesh.read(tmp_path).geometry()
    ref = refshim.RefMesh(tmp_path).geometry()
    assert np.array_equal(mine["cc"], ref["cc"])


# comment layouts the reference's stripper (main.cu:533-537) handles in particular ways: a '/' and a
# '*' left on both sides of an erased block start a new block; "//" inside a block; an unterminated
# block keeps the rest of the file; comments between list entries
COMMENT_EDITS = [
    lambda s: s.replace("(\n(", "(\n//* a */* (9 9 9) */ (", 1),
    lambda s: s.replace("(\n(", "(\n/* x // y */ // z\n(", 1),
    lambda s: s.replace("\n(", "\n/*/ odd */(", 1),
    lambda s: s.replace(")\n(", ")\n// between entries\n/* and */ (", 3),
    lambda s: s.rstrip() + "\n/* never closed ( ) (\n",
    lambda s: s.replace("FoamFile", "/*/*/ FoamFile", 1),
]


@needs_ref
@pytest.mark.parametrize("edit", range(len(COMMENT_EDITS)))
@pytest.mark.parametrize("name", ["points", "faces", "owner"])
def test_comment_layouts_like_reference(tmp_path, edit, name):
    m = anb.HostMesh.channel(4, 3, 2, jitter=0.1, seed=1)
    m.write(tmp_path)
    p = tmp_path / name
    p.write_text(COMMENT_EDITS[edit](p.read_text()))
    mine_err = ref_err = None
    try:
        mine = anb.HostMesh.read(tmp_path).geometry()
    except Exception as e:  # noqa: BLE001
        mine_err = str(e)
    try:
        ref = refshim.RefMesh(tmp_path).geometry()
    except RuntimeError as e:
        ref_err = str(e)
    if ref_err is not None:
        assert mine_err is not None and ref_err in mine_err, (mine_err, ref_err)
        return
    assert mine_err is None, mine_err
    for k in ("cc", "vol", "xf", "nf", "af"):
        assert np.array_equal(mine[k], ref[k]), k


def _mid_replace(s, old, new):
    """Replaces the first `old` after the middle of `s` (inside a large list)."""
    i = s.index(old, len(s) // 2)
    return s[:i] + new + s[i + len(old):]


# large files (several MB) are parsed in parallel chunks under a strict grammar; entries that
# leave it (extra tokens, trailing garbage, signs, comments) send the file to the serial reader
LARGE_EDITS = [
    ("points", None),
    ("points", lambda s: _mid_replace(s, ")\n(", " 7)\n(")),            # a fourth coordinate
    ("points", lambda s: _mid_replace(s, ")\n(", ")\n junk (")),        # garbage between entries
    ("faces", lambda s: _mid_replace(s, ")\n4(", " 5)\n4(")),          # an extra vertex
    ("faces", lambda s: _mid_replace(s, "\n4(", "\n// note\n4(")),      # a comment inside the list
    ("owner", lambda s: _mid_replace(s, "\n", "\n+3 ")),                 # a signed label
    ("neighbour", lambda s: _mid_replace(s, "\n", "\nx ")),              # a label list cut short
]


@needs_ref
@pytest.mark.parametrize("name,mutate", LARGE_EDITS)
def test_large_files_like_reference(tmp_path, name, mutate):
    m = anb.HostMesh.channel(60, 40, 40, jitter=0.1, seed=3)
    m.write(tmp_path)
    p = tmp_path / name
    assert p.stat().st_size > 2 << 20 or name in ("owner", "neighbour")
    if mutate is not None:
        p.write_text(mutate(p.read_text()))
    mine_err = ref_err = None
    try:
        r = anb.HostMesh.read(tmp_path)
        mine = r.geometry()
    except Exception as e:  # noqa: BLE001
        mine_err = str(e)
    try:
        ref = refshim.RefMesh(tmp_path).geometry()
    except RuntimeError as e:
        ref_err = str(e)
    if ref_err is not None:
        assert mine_err is not None and ref_err in mine_err, (mine_err, ref_err)
        return
    assert mine_err is None, mine_err
    for k in ("cc", "vol", "xf", "nf", "af"):
        assert np.array_equal(mine[k], ref[k]), k
    if mutate is None:
        a, b = m.topology(), r.topology()
        for k in ("points", "face_offsets", "face_points", "owner", "neighbour"):
            assert np.array_equal(a[k], b[k]), k


@needs_ref
@pytest.mark.parametrize("name,mutate", [
    ("faces", lambda s: s.replace("4(", "4 x(", 1)),            # Malformed faces list
    ("owner", lambda s: s.split("\n(")[0]),                       # no top-level list
    ("neighbour", lambda s: s.rsplit(")", 1)[0]),                  # unmatched parenthesis
])
def test_malformed_files_same_error(tmp_path, name, mutate):
    m = anb.HostMesh.channel(3, 2, 2)
    m.write(tmp_path)
    p = tmp_path / name
    p.write_text(mutate(p.read_text()))
    with pytest.raises(Exception) as mine:
        anb.HostMesh.read(tmp_path)
    with pytest.raises(RuntimeError) as ref:
        refshim.RefMesh(tmp_path)
    assert str(ref.value) in str(mine.value)


def test_missing_file_error(tmp_path):
    with pytest.raises(anb.AnbError, match="Could not open"):
        anb.HostMesh.read(tmp_path / "nope")
