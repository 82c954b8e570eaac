"""Runtime boundary conditions (.bc) and .case expansion against the reference's own code
(bc_runtime_config.cu, velocity_bc_eval.cu, patch_geometry.cu, main.cu:162-331)."""
import shutil
from pathlib import Path

import numpy as np
import pytest

import anabasis_b200 as anb
from tests import refshim

needs_ref = pytest.mark.skipif(not refshim.available(), reason="reference shim not built")
REF = Path("/root/reference")

BC_FILES = {
    "parabolic": """velocity patch_0_0 wall_noslip
velocity patch_1_0 parabolic_box_inlet 0.41 0.45 y z average_patch_normal
velocity patch_2_0 zero_gradient
velocity patch_3_0 wall_noslip
pressure patch_0_0 zero_gradient
pressure patch_1_0 zero_gradient
pressure patch_2_0 fixed_value 0.25
pressure patch_3_0 open
""",
    "local_normal_flow_rate": """# comment line
velocity patch_0_0 wall_noslip   # trailing comment
velocity patch_1_0 fixed_flow_rate -1.962977932911e-03 local_face_normal
velocity patch_2_0 zero_gradient
velocity patch_3_0 fixed_uniform_vector 0.1 -0.2 0.3
pressure patch_0_0 zero_gradient
pressure patch_1_0 zero_gradient
pressure patch_2_0 fixed_value 0
pressure patch_3_0 zero_gradient
""",
    "normal_speed": """velocity patch_0_0 wall_noslip
velocity patch_1_0 fixed_normal_speed -1.0
velocity patch_2_0 fixed_normal_speed 0.5 local_face_normal
velocity patch_3_0 parabolic_box_inlet 0.2 1.5 Z 1 local_face_normal
pressure patch_0_0 zero_gradient
pressure patch_1_0 zero_gradient
pressure patch_2_0 fixed_value -3.5e-2
""",
}

BAD_LINES = [
    "velocity patch_0_0",
    "velocity patch_0_0 wall_noslip extra",
    "velocity patch_0_0 fixed_uniform_vector 1 2",
    "velocity patch_0_0 fixed_uniform_vector 1 2 3x",
    "velocity patch_0_0 fixed_normal_speed 1 sideways",
    "velocity patch_0_0 parabolic_box_inlet 0.41 0.45 y y",
    "velocity patch_0_0 parabolic_box_inlet 0.41 0.45 y w",
    "velocity patch_0_0 warp_drive",
    "pressure patch_0_0 fixed_value",
    "pressure patch_0_0 zero_gradient 1",
    "pressure patch_0_0 suction",
    "temperature patch_0_0 fixed 300",
    "velocity patch_9_9 wall_noslip",
]


@pytest.fixture(scope="module")
def mesh(tmp_path_factory):
    d = tmp_path_factory.mktemp("bcmesh")
    m = anb.HostMesh.channel(24, 6, 5, jitter=0.12, seed=3, obstacle=True)
    m.write(d)
    return d


@needs_ref
@pytest.mark.parametrize("name", sorted(BC_FILES))
def test_bc_values_bit_identical(mesh, tmp_path, name):
    f = tmp_path / f"{name}.bc"
    f.write_text(BC_FILES[name])
    mine = anb.HostMesh.read(mesh).evaluate_bc(f)
    ref = refshim.RefMesh(mesh).bc_eval(f)
    for k in ("type_u", "type_v", "type_w", "type_p", "u", "v", "w", "p"):
        assert np.array_equal(mine[k], ref[k]), k


@needs_ref
@pytest.mark.skipif(not REF.exists(), reason="reference tree not mounted")
@pytest.mark.parametrize("bc", sorted(p.name for p in (REF / "bc_configs").glob("*.bc")) if REF.exists() else [])
def test_reference_bc_configs(mesh, bc):
    # the reference's own example configurations (patch_0_0..patch_3_0 exist in the channel mesh)
    path = REF / "bc_configs" / bc
    mine_err = ref_err = None
    try:
        mine = anb.HostMesh.read(mesh).evaluate_bc(path)
    except anb.AnbError as e:
        mine_err = str(e)
    try:
        ref = refshim.RefMesh(mesh).bc_eval(path)
    except RuntimeError as e:
        ref_err = str(e)
    if ref_err is not None:
        assert mine_err is not None and ref_err in mine_err
        return
    assert mine_err is None, mine_err
    for k in ("type_u", "type_v", "type_w", "type_p", "u", "v", "w", "p"):
        assert np.array_equal(mine[k], ref[k]), (bc, k)


@needs_ref
def test_fixed_flow_rate_planarity_check(mesh, tmp_path):
    # velocity_bc_eval.cu:122-134: a flow rate along the average normal of a patch that is not
    # planar (the four channel walls: the area vectors cancel) is rejected with the same message
    f = tmp_path / "nonplanar.bc"
    f.write_text(BC_FILES["parabolic"].replace("velocity patch_0_0 wall_noslip",
                                               "velocity patch_0_0 fixed_flow_rate 1e-3 average_patch_normal"))
    with pytest.raises(anb.AnbError) as mine:
        anb.HostMesh.read(mesh).evaluate_bc(f)
    with pytest.raises(RuntimeError) as ref:
        refshim.RefMesh(mesh).bc_eval(f)
    assert "planarity" in str(ref.value)
    assert str(ref.value) in str(mine.value)
    # the same flow rate along the local face normals is accepted by both, with equal values
    f.write_text(BC_FILES["parabolic"].replace("velocity patch_0_0 wall_noslip",
                                               "velocity patch_0_0 fixed_flow_rate 1e-3 local_face_normal"))
    a, b = anb.HostMesh.read(mesh).evaluate_bc(f), refshim.RefMesh(mesh).bc_eval(f)
    for k in ("u", "v", "w", "type_u"):
        assert np.array_equal(a[k], b[k]), k


@needs_ref
@pytest.mark.parametrize("line", BAD_LINES)
def test_bc_errors_same_message(mesh, tmp_path, line):
    f = tmp_path / "bad.bc"
    f.write_text("velocity patch_1_0 wall_noslip\n" + line + "\n")
    with pytest.raises(anb.AnbError) as mine:
        anb.HostMesh.read(mesh).evaluate_bc(f)
    with pytest.raises(RuntimeError) as ref:
        refshim.RefMesh(mesh).bc_eval(f)
    assert str(ref.value) in str(mine.value)


@needs_ref
@pytest.mark.skipif(not REF.exists(), reason="reference tree not mounted")
@pytest.mark.parametrize("case", sorted(p.name for p in (REF / "cases").glob("*.case")) if REF.exists() else [])
def test_case_expansion_matches_reference(tmp_path, case):
    # copy: the expansion writes <case>.generated.bc next to the case file
    a = tmp_path / "a" / case
    b = tmp_path / "b" / case
    for p in (a, b):
        p.parent.mkdir()
        shutil.copy(REF / "cases" / case, p)
    mine = anb.expand_case_args(["prog", "-case-config", str(a), "-nsteps", "7"])
    ref = refshim.expand_case(["prog", "-case-config", str(b), "-nsteps", "7"])
    norm = lambda v, d: [x.replace(str(d), "<dir>") for x in v]
    assert norm(mine, a.parent) == norm(ref, b.parent)
    ga, gb = a.with_name(case + ".generated.bc"), b.with_name(case + ".generated.bc")
    assert ga.exists() == gb.exists()
    if ga.exists():
        assert ga.read_text().replace(str(a), "") == gb.read_text().replace(str(b), "")


@needs_ref
@pytest.mark.parametrize("text", [
    "rho 1.0\nfrobnicate 3\n",                                    # unknown key
    "rho 1.0 2.0\n",                                              # wrong arity
    "bcConfig x.bc\nvelocity patch_0_0 wall_noslip\n",            # both bcConfig and inline BCs
])
def test_case_errors_same_message(tmp_path, text):
    for tag in ("a", "b"):
        (tmp_path / f"{tag}.case").write_text(text)
    with pytest.raises(anb.AnbError) as mine:
        anb.expand_case_args(["prog", "-case-config", str(tmp_path / "a.case")])
    with pytest.raises(RuntimeError) as ref:
        refshim.expand_case(["prog", "-case-config", str(tmp_path / "b.case")])
    assert str(ref.value).replace("b.case", "X") in str(mine.value).replace("a.case", "X")
