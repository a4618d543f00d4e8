"""Host-side checks that need no GPU: the C ABI library loads and exports every declared symbol, the
setup/grid/boundary readers derive what the reference derives, and bad inputs are rejected on the
host (so no kernel ever sees an out-of-range face)."""
import re
from pathlib import Path

import numpy as np
import pytest

import ostc
import ostc_cases as oc

ROOT = Path(__file__).resolve().parent.parent


def test_exports_every_declared_symbol(built):
    lib = ostc.load_library()
    header = (ROOT / "include" / "ostc.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|void|const char \*)\s*(ostc_\w+)\s*\(", header, re.M))
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(ostc.EXPORTS), declared ^ set(ostc.EXPORTS)


@pytest.mark.parametrize("recon,rs,ngg", [(4, 3, 3), (5, 4, 4), (4, 4, 3), (5, 3, 4)])
def test_probe_2d(built, tmp_path, recon, rs, ngg):
    case = oc.mixing_layer_2d(mx=33, my=17, reconstruction=recon, inviscid_scheme=rs)
    d = oc.write_case(case, tmp_path / "c")
    p = ostc.probe_case(str(d))
    assert p["ngg"] == ngg and p["inviscid_type"] == 1 and p["n_var"] == 5 and p["dimension"] == 2
    assert (p["mx"], p["my"], p["mz"]) == (33, 17, 1)
    assert p["n_faces"] == 4 and p["n_bc_launches"] == 4


def test_probe_3d_farfield(built, tmp_path):
    case = oc.mixing_layer_3d(mx=24, my=20, mz=16)
    d = oc.write_case(case, tmp_path / "c")
    p = ostc.probe_case(str(d))
    assert p["dimension"] == 3 and p["n_faces"] == 6 and p["ngg"] == 4
    assert p["reconstruction"] == 5 and p["inviscid_scheme"] == 4


def _case_dir(tmp_path, **kw):
    case = oc.mixing_layer_2d(mx=33, my=17, **kw)
    return case, oc.write_case(case, tmp_path / "c")


def test_missing_grid_is_io_error(built, tmp_path):
    _, d = _case_dir(tmp_path)
    (d / "grid" / "grid   0.dat").unlink()
    with pytest.raises(ostc.OstcError) as e:
        ostc.probe_case(str(d))
    assert e.value.code == -2


def test_unsupported_species_rejected(built, tmp_path):
    _, d = _case_dir(tmp_path)
    s = (d / "setup.txt").read_text()
    (d / "setup.txt").write_text(s.replace("int species = 0", "int species = 2"))
    with pytest.raises(ostc.OstcError, match="species = 2"):
        ostc.probe_case(str(d))
    # species = 1 with an AWENO scheme: the reference's mixture AWENO is an empty stub
    (d / "setup.txt").write_text(s.replace("int species = 0", "int species = 1"))
    with pytest.raises(ostc.OstcError, match="AWENO"):
        ostc.probe_case(str(d))


def test_mixture_probe_and_errors(built, tmp_path):
    case = oc.reacting_mixing_layer_3d(mx=12, my=10, mz=8)
    d = oc.write_case(case, tmp_path / "mix")
    info = ostc.probe_case(str(d))
    assert info["n_var"] == 14 and info["n_scalar"] == 9 and info["ngg"] == 4 and info["inviscid_type"] == 3
    setup = (d / "setup.txt").read_text()
    # the reference's 52 reads outside its stencil: rejected with the reason
    (d / "setup.txt").write_text(setup.replace("int inviscid_scheme = 72", "int inviscid_scheme = 52"))
    with pytest.raises(ostc.OstcError, match="outside its stencil"):
        ostc.probe_case(str(d))
    # the primitive reconstructions with the mixture AUSM+ / HLLC / Roe: two ghost layers
    for scheme, it in ((3, 0), (4, 0), (2, 2)):
        (d / "setup.txt").write_text(setup.replace("int inviscid_scheme = 72", f"int inviscid_scheme = {scheme}"))
        info = ostc.probe_case(str(d))
        assert info["ngg"] == 2 and info["inviscid_type"] == it, scheme
    # Lax-Friedrichs has no mixture form in the reference
    (d / "setup.txt").write_text(setup.replace("int inviscid_scheme = 72", "int inviscid_scheme = 1"))
    with pytest.raises(ostc.OstcError, match="Lax-Friedrichs"):
        ostc.probe_case(str(d))
    (d / "setup.txt").write_text(setup.replace("chemistry/H2_mech.inp", "chemistry/missing.inp"))
    with pytest.raises(ostc.OstcError, match="cannot open") as e:
        ostc.probe_case(str(d))
    assert e.value.code == -2  # OSTC_EIO


def test_face_outside_block_rejected(built, tmp_path):
    case, _ = _case_dir(tmp_path)
    case.faces[2] = oc.Face((0, 40, 0, 0, 0, 0), 3)
    d = oc.write_case(case, tmp_path / "bad")
    with pytest.raises(ostc.OstcError, match="outside"):
        ostc.probe_case(str(d))


def test_face_not_on_a_side_rejected(built, tmp_path):
    case, _ = _case_dir(tmp_path)
    case.faces[2] = oc.Face((0, 32, 5, 5, 0, 0), 3)
    d = oc.write_case(case, tmp_path / "bad")
    with pytest.raises(ostc.OstcError, match="side"):
        ostc.probe_case(str(d))


def test_setup_grammar(built, tmp_path):
    """Comments, '//' continuation inside arrays, structs and later overrides (Parameter.cpp:39-185)."""
    _, d = _case_dir(tmp_path)
    s = (d / "setup.txt").read_text()
    s = s.replace("int reconstruction = 4", "int reconstruction = 5 // overridden below\n"
                  "! a bang comment\n\nint reconstruction = 4")
    s += "array real some_values = { 1 2 // next line\n  3 4 }\nrange real core = {\n 0 1\n -1 1\n}\n"
    (d / "setup.txt").write_text(s)
    p = ostc.probe_case(str(d))
    assert p["ngg"] == 3 and p["reconstruction"] == 4


def test_unknown_boundary_type_rejected(built, tmp_path):
    case, _ = _case_dir(tmp_path)
    case.faces[0] = oc.Face(case.faces[0].raw, 5)  # label 5 = supersonic inflow, not on this path
    d = oc.write_case(case, tmp_path / "bad")
    with pytest.raises(ostc.OstcError, match="label 5"):
        ostc.probe_case(str(d))


def test_boundary_faces_probe(built, tmp_path):
    """Walls, inflows and back pressure parse on the host (BoundCond.cpp:157-214, 497-560, 704-768):
    accepted for air, with the refusals the reference makes (subsonic inflow / back pressure with
    species, a subsonic inflow without its total-state ratios) or that this path makes (radiative walls,
    fluctuating inflow, an inflow without struct)."""
    ok = [("wall", oc.mixing_layer_3d(mx=12, my=10, mz=8, ybc="wall")),
          ("adiabatic", oc.mixing_layer_2d(mx=33, my=17, ybc="wall", wall_thermal="adiabatic")),
          ("inflow", oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="inflow")),
          ("subsonic", oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="subsonic", ybc="outflow"))]
    for name, case in ok:
        p = ostc.probe_case(str(oc.write_case(case, tmp_path / name)))
        assert p["n_faces"] == len(case.faces), name
    bad = oc.reacting_mixing_layer_3d(mx=12, my=10, mz=8)
    bad.faces[1] = oc.Face(bad.faces[1].raw, 9)
    bad.bc_structs["back_pressure"] = {"type": ("string", "back_pressure"), "label": ("int", 9),
                                       "pressure": ("real", 101325.0)}
    with pytest.raises(ostc.OstcError, match="multi-species"):
        ostc.probe_case(str(oc.write_case(bad, tmp_path / "bp_mix")))
    rad = oc.mixing_layer_3d(mx=12, my=10, mz=8, ybc="wall")
    rad.bc_structs["wall"]["thermal_type"] = ("string", "equilibrium_radiation")
    with pytest.raises(ostc.OstcError, match="equilibrium_radiation"):
        ostc.probe_case(str(oc.write_case(rad, tmp_path / "rad")))
    # white noise (1) is on the path; stability-mode (2), receptivity (3) fluctuations and profile-file
    # inflows are refused
    fl = oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="inflow", inflow_noise=0.01)
    assert ostc.probe_case(str(oc.write_case(fl, tmp_path / "fl1")))["n_faces"] == len(fl.faces)
    for key, val in (("fluctuation_type", 2), ("fluctuation_type", 3), ("inflow_type", 1)):
        fl = oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="inflow")
        fl.bc_structs["inflow"][key] = ("int", val)
        with pytest.raises(ostc.OstcError, match=key):
            ostc.probe_case(str(oc.write_case(fl, tmp_path / f"fl_{key}_{val}")))
    # the digital filter: a 3-D block with enough spanwise planes and the Gaussian stress supplier
    df = oc.spatial_mixing_layer_3d(mx=12, my=10, mz=56, fluctuation_type=11)
    assert ostc.probe_case(str(oc.write_case(df, tmp_path / "df")))["n_faces"] == len(df.faces)
    with pytest.raises(ostc.OstcError, match="mz - 1 >= 50"):
        ostc.probe_case(str(oc.write_case(oc.spatial_mixing_layer_3d(mx=12, my=10, mz=20, fluctuation_type=11),
                                          tmp_path / "df_thin")))
    with pytest.raises(ostc.OstcError, match="3-D block"):
        ostc.probe_case(str(oc.write_case(oc.spatial_mixing_layer_3d(mx=12, my=10, mz=1, fluctuation_type=11),
                                          tmp_path / "df_2d")))
    # a mixing-layer problem (problem_type 1) parses its streams; without them it is refused
    ml = oc.spatial_mixing_layer_3d(mx=12, my=10, mz=6, fluctuation_type=1)
    assert ostc.probe_case(str(oc.write_case(ml, tmp_path / "ml")))["n_faces"] == len(ml.faces)
    del ml.mixing_layer["lower"]["temperature"]
    with pytest.raises(ostc.OstcError, match="temperature"):
        ostc.probe_case(str(oc.write_case(ml, tmp_path / "ml_bad")))
    for key in ("pt_pRef_ratio", "Tt_TRef_ratio"):
        sub = oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="subsonic", ybc="outflow")
        del sub.bc_structs["subsonic_inflow"][key]
        with pytest.raises(ostc.OstcError, match=key):
            ostc.probe_case(str(oc.write_case(sub, tmp_path / ("sub_" + key))))
    nostruct = oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="inflow")
    del nostruct.bc_structs["inflow"]
    with pytest.raises(ostc.OstcError, match="needs a struct"):
        ostc.probe_case(str(oc.write_case(nostruct, tmp_path / "ns")))
