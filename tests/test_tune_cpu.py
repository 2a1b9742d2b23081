"""The smoother autotuner's candidate lists (fhd_tune_candidates, host only):
which plans exist for which levels, and that every tile it would time
divides the level and fits the device -- the geometry rules the GPU test
then exercises by forcing each candidate."""
import pytest

import lowmachfhd_b200 as L

SMEM_SM = 233472  # B200 shared memory per SM


def kinds(c):
    return {x["kind"] for x in c}


def test_fp32_visc1_large_level_has_every_kind():
    c = L.tune_candidates("stag", 3, [256, 256, 256], "mixed", 1)
    assert kinds(c) == {"colour", "tiled", "rowtile"}
    rows = [x for x in c if x["kind"] == "rowtile"]
    # one CTA per SM with the deep ring for 4- and 8-row tiles (256 or 512
    # compute threads); the short ring only where two CTAs fit on one SM
    assert {(x["y"], x["per_sm"], x["threads"]) for x in rows} == {(4, 1, 256), (8, 1, 256), (4, 2, 256),
                                                                  (4, 1, 512), (8, 1, 512)}
    for x in rows:
        assert 256 % x["y"] == 0 and x["zruns"] >= 1
        assert x["per_sm"] * (x["smem"] + 1024) <= SMEM_SM
        assert x["smem"] <= 232448
    for x in c:
        if x["kind"] == "tiled":
            assert 256 % x["x"] == 0 and x["x"] % 4 == 0 and x["x"] <= 64
            assert 256 % x["y"] == 0 and x["y"] % 2 == 0 and x["y"] <= 8
        if x["kind"] == "colour":
            assert x["x"] * x["y"] == 256


@pytest.mark.parametrize("prec,visc", [("fp64", 1), ("mixed", -1), ("mixed", 2)])
def test_rowtile_only_for_fp32_constant_viscosity(prec, visc):
    c = L.tune_candidates("stag", 3, [128, 128, 128], prec, visc)
    assert "rowtile" not in kinds(c)
    assert {"colour", "tiled"} <= kinds(c)
    if prec == "fp64":
        for x in c:
            if x["kind"] == "tiled":
                assert x["x"] % 2 == 0


def test_two_dimensional_levels_use_colour_blocks():
    c = L.tune_candidates("stag", 2, [256, 256], "mixed", 1)
    assert kinds(c) == {"colour"}
    assert len(c) == 4
    # a 32-wide level (16 cells of a colour per row) skips blocks wider than 32
    c = L.tune_candidates("stag", 2, [32, 32], "mixed", 1)
    assert all(x["x"] <= 32 for x in c)


def test_pressure_levels():
    c = L.tune_candidates("cc", 3, [64, 64, 64], "mixed", 1)
    assert kinds(c) == {"colour", "tiled"}
    c = L.tune_candidates("cc", 3, [24, 24, 22], "fp64", 1)
    assert {"colour", "tiled"} <= kinds(c)
    for x in c:
        if x["kind"] == "tiled":
            assert 24 % x["x"] == 0 and 24 % x["y"] == 0


def test_odd_extent_has_no_fused_candidates():
    c = L.tune_candidates("stag", 3, [24, 24, 23], "mixed", 1)
    assert kinds(c) == {"colour"}


def test_bad_arguments():
    with pytest.raises(L.FhdError):
        L.tune_candidates("stag", 4, [8, 8, 8])
    with pytest.raises(L.FhdError):
        L.tune_candidates("stag", 3, [1, 8, 8])


K96S = L.tune_key("stag", 3, [96, 96, 96], "mixed", 1)
K96C = L.tune_key("cc", 3, [96, 96, 96], "mixed", 1)


def test_table_key_names_version_and_device():
    ver = K96S.split(":")[0]
    assert ver[0] == "v" and int(ver[1:]) >= 3
    assert K96S == f"{ver}:0:s:4:3:1:96x96x96:148:232448:233472"
    assert L.tune_key("cc", 3, [96, 96, 96], "fp64", 2, sms=132, smem_optin=232448, smem_sm=233472,
                      device=1) == f"{ver}:1:c:8:3:0:96x96x96:132:232448:233472"
    with pytest.raises(L.FhdError):
        L.tune_key("stag", 4, [8, 8, 8])


def test_table_import_export_roundtrip():
    text = f"{K96S} 11\n{K96C} 2\n"
    assert L.tune_import(text) == 2
    out = L.tune_export()
    for line in text.splitlines():
        assert line in out.splitlines()
    # re-importing replaces, and an empty text adds nothing
    assert L.tune_import(f"{K96S} 3\n") == 1
    assert f"{K96S} 3" in L.tune_export().splitlines()
    assert L.tune_import("") == 0


def test_table_import_skips_other_versions():
    ver = K96S.split(":")[0]
    other = "v1:" + K96S[len(ver) + 1:].replace("96x96x96", "88x88x88")
    assert L.tune_import(f"{other} 4\n") == 0
    assert other not in L.tune_export()


@pytest.mark.parametrize("bad", [f"{K96S}\n", "nonsense 1\n", f"{K96S} x\n", K96S.replace(":s:", ":q:") + " 1\n",
                                 f"{K96S} 1 2\n", "0:s:4:3:1:96x96x96 1\n"])
def test_table_import_rejects_malformed_lines(bad):
    before = L.tune_export()
    with pytest.raises(L.FhdError):
        L.tune_import(L.tune_key("stag", 3, [40, 40, 40]) + " 1\n" + bad)
    assert L.tune_export() == before
