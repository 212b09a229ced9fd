"""The launch-shape tuner's host logic (volcano_ca_mc_b200.tuner): shape classes, candidates, the
choice rule and the table lookup, on the CPU (timing the candidates needs a GPU)."""
from volcano_ca_mc_b200 import capi, tuner


def test_shape_class_and_candidates():
    assert tuner.shape_class(1024, 1024, 256, "pentagonal") == "3d-pentagonal-28"
    assert tuner.shape_class(512, 1, 256, "moore") == "xz-moore-17"
    assert tuner.shape_class(300, 200, 1, "hexagonal") == "xy-hexagonal-16"
    assert len(tuner.candidates(64, 64, 32)) == 10
    assert tuner.candidates(512, 1, 256) == [(0, 0, 0), (0, 0, 2)]


def test_choice_keeps_the_default_within_the_margin():
    assert tuner.choose({"4x4/b0": 4.22, "8x2/b0": 4.12, "2x8/b0": 4.5}) == "4x4/b0"  # 2.4 % only
    assert tuner.choose({"4x4/b0": 4.22, "8x2/b0": 4.00}) == "8x2/b0"                  # 5.2 %
    assert tuner.choose({"4x4/b0": 4.0, "4x4/b2": 4.3}) == "4x4/b0"


def test_lookup_exact_nearest_and_absent():
    table = {"classes": {"3d-moore-20": {"tile": [8, 2], "rules_blocks_per_sm": 2},
                         "3d-moore-24": {"tile": [2, 8], "rules_blocks_per_sm": 0}}}
    assert tuner.lookup(128, 128, 64, "moore", table) == (8, 2, 2)       # 2^20: exact
    assert tuner.lookup(256, 256, 128, "moore", table) == (2, 8, 0)      # 2^23: nearest is 2^24
    assert tuner.lookup(128, 128, 64, "pentagonal", table) == (0, 0, 0)  # no entry of that neighbourhood
    assert tuner.lookup(512, 1, 256, "moore", table) == (0, 0, 0)        # 2D: no 2D entries
    p = capi.CaParams(128, 128, 64, neighborhood="moore")
    tuner.apply(p, table)
    assert (p.tile_y, p.tile_z, p.rules_blocks_per_sm) == (8, 2, 2)


def test_committed_table_is_well_formed():
    table = tuner.load_table()
    assert table.get("classes"), "volcano_ca_mc_b200/tuning.json holds no classes"
    shapes = {f"{ty}x{tz}" for ty, tz in tuner.TILES_3D}
    for cls, e in table["classes"].items():
        assert cls.startswith("3d-")
        assert f"{e['tile'][0]}x{e['tile'][1]}" in shapes and e["rules_blocks_per_sm"] in tuner.BLOCKS
        assert tuner.choose(e["ms"]) == f"{e['tile'][0]}x{e['tile'][1]}/b{e['rules_blocks_per_sm']}", cls
