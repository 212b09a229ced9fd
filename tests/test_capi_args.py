"""Argument checks and empty inputs of the C ABI.

Invalid configurations are refused with VCA_ERR_ARG (status 1, the reference's ConfigError) before
any device work, so those checks run without a GPU; the footprints are host arithmetic.  The GPU
part covers the refusals that need a handle (vents outside the grid, negative heights, terrain in
classic mode) and the empty cases: a lava run without vents stops at once with "no lava"
(countInitialState, engine/src/ca/LavaCA.hpp:1272-1279), an MC stage on an empty domain still
counts its sweeps (PottsMC.cpp:516-533), and flow sums over zero flows."""
import numpy as np
import pytest

from volcano_ca_mc_b200 import capi


def _refused(make, match):
    with pytest.raises(capi.VcaError, match=r"\(status 1\).*" + match):
        make()


@pytest.mark.parametrize("dims,kw,match", [
    ((10, 1, 1), {}, "2D .*or 3D"),
    ((40, 30, 1), {}, "x-z cross-section"),
    ((40, 1, 40), {"max_steps": 70000}, "max_steps"),
    ((20, 20, 20), {"neighborhood": "hexagonal"}, "hexagonal"),
    ((2000, 2000, 1000), {}, "2 000 000 000"),
])
def test_ca_create_refuses(dims, kw, match):
    _refused(lambda: capi.LavaCA(capi.CaParams(*dims, **kw)), match)
    _refused(lambda: capi.ca_footprint(capi.CaParams(*dims, **kw)), match)


@pytest.mark.parametrize("kw,match", [({"Q": 1}, "Q must be"), ({"J": 0.0}, "J must be"), ({"kT": -1.0}, "kT"),
                                      ({"neighborhood": "hexagonal"}, "hexagonal")])
def test_mc_create_refuses(kw, match):
    _refused(lambda: capi.PottsMC(capi.McParams(20, 20, 20, **kw)), match)


def test_footprints_grow_with_the_space():
    small = capi.ca_footprint(capi.CaParams(64, 64, 32))
    big = capi.ca_footprint(capi.CaParams(256, 256, 128))
    assert 0 < small < big
    # the full-size grid: 2 x 13 B of state per cell plus schedule and derived planes, about 9 GB
    c3 = capi.ca_footprint(capi.CaParams(1024, 1024, 256, neighborhood="pentagonal"))
    assert 7e9 < c3 < 11e9
    assert 0 < capi.mc_footprint(capi.McParams(64, 64, 32)) < capi.mc_footprint(capi.McParams(256, 256, 128))


@pytest.mark.gpu
def test_handle_refusals():
    ca = capi.LavaCA(capi.CaParams(32, 1, 24))
    heights = np.full(32, 4, np.int32)
    heights[3] = -1
    _refused(lambda: ca.apply_terrain(heights), "negative height")
    ca.apply_terrain(np.full(32, 4, np.int32))
    _refused(lambda: ca.place_seeds([(40, 0, 5, 1)]), "outside the grid")
    ca.close()
    classic = capi.LavaCA(capi.CaParams(16, 16, 8, mode="classic"))
    _refused(lambda: classic.apply_terrain(np.zeros(256, np.int32)), "lava mode only")
    classic.close()


@pytest.mark.gpu
def test_empty_inputs():
    ca = capi.LavaCA(capi.CaParams(48, 1, 32, max_steps=50))
    ca.apply_terrain(np.full(48, 6, np.int32))
    ca.place_seeds([])
    ca.run()
    info = ca.info()
    assert (info.steps, capi.STOP_NAMES[info.stop_reason]) == (0, "no lava")
    lava, basalt, reach2 = ca.flow_stats(0)
    assert lava.tolist() == basalt.tolist() == reach2.tolist() == [0]

    mc = capi.PottsMC(capi.McParams(48, 1, 32, Q=16))
    mc.set_domain_from_ca(ca)  # no basalt: an empty domain
    mc.initialize()
    mc.sweep(5)
    mi = mc.info()
    assert (mi.sweeps, mi.attempts, mi.domain_cells) == (5, 0, 0)
    assert mc.energy() == 0.0
    assert not mc.crystals().any()
    mc.close()
    ca.close()


@pytest.mark.parametrize("dims,match", [
    ((1024, 1024, 256), "null spins"),           # exactly 2^28 cells: within the limit
    ((15790321, 17, 1), "exceed the fixed scratch"),  # 2^28 + 1 cells
])
def test_noalloc_size_limit(dims, match):
    """The 2^28-cell limit of vca_mc_energy_noalloc is checked before the pointers, so null pointers
    show which side of the limit a size falls on without any grid or device."""
    _refused(lambda: capi.mc_energy_noalloc(0, *dims, 0), match)


@pytest.mark.parametrize("dims,tile,match", [
    ((40, 20, 20), (4, 2), "16 cells"),
    ((40, 20, 20), (3, 5), "16 cells"),
    ((64, 1, 40), (4, 4), "tile_y = 1"),
    ((64, 40, 1), (4, 4), "tile_z = 1"),
])
def test_ca_tile_shape_refusals(dims, tile, match):
    mode = "classic" if dims[2] == 1 else "lava"  # a 2D lava space is the x-z section
    _refused(lambda: capi.LavaCA(capi.CaParams(*dims, mode=mode, tile_y=tile[0], tile_z=tile[1])), match)
