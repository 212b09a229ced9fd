"""vca_mc_energy_noalloc (the allocation-free energy entry point) against vca_mc_energy on the same
spins: a grid in torch device memory, two calls in a row on torch's current stream, each equal to
the handle's energy (exact: both count unlike pairs in integers, tolerance 0).  Collected last so
that it also runs after every other GPU test in the same process."""
from __future__ import annotations

import numpy as np
import pytest

from volcano_ca_mc_b200 import capi

pytestmark = pytest.mark.gpu

CASES = [
    # (nx, ny, nz, neighborhood, boundary, full domain, sweeps)
    (24, 20, 16, "moore", "periodic", True, 5),
    (33, 31, 20, "von_neumann", "periodic", False, 4),
    (36, 28, 20, "pentagonal", "periodic", False, 3),
    (64, 1, 40, "hexagonal", "absorbing", True, 6),
    (128, 128, 96, "moore", "periodic", True, 2),  # 384 blocks: the last block adds > 256 partials
]


def handle_energy_and_spins(nx, ny, nz, nb, bc, full, sweeps, seed=5):
    mc = capi.PottsMC(capi.McParams(nx, ny, nz, neighborhood=nb, boundary=bc, domain_full=full, seed=seed, Q=16,
                                    kT=0.5))
    if full:
        mc.set_domain(None)
    else:
        rng = np.random.default_rng(seed)
        mc.set_domain((rng.random(nx * ny * nz) < 0.6).astype(np.uint8))
    mc.initialize()
    mc.sweep(sweeps)
    e, spins = mc.energy(), mc.crystals()
    mc.close()
    return e, spins


@pytest.mark.parametrize("nx,ny,nz,nb,bc,full,sweeps", CASES)
def test_noalloc_energy_matches_handle(nx, ny, nz, nb, bc, full, sweeps):
    import torch

    expected, spins = handle_energy_and_spins(nx, ny, nz, nb, bc, full, sweeps)
    dev = torch.from_numpy(spins).cuda()
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(2):
        capi.mc_energy_noalloc(dev.data_ptr(), nx, ny, nz, out.data_ptr() + 8 * k, neighborhood=nb, boundary=bc,
                               domain_full=full, seed=5, mcs=sweeps, J=1.0, stream=stream)
    torch.cuda.synchronize()
    got = out.cpu().tolist()
    assert got[0] == expected and got[1] == expected, (got, expected)


def test_noalloc_large_then_small_call():
    """A 384-block call followed by a 1-block call on the same stream: the ticket target changes
    between them, and each result must still equal the handle's energy."""
    import torch

    big = handle_energy_and_spins(128, 128, 96, "moore", "periodic", True, 2)
    small = handle_energy_and_spins(24, 20, 8, "von_neumann", "absorbing", True, 3)
    dev_big = torch.from_numpy(big[1]).cuda()
    dev_small = torch.from_numpy(small[1]).cuda()
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    capi.mc_energy_noalloc(dev_big.data_ptr(), 128, 128, 96, out.data_ptr(), neighborhood="moore", boundary="periodic",
                           domain_full=True, seed=5, mcs=2, J=1.0, stream=stream)
    capi.mc_energy_noalloc(dev_small.data_ptr(), 24, 20, 8, out.data_ptr() + 8, neighborhood="von_neumann",
                           boundary="absorbing", domain_full=True, seed=5, mcs=3, J=1.0, stream=stream)
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [big[0], small[0]]


def test_noalloc_rejects_oversized_grid():
    import torch

    spins = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.VcaError, match="exceed the fixed scratch"):
        capi.mc_energy_noalloc(spins.data_ptr(), 1024, 1024, 257, out.data_ptr())


def test_noalloc_rejects_host_pointer():
    import torch

    host = np.zeros(64, np.int32)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.VcaError):
        capi.mc_energy_noalloc(host.ctypes.data, 8, 8, 1, out.data_ptr())
