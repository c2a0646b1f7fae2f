"""flb_total_mass_noalloc (the allocation-free mass sum) against flb_total_mass.

Collected last on purpose: the entry point's scratch lives in a fixed device
array that stays resident once the library is loaded, and it must give the
same sum both in a fresh process and after every other test has run.
"""
import numpy as np
import pytest

from flowlb_b200 import cases
from flowlb_b200 import engine as E


def _device_fields(torch, s, n):
    mass = torch.empty(n, dtype=torch.float64, device="cuda")
    excess = torch.empty(n, dtype=torch.float64, device="cuda")
    flags = torch.empty(n, dtype=torch.uint8, device="cuda")
    s.read_device(E.FIELD_MASS, mass.data_ptr())
    s.read_device(E.FIELD_EXCESS, excess.data_ptr())
    s.read_device(E.FIELD_FLAGS, flags.data_ptr())
    s.sync()
    return mass, excess, flags


@pytest.mark.gpu
@pytest.mark.parametrize("fs_mode", [E.FS_REFERENCE, E.FS_CONSERVATIVE], ids=["reference", "conservative"])
@pytest.mark.parametrize("shape", [(64, 48), (257, 131)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_noalloc_mass_matches_handle_mass(require_gpu, fs_mode, shape):
    import torch
    nx, ny = shape
    case = cases.small_dam_break(nx, ny)
    s = E.Solver(case.flags, free_surface=True, precision=32, mass_precision=64, tau=case.tau, fx=case.fx,
                 fy=case.fy, fs_mode=fs_mode, u_max=0.25)
    s.step(37)
    expect = s.total_mass()
    mass, excess, flags = _device_fields(torch, s, nx * ny)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row on the same scratch
    for k in range(2):
        E.total_mass_noalloc(mass.data_ptr(), excess.data_ptr(), flags.data_ptr(), nx, ny, fs_mode,
                             out[k:].data_ptr(), stream)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    # same cells, same per-block tree and the same fixed-order final sum: the
    # results agree to the last bit (a change of reduction order would show
    # here); the message gives the relative difference for diagnosis
    for k in range(2):
        assert got[k] == expect, (k, got[k], expect, abs(got[k] - expect) / abs(expect))
    assert got[0] == got[1]
    # and it does not depend on the solver's own state or scratch
    s.step(5)
    mass2, excess2, flags2 = _device_fields(torch, s, nx * ny)
    E.total_mass_noalloc(mass2.data_ptr(), excess2.data_ptr(), flags2.data_ptr(), nx, ny, fs_mode,
                         out.data_ptr(), stream)
    torch.cuda.synchronize()
    assert float(out[0].item()) == s.total_mass()


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Validated before any CUDA call, so it needs no device: a grid larger
    than FLB_NOALLOC_MAX_CELLS (16,777,216 cells) is refused, as are bad modes
    and null pointers."""
    fake = 256  # never dereferenced: every case below is rejected on the host
    with pytest.raises(E.FlowLBError) as ei:
        E.total_mass_noalloc(fake, fake, fake, 4097, 4096, E.FS_CONSERVATIVE, fake)
    assert ei.value.status == 1
    with pytest.raises(E.FlowLBError):
        E.total_mass_noalloc(fake, fake, fake, 64, 64, 7, fake)
    with pytest.raises(E.FlowLBError):
        E.total_mass_noalloc(0, fake, fake, 64, 64, E.FS_CONSERVATIVE, fake)
