"""cfg_xz_c2r_noalloc: the allocation-free inverse x-z plane transform, for
callers that cannot allocate device memory (device memory pre-assigned to
another owner, or a step loop that cannot take cudaMalloc's synchronisation).

Checked through the C ABI against the existing entry point cfg_xz_c2r, on
two calls in a row (the shared fixed scratch keeps the first call's contents),
at the FP64 tolerance of the other transform tests.  This file is collected
last so that a run stopping at its first failure has run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _check_calls(cf, L, nx, nz, ncalls, rng):
    import torch
    grid = cf.Grid(nx, 17, nz, lx=4 * np.pi, lz=2 * np.pi, stretch=1.5)
    flow = cf.ChannelFlow(grid, precision=cf.FP64, device=0)
    nxh, nx2, nz2 = nx // 2 + 1, grid.nx2, grid.nz2
    for trial in range(ncalls):
        c = (rng.standard_normal((nz, nxh)) + 1j * rng.standard_normal((nz, nxh))) * (trial + 1)
        ref = flow.xz_fft_complex_to_real(c)
        cd = torch.from_numpy(np.ascontiguousarray(c.ravel(order="F")).view(np.float64).copy()).cuda()
        out = torch.full((nx2 * nz2,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        r = L.cfg_xz_c2r_noalloc(nx, nz, nx2, nz2, cd.data_ptr(), out.data_ptr(), None)
        torch.cuda.synchronize()
        assert r == 0
        got = out.cpu().numpy().reshape((nx2, nz2), order="F")
        assert rel(got, ref) < 1e-12, (nx, nz, trial, rel(got, ref))
    flow.close()


def test_noalloc_matches_cfg_xz_c2r_twice(cf):
    L = cf.load_library()
    rng = np.random.default_rng(2024)
    # two calls in a row on one plane size (the second reuses the twiddle
    # tables the first wrote), then another size and back
    _check_calls(cf, L, 32, 24, 2, rng)
    _check_calls(cf, L, 48, 16, 1, rng)
    _check_calls(cf, L, 32, 24, 1, rng)


def test_noalloc_rejects_oversized_plane(cf):
    L = cf.load_library()
    # (nx/2+1)*nz2 = 1025*1536 exceeds the 262144-element scratch
    assert L.cfg_xz_c2r_noalloc(2048, 1024, 3072, 1536, 1, 1, None) == -7
    assert L.cfg_xz_c2r_noalloc(1024, 1024, 1536, 1536, 1, 1, None) == -7
