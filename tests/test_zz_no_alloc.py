"""The allocation-free OC update (``tp3d_oc_update_noalloc``).

Some callers cannot allocate device memory per call: applications whose device
memory is reserved up front by their own allocator, or code that cannot accept
the implicit device synchronisation of cudaMalloc / cudaFree.  For them the
library offers an OC update whose scratch is a static device array.  These
tests call it through the C ABI, three times in a row on different designs
(a small grid, a filter radius at the stencil's limit, and a grid of exactly
the static maximum of elements), and compare it with the allocating entry
point ``tp3d_oc_update``: both run the same kernel on the same launch grid,
so the results must agree bit for bit.  This file is collected last so that a
run that stops at the first failure has already run every other test; it also
passes on its own in a fresh process (the first call does the per-device
set-up).
"""

import numpy as np
import pytest
import torch

from oracle import simp_oracle as O


def _problem(nx, ny, nz, rmin, seed):
    """A seeded OC input: design, filtered sensitivities of the cantilever masks."""
    import pytopo3d_b200 as P

    rng = np.random.default_rng(seed)
    shape = (ny, nx, nz)
    solid, void, free = O.prepare_masks(nx, ny, nz)
    x = rng.uniform(0.1, 0.9, size=shape)
    x[solid], x[void] = 1.0, 0.0
    H, Hs = P.build_filter(nx, ny, nz, rmin)
    _, _, dp = P.build_physical_density(x, H, Hs, 2.0, 0.5, solid, void)
    dc = -np.abs(rng.normal(size=shape))
    dc_dx = P.apply_density_filter_chain_rule(dc, dp, H, Hs)
    dv_dx = P.apply_density_filter_chain_rule(free.astype(float), dp, H, Hs)
    Hs = Hs.cpu().numpy() if isinstance(Hs, torch.Tensor) else np.asarray(Hs)
    return x, dc_dx, dv_dx, Hs, solid, void, 0.3 * int(free.sum())


def _flat(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a).transpose(2, 1, 0)).reshape(-1)).to("cuda", dtype)


def _run(L, fn, dims, rmin, args, scratch=None):
    from pytopo3d_b200 import _lib

    nx, ny, nz = dims
    x, dc, dv, Hs, solid, void, target = args
    xd, dcd, dvd = _flat(x), _flat(dc), _flat(dv)
    Hsd = torch.as_tensor(Hs).to("cuda")
    sd, vd = _flat(solid, torch.uint8), _flat(void, torch.uint8)
    xn, rn = torch.empty_like(xd), torch.empty_like(xd)
    stats = torch.empty(8, dtype=torch.float64, device="cuda")
    common = [nx, ny, nz, rmin, xd.data_ptr(), dcd.data_ptr(), dvd.data_ptr(), Hsd.data_ptr(), sd.data_ptr(),
              vd.data_ptr(), 0.2, target, 2.0, 0.5, 80, 1e-8, xn.data_ptr(), rn.data_ptr(), stats.data_ptr()]
    if scratch is None:
        rc = fn(*common, _lib.stream_ptr())
    else:
        rc = fn(*common, scratch.data_ptr(), _lib.stream_ptr())
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return xn.cpu().numpy(), rn.cpu().numpy(), stats.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_oc_update_matches_allocating_entry_point():
    from pytopo3d_b200 import _lib

    L = _lib.lib()
    cap = L.tp3d_oc_noalloc_max_elements()
    # calls in a row on different sizes and radii: rmin 6.9 fills the largest
    # column table (offsets up to 6), 64x64x64 is exactly the element limit
    cases = [((16, 8, 8), 2.5, 1), ((23, 9, 7), 6.9, 2), ((64, 64, 64), 1.5, 3)]
    assert 64 * 64 * 64 == cap
    for dims, rmin, seed in cases:
        args = _problem(*dims, rmin, seed)
        nbytes = L.tp3d_oc_scratch_bytes(*dims, rmin)
        scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        ref = _run(L, L.tp3d_oc_update, dims, rmin, args, scratch)
        got = _run(L, L.tp3d_oc_update_noalloc, dims, rmin, args)
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)
        assert np.isfinite(got[2][2]) and got[2][2] >= 1  # bisection steps recorded


def test_noalloc_rejects_grids_above_its_static_limit():
    from pytopo3d_b200 import _lib

    L = _lib.lib()
    cap = L.tp3d_oc_noalloc_max_elements()
    assert cap == 1 << 18
    # rejected on the host, before any device work
    rc = L.tp3d_oc_update_noalloc(cap, 2, 1, 1.5, 1, 1, 1, 1, None, None, 0.2, 1.0, 2.0, 0.5, 80, 1e-8, 1, 1, 1,
                                  None)
    assert rc == _lib.TP3D_ERR_ARG
    assert "262144" in _lib.last_error()
