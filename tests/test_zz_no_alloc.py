"""The allocation-free cell binning entry point (simox_cell_sort_noalloc).

It exists for callers that cannot let a library allocate device memory:
programs whose GPU memory is owned by another allocator (a caching pool, an
arena reserved at start-up) or per-step loops where cudaMalloc/cudaFree
would synchronise the device.  Its only scratch is a fixed device array in
the library.  Here its output, called through the C ABI on two different
systems in a row (so stale scratch from the first call would show), must
equal what the allocating entry point simox_cell_sort + simox_get_cells
returns for the same positions: bit-exact, as binning is integer work.  The
test allocates its own device buffers (with torch); the entry point does not.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from simox_b200 import _abi, systems as S

pytestmark = pytest.mark.gpu


def _reference_cells(s, stride):
    from simox_b200 import api
    with api.from_system(s) as g:
        g.cell_sort()
        return g.get_cells(link_stride=stride)


def _noalloc_cells(lib, s, stride):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(s.x)).cuda()
    nc = [int(b // s.rcut) for b in s.box]
    ncell = nc[0] * nc[1] * nc[2]
    npt = torch.full((ncell,), -1, dtype=torch.int32, device="cuda")
    link = torch.zeros((ncell, stride), dtype=torch.int32, device="cuda")
    box = (C.c_double * 3)(*[float(b) for b in s.box])
    torch.cuda.synchronize()
    st = lib.simox_cell_sort_noalloc(C.c_void_p(x.data_ptr()), s.n, box, float(s.rcut),
                                     C.c_void_p(npt.data_ptr()), C.c_void_p(link.data_ptr()), stride, None)
    assert st == 0, _abi.status_text(st)
    return npt.cpu().numpy(), link.cpu().numpy()


def _same(ref, got):
    npt_r, link_r = ref
    npt_g, link_g = got
    assert np.array_equal(npt_r, npt_g)
    for c in range(len(npt_r)):
        assert np.array_equal(link_r[c, : npt_r[c]], link_g[c, : npt_g[c]]), c


def test_noalloc_matches_cell_sort_on_two_calls(simox_lib):
    stride = 500
    a = S.al_slab_oxygen(seed=3)                                   # 2,700 atoms, 4x4x4 cells
    b = S.small_alo(seed=8, n=900, box=(41.0, 31.5, 52.0), fft=(16, 16, 16))   # 4x3x5 cells
    for s in (a, b):
        _same(_reference_cells(s, stride), _noalloc_cells(simox_lib, s, stride))


def test_noalloc_rejects_sizes_beyond_its_scratch(simox_lib):
    import torch
    # small real device buffers: if a later change reordered the argument
    # checks after the launches, a wrong status would show, not a bad address
    npt = torch.zeros(1, dtype=torch.int32, device="cuda")
    link = torch.zeros(1, dtype=torch.int32, device="cuda")
    p_npt, p_link = C.c_void_p(npt.data_ptr()), C.c_void_p(link.data_ptr())
    box = (C.c_double * 3)(1000.0, 1000.0, 1000.0)     # 100^3 cells > 65,536
    st = simox_lib.simox_cell_sort_noalloc(None, 0, box, 10.0, p_npt, p_link, 500, None)
    assert st == _abi.SIMOX_E_SCRATCH_LIMIT
    box = (C.c_double * 3)(40.0, 40.0, 40.0)
    st = simox_lib.simox_cell_sort_noalloc(None, 0, box, 10.0, p_npt, p_link, 5000, None)
    assert st == _abi.SIMOX_E_SCRATCH_LIMIT
    torch.cuda.synchronize()
    assert int(npt.item()) == 0 and int(link.item()) == 0


def test_noalloc_grid_rule_agrees_with_create(simox_lib):
    """Both entry points reject a cell grid with one cell on an axis."""
    import torch
    from simox_b200 import api
    s = S.small_alo(seed=8, n=200, box=(41.0, 31.5, 52.0), fft=(16, 16, 16))
    s.box = np.array([41.0, 31.5, 15.0])                      # 4 x 3 x 1 cells
    s.x[:, 2] = np.clip(s.x[:, 2], -7.4, 7.4)
    with pytest.raises(api.SimoxError) as ei:
        api.from_system(s)
    assert ei.value.code == _abi.SIMOX_E_CELL_TOO_SMALL
    npt = torch.zeros(12, dtype=torch.int32, device="cuda")
    link = torch.zeros((12, 500), dtype=torch.int32, device="cuda")
    x = torch.from_numpy(np.ascontiguousarray(s.x)).cuda()
    box = (C.c_double * 3)(*[float(b) for b in s.box])
    st = simox_lib.simox_cell_sort_noalloc(C.c_void_p(x.data_ptr()), s.n, box, float(s.rcut),
                                           C.c_void_p(npt.data_ptr()), C.c_void_p(link.data_ptr()), 500, None)
    assert st == _abi.SIMOX_E_CELL_TOO_SMALL
