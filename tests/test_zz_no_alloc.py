"""fsl_cell_list_noalloc: the cell list for callers that cannot allocate device
memory (frameworks that own the device memory, loops that must not stall
in-flight GPU work).  Its output must equal the
handle-based fsl_cell_list exactly (cell lists are integer results, compared
bit for bit), on two calls in a row that share the library's scratch array.

This file is collected last so that a failure here comes after every other
test has run.
"""
import ctypes

import numpy as np
import pytest

from helpers import uniform_positions

pytestmark = pytest.mark.gpu


def _noalloc(L, lx, ly, lz, cutoff, q, m, torch):
    n = q.shape[1]
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    cell_of = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    start = torch.full((m + 1,), -7, dtype=torch.int32, device="cuda")
    srt = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.fsl_cell_list_noalloc(lx, ly, lz, cutoff, n, qd.data_ptr(), cell_of.data_ptr(),
                                 start.data_ptr(), srt.data_ptr(), stream)
    torch.cuda.synchronize()
    return rc, cell_of.cpu().numpy()[:n], start.cpu().numpy(), srt.cpu().numpy()[:n]


def test_noalloc_matches_handle_entry_point(fsl):
    import torch
    from fluam_b200 import _lib
    L = _lib.load()
    box = (20.0, 16.0, 24.0)
    cutoff = 1.5
    q1 = uniform_positions(5000, box, 31)
    q1[:, :40] += 57.0  # unwrapped coordinates
    q2 = uniform_positions(3000, box, 32) * 0.4  # denser, fewer particles: stale scratch
    for q in (q1, q2):
        cfg = fsl.make_config((20, 16, 24), box, kT=0.01, dt=0.01, cutoff=cutoff)
        ref = fsl.StokesLimit(cfg, q)
        c_ref, s_ref, p_ref = ref.cell_list()
        m = len(s_ref) - 1
        ref.close()
        rc, c, s, p = _noalloc(L, *box, cutoff, q, m, torch)
        assert rc == 0, _lib.last_error()
        np.testing.assert_array_equal(c, c_ref)
        np.testing.assert_array_equal(s, s_ref)
        np.testing.assert_array_equal(p, p_ref)


def test_noalloc_rejects_sizes_beyond_its_scratch(fsl):
    import torch
    from fluam_b200 import _lib
    L = _lib.load()
    q = np.zeros((3, 4))
    # 160^3 > 2^20 neighbour-grid cells
    rc, *_ = _noalloc(L, 240.0, 240.0, 240.0, 1.5, q, 27, torch)
    assert rc == -1 and "1048576" in _lib.last_error()
    rc = L.fsl_cell_list_noalloc(10.0, 10.0, 10.0, 1.5, (1 << 18) + 1, None, None, None, None,
                                 None)
    assert rc == -1 and "262144" in _lib.last_error()
