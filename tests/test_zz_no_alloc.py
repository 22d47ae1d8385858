"""rw_cell_sort_noalloc: the cell-key sort for callers that cannot allocate device
memory (a host whose allocator belongs to another framework, a loop that must not
block in cudaMalloc, a plugin host that forbids allocations).  The caller passes device
inputs and outputs; the entry point uses only the library's fixed scratch array.

Checked against the library's normal path: the first neighbour search of
rw_create_from_case sorts the same keys, and rw_get_array(RW_ARR_PART_IDX) returns its
permutation.  Integer work, so the comparison is exact, on two calls in a row."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(L, keys_d, n, max_key, out_k, out_p, stream):
    return L.rw_cell_sort_noalloc(ct.c_void_p(keys_d.data_ptr()), n, max_key, ct.c_void_p(out_k.data_ptr()),
                                  ct.c_void_p(out_p.data_ptr()), ct.c_void_p(stream))


def test_noalloc_sort_matches_neighbor_search():
    import torch

    from retainwall_code_b200 import LoquatSph, _lib, cases as C

    L = _lib.lib()
    case = C.retaining_wall(nx=40, ny=20, nz=30, dx=0.0025)
    sim = LoquatSph(case=case)
    perm = sim.get("part_idx")                  # permutation of the library's own sort
    keys_sorted = sim.get("cellpos")[:, 3].copy()
    info = sim.info()
    sim.close()
    n = info.np
    assert n <= (1 << 20)
    keys_in = np.empty_like(keys_sorted)
    keys_in[perm] = keys_sorted                  # keys in the case's original order
    dev = torch.device("cuda", 0)
    keys_d = torch.from_numpy(keys_in).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        out_k = torch.full((n,), -7, dtype=torch.int32, device=dev)
        out_p = torch.full((n,), -7, dtype=torch.int32, device=dev)
        st = _call(L, keys_d, n, info.ncell - 1, out_k, out_p, stream)
        assert st == 0, (call, st)
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(out_p.cpu().numpy(), perm, err_msg=f"call {call}: permutation")
        np.testing.assert_array_equal(out_k.cpu().numpy(), keys_sorted, err_msg=f"call {call}: keys")
    assert torch.equal(keys_d.cpu(), torch.from_numpy(keys_in))  # input untouched


def test_noalloc_sort_rejects_oversize():
    from retainwall_code_b200 import _lib

    L = _lib.lib()
    big = (1 << 20) + 1
    assert L.rw_cell_sort_noalloc(ct.c_void_p(8), big, 100, ct.c_void_p(8), ct.c_void_p(8), None) == 1
    assert L.rw_cell_sort_noalloc(ct.c_void_p(8), 10, 1 << 24, ct.c_void_p(8), ct.c_void_p(8), None) == 1
