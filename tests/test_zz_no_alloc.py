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


@pytest.mark.parametrize("max_key,n", [(200, 5000), ((1 << 24) - 1, 300_001), ((1 << 16) + 5, 2048 * 7 + 1)],
                         ids=["one-pass", "three-pass", "three-pass-small"])
def test_noalloc_sort_pass_counts(max_key, n):
    """Key ranges that take one pass (max_key < 2^8) and three passes (max_key >= 2^16):
    with an odd pass count the first pass writes the caller's outputs and reads its
    values from an identity in the scratch.  Random keys, n not a multiple of the
    2048-key tile, two calls in a row (the scratch keeps the previous call's contents);
    the result equals numpy's stable argsort."""
    import torch

    from retainwall_code_b200 import _lib

    L = _lib.lib()
    rng = np.random.default_rng(max_key % 1000 + n)
    keys = rng.integers(0, max_key + 1, n, dtype=np.int64).astype(np.int32)
    keys[: n // 10] = max_key  # many ties at the top key
    perm = np.argsort(keys, kind="stable").astype(np.int32)
    dev = torch.device("cuda", 0)
    keys_d = torch.from_numpy(keys).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        out_k = torch.full((n,), -7, dtype=torch.int32, device=dev)
        out_p = torch.full((n,), -7, dtype=torch.int32, device=dev)
        st = _call(L, keys_d, n, max_key, out_k, out_p, stream)
        assert st == 0, (call, st)
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(out_p.cpu().numpy(), perm, err_msg=f"call {call}: permutation")
        np.testing.assert_array_equal(out_k.cpu().numpy(), keys[perm], err_msg=f"call {call}: keys")
