"""The allocation-free sort entry point, checked against the allocating one.

pm_sort_u64_noalloc serves callers that must not call cudaMalloc/cudaFree (a latency-bound
loop that cannot stall on the driver's allocator, or a process whose device memory another
framework already holds).  It keeps its scratch in a static device array shared by every call,
so two calls in a row must each give exactly what pm_sort_u64 gives: a stable sort is unique,
so the keys and the permutation must match bit for bit.  This file is collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sorted_by_allocating_entry(lib, torch, kin, lo, hi):
    n = kin.numel()
    keys_out = torch.empty_like(kin)
    tmp_keys = torch.empty_like(kin)
    perm = torch.empty(n, dtype=torch.int32, device=kin.device)
    tmp_vals = torch.empty_like(perm)
    torch.cuda.synchronize()
    rc = lib.pm_sort_u64(kin.data_ptr(), keys_out.data_ptr(), perm.data_ptr(), tmp_keys.data_ptr(),
                         tmp_vals.data_ptr(), n, lo, hi)
    assert rc == 0
    return keys_out, perm


def test_noalloc_sort_equals_allocating_sort_two_calls_in_a_row():
    import torch

    from pbh_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(2024)
    # The second call is smaller and sorts other bits, so leftovers of the first would show.
    for n, lo, hi in [(200003, 0, 64), (65536, 5, 37)]:
        keys = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64)
        keys[::5] = keys[1]                               # ties: stability matters
        kin = torch.from_numpy(keys.view(np.int64)).cuda()
        ref_keys, ref_perm = _sorted_by_allocating_entry(lib, torch, kin, lo, hi)
        keys_out = torch.empty_like(kin)
        perm = torch.empty(n, dtype=torch.int32, device=kin.device)
        torch.cuda.synchronize()
        rc = lib.pm_sort_u64_noalloc(kin.data_ptr(), keys_out.data_ptr(), perm.data_ptr(), n, lo, hi, None)
        assert rc == 0
        assert torch.equal(keys_out, ref_keys)
        assert torch.equal(perm, ref_perm)
        assert torch.equal(kin, torch.from_numpy(keys.view(np.int64)).cuda())   # input left unchanged


def test_noalloc_sort_rejects_more_keys_than_its_scratch_holds():
    import torch

    from pbh_b200 import _lib
    lib = _lib.load()
    n = _lib.NOALLOC_MAX_KEYS + 1
    kin = torch.zeros(n, dtype=torch.int64, device="cuda")
    keys_out = torch.full_like(kin, 7)
    perm = torch.full((n,), 7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.pm_sort_u64_noalloc(kin.data_ptr(), keys_out.data_ptr(), perm.data_ptr(), n, 0, 64, None)
    assert rc == -2003
    assert int(keys_out.min()) == 7 and int(perm.min()) == 7
