"""The no-allocation sort entry point against the workspace sort.

Collected last on purpose: the first call on a device does the entry point's
set-up, and it must also work after every other test has used the library.
"""
import ctypes as C

import numpy as np
import pytest

from dyphur_b200 import capi


def test_noalloc_rejects_oversize_without_gpu_work():
    n = capi.SORT_NOALLOC_MAX_KEYS + 1
    assert capi.lib().dyph_sort_by_key_u64_u32_noalloc(None, None, n, None) == capi.ERR_TOO_LARGE
    assert b"no-allocation" in capi.lib().dyph_status_string(capi.ERR_TOO_LARGE)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [3000, 100003, capi.SORT_NOALLOC_MAX_KEYS])
def test_noalloc_sort_matches_workspace_sort_twice(n):
    import torch
    from dyphur_b200 import device
    device.require_device()
    lib = capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(n)
    for call in range(2):  # two calls in a row reuse the same scratch
        keys = rng.integers(0, 2**63, n, dtype=np.int64)
        keys[:: 5 + call] = keys[call]  # duplicates: the sort must stay stable
        vals = rng.permutation(n).astype(np.int32)
        k1, v1 = torch.from_numpy(keys).cuda(), torch.from_numpy(vals).cuda()
        k2, v2 = k1.clone(), v1.clone()
        capi.check(lib.dyph_sort_by_key_u64_u32_noalloc(k1.data_ptr(), v1.data_ptr(), n, stream))
        ws_bytes = lib.dyph_sort_workspace_bytes(n)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
        capi.check(lib.dyph_sort_by_key_u64_u32(k2.data_ptr(), v2.data_ptr(), n, ws.data_ptr(), ws_bytes, stream))
        torch.cuda.synchronize()
        assert torch.equal(k1, k2) and torch.equal(v1, v2)
        order = np.argsort(keys.view(np.uint64), kind="stable")
        assert np.array_equal(k1.cpu().numpy(), keys[order])
        assert np.array_equal(v1.cpu().numpy(), vals[order])


@pytest.mark.gpu
def test_noalloc_oversize_leaves_input_untouched():
    import torch
    from dyphur_b200 import device
    device.require_device()
    n = capi.SORT_NOALLOC_MAX_KEYS + 1
    k = torch.arange(n, 0, -1, dtype=torch.int64, device="cuda")
    v = torch.arange(n, dtype=torch.int32, device="cuda")
    k0 = k.clone()
    st = capi.lib().dyph_sort_by_key_u64_u32_noalloc(k.data_ptr(), v.data_ptr(), n,
                                                     torch.cuda.current_stream().cuda_stream)
    assert st == capi.ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert torch.equal(k, k0)
