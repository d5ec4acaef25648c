"""The sort entry point that allocates nothing (apo2_radix_sort_pairs_static).

It serves callers that cannot allocate device memory where they sort, e.g. under a memory
owner that forbids other allocations, or where an allocation's implicit synchronisation would
stall other work: its scratch is a fixed array inside the library. This file is collected last
so that a stop at its first failure has already run every other test; it also passes alone
in a fresh process. Integer sort: results must be identical to apo2_radix_sort_pairs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _keys(n, seed):
    rng = np.random.default_rng(seed)
    keys = (rng.integers(0, 1 << 20, size=n, dtype=np.int64) << np.int64(30)) | rng.integers(0, 8, size=n)
    return keys, np.arange(n, dtype=np.int32)


def _sort_with_scratch(lib, torch, keys, vals):
    k = torch.from_numpy(keys).cuda()
    v = torch.from_numpy(vals).cuda()
    scratch = torch.empty(int(lib.apo2_radix_sort_scratch_bytes(k.numel())), dtype=torch.uint8, device="cuda")
    assert lib.apo2_radix_sort_pairs(k.data_ptr(), v.data_ptr(), k.numel(), scratch.data_ptr(), None) == 0
    torch.cuda.synchronize()
    return k.cpu().numpy(), v.cpu().numpy()


def test_static_sort_matches_allocating_sort_twice():
    import torch

    import apo_b200
    lib = apo_b200.load_library()
    for call, (n, seed) in enumerate([(MAX_PAIRS, 1), (300_001, 2)]):
        keys, vals = _keys(n, seed)
        ref_k, ref_v = _sort_with_scratch(lib, torch, keys, vals)
        k = torch.from_numpy(keys).cuda()
        v = torch.from_numpy(vals).cuda()
        torch.cuda.synchronize()
        assert lib.apo2_radix_sort_pairs_static(k.data_ptr(), v.data_ptr(), n, None) == apo_b200.APO2_OK, call
        torch.cuda.synchronize()
        assert np.array_equal(k.cpu().numpy(), ref_k), call
        assert np.array_equal(v.cpu().numpy(), ref_v), call


def test_static_sort_rejects_sizes_above_its_scratch():
    import torch

    import apo_b200
    lib = apo_b200.load_library()
    k = torch.zeros(8, dtype=torch.int64, device="cuda")
    v = torch.zeros(8, dtype=torch.int32, device="cuda")
    # the size check comes before any device work, so the short buffers are never touched
    assert lib.apo2_radix_sort_pairs_static(k.data_ptr(), v.data_ptr(), MAX_PAIRS + 1, None) == apo_b200.APO2_ERR_TOO_LARGE
