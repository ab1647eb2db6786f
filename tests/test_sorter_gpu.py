"""GpuRadixSorter contract (src/gpu/radix-sort.ts:91-216) on the device sort:
results must equal a stable CPU sort bit for bit."""
import numpy as np
import pytest

import droplet_b200 as dl

pytestmark = pytest.mark.gpu


def _stable(keys, vals):
    o = np.argsort(keys, kind="stable")
    return keys[o], (o.astype(np.uint32) if vals is None else vals[o])


@pytest.fixture(scope="module")
def sorter(device):
    s = dl.GpuRadixSorter(device)
    yield s
    s.destroy()


@pytest.mark.parametrize("n,bits,with_vals", [(1, 32, True), (3839, 32, True), (3840, 8, True),
                                               (100_003, 14, True), (1_000_000, 32, False),
                                               (2_500_000, 5, True), (777_777, 24, False)])
def test_sort_matches_stable_cpu_sort(sorter, n, bits, with_vals):
    import torch
    rng = np.random.default_rng(n + bits)
    hk = rng.integers(0, 2 ** bits, n, dtype=np.uint64).astype(np.uint32)
    hv = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) if with_vals else None
    k = torch.from_numpy(hk.view(np.int32).copy()).cuda()
    v = torch.from_numpy(hv.view(np.int32).copy()).cuda() if with_vals else None
    ok, ov = sorter.sort(k, v, n, bits)
    torch.cuda.synchronize()
    rk, rv = _stable(hk, hv)
    gk = ok[:n].cpu().view(torch.int32).numpy().view(np.uint32)
    gv = ov[:n].cpu().view(torch.int32).numpy().view(np.uint32)
    assert np.array_equal(gk, rk)
    assert np.array_equal(gv, rv)
    passes = (bits + 7) // 8
    # even pass counts end in the caller's arrays, odd ones in the pong buffers
    assert (ok.data_ptr() == k.data_ptr()) == (passes % 2 == 0)


@pytest.mark.parametrize("digit_bits", [6, 7])
def test_narrow_digits_give_the_same_order(sorter, digit_bits):
    import torch
    rng = np.random.default_rng(7)
    n = 300_000
    hk = rng.integers(0, 2 ** 20, n, dtype=np.uint64).astype(np.uint32)
    hv = np.arange(n, dtype=np.uint32)[::-1].copy()
    sorter.set_digit_bits(digit_bits)
    try:
        ok, ov = sorter.sort(torch.from_numpy(hk.view(np.int32).copy()).cuda(),
                             torch.from_numpy(hv.view(np.int32).copy()).cuda(), n, 20)
    finally:
        sorter.set_digit_bits(8)
    rk, rv = _stable(hk, hv)
    assert np.array_equal(ok[:n].cpu().view(torch.int32).numpy().view(np.uint32), rk)
    assert np.array_equal(ov[:n].cpu().view(torch.int32).numpy().view(np.uint32), rv)


def test_empty_and_bad_arguments(sorter):
    import torch
    k = torch.zeros(4, dtype=torch.int32, device="cuda")
    ok, ov = sorter.sort(k, k.clone(), 0, 32)
    assert ok.data_ptr() == k.data_ptr()
    with pytest.raises(dl.DropletError):
        sorter.sort(k, None, 4, 33)
    with pytest.raises(dl.DropletError):
        sorter.sort(k, None, 8, 32)          # n larger than the tensors
    with pytest.raises(dl.DropletError):
        sorter.set_digit_bits(9)
