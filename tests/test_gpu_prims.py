"""GPU tests of the device scan and radix sort on adversarial sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 2, 31, 1023, 1024, 1025, 2047, 2048, 2049, 65536 + 7, 3_000_001]


@pytest.mark.parametrize("n", SIZES)
def test_exclusive_scan(engine, n):
    import torch
    rng = np.random.default_rng(n)
    a = rng.integers(0, 1000, size=n).astype(np.int32)
    d = torch.from_numpy(a).cuda()
    out, tot = engine.exclusive_scan_i32(d)
    ref = np.concatenate([[0], np.cumsum(a, dtype=np.int64)])
    assert tot == int(ref[-1])
    assert np.array_equal(out.cpu().numpy(), ref[:-1])


@pytest.mark.parametrize("lo,hi", [(-1000, 0), (-2_000_000_000, 2_000_000_000)])
def test_exclusive_scan_signed(engine, lo, hi):
    """Negative tile aggregates and prefixes cross the look-back as signed values."""
    import torch
    rng = np.random.default_rng(7)
    a = rng.integers(lo, hi, size=3_000_017).astype(np.int32)
    out, tot = engine.exclusive_scan_i32(torch.from_numpy(a).cuda())
    ref = np.concatenate([[0], np.cumsum(a, dtype=np.int64)])
    assert tot == int(ref[-1])
    assert np.array_equal(out.cpu().numpy(), ref[:-1])


def test_exclusive_scan_large_values(engine):
    import torch
    a = np.full(5_000_000, 2_000_000_000, dtype=np.int32)
    out, tot = engine.exclusive_scan_i32(torch.from_numpy(a).cuda())
    assert tot == 2_000_000_000 * 5_000_000
    assert int(out[-1].item()) == 2_000_000_000 * (5_000_000 - 1)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("bits", [16, 40, 64])
def test_radix_sort_stable(engine, n, bits):
    import torch
    rng = np.random.default_rng(n + bits)
    hi = 1 << min(bits, 62)
    keys = rng.integers(0, min(hi, 50), size=n, dtype=np.int64) if bits == 16 else rng.integers(0, hi, size=n, dtype=np.int64)
    vals = np.arange(n, dtype=np.int32)
    dk, dv = torch.from_numpy(keys.copy()).cuda(), torch.from_numpy(vals.copy()).cuda()
    engine.radix_sort_u64(dk, dv, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(dk.cpu().numpy(), keys[order])
    assert np.array_equal(dv.cpu().numpy(), vals[order])


def test_radix_sort_full_unsigned_range(engine):
    import torch
    rng = np.random.default_rng(1)
    keys = rng.integers(0, 1 << 63, size=100_000, dtype=np.int64).view(np.uint64) * np.uint64(2) + np.uint64(1)
    vals = np.arange(len(keys), dtype=np.int32)
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.copy()).cuda()
    engine.radix_sort_u64(dk, dv, 64)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(dv.cpu().numpy(), vals[order])
