"""GPU tests of bb_radix_sort_pairs (the step's onesweep sort on caller device arrays) against
a stable numpy sort: bit-exact keys and values, ties kept in input order."""
import ctypes

import numpy as np
import pytest

import beatbox as bb

pytestmark = pytest.mark.gpu


def dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def sort_on_gpu(fn, keys, vals, bits):
    import torch

    kin = torch.from_numpy(keys.view(np.int32)).cuda()
    vin = torch.from_numpy(vals.view(np.int32)).cuda()
    kout = torch.full_like(kin, -1)
    vout = torch.full_like(vin, -1)
    torch.cuda.synchronize()
    code = fn(dptr(kin), dptr(vin), dptr(kout), dptr(vout), len(keys), bits, None)
    assert code == bb.OK, bb.load_library().bb_last_error_string()
    torch.cuda.synchronize()
    flags = ctypes.c_uint32(0xFFFFFFFF)
    static = 1 if fn is bb.load_library().bb_radix_sort_pairs_static else 0
    assert bb.load_library().bb_radix_sort_error_flags(static, None, ctypes.byref(flags)) == bb.OK
    assert flags.value == 0  # the look-back waits all ended
    return kout.cpu().numpy().view(np.uint32), vout.cpu().numpy().view(np.uint32), kin, vin


def expected(keys, vals, bits):
    mask = np.uint32((1 << bits) - 1) if bits < 32 else np.uint32(0xFFFFFFFF)
    order = np.argsort(keys & mask, kind="stable")
    return keys[order], vals[order]


@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 4095, 4096, 4097, 100_003, 1_000_003])
@pytest.mark.parametrize("bits", [8, 30, 32])
def test_radix_sort_pairs_matches_stable_sort(n, bits):
    lib = bb.load_library()
    rng = np.random.default_rng(n + bits)
    hi = 1 << min(bits, 31)
    keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    keys[: n // 3] = keys[0]  # many duplicates exercise stability
    vals = np.arange(n, dtype=np.uint32)
    gk, gv, kin, vin = sort_on_gpu(lib.bb_radix_sort_pairs, keys, vals, bits)
    ek, ev = expected(keys, vals, bits)
    assert np.array_equal(gv, ev)
    assert np.array_equal(gk, ek)
    # inputs untouched
    assert np.array_equal(kin.cpu().numpy().view(np.uint32), keys)


def test_radix_sort_pairs_on_unaligned_views():
    """Inputs that start 4 bytes into a buffer (no 16-byte alignment) sort the same."""
    import torch

    lib = bb.load_library()
    n = 70_001
    rng = np.random.default_rng(7)
    keys = rng.integers(0, 1 << 31, n + 1, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n + 1, dtype=np.uint32)
    kin = torch.from_numpy(keys.view(np.int32)).cuda()[1:]
    vin = torch.from_numpy(vals.view(np.int32)).cuda()[1:]
    kout, vout = torch.full_like(kin, -1), torch.full_like(vin, -1)
    torch.cuda.synchronize()
    assert lib.bb_radix_sort_pairs(dptr(kin), dptr(vin), dptr(kout), dptr(vout), n, 32, None) == bb.OK
    torch.cuda.synchronize()
    ek, ev = expected(keys[1:], vals[1:], 32)
    assert np.array_equal(kout.cpu().numpy().view(np.uint32), ek)
    assert np.array_equal(vout.cpu().numpy().view(np.uint32), ev)


def test_radix_sort_pairs_rejects_bad_arguments():
    lib = bb.load_library()
    assert lib.bb_radix_sort_pairs(None, None, None, None, 0, 30, None) == bb.OK
    assert lib.bb_radix_sort_pairs(None, None, None, None, 16, 30, None) == bb.E_INVALID
    assert lib.bb_radix_sort_pairs(None, None, None, None, 16, 0, None) == bb.E_INVALID
