"""GPU test of bb_radix_sort_pairs_static, the sort entry point whose scratch is a fixed
device array in the library: same output as bb_radix_sort_pairs on two calls in a row, no
change in free device memory across those calls, and sizes above the limit rejected.

The file name puts it last in collection order, so it also runs after every other GPU test
in the same process (the static scratch must not depend on a fresh context)."""
import ctypes

import numpy as np
import pytest

import beatbox as bb

pytestmark = pytest.mark.gpu


def dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def case(n, bits, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << min(bits, 31), n, dtype=np.uint64).astype(np.uint32)
    if bits == 32:
        keys |= (rng.integers(0, 2, n, dtype=np.uint64).astype(np.uint32) << np.uint32(31))
    keys[: n // 4] = keys[n // 2]  # duplicates: ties must keep input order
    vals = rng.permutation(n).astype(np.uint32)
    return keys, vals


def test_static_sort_matches_allocating_sort_twice_in_a_row():
    import torch

    lib = bb.load_library()
    assert bb.SORT_STATIC_MAX_KEYS == 262144
    cases = [(bb.SORT_STATIC_MAX_KEYS, 32, 1), (100_003, 30, 2)]
    bufs = []
    for n, bits, seed in cases:
        k, v = case(n, bits, seed)
        kin = torch.from_numpy(k.view(np.int32)).cuda()
        vin = torch.from_numpy(v.view(np.int32)).cuda()
        outs = [torch.full_like(kin, -1) for _ in range(4)]
        bufs.append((n, bits, k, v, kin, vin, outs))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # first call per device looks the scratch address up; later calls only launch work
    n, bits, _, _, kin, vin, outs = bufs[1]
    assert lib.bb_radix_sort_pairs_static(dptr(kin), dptr(vin), dptr(outs[2]), dptr(outs[3]), n, bits,
                                          stream) == bb.OK
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for n, bits, _, _, kin, vin, outs in bufs:  # two static calls back to back, no sync between
        assert lib.bb_radix_sort_pairs_static(dptr(kin), dptr(vin), dptr(outs[0]), dptr(outs[1]), n, bits,
                                              stream) == bb.OK, lib.bb_last_error_string()
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    flags = ctypes.c_uint32(0xFFFFFFFF)
    assert lib.bb_radix_sort_error_flags(1, stream, ctypes.byref(flags)) == bb.OK
    assert flags.value == 0  # the second static sort's look-back waits all ended
    for n, bits, k, v, kin, vin, outs in bufs:
        assert lib.bb_radix_sort_pairs(dptr(kin), dptr(vin), dptr(outs[2]), dptr(outs[3]), n, bits,
                                       stream) == bb.OK, lib.bb_last_error_string()
    torch.cuda.synchronize()
    for n, bits, k, v, kin, vin, outs in bufs:
        sk, sv, ak, av = (o.cpu().numpy().view(np.uint32) for o in outs)
        assert np.array_equal(sk, ak) and np.array_equal(sv, av)
        mask = np.uint32(0xFFFFFFFF) if bits == 32 else np.uint32((1 << bits) - 1)
        order = np.argsort(k & mask, kind="stable")
        assert np.array_equal(sv, v[order]) and np.array_equal(sk, k[order])


def test_static_sort_rejects_sizes_above_its_limit():
    lib = bb.load_library()
    big = bb.SORT_STATIC_MAX_KEYS + 1
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    fake2 = ctypes.c_void_p(512)
    assert lib.bb_radix_sort_pairs_static(fake, fake2, ctypes.c_void_p(1024), ctypes.c_void_p(2048), big, 32,
                                          None) == bb.E_INVALID
    assert b"BB_SORT_STATIC_MAX_KEYS" in lib.bb_last_error_string()
    assert lib.bb_radix_sort_pairs_static(None, None, None, None, 0, 32, None) == bb.OK
