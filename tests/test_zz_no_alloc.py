"""The allocation-free cell-key sort (dfsph_sort_cell_keys_noalloc), called through the C ABI.

Callers that may not allocate device memory (a host framework that owns every allocation, a plugin
handed fixed device buffers) sort their cell keys with this entry point; its scratch is a fixed
device array inside the library. Its result must equal the sorted order the allocating solver path
produces for the same particles (dfsph_neighbors_search, read back as the sorted id order), on two
calls in a row (the second call reuses the scratch the first one left behind). This file is named
to be collected last."""
import ctypes as C

import numpy as np
import pytest

from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.scene import synthetic_scene

pytestmark = pytest.mark.gpu


def _spread10(v):
    v = v.astype(np.uint64) & 0x3FF
    v = (v | (v << 16)) & 0x030000FF
    v = (v | (v << 8)) & 0x0300F00F
    v = (v | (v << 4)) & 0x030C30C3
    v = (v | (v << 2)) & 0x09249249
    return v


def _cell_keys(d: DFSPHCUDA, x: np.ndarray) -> np.ndarray:
    """Morton cell keys of positions, computed on the host with the solver's grid and the same FP32
    operations as the device (floor(x / H + offset))."""
    H = np.float32(4.0 * d.scene.config.particleRadius)
    off = np.array([d.get_param(f"grid_offset_{a}") for a in "xyz"], dtype=np.float32)
    c = np.floor(x.astype(np.float32) / H + off).astype(np.int64)
    return (_spread10(c[:, 0]) | (_spread10(c[:, 1]) << 1) | (_spread10(c[:, 2]) << 2)).astype(np.uint32)


def test_noalloc_sort_matches_solver_sorted_order():
    import torch

    scene = synthetic_scene(2)  # 250,047 particles: below the 262,144-key limit
    d = DFSPHCUDA(scene)
    d.neighbors_search()
    ref_perm = d.field("id", order=_capi.ORDER_SORTED)  # stable sort of upload order by cell key
    keys = _cell_keys(d, scene.fluid)
    n = keys.size
    assert n <= _capi.NOALLOC_MAX_KEYS

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    keys_in = torch.from_numpy(keys.view(np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        keys_out = torch.full((n,), -1, dtype=torch.int32, device=dev)
        perm_out = torch.full((n,), -1, dtype=torch.int32, device=dev)
        code = lib.dfsph_sort_cell_keys_noalloc(C.c_void_p(keys_in.data_ptr()), C.c_void_p(keys_out.data_ptr()),
                                                C.c_void_p(perm_out.data_ptr()), n, 30,
                                                C.c_void_p(stream.cuda_stream))
        assert code == _capi.DFSPH_OK, lib.dfsph_last_error(None)
        perm = perm_out.cpu().numpy().view(np.uint32)
        sorted_keys = keys_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(perm, ref_perm), f"call {call}: permutation differs from the solver's"
        assert np.array_equal(sorted_keys, keys[ref_perm]), f"call {call}: keys differ"
    d.close()


def _noalloc_sort(keys: np.ndarray, key_bits: int):
    import torch

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    n = keys.size
    keys_in = torch.from_numpy(keys.view(np.int32)).to(dev)
    keys_out = torch.full((n,), -1, dtype=torch.int32, device=dev)
    perm_out = torch.full((n,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    code = lib.dfsph_sort_cell_keys_noalloc(C.c_void_p(keys_in.data_ptr()), C.c_void_p(keys_out.data_ptr()),
                                            C.c_void_p(perm_out.data_ptr()), n, key_bits,
                                            C.c_void_p(stream.cuda_stream))
    assert code == _capi.DFSPH_OK, lib.dfsph_last_error(None)
    return keys_out.cpu().numpy().view(np.uint32), perm_out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n,key_bits,high", [(1, 8, False), (2047, 8, False), (2049, 24, False),
                                             (100_003, 24, True), (262_144, 30, True), (77_777, 32, False),
                                             (5000, 13, True)])
def test_noalloc_sort_equals_stable_argsort(n, key_bits, high):
    """1, 2, 3 and 4 digit passes (odd counts write the caller's buffers on the first pass), one key,
    partial tiles and a full last tile, and keys with bits set above key_bits (carried, not
    ordered): equal to numpy's stable argsort of the low key_bits bits, twice in a row."""
    rng = np.random.default_rng(n + key_bits)
    low = rng.integers(0, 1 << min(key_bits, 31), size=n, dtype=np.int64)
    if key_bits == 32:
        low = rng.integers(0, 1 << 32, size=n, dtype=np.int64)
    low[: n // 3] = low[n // 3: 2 * (n // 3)]  # many equal keys: stability matters
    keys = low.astype(np.uint64)
    if high and key_bits < 32:
        keys |= rng.integers(0, 1 << (32 - key_bits), size=n).astype(np.uint64) << key_bits
    keys = keys.astype(np.uint32)
    mask = np.uint32(0xFFFFFFFF if key_bits == 32 else (1 << key_bits) - 1)
    ref = np.argsort(keys & mask, kind="stable").astype(np.uint32)
    for _ in range(2):
        ko, po = _noalloc_sort(keys, key_bits)
        assert np.array_equal(po, ref)
        assert np.array_equal(ko, keys[ref])


def test_noalloc_sort_rejects_overlap_and_capture():
    import torch

    lib = _capi.load()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(3000, dtype=torch.int32, device=dev)
    p = buf.data_ptr()
    # keys_out overlapping keys_in
    code = lib.dfsph_sort_cell_keys_noalloc(C.c_void_p(p), C.c_void_p(p + 4 * 500), C.c_void_p(p + 4 * 2000), 1000,
                                            8, None)
    assert code == _capi.DFSPH_E_INVALID and b"overlap" in lib.dfsph_last_error(None)
    keys = torch.zeros(1000, dtype=torch.int32, device=dev)
    ko = torch.zeros(1000, dtype=torch.int32, device=dev)
    po = torch.zeros(1000, dtype=torch.int32, device=dev)
    s = torch.cuda.Stream(dev)
    g = torch.cuda.CUDAGraph()
    codes = []
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            codes.append(lib.dfsph_sort_cell_keys_noalloc(C.c_void_p(keys.data_ptr()), C.c_void_p(ko.data_ptr()),
                                                          C.c_void_p(po.data_ptr()), 1000, 8,
                                                          C.c_void_p(s.cuda_stream)))
            ko.add_(1)  # the captured graph must not be empty
    assert codes == [_capi.DFSPH_E_STATE]
    assert b"stream capture" in lib.dfsph_last_error(None)
    del g
    torch.cuda.synchronize()


def test_noalloc_sort_rejects_oversize_input():
    lib = _capi.load()
    n = _capi.NOALLOC_MAX_KEYS + 1
    code = lib.dfsph_sort_cell_keys_noalloc(C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), n, 30, None)
    assert code == _capi.DFSPH_E_INVALID
    assert b"exceeds the maximum" in lib.dfsph_last_error(None)
