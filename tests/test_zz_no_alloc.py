"""The no-allocation entry point, checked against the regular counting path
and the oracle, and shown to leave the device's free memory unchanged.

stc_count_oriented_csr_noalloc serves callers that cannot let a library call
cudaMalloc (they hand out all device memory from their own pool, or run under
a budget where a foreign allocation would fail); it keeps its scratch in a
fixed device array instead.  This file runs last so that a failure here
leaves every other test already run, and it builds everything it needs itself
so that it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import signed_triangle_counting_b200 as stc
from signed_triangle_counting_b200 import _capi, synth

pytestmark = pytest.mark.gpu


def oriented_csr(el):
    """Forward CSR oriented from lower to higher id (first occurrence of a
    duplicate kept, self-loops dropped), as host arrays."""
    src, dst, sign = el.src.astype(np.uint64), el.dst.astype(np.uint64), el.sign
    keep = src != dst
    src, dst, sign = src[keep], dst[keep], sign[keep]
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    key = (lo << np.uint64(32)) | hi
    uniq, first = np.unique(key, return_index=True)
    tails = (uniq >> np.uint64(32)).astype(np.int64)
    heads = (uniq & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    signs = sign[first].astype(np.int8)
    n = int(max(el.src.max(), el.dst.max())) + 1
    offsets = np.zeros(n + 1, np.uint64)
    np.cumsum(np.bincount(tails, minlength=n), out=offsets[1:])
    return n, offsets, heads, signs


def to_device(offsets, heads, signs):
    import torch
    pad = 4  # the engine reads whole 16-byte chunks
    d_off = torch.from_numpy(offsets.view(np.int64)).cuda()
    d_heads = torch.zeros(len(heads) + pad, dtype=torch.int32, device="cuda")
    d_heads[: len(heads)] = torch.from_numpy(heads.view(np.int32)).cuda()
    d_signs = torch.zeros(len(signs) + pad, dtype=torch.int8, device="cuda")
    d_signs[: len(signs)] = torch.from_numpy(signs).cuda()
    return d_off, d_heads, d_signs


def noalloc_count(n, m, d_off, d_heads, d_signs):
    import torch
    out = _capi.stc_counts()
    st = _capi.lib().stc_count_oriented_csr_noalloc(
        C.c_void_p(d_off.data_ptr()), C.c_void_p(d_heads.data_ptr()), C.c_void_p(d_signs.data_ptr()),
        n, m, C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(out))
    return st, (out.t0, out.t1, out.t2, out.t3)


@pytest.mark.parametrize("family", ["rmat", "delaunay", "skew"])
def test_noalloc_matches_regular_path_twice(family):
    if family == "rmat":
        el = synth.rmat(41, 14, 1 << 14, 16 << 14, p_pos=0.5)
    elif family == "delaunay":
        el = synth.delaunay(42, 30000, 0.2, 0.6)
    else:
        el = synth.skew(43, 1 << 16, 1 << 17, 4, 3000, 30000, 0.8)
    import torch
    with stc.Context(0) as ctx:
        want = ctx.count(el.src, el.dst, el.sign).as_tuple()
    assert sum(want) > 0
    assert want == oracle.count_arrays(el.src, el.dst, el.sign)
    n, offsets, heads, signs = oriented_csr(el)
    d_off, d_heads, d_signs = to_device(offsets, heads, signs)
    # A first call loads the module and looks up the scratch address; after
    # it, calls take no device memory: the free memory the driver reports is
    # the same before and after two more calls.
    st, got = noalloc_count(n, len(heads), d_off, d_heads, d_signs)
    assert st == _capi.STC_OK and got == want
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(2):  # the shared scratch must start clean on every call
        st, got = noalloc_count(n, len(heads), d_off, d_heads, d_signs)
        assert st == _capi.STC_OK
        assert got == want
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_rejects_bad_input():
    el = synth.er(44, 500, 3000, 0.5)
    n, offsets, heads, signs = oriented_csr(el)
    d_off, d_heads, d_signs = to_device(offsets, heads, signs)
    st, _ = noalloc_count((1 << 22) + 1, len(heads), d_off, d_heads, d_signs)
    assert st == _capi.STC_ERR_LIMIT
    bad = heads.copy()
    bad[0] = 0  # a head that is not above its tail
    d_off, d_bad, d_signs = to_device(offsets, bad, signs)
    st, _ = noalloc_count(n, len(heads), d_off, d_bad, d_signs)
    assert st == _capi.STC_ERR_INVALID_ARGUMENT
    # and a good call right after still counts correctly
    d_off, d_heads, d_signs = to_device(offsets, heads, signs)
    with stc.Context(0) as ctx:
        want = ctx.count(el.src, el.dst, el.sign).as_tuple()
    st, got = noalloc_count(n, len(heads), d_off, d_heads, d_signs)
    assert st == _capi.STC_OK and got == want
