"""The bounded device-side waits: every decoupled look-back of the radix sort
gives up after a poll limit, records a timeout, writes nothing outside its
buffers, and the entry point that launched it returns PRT_ERR_TIMEOUT.

The waits are made to run out by the library's test hook
(prt_debug_wait_limit with never_published=1: every look-back sees no
predecessor published and polls a few hundred times), so nothing hangs and
nothing faults; afterwards the same context must still give bit-exact
results."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.fixture
def blind_waits():
    from parlllelrtree_b200 import _lib

    L = _lib.lib()
    assert L.prt_debug_wait_limit(256, 1) == 0
    try:
        yield L
    finally:
        L.prt_debug_wait_limit(0, 0)


def _guarded(n, dtype, fill):
    """A buffer between two guard regions, to see that nothing writes past it."""
    g = torch.full((n + 2 * 4096,), fill, dtype=dtype, device="cuda")
    return g, g[4096:4096 + n]


def test_build_wait_times_out(cuda, blind_waits):
    from parlllelrtree_b200 import _lib

    L = blind_waits
    b = torch.from_numpy(dg.mixture_boxes(2_000_000, seed=11)).cuda()
    for fn, args in (("prt_build_bottomup", (16, 1)), ("prt_build_topdown", (16,))):
        h = C.c_void_p()
        rc = getattr(L, fn)(_ptr(b), _lib.COORD["f32"], None, len(b), *args, _stream(), C.byref(h))
        assert rc == _lib.PRT_ERR_TIMEOUT, (fn, rc, L.prt_last_error())
        assert b"timed out" in L.prt_last_error()
        assert not h.value  # no tree is handed out
    torch.cuda.synchronize()  # no fault left behind


def test_sorted_join_and_batched_overlay_time_out(cuda, blind_waits):
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib

    L = blind_waits
    # the tree is built with the default limit, then the waits are blinded
    L.prt_debug_wait_limit(0, 0)
    boxes = torch.from_numpy(dg.mixture_boxes(200_000, seed=12, mean_side=2e-3)).cuda()
    tree = prt.build_bottomup(boxes, fanout=16)
    q = torch.from_numpy(dg.window_queries(50_000, seed=13, side_hi=5e-3)).cuda()
    n = len(tree.join(q))
    assert n > 3072 * 4  # several sort tiles
    L.prt_debug_wait_limit(256, 1)
    guard, out = _guarded(2 * (n + 16), torch.int32, -7)
    cnt = C.c_int64(0)
    rc = L.prt_join_sorted(tree._h, _ptr(q), tree.coord, len(q), _ptr(out), n + 16, C.byref(cnt), _stream())
    assert rc == _lib.PRT_ERR_TIMEOUT, L.prt_last_error()
    torch.cuda.synchronize()
    assert (guard[:4096] == -7).all() and (guard[-4096:] == -7).all()

    # the batched overlay sorts its pairs by size: its timeout is reported too
    A = dg.star_layer(3000, seed=14, r_lo=0.01, r_hi=0.05)
    B = dg.star_layer(3000, seed=15, r_lo=0.01, r_hi=0.05)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    L.prt_debug_wait_limit(0, 0)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr())
    l2p = t.leaf_order()
    assert len(pairs) > 3072 * 2
    L.prt_debug_wait_limit(256, 1)
    with pytest.raises(prt.PrtError) as ei:
        prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="batched")
    assert ei.value.code == _lib.PRT_ERR_TIMEOUT
    torch.cuda.synchronize()


def test_context_usable_after_timeouts(cuda):
    """After the timed-out calls the default limit is back and results are exact."""
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib

    _lib.lib().prt_debug_wait_limit(256, 1)
    h = C.c_void_p()
    b = dg.mixture_boxes(500_000, seed=16)
    bd = torch.from_numpy(b).cuda()
    rc = _lib.lib().prt_build_bottomup(_ptr(bd), _lib.COORD["f32"], None, len(b), 16, 1, _stream(), C.byref(h))
    assert rc == _lib.PRT_ERR_TIMEOUT
    _lib.lib().prt_debug_wait_limit(0, 0)
    keys, _ = oracle.keys_morton32(b)
    perm = oracle.stable_argsort(keys)
    t = prt.build_bottomup(bd, fanout=16)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
    t2 = prt.build_topdown(bd, fanout=16)
    assert np.array_equal(t2.leaf_order().cpu().numpy(), oracle.td_order(b, 16))
