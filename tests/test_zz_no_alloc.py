"""prt_join_noalloc: the join for callers that may not allocate device memory
(a host whose own pool owns the device memory budget and rejects any other
allocation, or an embedding that forbids the library's cudaMalloc calls).  It keeps
its scratch in a fixed array inside the library, so these tests call it
through the C ABI and compare its pairs with prt_join's on two calls in a row
(the second call must not see the first call's leftovers), and check that a
frontier beyond the fixed maximum is refused with an error.

This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _sorted_pairs(p):
    a = p.cpu().numpy().astype(np.int64)
    return a[np.lexsort((a[:, 0], a[:, 1]))]


@pytest.mark.parametrize("build", ["bottomup", "topdown"])
def test_join_noalloc_matches_join_on_two_calls(cuda, build):
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib
    from parlllelrtree_b200 import datagen as dg

    L = _lib.lib()
    boxes = torch.from_numpy(dg.mixture_boxes(300000, seed=3, mean_side=2e-3)).cuda()
    fn = prt.build_bottomup if build == "bottomup" else prt.build_topdown
    tree = fn(boxes, fanout=16)
    for call, seed in enumerate((4, 5)):
        q = torch.from_numpy(dg.window_queries(20000, seed=seed, side_hi=5e-3)).cuda()
        ref = _sorted_pairs(tree.join(q))
        cap = len(ref) + 64
        out = torch.full((cap, 2), -1, dtype=torch.int32, device="cuda")
        count = C.c_int64(-1)
        rc = L.prt_join_noalloc(tree._h, _ptr(q), tree.coord, len(q), _ptr(out), cap, C.byref(count), _stream())
        assert rc == 0, L.prt_last_error()
        assert count.value == len(ref), call
        got = _sorted_pairs(out[: count.value])
        # integer pairs: exact equality (the pair order is not defined)
        assert np.array_equal(got, ref), call
        assert (out[count.value:] == -1).all()


def test_join_noalloc_refuses_frontier_beyond_its_maximum(cuda):
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib
    from parlllelrtree_b200 import datagen as dg

    L = _lib.lib()
    boxes = torch.from_numpy(dg.mixture_boxes(200000, seed=6)).cuda()
    tree = prt.build_bottomup(boxes, fanout=16)
    # 400 windows covering everything: the leaf-level frontier holds every
    # leaf node for every query, 400 x 12,500 = 5M items > 4,194,304
    q = torch.tensor([[-1.0, -1.0, 2.0, 2.0]] * 400, dtype=torch.float32, device="cuda")
    out = torch.empty((16, 2), dtype=torch.int32, device="cuda")
    count = C.c_int64(0)
    rc = L.prt_join_noalloc(tree._h, _ptr(q), tree.coord, len(q), _ptr(out), 16, C.byref(count), _stream())
    assert rc == _lib.PRT_ERR_CAPACITY
    assert b"fixed scratch" in L.prt_last_error()
