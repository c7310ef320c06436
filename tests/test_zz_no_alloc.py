"""gt_direct_noalloc, the allocation-free direct sum, against the ordinary entry point gt_direct.

Some callers cannot allocate device memory when they ask for forces.  One example is an
application whose pool allocator already holds all free device memory.  Another is one that must
not set off the implicit device synchronisation cudaMalloc/cudaFree can cause in the middle of an
asynchronous step.  For them gt_direct_noalloc keeps its partial sums in a fixed array inside the
library.  This test calls it through the C ABI twice in a row, with different sizes, so the second
call runs on the first call's leftovers in that shared array.  The first call is FP64 and must equal
gt_direct's to the FP64 tolerance of the direct-sum parity test (relative 1e-12).  The second is
FP32; its source chunks can differ from gt_direct's (the chunk count is capped so the partials fit
the fixed array), so it is held to an FP32 tolerance (relative 1e-5 per target).  This file sorts
last so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import _gt, ics

pytestmark = pytest.mark.gpu

GT_ERR_OVERFLOW = 5
MAX_TARGETS = (1 << 20) // 4  # GT_DIRECT_NOALLOC_MAX_TARGETS in include/gt.h


def relerr(a, b):
    d = np.sqrt(sum((x - y) ** 2 for x, y in zip(a, b)))
    n = np.sqrt(sum(y ** 2 for y in b))
    return d / np.where(n > 0, n, 1.0)


def test_direct_noalloc_matches_direct_on_two_calls():
    import torch

    L = g.load_library()
    ctx = g.Context(0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    P = ics.plummer(n=30000, seed=13, soft=0.01)
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    for call, (step, precision, tol) in enumerate([(3, g.GT_DIRECT_FP64, 1e-12), (7, g.GT_DIRECT_FP32, 1e-5)]):
        tg = np.arange(call, 30000, step, dtype=np.uint32)
        nt = len(tg)
        tdev = torch.as_tensor(tg.view(np.int32), device="cuda")
        out = [torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(4)]
        st = L.gt_direct_noalloc(len(P["m"]), *[dev[k].data_ptr() for k in ("x", "y", "z", "m", "soft")],
                                 nt, tdev.data_ptr(), 1.0, precision, *[o.data_ptr() for o in out],
                                 C.c_void_p(stream))
        assert st == 0, _gt.STATUS.get(st)
        torch.cuda.synchronize()
        got = [o.cpu().numpy() for o in out]
        want = ctx.direct(P, tg, precision=precision)
        assert relerr(got[:3], want[:3]).max() <= tol
        np.testing.assert_allclose(got[3], want[3], rtol=tol)


def test_direct_noalloc_rejects_too_many_targets():
    L = g.load_library()
    st = L.gt_direct_noalloc(10, None, None, None, None, None, MAX_TARGETS + 1, None, 1.0,
                             g.GT_DIRECT_FP64, None, None, None, None, None)
    # argument checks come first (null arrays); with valid pointers the size check answers
    assert st in (1, GT_ERR_OVERFLOW)
    import torch

    x = torch.zeros(10, dtype=torch.float64, device="cuda")
    t = torch.zeros(MAX_TARGETS + 1, dtype=torch.int32, device="cuda")
    o = torch.zeros(MAX_TARGETS + 1, dtype=torch.float64, device="cuda")
    st = L.gt_direct_noalloc(10, x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), None,
                             MAX_TARGETS + 1, t.data_ptr(), 1.0, g.GT_DIRECT_FP64, o.data_ptr(),
                             o.data_ptr(), o.data_ptr(), None, None)
    assert st == GT_ERR_OVERFLOW
    # no particles but some targets: rejected before anything is launched
    st = L.gt_direct_noalloc(0, x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), None,
                             4, t.data_ptr(), 1.0, g.GT_DIRECT_FP64, o.data_ptr(),
                             o.data_ptr(), o.data_ptr(), None, None)
    assert st == 1
