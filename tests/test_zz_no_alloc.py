"""The decision entry point that allocates nothing (rfd_decide_noalloc).

Some callers cannot allocate device memory while they run - a robot control loop where an
allocation may stall or fail, or a process held to a memory budget fixed at start-up.
For them librfd.so keeps all working memory of this one decision in a fixed device array.
This file is collected last so that a failure here never hides the other tests.  It checks
the entry point through the C ABI against rfd_decide (the allocating path) bit for bit,
on consecutive calls that reuse the array, and the size check that needs no GPU work.
"""
import numpy as np
import pytest


@pytest.mark.gpu
def test_noalloc_decision_matches_allocating_path(ctx, built):
    import torch
    stream = torch.cuda.current_stream()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    cases = [built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 41, 3000),
             built.gen_pair(0, 2, 900, 1300, 1.0, 0.05, 42, 900)]
    for P, Q in cases:
        r = ctx.distance(P, Q, precise=True)
        dP = torch.from_numpy(P).cuda()
        dQ = torch.from_numpy(Q).cuda()
        torch.cuda.synchronize()
        # two calls in a row on the same array: reachable, then unreachable
        for radius in (r["distance"] * (1 + 1e-7), r["distance"] * (1 - 1e-7)):
            out.fill_(-7.0)
            built.decide_noalloc(dP.data_ptr(), len(P), dQ.data_ptr(), len(Q), P.shape[1], radius,
                                 stream.cuda_stream, out.data_ptr())
            stream.synchronize()
            got = out.item()
            want_reach, want_ub = ctx.decide(P, Q, radius)
            assert got == want_ub, (radius, got, want_ub)
            assert (got == 1.0) == want_reach


@pytest.mark.gpu
def test_noalloc_rejects_pairs_beyond_the_array(ctx, built):
    import torch
    dP = torch.zeros((40000, 3), dtype=torch.float64, device="cuda")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    with pytest.raises(built.RfdError) as e:
        built.decide_noalloc(dP.data_ptr(), 40000, dP.data_ptr(), 40000, 3, 1.0,
                             torch.cuda.current_stream().cuda_stream, out.data_ptr())
    assert e.value.code == built.RFD_ERR_LIMIT
