"""The decision entry point that allocates nothing (rfd_decide_noalloc).

Some callers cannot allocate device memory while they run - a robot control loop where an
allocation may stall or fail, or a process held to a memory budget fixed at start-up.
For them librfd.so keeps all working memory of this one decision in a fixed device array.
This file is collected last so that a failure here never hides the other tests.  It checks
the entry point through the C ABI against rfd_decide (the allocating path) and against the
CPU oracle, bit for bit, on consecutive calls that reuse the array (including a first curve
of 32k + 1 points, one strip more than a multiple of 32 rows); the size check that needs no
GPU work; and that a wait which runs out of its budget shows as NaN, after which the next
call is correct again.
"""
import numpy as np
import pytest

import oracle


@pytest.mark.gpu
def test_noalloc_decision_matches_allocating_path(ctx, built):
    import torch
    stream = torch.cuda.current_stream()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    cases = [built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 41, 3000),
             built.gen_pair(0, 2, 900, 1300, 1.0, 0.05, 42, 900),
             built.gen_pair(0, 3, 32 * 40 + 1, 1100, 1.0, 0.05, 43, 0)]
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
            o_reach, o_ub = oracle.decide(P, Q, radius, threads=oracle.max_threads())
            assert got == o_ub, (radius, got, o_ub)
            assert (got == 1.0) == o_reach


@pytest.mark.gpu
def test_noalloc_timeout_shows_as_nan_then_recovers(ctx, built, monkeypatch):
    import torch
    P, Q = built.gen_pair(1, 3, 2000, 1900, 100.0, 0.1, 44, 0)
    dP = torch.from_numpy(P).cuda()
    dQ = torch.from_numpy(Q).cuda()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    radius = ctx.distance(P, Q, precise=True)["distance"] * (1 + 1e-7)
    torch.cuda.synchronize()
    # a budget of a few hundred cycles: the second strip cannot get its first row chunk in time
    monkeypatch.setenv("RFD_SPIN_CYCLES", "300")
    out.fill_(-7.0)
    built.decide_noalloc(dP.data_ptr(), len(P), dQ.data_ptr(), len(Q), 3, radius,
                         stream.cuda_stream, out.data_ptr())
    stream.synchronize()
    assert np.isnan(out.item())
    monkeypatch.delenv("RFD_SPIN_CYCLES")
    out.fill_(-7.0)
    built.decide_noalloc(dP.data_ptr(), len(P), dQ.data_ptr(), len(Q), 3, radius,
                         stream.cuda_stream, out.data_ptr())
    stream.synchronize()
    assert out.item() == oracle.decide(P, Q, radius, threads=oracle.max_threads())[1] == 1.0


@pytest.mark.gpu
def test_noalloc_rejects_pairs_beyond_the_array(ctx, built):
    import torch
    dP = torch.zeros((40000, 3), dtype=torch.float64, device="cuda")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    with pytest.raises(built.RfdError) as e:
        built.decide_noalloc(dP.data_ptr(), 40000, dP.data_ptr(), 40000, 3, 1.0,
                             torch.cuda.current_stream().cuda_stream, out.data_ptr())
    assert e.value.code == built.RFD_ERR_LIMIT
