"""The bounded-wait failure path, made to happen on purpose.

Every inter-warp wait of the kernels (a strip waiting for the row of the strip above it, a
helper warp waiting for its tile request, the continuous search waiting for a queue entry)
is bounded by a clock budget; past it the kernel sets an error word, every warp leaves and
the call reports RFD_ERR_TIMEOUT.  The reference's spins are unbounded
(src/intersection_algorithm_in_parallel.cu:304-306, :332-334).  Here the budget is cut to a
few hundred SM cycles, far less than a strip needs before its first row chunk is ready, so
the waits run out: nothing faults, the context stays usable, and the next call with the
normal budget is bit-identical to the oracle.
"""
import pytest

import oracle

TINY = 300  # SM clock cycles


def _pair(built):
    return built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 61, 0)


@pytest.mark.gpu
def test_distance_times_out_then_recovers(built):
    P, Q = _pair(built)
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
    c = built.Context(0)
    try:
        c.set_wait_budget(TINY)
        for kw in (dict(precise=True), dict(precise=True, dense=True)):
            with pytest.raises(built.RfdError) as e:
                c.distance(P, Q, **kw)
            assert e.value.code == built.RFD_ERR_TIMEOUT
        c.set_wait_budget(0)  # the default budget again, same context and workspace
        got = c.distance(P, Q, precise=True)
        assert got["distance"] == want["distance"]
        assert got["dfd"] == want["dfd"] and got["vefd"] == want["vefd"]
        assert got["probes"] == want["probes"]
    finally:
        c.close()


@pytest.mark.gpu
def test_decision_and_batch_time_out_then_recover(built):
    P, Q = _pair(built)
    r = 0.5 * (oracle.dfd_sq(P, Q) ** 0.5 + oracle.endpoint(P, Q))
    want_reach, want_ub = oracle.decide(P, Q, r, threads=oracle.max_threads())
    c = built.Context(0)
    try:
        c.set_wait_budget(TINY)
        with pytest.raises(built.RfdError) as e:
            c.decide(P, Q, r)
        assert e.value.code == built.RFD_ERR_TIMEOUT
        pairs = [built.gen_pair(0, 2, 700 + 37 * k, 650, 1.0, 0.05, 62, k) for k in range(6)]
        with pytest.raises(built.RfdError) as e:
            c.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=True)
        assert e.value.code == built.RFD_ERR_TIMEOUT
        c.set_wait_budget(0)
        assert c.decide(P, Q, r) == (want_reach, want_ub)
        res = c.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=True)
        for (p, q), g in zip(pairs, res):
            assert g["distance"] == oracle.distance(p, q, stop_mode=1, quirks=False)["distance"]
    finally:
        c.close()


@pytest.mark.gpu
def test_environment_sets_the_budget_of_new_contexts(built, monkeypatch):
    P, Q = _pair(built)
    monkeypatch.setenv("RFD_SPIN_CYCLES", str(TINY))
    c = built.Context(0)
    try:
        with pytest.raises(built.RfdError) as e:
            c.bounds(P, Q)
        assert e.value.code == built.RFD_ERR_TIMEOUT
    finally:
        c.close()
    monkeypatch.delenv("RFD_SPIN_CYCLES")
    c = built.Context(0)
    try:
        dfd, vefd = c.bounds(P, Q, quirks=False)
        assert dfd == oracle.dfd_sq(P, Q) ** 0.5
    finally:
        c.close()
