"""The launch-window plan of the team strips, restated and checked exhaustively on the CPU.

run_batch (robotfd_b200/csrc/rfd_engine.cu) runs a pair's VE-FD and decision strips in launch
windows of W strips when one boundary row per strip does not fit: strip s writes ring row
s % ring, team_window_fill_kernel resets the rows a window's strips write before its launch,
and the next window starts after the previous one ends.  A split pair (meet in the middle)
has two halves, each with a ring of its own: the forward half's k strips (ring min(W + 1, k),
every strip hands a row on, the last one to the meet) and the mirror's S - k strips (ring
min(W + 1, S - k), likewise); window g runs strips gW .. gW + W - 1 of both halves.  An
unsplit pair's ring is min(W + 1, S - 1) (ring_of) and its last strip hands nothing on.

Checked for every small S, W and split: within a window the strips write distinct rows; no
window resets the row its first strip reads (written by the strip before it, in an earlier
window); every strip reads the row its predecessor wrote, not overwritten since; and the
rows the meet reads (each half's last strip's) are not reset or overwritten by any later
window.
"""


def ring_of(strips, rows):
    return max(1, min(strips - 1, rows))


def plan(S, W, k):
    """Halves as (name, strips, writers, ring): writers = strips that hand a row on."""
    if k:
        return [("fwd", k, k, min(W + 1, k)), ("mir", S - k, S - k, min(W + 1, S - k))]
    return [("all", S, S - 1, ring_of(S, W + 1))]


def check(S, W, k):
    halves = plan(S, W, k)
    nwin = -(-max(h[1] for h in halves) // W)
    for name, strips, writers, ring in halves:
        row = {}  # ring row -> strip whose value it holds (None after a reset)
        for g in range(nwin):
            s0, s1 = g * W, min(g * W + W, strips)
            resets = {s % ring for s in range(s0, min(s0 + W, writers))}
            if s0 > 0 and s0 < strips:
                assert (s0 - 1) % ring not in resets, (S, W, k, name, g)
            for r in resets:
                row[r] = None
            written = [s % ring for s in range(s0, min(s1, writers))]
            assert len(written) == len(set(written)), (S, W, k, name, g)
            for s in range(s0, s1):
                if s > 0:
                    assert row.get((s - 1) % ring) == s - 1, (S, W, k, name, s)
                if s < writers:
                    row[s % ring] = s
        if k:  # the meet reads each half's last strip's row after the last window
            assert row.get((writers - 1) % ring) == writers - 1, (S, W, k, name)


def test_window_plan_exhaustive():
    for S in range(2, 70):
        for W in range(1, S + 2):
            check(S, W, 0)
            for k in {S // 2} | ({1, S - 1} if S > 2 else set()):
                if 1 <= k <= S - 1:
                    check(S, W, k)
