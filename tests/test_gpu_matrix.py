"""Many-to-many distances (rfd_distance_matrix) on the GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def curves(built, d, k0):
    return [built.gen_pair(k % 2, d, 80 + 37 * k, 60 + 11 * k, 100.0 if k % 2 else 1.0, 0.1, 73, k0 + k)[k % 2]
            for k in range(9)]


@pytest.mark.parametrize("d", [2, 3])
def test_matrix_matches_batch(ctx, built, d):
    cs = curves(built, d, 10 * d)
    n = len(cs)
    M, res = ctx.distance_matrix(cs, precise=True, with_results=True)
    assert np.array_equal(M, M.T) and np.all(np.diag(M) == 0.0)
    pairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
    want = ctx.distance_batch([cs[i] for i, _ in pairs], [cs[j] for _, j in pairs], precise=True)
    for k, (i, j) in enumerate(pairs):
        assert M[i, j] == want[k]["distance"] and res[k]["distance"] == want[k]["distance"]
    # a budget of one byte: one batch call per pair, the same results
    M1 = ctx.distance_matrix(cs, precise=True, budget_bytes=1.0)
    assert np.array_equal(M, M1)


def test_matrix_rejects_mixed_dims(ctx, built):
    cs = curves(built, 2, 0)[:3] + curves(built, 3, 0)[:1]
    with pytest.raises(built.RfdError):
        ctx.distance_matrix(cs)
