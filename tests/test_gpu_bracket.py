"""Learned bracket on the GPU: features, the tensor-core MLP against its CPU oracle, and
solves that use a bracket (which only changes the probe sequence, never the answer)."""
import numpy as np
import pytest

from oracle import mlp_oracle

pytestmark = pytest.mark.gpu

# BF16 operands with FP32 accumulation against a float64 reference with the same BF16
# rounding points: only the accumulation order and precision differ (a few 1e-7 relative per
# dot product), which now and then moves a value across a BF16 rounding boundary (one BF16 ulp,
# 2^-8 relative) when activations are rounded between layers.  Relative error of a whole
# output / gradient tensor.
FWD_TOL = 1e-3
GRAD_TOL = 2e-3


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_oracle(built, torch):
    model = built.Model(0, seed=7)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(300, 400)).astype(np.float32)
    X[:, 386:] = 0
    dX = torch.from_numpy(X).cuda()
    dY = torch.empty((300, 2), dtype=torch.float32, device="cuda")
    model.forward(dX.data_ptr(), 300, dY.data_ptr())
    want, _, _ = mlp_oracle.forward(model.get_params(), X)
    err = rel(dY.cpu().numpy(), want)
    assert err < FWD_TOL, err


@pytest.mark.parametrize("B", [37, 512])
def test_gradients_match_oracle(built, torch, B):
    model = built.Model(0, seed=3)
    rng = np.random.default_rng(B)
    X = rng.normal(size=(B, 400)).astype(np.float32)
    X[:, 386:] = 0
    T = rng.normal(size=B).astype(np.float32)
    # the device copies must outlive the call: a freed temporary's block is reused
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    g, loss = model.gradients(dX.data_ptr(), dT.data_ptr(), B)
    want_loss, want = mlp_oracle.loss_and_grads(model.get_params(), X, T.astype(np.float64))
    assert abs(loss - want_loss) <= 1e-2 * abs(want_loss)
    o = 0
    for (n, k) in mlp_oracle.SIZES:
        for size in (n * k, n):
            err = rel(g[o:o + size], want[o:o + size])
            assert err < GRAD_TOL, (n, k, size, err)
            o += size


def test_training_reduces_pinball_loss(built, torch):
    model = built.Model(0, seed=11)
    rng = np.random.default_rng(5)
    X = rng.normal(size=(2048, 400)).astype(np.float32)
    X[:, 386:] = 0
    T = (X[:, 0] * 2 - X[:, 1] + 0.1 * rng.normal(size=2048)).astype(np.float32)
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    losses = [model.train_step(dX.data_ptr(), dT.data_ptr(), 2048, 1e-3) for _ in range(150)]
    assert losses[-1] < 0.5 * losses[0]
    # the 5% / 95% quantile outputs bracket most targets after training
    dY = torch.empty((2048, 2), dtype=torch.float32, device="cuda")
    model.forward(dX.data_ptr(), 2048, dY.data_ptr())
    Y = dY.cpu().numpy()
    inside = np.mean((Y[:, 0] <= T) & (T <= Y[:, 1]))
    assert inside > 0.7


def resample_ref(X, m=64):
    seg = np.linalg.norm(np.diff(X, axis=0), axis=1)
    cum = np.concatenate([[0.0], np.cumsum(seg)])
    s = np.linspace(0.0, cum[-1], m)
    out = np.stack([np.interp(s, cum, X[:, k]) for k in range(X.shape[1])], 1)
    out[0], out[-1] = X[0], X[-1]
    if X.shape[1] == 2:
        out = np.concatenate([out, np.zeros((m, 1))], 1)
    return out


def test_features_match_numpy(ctx, built):
    pairs = [built.gen_pair(1, 3, 1000, 700, 100.0, 0.1, 3, 1),
             built.gen_pair(0, 2, 90, 3000, 1.0, 0.05, 3, 2),
             built.gen_pair(1, 2, 70000, 400, 100.0, 0.1, 3, 3)]
    ep = np.array([0.5, 0.7, 1.1])
    ve = np.array([0.6, 0.8, 1.3])
    F = ctx.features([p for p, _ in pairs], [q for _, q in pairs], ep, ve)
    for k, (P, Q) in enumerate(pairs):
        pts = np.concatenate([resample_ref(P), resample_ref(Q)])
        c = pts.mean(0)
        sc = np.sqrt(((pts - c) ** 2).sum(1).max())
        want = ((pts - c) / sc).ravel()
        np.testing.assert_allclose(F[k, :384], want, atol=2e-5)
        assert abs(F[k, 384] - np.log(ep[k] / sc)) < 1e-4
        assert abs(F[k, 385] - np.log(ve[k] / sc)) < 1e-4
        assert np.all(F[k, 386:] == 0)


def test_bracketed_solves_agree_with_plain(ctx, built):
    pairs = [built.gen_pair(k % 2, 2 + k % 2, 300 + 97 * k, 250 + 131 * k, 100.0 if k % 2 else 1.0,
                            0.1, 21, k) for k in range(24)]
    Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
    plain = ctx.distance_batch(Ps, Qs, precise=True)
    tol = 2.0 ** -33
    # an untrained network: its brackets are arbitrary, verification must repair them
    model = built.Model(0, seed=99)
    got = ctx.distance_batch(Ps, Qs, precise=True, model=model)
    for a, b in zip(plain, got):
        assert abs(a["distance"] - b["distance"]) <= 2 * tol * a["distance"]
        assert b["lb"] <= b["distance"] <= b["ub"]
    # explicit brackets: right, too low, too high
    br = []
    for r in plain:
        fd = r["distance"]
        br.append([fd * (1 - 1e-9), fd * (1 + 1e-9)])
    br[0] = [plain[0]["vefd"] * 0.5, plain[0]["vefd"] * 0.6]
    br[1] = [plain[1]["dfd"] * 2, plain[1]["dfd"] * 3]
    got = ctx.distance_batch(Ps, Qs, precise=True, brackets=np.array(br))
    for k, (a, b) in enumerate(zip(plain, got)):
        assert abs(a["distance"] - b["distance"]) <= 2 * tol * a["distance"], k
    assert sum(b["probes"] for b in got[2:]) < sum(a["probes"] for a in plain[2:])


@pytest.mark.parametrize("M,N,K,layout", [(37, 256, 400, "nt"), (512, 256, 256, "nt"),
                                          (256, 400, 37, "tn"), (2, 256, 512, "tn"),
                                          (512, 256, 2, "nn"), (100, 70, 50, "nn")])
def test_gemm_matches_torch(built, torch, M, N, K, layout):
    """GEMM kernel vs a plain PyTorch FP32 product of the same BF16-rounded operands."""
    g = torch.Generator().manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, generator=g)
    B = torch.randn(K, N, generator=g)
    want = A.bfloat16().double() @ B.bfloat16().double()
    if layout == "nt":    # A row-major [M][K], B stored as [N][K]
        a_buf, a_sr, a_sc = A.contiguous(), K, 1
        b_buf, b_sr, b_sc = B.t().contiguous(), 1, K
    elif layout == "tn":  # A stored as [K][M], B row-major [K][N]
        a_buf, a_sr, a_sc = A.t().contiguous(), 1, M
        b_buf, b_sr, b_sc = B.contiguous(), N, 1
    else:
        a_buf, a_sr, a_sc = A.contiguous(), K, 1
        b_buf, b_sr, b_sc = B.contiguous(), N, 1
    da, db = a_buf.cuda(), b_buf.cuda()
    dc = torch.empty(M, N, device="cuda")
    built.gemm_bf16(M, N, K, da.data_ptr(), a_sr, a_sc, db.data_ptr(), b_sr, b_sc, dc.data_ptr())
    got = dc.cpu().double()
    # FP32 accumulation of K products against float64
    assert float((got - want).abs().max()) <= 1e-5 * float(want.abs().max()) * max(1, K) ** 0.5


def test_trained_network_saves_probes(ctx, built):
    """The shipped network on held-out uneven-batch pairs (seed 4), against the plain method
    and against the same search without the network: the threshold probe over VE-FD alone
    (a bracket at the VE-FD bound, i.e. plain bisection above the threshold when it fails).
    The threshold probe ends about 97 % of these pairs in one probe with or without the
    network; the network is judged on the rest, the tail pairs, where it must save probes
    and where its [q05, q95] must hold the true log10(FD/VEFD - 1) most of the time."""
    import torch
    from robotfd_b200 import train_bracket
    pairs = train_bracket.pairs_of(4096, 4, 0, 4096)
    Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
    plain = ctx.distance_batch(Ps, Qs, precise=True)
    model = built.Model.pretrained(0)
    try:
        got = ctx.distance_batch(Ps, Qs, precise=True, model=model)
        br = np.array([[r["vefd"] * (1 - 1e-15), r["vefd"]] for r in plain])
        alone = ctx.distance_batch(Ps, Qs, precise=True, brackets=br)
        cover, _, _ = train_bracket.coverage(ctx, model, Ps, Qs, plain)
    finally:
        model.close()
    tol = 2.0 ** -33
    for a, b, c in zip(plain, got, alone):
        for r in (b, c):
            assert abs(a["distance"] - r["distance"]) <= 2 * tol * a["distance"]
            assert r["lb"] <= r["distance"] <= r["ub"] and r["ub"] - r["lb"] <= tol * r["ub"]
        assert b["flags"] & built.FLAG_BRACKET_USED
    mean_plain = np.mean([a["probes"] for a in plain])
    assert np.mean([b["probes"] for b in got]) < 0.1 * mean_plain
    tail = [k for k, c in enumerate(alone) if c["probes"] > 1]
    assert len(tail) > 50
    net = np.mean([got[k]["probes"] for k in tail])
    thr = np.mean([alone[k]["probes"] for k in tail])
    assert net < thr - 0.5, (net, thr)             # measured saving on the tail
    assert np.mean(cover) > 0.6, np.mean(cover)    # calibrated quantiles (held-out tail pairs)
