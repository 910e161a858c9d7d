"""Host logic of the bracket training script (CPU): the normalisation fold and the target."""
import numpy as np

from oracle import mlp_oracle
from robotfd_b200 import train_bracket as tb


def forward_f64(params, X):
    a = np.asarray(X, dtype=np.float64)
    layers = mlp_oracle.unpack(params.astype(np.float64))
    for li, (W, b) in enumerate(layers):
        z = a @ W.T + b
        a = mlp_oracle.gelu(z) if li < 3 else z
    return a


def test_fold_matches_normalised_network():
    rng = np.random.default_rng(0)
    n = sum(o * i + o for o, i in mlp_oracle.SIZES)
    params = (rng.normal(size=n) * 0.05).astype(np.float32)
    X = rng.normal(size=(64, 400)) * 3 + 1
    mu = rng.normal(size=400)
    sd = rng.uniform(0.5, 2.0, size=400)
    ymu, ysd = -10.3, 1.7
    want = forward_f64(params, (X - mu) / sd) * ysd + ymu
    got = forward_f64(tb.fold(params, mu, sd, ymu, ysd), X)
    # the folded parameters are stored as float32
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


def test_target():
    base = {"distance": 1.0 + 1e-10, "vefd": 1.0, "flags": 0}
    assert abs(tb.target(base) - np.log10(1e-10 + 1e-13)) < 1e-5
    assert tb.target(dict(base, distance=1.0)) == -13.0
    assert np.isnan(tb.target(dict(base, vefd=0.0)))
    assert np.isnan(tb.target(dict(base, flags=128)))
