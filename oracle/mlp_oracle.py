"""CPU oracle of the learned-bracket network (TEST INFRASTRUCTURE ONLY).

Restates robotfd_b200/csrc/rfd_mlp.cu in numpy: the same layer shapes, the tanh GELU, the
pinball loss of the 5% / 95% quantiles and the gradients of every parameter.  Every GEMM
operand is rounded to BF16 exactly where the GPU rounds it (weights, layer inputs,
upstream gradients); products accumulate in float64 here and in FP32 on the GPU, so the
two agree to BF16-rounding tolerance, which is what the gradient check asserts.
"""
import numpy as np

IN, H, OUT = 400, 256, 2
TAU = (0.05, 0.95)
SIZES = [(H, IN), (H, H), (H, H), (OUT, H)]


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(params):
    out, o = [], 0
    for (n, k) in SIZES:
        W = params[o:o + n * k].reshape(n, k)
        o += n * k
        b = params[o:o + n]
        o += n
        out.append((W, b))
    assert o == params.size
    return out


def gelu(z):
    u = 0.7978845608028654 * (z + 0.044715 * z ** 3)
    return 0.5 * z * (1.0 + np.tanh(u))


def gelu_grad(z):
    u = 0.7978845608028654 * (z + 0.044715 * z ** 3)
    th = np.tanh(u)
    return 0.5 * (1 + th) + 0.5 * z * (1 - th * th) * 0.7978845608028654 * (1 + 3 * 0.044715 * z * z)


def forward(params, X):
    layers = unpack(params)
    a = np.asarray(bf16(X), dtype=np.float64)
    Zs, As = [], [a]
    for li, (W, b) in enumerate(layers):
        z = a @ np.asarray(bf16(W), dtype=np.float64).T + np.asarray(b, dtype=np.float64)
        if li < 3:
            Zs.append(z)
            a = np.asarray(bf16(gelu(z)), dtype=np.float64)
            As.append(a)
        else:
            return z, Zs, As
    raise AssertionError


def loss_and_grads(params, X, T):
    layers = unpack(params)
    Y, Zs, As = forward(params, X)
    B = X.shape[0]
    u = T[:, None] - Y
    tau = np.array(TAU)[None, :]
    ind = (u < 0).astype(np.float64)
    loss = float(np.sum(u * (tau - ind)) / B)
    d = -(tau - ind) / B
    grads = [None] * 4
    for li in range(3, -1, -1):
        W, _ = layers[li]
        dq = np.asarray(bf16(d), dtype=np.float64)
        gW = dq.T @ As[li]
        gb = d.sum(0)
        grads[li] = (gW, gb)
        if li > 0:
            dh = dq @ np.asarray(bf16(W), dtype=np.float64)
            d = dh * gelu_grad(Zs[li - 1])
    flat = np.concatenate([np.concatenate([g.ravel(), b]) for g, b in grads])
    return loss, flat
