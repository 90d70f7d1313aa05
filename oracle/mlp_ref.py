"""FP64 numpy restatement of the scattering-source surrogate network, for
checking the GPU training kernels.  TEST INFRASTRUCTURE ONLY: imported by
tests/, never by the product.

Network: x[NF] -> tanh(W0 x + b0) -> tanh(W1 . + b1) -> tanh(W2 . + b2)
-> W3 . + b3 = y[nout]; weights W_l are [out][in] row-major.  Loss: mean
over the batch of the sum over outputs of (y - t)^2.
"""
import numpy as np


def forward(params, x):
    """params: [(W0, b0), ..., (W3, b3)]; x: [n][NF].  Returns the
    activations of every layer (input first) and the output."""
    acts = [x]
    h = x
    for li, (w, b) in enumerate(params):
        z = h @ w.T + b
        h = np.tanh(z) if li < len(params) - 1 else z
        acts.append(h)
    return acts


def loss_and_grads(params, x, t):
    """Loss and gradients (same structure as params) for one batch."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    p64 = [(np.asarray(w, np.float64), np.asarray(b, np.float64)) for w, b in params]
    acts = forward(p64, x)
    n = x.shape[0]
    y = acts[-1]
    loss = np.sum((y - t) ** 2) / n
    dh = 2.0 * (y - t) / n
    grads = [None] * len(p64)
    for li in range(len(p64) - 1, -1, -1):
        w, _ = p64[li]
        if li < len(p64) - 1:
            dh = dh * (1.0 - acts[li + 1] ** 2)  # tanh'
        grads[li] = (dh.T @ acts[li], dh.sum(axis=0))
        dh = dh @ w
    return loss, grads


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest, ties to even),
    returned as float32."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def infer_bf16(params, feat, xm, xs, ym, ys):
    """The inference the GPU runs, restated in numpy: standardised features
    and every hidden activation rounded to BF16, BF16-rounded weights, FP32
    biases, products summed in FP64 (the GPU sums in FP32), exact tanh (the
    GPU's tcgen05 path uses the hardware approximation), sources
    exp(y * ys + ym)."""
    h = bf16((np.asarray(feat, np.float32) - xm) / xs).astype(np.float64)
    for li, (w, b) in enumerate(params):
        z = h @ bf16(w).astype(np.float64).T + np.asarray(b, np.float32).astype(np.float64)
        if li < len(params) - 1:
            h = bf16(np.tanh(z).astype(np.float32)).astype(np.float64)
        else:
            h = z.astype(np.float32)
    y = h * np.asarray(ys, np.float32) + np.asarray(ym, np.float32)   # float32, as the GPU
    return np.exp(y.astype(np.float64))
