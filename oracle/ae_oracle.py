"""CPU oracle of the learned snapshot compressor (test infrastructure only).

Float64 restatement of the autoencoder the library trains and runs (layer
table in konglong_b200/csrc/ae.cu): every layer is y = act(x @ W + b) on the
previous layer's output memory viewed as [rows][K] (Morton block layout),
leaky ReLU with slope 0.1, MSE loss against the input block.  With
`bf16=True` the operands of every matrix product are rounded to BF16 (round
to nearest even) as the tensor-core kernels round them, so the GPU result
differs from this oracle only by FP32 accumulation; with `bf16=False` it is
the plain FP64 reference the errors are stated against.  There is no
reference-code counterpart: bgprtm has no learned compressor (its
WaveFieldCompress is the non-learned fallback).
"""
import numpy as np

LAYERS = [(8, 16, 64, True), (128, 16, 8, True), (16, 16, 8, True), (128, 64, 1, False),
          (64, 128, 1, True), (16, 16, 8, True), (16, 128, 8, True), (16, 8, 64, False)]
SLOPE = 0.1


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(params):
    out, o = [], 0
    for K, N, _, _ in LAYERS:
        W = np.asarray(params[o:o + K * N], np.float64).reshape(K, N)
        o += K * N
        b = np.asarray(params[o:o + N], np.float64)
        o += N
        out.append((W, b))
    return out


def _mm(a, b, round_bf16):
    if round_bf16:
        return bf16(a) @ bf16(b)
    return np.asarray(a, np.float64) @ np.asarray(b, np.float64)


def forward(params, blocks, round_bf16=False, upto=len(LAYERS)):
    """Activations of every layer for blocks [n][512]: list of (pre, post)."""
    n = blocks.shape[0]
    x = np.asarray(blocks, np.float64)
    acts = []
    for l, ((W, b), (K, N, R, act)) in enumerate(zip(unpack(params), LAYERS)):
        if l == upto:
            break
        xin = x.reshape(n * R, K)
        pre = _mm(xin, W, round_bf16) + b
        post = np.where(pre > 0, pre, SLOPE * pre) if act else pre
        acts.append((xin, pre, post))
        x = post
    return acts


def loss_grad(params, blocks, round_bf16=False):
    """MSE loss of the reconstruction and d loss / d params (library layout)."""
    n = blocks.shape[0]
    acts = forward(params, blocks, round_bf16)
    y = acts[-1][2].reshape(n, -1)
    x0 = np.asarray(blocks, np.float64)
    tot = x0.size
    loss = float(np.sum((y - x0) ** 2) / tot)
    dy = (2.0 * (y - x0) / tot).reshape(acts[-1][2].shape)
    grads = [None] * len(LAYERS)
    for l in range(len(LAYERS) - 1, -1, -1):
        K, N, R, act = LAYERS[l]
        xin, pre, _ = acts[l]
        W, _ = unpack(params)[l]
        dp = np.where(pre > 0, dy, SLOPE * dy) if act else dy
        gW = _mm(xin.T, dp, round_bf16)
        gb = dp.sum(axis=0)
        grads[l] = (gW, gb)
        dx = _mm(dp, W.T, round_bf16)
        if l > 0:
            dy = dx.reshape(acts[l - 1][2].shape)
    flat = np.concatenate([np.concatenate([g.ravel(), b]) for g, b in grads])
    return loss, flat


def reconstruct(params, blocks, round_bf16=False):
    n = blocks.shape[0]
    acts = forward(params, blocks, round_bf16)
    return acts[-1][2].reshape(n, -1), acts[3][2].reshape(n, -1)
