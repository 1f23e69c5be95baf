"""Learned snapshot compressor: host side of the rtm_ae_* C ABI.

A 3-D convolutional autoencoder on 8^3-cell wavefield blocks (4 encoder +
4 decoder layers, 16 channels, 512 cells -> 64 latent values (stored as BF16,
the decoder's operand precision) + the block's
max |w|, 15.5:1), trained on blocks of the engine's own forward wavefields and
run inside the RTM loop as snapshot format RTM_SNAP_AE.  Training and
inference run in the library's BF16 tensor-core kernels (FP32 accumulation,
FP32 master weights, Adam); this module only prepares data and drives them.
"""
import ctypes as C

import numpy as np

from . import _lib

LAYERS = [(8, 16, 64, True), (128, 16, 8, True), (16, 16, 8, True), (128, 64, 1, False),
          (64, 128, 1, True), (16, 16, 8, True), (16, 128, 8, True), (16, 8, 64, False)]  # K, N, rows/block, act
LATENT = 64
BLOCK = 512


def morton_perm():
    """perm[m] = (y*8 + x)*8 + z of the cell with Morton index m (bits z y x
    from the least significant end), the block layout of the library."""
    perm = np.zeros(BLOCK, np.int64)
    for y in range(8):
        for x in range(8):
            for z in range(8):
                m = 0
                for b in range(3):
                    m |= ((z >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((x >> b) & 1) << (3 * b + 2)
                perm[m] = (y * 8 + x) * 8 + z
    return perm


_PERM = morton_perm()


def volume_to_blocks(w):
    """Volume [ny][nx][nz] -> (blocks [nb][512] Morton order, scale-normalised,
    scales [nb]); blocks ordered (by, bx, bz) with bz fastest, zero padding."""
    ny, nx, nz = w.shape
    py, px, pz = -ny % 8, -nx % 8, -nz % 8
    v = np.pad(np.asarray(w, np.float32), ((0, py), (0, px), (0, pz)))
    by, bx, bz = v.shape[0] // 8, v.shape[1] // 8, v.shape[2] // 8
    b = v.reshape(by, 8, bx, 8, bz, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, BLOCK)[:, _PERM]
    s = np.abs(b).max(axis=1)
    out = np.where(s[:, None] > 0, b / np.where(s > 0, s, 1.0)[:, None], 0.0).astype(np.float32)
    return out, s.astype(np.float32)


def blocks_to_volume(blocks, scales, shape):
    ny, nx, nz = shape
    by, bx, bz = -(-ny // 8), -(-nx // 8), -(-nz // 8)
    b = np.empty_like(blocks)
    b[:, _PERM] = blocks * scales[:, None]
    v = b.reshape(by, bx, bz, 8, 8, 8).transpose(0, 3, 1, 4, 2, 5).reshape(by * 8, bx * 8, bz * 8)
    return np.ascontiguousarray(v[:ny, :nx, :nz])


def fallback_selection(scales, tau, max_fraction):
    """Blocks a learned snapshot also keeps as FP16 (rtm_set_compressor_fallback):
    the candidates (scale > 0 and > tau x the largest) whose scale exceeds the
    (cap+1)-th largest candidate scale, cap = ceil(max_fraction x blocks); all
    candidates when there are at most cap.  Returns ascending block indices."""
    s = np.asarray(scales, np.float32)
    if max_fraction <= 0 or s.size == 0:
        return np.zeros(0, np.int64)
    cap = max(1, int(np.ceil(float(np.float32(max_fraction)) * s.size)))
    cand = (s > 0) & (s > np.float32(tau) * s.max())
    if cand.sum() > cap:
        cand &= s > np.sort(s[cand])[::-1][cap]
    return np.flatnonzero(cand)


def apply_fallback(rec, w, scales, sel):
    """Overwrite the selected 8^3 blocks of the decoded volume `rec` with the
    FP16 copy of w / scale, times scale, as the device load does."""
    rec = np.array(rec, np.float32, copy=True)
    ny, nx, nz = rec.shape
    nbz, nbx = -(-nz // 8), -(-nx // 8)
    for b in np.asarray(sel):
        bz, bx, by = b % nbz, (b // nbz) % nbx, b // (nbz * nbx)
        sl = (slice(by * 8, by * 8 + 8), slice(bx * 8, bx * 8 + 8), slice(bz * 8, bz * 8 + 8))
        sc = np.float32(scales[b])
        rec[sl] = (np.asarray(w[sl], np.float32) / sc).astype(np.float16).astype(np.float32) * sc
    return rec


def init_params(seed=5):
    """Glorot-uniform weights, zero biases, in the library's parameter layout."""
    rng = np.random.default_rng(seed)
    out = []
    for K, N, _, _ in LAYERS:
        a = np.sqrt(6.0 / (K + N))
        out.append(rng.uniform(-a, a, (K, N)).astype(np.float32).ravel())
        out.append(np.zeros(N, np.float32))
    return np.concatenate(out)


def init_params_average():
    """Parameters with which the network computes the 16:1 2^3-average code
    exactly (up to BF16 rounding): the latent holds the 64 averages (scaled),
    the decoder repeats each over its 2^3 cube.  A leaky ReLU passes a value
    x linearly through two channels, x = (lr(x) - lr(-x)) / (1 + slope), so
    every layer carries the averages as (+, -) channel pairs: E1 forms them
    from the 8 children of each 2^3 cube, E2 / E3 and D1 / D2 / D3 re-split
    them (each re-split scales them by 1 + slope), E4 writes the 64 values
    to the latent and D4 removes the accumulated scale.  All weights are +-1,
    +-1/8 or the one D4 factor; biases are zero.  Training from here starts
    at the non-learned code's error."""
    g = 1.0 + 0.1  # the leaky ReLU's (+, -) pair gain, slope 0.1
    W = [np.zeros((K, N), np.float64) for K, N, _, _ in LAYERS]
    for k in range(8):  # E1: rows = 2^3 cubes, K = their 8 children
        W[0][k, 0], W[0][k, 1] = 1.0 / 8, -1.0 / 8
    for c in range(8):  # E2: K = 8 cubes x 16 channels -> (+, -) of cube c in channels 2c, 2c+1
        W[1][c * 16, 2 * c], W[1][c * 16 + 1, 2 * c] = 1.0, -1.0
        W[1][c * 16, 2 * c + 1], W[1][c * 16 + 1, 2 * c + 1] = -1.0, 1.0
    for c in range(8):  # E3 and D2: pointwise re-split of the 8 pairs
        for l in (2, 5):
            W[l][2 * c, 2 * c], W[l][2 * c + 1, 2 * c] = 1.0, -1.0
            W[l][2 * c, 2 * c + 1], W[l][2 * c + 1, 2 * c + 1] = -1.0, 1.0
    for r in range(8):  # E4: K = 8 rows x 16 channels -> latent 8 r + c; D1 back to (+, -) pairs
        for c in range(8):
            W[3][r * 16 + 2 * c, 8 * r + c], W[3][r * 16 + 2 * c + 1, 8 * r + c] = 1.0, -1.0
            W[4][8 * r + c, r * 16 + 2 * c], W[4][8 * r + c, r * 16 + 2 * c + 1] = 1.0, -1.0
    for c in range(8):  # D3: pair c -> the (+, -) channels of child cube c
        W[6][2 * c, c * 16], W[6][2 * c + 1, c * 16] = 1.0, -1.0
        W[6][2 * c, c * 16 + 1], W[6][2 * c + 1, c * 16 + 1] = -1.0, 1.0
    # D4: every one of a cube's 8 cells is its average; six (+, -) re-splits
    # (E2, E3, E4, D2, D3, D4) have scaled it by g each
    for k in range(8):
        W[7][0, k], W[7][1, k] = 1.0 / g ** 6, -1.0 / g ** 6
    out = []
    for w, (K, N, _, _) in zip(W, LAYERS):
        out.append(w.astype(np.float32).ravel())
        out.append(np.zeros(N, np.float32))
    return np.concatenate(out)


def naive_16to1(blocks):
    """Reference 16:1 code without learning: 2^3 averages (64 values) in FP16."""
    return np.repeat(blocks.reshape(-1, 64, 8).mean(axis=2, keepdims=True).astype(np.float16).astype(np.float32),
                     8, axis=2).reshape(-1, BLOCK)


class AutoEncoder:
    def __init__(self, params=None, seed=5):
        self.L = _lib.lib()
        a = C.c_void_p()
        _lib.check(self.L.rtm_ae_create(C.byref(a)), "rtm_ae_create")
        self.a = a
        self.nparams = self.L.rtm_ae_nparams()
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if getattr(self, "a", None):
            self.L.rtm_ae_destroy(self.a)
            self.a = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        _lib.check(self.L.rtm_ae_set_params(self.a, p), "rtm_ae_set_params")

    def params(self):
        p = np.zeros(self.nparams, np.float32)
        _lib.check(self.L.rtm_ae_get_params(self.a, p), "rtm_ae_get_params")
        return p

    def loss_grad(self, blocks):
        b = np.ascontiguousarray(blocks, np.float32)
        loss = C.c_float()
        g = np.zeros(self.nparams, np.float32)
        _lib.check(self.L.rtm_ae_loss_grad(self.a, b, b.shape[0], C.byref(loss), g), "rtm_ae_loss_grad")
        return loss.value, g

    def train_step(self, blocks, lr):
        b = np.ascontiguousarray(blocks, np.float32)
        loss = C.c_float()
        _lib.check(self.L.rtm_ae_train_step(self.a, b, b.shape[0], float(lr), C.byref(loss)), "rtm_ae_train_step")
        return loss.value

    def reconstruct(self, blocks):
        b = np.ascontiguousarray(blocks, np.float32)
        out = np.zeros_like(b)
        lat = np.zeros((b.shape[0], LATENT), np.float32)
        _lib.check(self.L.rtm_ae_reconstruct(self.a, b, b.shape[0], out, lat), "rtm_ae_reconstruct")
        return out, lat

    def fit(self, blocks, steps=2000, batch=256, lr=2e-3, seed=0, lr_final=2e-4, weights=None, uniform=0.5):
        """Adam on random batches of `blocks` with a cosine-decayed learning
        rate; `weights` (e.g. the blocks' energy, scale^2) sets the sampling
        probability, so the loss follows the volume-level error the imaging
        condition sees, mixed with a fraction `uniform` of uniform sampling.
        Returns the batch losses."""
        rng = np.random.default_rng(seed)
        prob = None
        if weights is not None:
            w = np.asarray(weights, np.float64)
            prob = (1.0 - uniform) * w / w.sum() + uniform / w.size
        losses = []
        for k in range(steps):
            idx = rng.choice(blocks.shape[0], batch, p=prob) if prob is not None else \
                rng.integers(0, blocks.shape[0], batch)
            lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(1, steps - 1)))
            losses.append(self.train_step(blocks[idx], lr_k))
        return np.asarray(losses)


def volume_nrmse(ae, w):
    """NRMSE of the learned code of volume w (host round trip), the error the
    imaging condition sees."""
    b, sc = volume_to_blocks(w)
    rec, _ = ae.reconstruct(b)
    v = blocks_to_volume(rec, sc, w.shape)
    return float(np.linalg.norm((v - w).ravel()) / max(np.linalg.norm(w.ravel()), 1e-30))


def training_blocks(shot, propagator_cls, coeff_fn, nblocks=20000, every=20, seed=5, min_scale_frac=1e-3):
    """Blocks of forward wavefields of `shot`'s model (the engine's own
    modelling run, a snapshot every `every` steps), dropping blocks the wave
    has not reached (max |w| below min_scale_frac of the run's peak).  Returns
    (blocks [n][512] normalised, scales [n])."""
    from . import workloads as W
    from .spec import FIELD_W1
    s = shot.spec
    p = propagator_cls(s)
    if s.use_q:
        p.set_q_coeffs(*W.q_coefficients(s.dt, shot.fpeak))
    p.set_model(**shot.model_arrays())
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, coeff_fn)
    p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
    p.reset()
    out, scales = [], []
    for _ in range(shot.nt // every):
        p.modelling(every, -1, 1)
        b, sc = volume_to_blocks(p.get(FIELD_W1).reshape(s.shape))
        out.append(b), scales.append(sc)
    p.close()
    b, sc = np.concatenate(out), np.concatenate(scales)
    keep = sc > min_scale_frac * sc.max()
    b, sc = b[keep], sc[keep]
    rng = np.random.default_rng(seed)
    if b.shape[0] > nblocks:
        idx = rng.choice(b.shape[0], nblocks, replace=False)
        b, sc = b[idx], sc[idx]
    return b, sc
