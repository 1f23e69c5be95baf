"""Learned compressor, CPU side: the oracle's gradient against finite
differences, the Morton block layout and the volume <-> block round trip."""
import numpy as np

from konglong_b200 import compressor as AE
from oracle import ae_oracle as O


def test_layer_table_matches_library_layout():
    assert AE.LAYERS == O.LAYERS
    # every layer consumes the previous layer's output memory exactly
    rows_out = [R * N for K, N, R, _ in AE.LAYERS]
    rows_in = [R * K for K, N, R, _ in AE.LAYERS]
    assert rows_in[0] == AE.BLOCK and rows_out[-1] == AE.BLOCK
    assert rows_in[1:] == rows_out[:-1]
    assert rows_out[3] == AE.LATENT
    assert AE.init_params().size == sum(K * N + N for K, N, _, _ in AE.LAYERS)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = AE.init_params(3).astype(np.float64) + 0.01 * rng.standard_normal(AE.init_params().size)
    blocks = rng.uniform(-1, 1, (2, AE.BLOCK))
    loss, g = O.loss_grad(p, blocks)
    idx = rng.choice(p.size, 40, replace=False)
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = O.loss_grad(q, blocks)
        q[i] -= 2 * h
        lm, _ = O.loss_grad(q, blocks)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_morton_layout_and_round_trip():
    perm = AE.morton_perm()
    assert sorted(perm.tolist()) == list(range(AE.BLOCK))
    # the 8 children of each 2^3 cube are consecutive: Morton m // 8 groups
    # cells whose (y, x, z) // 2 agree
    loc = np.stack([perm // 64, (perm // 8) % 8, perm % 8], 1)
    for g in range(64):
        c = loc[8 * g:8 * g + 8] // 2
        assert (c == c[0]).all()
    rng = np.random.default_rng(1)
    w = rng.standard_normal((19, 13, 21)).astype(np.float32)
    b, s = AE.volume_to_blocks(w)
    assert b.shape == (3 * 2 * 3, AE.BLOCK) and np.abs(b).max() <= 1.0 + 1e-6
    np.testing.assert_allclose(AE.blocks_to_volume(b, s, w.shape), w, rtol=1e-6, atol=1e-6)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -3.14159, 0.0], np.float32)
    r = O.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6  # ties to even
    assert abs(r[3] + 3.140625) < 1e-7 and r[4] == 0.0


def test_fallback_selection_is_the_top_candidates():
    """The FP16 fallback keeps the candidate blocks (scale > tau x max) above the
    (cap+1)-th largest candidate scale: never more than cap, ties left out."""
    rng = np.random.default_rng(3)
    s = np.exp(rng.standard_normal(5000) * 3).astype(np.float32)
    s[:40] = s.max()  # a tie at the top
    s[40:90] = 0.0
    for tau, frac in [(1e-3, 0.05), (0.0, 0.2), (0.5, 0.5), (1e-3, 1.0), (1e-3, 0.005)]:
        sel = AE.fallback_selection(s, tau, frac)
        cap = int(np.ceil(float(np.float32(frac)) * s.size))  # as the library: float max_fraction, double product
        cand = np.flatnonzero((s > 0) & (s > np.float32(tau) * s.max()))
        assert sel.size <= cap and np.isin(sel, cand).all()
        rest = np.setdiff1d(cand, sel)
        if rest.size:  # everything kept is larger than everything left out
            assert s[sel].min(initial=np.inf) > s[rest].max()
            assert (s[cand] >= s[rest].max()).sum() > cap  # and the next value would overflow
    assert AE.fallback_selection(s, 1e-3, 0.005).size == 0  # 40 tied maxima > cap 25
    w = rng.standard_normal((9, 17, 12)).astype(np.float32)
    _, sc = AE.volume_to_blocks(w)
    rec = AE.apply_fallback(np.zeros_like(w), w, sc, np.arange(sc.size))
    assert np.abs(rec - w).max() <= 1e-3 * np.abs(w).max()


def test_average_code_initialisation_reproduces_the_average_code():
    """init_params_average makes the network compute the 16:1 2^3-average
    code: through the BF16-emulating oracle its reconstruction equals the
    non-learned code up to BF16 rounding (0.5 %), its latents are the 64
    averages times the (+, -) pair gain 1.1^3."""
    rng = np.random.default_rng(2)
    b = rng.standard_normal((48, AE.BLOCK)).astype(np.float32)
    b /= np.abs(b).max(axis=1, keepdims=True)
    rec, lat = O.reconstruct(AE.init_params_average(), b, round_bf16=True)
    naive = AE.naive_16to1(b)
    assert np.linalg.norm(rec - naive) / np.linalg.norm(naive) < 1e-2
    avg = b.reshape(-1, 64, 8).mean(axis=2)
    np.testing.assert_allclose(lat, 1.1 ** 3 * avg, rtol=2e-2, atol=2e-3)
