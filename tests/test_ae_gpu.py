"""Learned snapshot compressor on the GPU: tensor-core forward and gradients
against the CPU oracle, training on the engine's own forward wavefields, the
gain of the trained network over the code without learning, and the learned
snapshots inside an RTM shot next to the plain FP32 store (the reference
image their error is measured against) and COMPRESS_16, with and without the
FP16 fallback of the high-energy blocks."""
import numpy as np
import pytest

from konglong_b200 import compressor as AE
from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import FIELD_W0, SNAP_AE, SNAP_C16, SNAP_FP32
from oracle import ae_oracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    """Blocks of VTI compact-FD forward runs (the 512x512x400 workload's model
    family at 0.2 scale): training blocks from two models, held-out blocks
    from a third."""
    tr = [AE.training_blocks(W.vti_cfd(scale=0.2, seed=sd, nt=400), Propagator, spread_coeffs,
                             nblocks=6000, every=10)[0] for sd in (2, 3)]
    held = AE.training_blocks(W.vti_cfd(scale=0.2, seed=9, nt=400), Propagator, spread_coeffs,
                              nblocks=2000, every=10)[0]
    return np.concatenate(tr), held


def test_forward_matches_oracle(data):
    ae = AE.AutoEncoder(seed=5)
    p, b = ae.params(), data[0][:64]
    out, lat = ae.reconstruct(b)
    ref, ref_lat = O.reconstruct(p, b, round_bf16=True)
    # same BF16 operands; the FP32 (GPU) and FP64 (oracle) sums of a layer can
    # round an activation to neighbouring BF16 values in the next layer
    assert rel_l2(out, ref) < 2e-3 and rel_l2(lat, ref_lat) < 2e-3
    exact, _ = O.reconstruct(p, b, round_bf16=False)
    assert rel_l2(out, exact) < 2e-2  # BF16 operands vs FP64


def test_gradients_match_oracle(data):
    ae = AE.AutoEncoder(seed=5)
    p, b = ae.params(), data[0][:32]
    loss, g = ae.loss_grad(b)
    l_ref, g_ref = O.loss_grad(p, b, round_bf16=True)
    assert abs(loss - l_ref) <= 1e-4 * l_ref
    assert rel_l2(g, g_ref) < 2e-3
    l64, g64 = O.loss_grad(p, b, round_bf16=False)
    assert abs(loss - l64) <= 1e-3 * l64 and rel_l2(g, g64) < 2e-2


def test_training_gain_over_untrained_and_naive_code(data):
    train, held = data
    ae = AE.AutoEncoder(seed=5)
    before = rel_l2(ae.reconstruct(held)[0], held)
    losses = ae.fit(train, steps=1500, batch=256, lr=3e-3)
    after = rel_l2(ae.reconstruct(held)[0], held)
    naive = rel_l2(AE.naive_16to1(held), held)
    assert losses[-50:].mean() < 0.1 * losses[:10].mean()
    # held-out blocks of another model, same 16:1 ratio as the averaging code
    assert after < 0.2 * before
    assert after < 0.6 * naive, (after, naive)


def test_learned_snapshots_in_rtm(data):
    train, _ = data
    ae = AE.AutoEncoder(seed=5)
    ae.fit(train, steps=1500, batch=256, lr=3e-3)
    sh = W.vti_cfd(scale=0.2, seed=9, nt=300)
    s = sh.spec
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([sh.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(sh.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    m = Propagator(s)
    m.set_model(**sh.model_arrays())
    m.set_injection(src, sh.wavelet[None, :], s.dt_dxyz)
    m.set_extraction(rcv, 300)
    m.reset()
    m.modelling(300, -1, 1)
    rec = m.traces()
    # the device store / load of one snapshot equals the host round trip
    w = np.ascontiguousarray(m.get(FIELD_W0).reshape(s.shape))
    m.set_compressor(ae)
    m.snapshot_setup(SNAP_AE, 1)
    m.put(FIELD_W0, w)
    m.snapshot_store(0)
    dev = m.snapshot_load(0).reshape(s.shape)
    b, sc = AE.volume_to_blocks(w)
    host = AE.blocks_to_volume(ae.reconstruct(b)[0], sc, s.shape)
    assert rel_l2(dev, host) < 1e-6
    # with the FP16 fallback of the high-energy blocks
    m.set_compressor_fallback(1e-3, 0.05)
    m.snapshot_setup(SNAP_AE, 1)
    m.put(FIELD_W0, w)
    m.snapshot_store(0)
    dev = m.snapshot_load(0).reshape(s.shape)
    sel = AE.fallback_selection(sc, 1e-3, 0.05)
    assert 0 < sel.size <= int(np.ceil(0.05 * sc.size))
    assert rel_l2(dev, AE.apply_fallback(host, w, sc, sel)) < 1e-6
    assert rel_l2(dev, w) < 0.5 * rel_l2(host, w)
    m.close()
    imgs = {}
    runs = [(SNAP_FP32, 0), (SNAP_C16, 0), (SNAP_AE, 0), (SNAP_AE, 0.05), (SNAP_AE, 0.15)]
    for fmt, frac in runs:
        q = Propagator(s)
        q.set_model(**sh.model_arrays())
        if fmt == SNAP_AE:
            q.set_compressor(ae)
            q.set_compressor_fallback(1e-3, frac)
        imgs[fmt, frac] = q.rtm_shot(src, sh.wavelet[None, :], rcv, rec, 300, 210, 5, snap_fmt=fmt, ntaper_t=3,
                                     ntaper_z=4)[0].reshape(s.shape)
        q.close()
    fb = {frac: rel_l2(imgs[SNAP_AE, frac], imgs[SNAP_FP32, 0]) for frac in (0.05, 0.15)}
    print("learned snapshots + FP16 fallback, image NRMSE vs FP32 store: "
          + ", ".join(f"{100 * f:.0f}% of blocks {e:.4f}" for f, e in fb.items()))
    assert fb[0.15] <= fb[0.05] < rel_l2(imgs[SNAP_AE, 0], imgs[SNAP_FP32, 0])
    imgs = {fmt: imgs[fmt, 0] for fmt in (SNAP_FP32, SNAP_C16, SNAP_AE)}
    ref = imgs[SNAP_FP32]
    assert np.isfinite(imgs[SNAP_AE]).all() and np.abs(ref).max() > 0
    assert rel_l2(imgs[SNAP_C16], ref) < 2e-3
    # below the near-surface mute (source and receiver depth + 10 cells)
    z0 = s.nbnd[4] + 12
    deep = rel_l2(imgs[SNAP_AE][:, :, z0:], ref[:, :, z0:])
    full = rel_l2(imgs[SNAP_AE], ref)
    print(f"learned-snapshot image NRMSE vs FP32 store: full {full:.3f}, below z={z0}: {deep:.3f}")
    # measured: full 0.96, below the mute 0.46-0.51 (the 16:1 code does not hold
    # the near-source blocks, which carry most of the energy); the learned code
    # alone is not the product form: it runs with the FP16 fallback (above, and
    # the ablation below)
    assert full < 1.0 and deep < 0.7


def test_ablation_at_equal_bytes(data):
    """What the trained network adds at the same bytes per block: every code
    below keeps the same FP16 copies of the 5 % highest-energy blocks and
    spends 32 floats + the block scale on each other block.  The residual
    error of a held-out snapshot (a compact-FD VTI forward wavefield of a model
    not trained on) with: the trained code; the same network untrained; the
    16:1 2^3-average code; no code (those blocks zero)."""
    train, _ = data
    ae = AE.AutoEncoder(seed=5)
    raw = AE.AutoEncoder(seed=5)
    ae.fit(train, steps=1500, batch=256, lr=3e-3)
    sh = W.vti_cfd(scale=0.2, seed=11, nt=400)
    s = sh.spec
    m = Propagator(s)
    m.set_model(**sh.model_arrays())
    k1, k2 = W.spread_band(s)
    m.set_injection(W.make_traceset([sh.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs),
                    sh.wavelet[None, :], s.dt_dxyz)
    m.reset()
    m.modelling(300, -1, 1)
    w = np.ascontiguousarray(m.get(FIELD_W0).reshape(s.shape))
    m.close()
    b, sc = AE.volume_to_blocks(w)
    sel = AE.fallback_selection(sc, 1e-3, 0.05)
    codes = {"trained": ae.reconstruct(b)[0], "untrained": raw.reconstruct(b)[0],
             "naive 16:1": AE.naive_16to1(b), "zero": np.zeros_like(b)}
    err = {k: rel_l2(AE.apply_fallback(AE.blocks_to_volume(v, sc, s.shape), w, sc, sel), w) for k, v in codes.items()}
    print("held-out snapshot NRMSE with the 5 % FP16 fallback: " + ", ".join(f"{k} {v:.2e}" for k, v in err.items()))
    # measured: trained 0.59, untrained 0.73, naive 16:1 0.15, zero 0.73.  Training
    # helps, but at equal bytes the 2^3-average code (64 FP16 values per block)
    # beats the 32-float latent on these band-limited wavefields: the learned
    # code does not earn its place over it.  Bounds: the trained network must
    # beat no code and the untrained network; the ordering against the naive
    # code is recorded as it stands.
    assert err["trained"] < 0.9 * err["untrained"]
    assert err["trained"] < 0.9 * err["zero"]
    assert err["naive 16:1"] < err["trained"]


def test_fused_volume_codec_equals_layered(data):
    """The fused encode / decode kernels that the snapshot store uses (one
    warp per block, the layers in shared memory) give the bits of the
    layer-by-layer GEMM path: the stored BF16 latents and the scales of a
    device volume equal rtm_ae_reconstruct's FP32 latents rounded to BF16 (the
    decoder's operand rounding) and its scales on the host-blocked volume, and
    the decoded volume equals that reconstruction times the scales; partial
    blocks at every face included."""
    import torch
    from konglong_b200 import _lib
    train, _ = data
    ae = AE.AutoEncoder(seed=5)
    ae.fit(train, steps=300, batch=256, lr=3e-3)
    rng = np.random.default_rng(3)
    L = _lib.lib()
    for shape in [(19, 27, 45), (16, 24, 64), (8, 9, 70)]:
        ny, nx, nz = shape
        w = (rng.standard_normal(shape) * np.linspace(0.1, 3.0, nz)).astype(np.float32)
        w[:, :, 5] = 0.0
        b, sc = AE.volume_to_blocks(w)
        rec, lat = ae.reconstruct(b)
        nb = b.shape[0]
        dv = torch.from_numpy(w).cuda()
        dl = torch.zeros(nb * AE.LATENT, device="cuda", dtype=torch.bfloat16)
        ds = torch.zeros(nb, device="cuda")
        out = torch.zeros_like(dv)
        _lib.check(L.rtm_ae_compress_volume(ae.a, dv.data_ptr(), nx, ny, nz, dl.data_ptr(), ds.data_ptr(), None),
                   "rtm_ae_compress_volume")
        _lib.check(L.rtm_ae_decompress_volume(ae.a, dl.data_ptr(), ds.data_ptr(), nx, ny, nz, out.data_ptr(), None),
                   "rtm_ae_decompress_volume")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ds.cpu().numpy(), sc)
        np.testing.assert_array_equal(dl.float().cpu().numpy().reshape(nb, AE.LATENT), O.bf16(lat).astype(np.float32))
        np.testing.assert_array_equal(out.cpu().numpy(), AE.blocks_to_volume(rec, sc, shape))
    ae.close()
