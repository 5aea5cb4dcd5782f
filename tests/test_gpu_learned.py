"""Learned coarse-grid PME correction: training kernels against the FP64
oracle, what the trained network gains over the coarse grid alone, and the
full-grid check with its fallback during stepping."""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol

pytestmark = pytest.mark.gpu


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def small_engine(coarse=12, grid=36, frames=24):
    s = systems.water_box(1500, 3.6, seed=11, name="water_learned")
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa_from_tol(1.0, 1e-5), dt=1e-6)
    e.load(s, pme_grid=(grid, grid, grid))
    lp = E.LearnedPME(e, coarse_grid=(coarse, coarse, coarse), max_frames=frames)
    return s, e, lp


def split_params(v):
    """Views of a parameter vector by block (W1 b1 W2 b2 W3 b3 W4 b4)."""
    K, N = [80, 128, 128, 128], [128, 128, 128, 8]
    out, off = [], 0
    for l in range(4):
        out.append(v[off:off + K[l] * N[l]].reshape(K[l], N[l]))
        off += K[l] * N[l]
        out.append(v[off:off + N[l]])
        off += N[l]
    return out


def test_training_gradients_match_oracle(oracle):
    s, e, lp = small_engine()
    rng = np.random.default_rng(3)
    rows = 512
    x = rng.normal(size=(rows, 68)).astype(np.float32)
    t = rng.normal(size=(rows, 3)).astype(np.float32)
    state = lp.weights()
    params = state[: E.MLP_NPARAM].copy()
    # a trained-looking network: larger output layer than the initial 0.1 scale
    blocks = split_params(params)
    blocks[6][:, :3] = rng.normal(scale=0.1, size=(128, 3))
    blocks[7][:3] = rng.normal(scale=0.1, size=3)
    for b in (1, 3, 5):
        blocks[b][:] = rng.normal(scale=0.05, size=blocks[b].shape)
    state[: E.MLP_NPARAM] = params
    lp.set_weights(state)
    loss, g = lp.gradients(x, t)
    # the kernels see BF16 weights and inputs; the oracle gets the same values
    ref_loss, ref_g = oracle.mlp_grads(bf16(x), t, bf16(params))
    assert abs(loss - ref_loss) < 1e-2 * ref_loss, (loss, ref_loss)
    for k, (a, b) in enumerate(zip(split_params(g.astype(np.float64)), split_params(ref_g))):
        if k == 6:
            a, b = a[:, :3], b[:, :3]
        if k == 7:
            a, b = a[:3], b[:3]
        if k == 0:
            a, b = a[:68], b[:68]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < 3e-2, (k, rel)
    # unused outputs and padded inputs get no gradient
    gb = split_params(g)
    assert np.all(gb[6][:, 3:] == 0) and np.all(gb[7][3:] == 0)


def test_trained_network_beats_coarse_grid():
    s, e, lp = small_engine(frames=20)
    for _ in range(20):
        e.step(20)
        lp.collect()
    loss = lp.train(epochs=40, batch=4096, lr=1e-3, seed=1)
    assert np.isfinite(loss)
    e.step(40)   # a held-out state
    coarse, learned = lp.eval()
    assert coarse > 1e-3
    assert learned < 0.8 * coarse, (coarse, learned)


def test_learned_step_check_and_fallback():
    s, e, lp = small_engine(frames=4)
    for _ in range(4):
        e.step(10)
        lp.collect()
    lp.train(epochs=5, batch=4096)
    lp.enable(True, check_interval=10, tolerance=10.0)
    e.step(25)
    st = lp.status()
    assert st["active"] and not st["fell_back"] and 0.0 <= st["last_rel"] < 10.0
    en = e.energies()
    assert np.isfinite(en["total"]) and en["pme_recip"] != 0.0
    # an unreachable bound: the first check falls back to plain PME
    lp.enable(True, check_interval=10, tolerance=1e-12)
    e.step(12)
    st = lp.status()
    assert st["fell_back"] and not st["active"]
    assert e.status() & 0x20
    e.step(5)
    assert np.isfinite(e.energies()["total"])


def test_inference_kernels_match_oracle(oracle):
    """The tcgen05 (TMEM) inference kernel and the warp-level mma.sync one
    against the FP64 forward pass, on BF16-rounded inputs and weights; 3,000
    rows leave a partial last 128-row tile."""
    s, e, lp = small_engine(frames=1)
    e.step(5)
    lp.collect()
    rng = np.random.default_rng(7)
    state = lp.weights()
    params = state[: E.MLP_NPARAM].copy()
    blocks = split_params(params)
    blocks[6][:, :3] = rng.normal(scale=0.1, size=(128, 3))
    blocks[7][:3] = rng.normal(scale=0.1, size=3)
    for b in (1, 3, 5):
        blocks[b][:] = rng.normal(scale=0.05, size=blocks[b].shape)
    state[: E.MLP_NPARAM] = params
    lp.set_weights(state)
    mean = state[E.MLP_NPARAM:E.MLP_NPARAM + 68].astype(np.float32)
    std = state[E.MLP_NPARAM + 68:E.MLP_NPARAM + 136].astype(np.float32)
    feats = (mean + std * rng.normal(size=(3000, 68))).astype(np.float32)
    xn = (feats - mean) * (np.float32(1.0) / std)
    ref = oracle.mlp_forward(bf16(xn), bf16(params))
    y_tc = lp.predict(feats, impl=0).astype(np.float64)
    y_mma = lp.predict(feats, impl=1).astype(np.float64)
    scale = np.sqrt((ref ** 2).mean())
    assert np.sqrt(((y_mma - ref) ** 2).mean()) < 2e-2 * scale
    assert np.sqrt(((y_tc - ref) ** 2).mean()) < 2e-2 * scale
    assert np.sqrt(((y_tc - y_mma) ** 2).mean()) < 1e-2 * scale


def test_tensor_core_wait_timeout_is_reported_and_engine_recovers():
    """The tcgen05 inference kernel's waits on its MMA completion are bounded.
    In the self-test mode (impl 2) its first layer's MMAs are withheld, so the
    waits run out with nothing in flight: the call returns LIMA_ERR_TIMEOUT,
    the kernel has released its tensor memory, and the engine keeps working —
    the same rows predict as before and the engine steps on."""
    from lima_b200 import LimaError

    s, e, lp = small_engine(frames=2)
    e.step(5)
    lp.collect()
    lp.train(epochs=1, batch=1024, seed=1)
    rng = np.random.default_rng(3)
    feats = rng.normal(size=(100, 68)).astype(np.float32)   # one CTA's tile
    before = lp.predict(feats, impl=0)
    with pytest.raises(LimaError) as ex:
        lp.predict(feats, impl=2)
    assert ex.value.code == 5      # LIMA_ERR_TIMEOUT
    after = lp.predict(feats, impl=0)
    assert np.array_equal(before, after)
    e.step(10)
    assert np.isfinite(e.energies()["total"])
