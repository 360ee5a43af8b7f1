"""The neural radiance cache: its encoding, loss and every gradient (MLP
weights and hash-grid entries) against an FP64 NumPy evaluation on the same
BF16-rounded values; online training lowers the loss."""
import numpy as np
import pytest

from nectarrender_b200 import nrc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

T = 1 << nrc.LOG2T


def bf(a):
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def geometry():
    b = np.exp((np.log(2048.0) - np.log(16.0)) / 15)
    scale = [float(np.floor(np.float32(16.0 * b ** l))) for l in range(16)]
    dense = [(s + 2.0) ** 3 <= T for s in scale]
    return scale, dense


def index(l, x, y, z, scale, dense):
    x, y, z = (np.asarray(v, np.uint64) for v in (x, y, z))
    if dense[l]:
        r = np.uint64(int(scale[l]) + 2)
        return ((x + r * (y + r * z)) & np.uint64(T - 1)).astype(np.int64)
    h = (x * np.uint64(1)) ^ ((y * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) ^ \
        ((z * np.uint64(805459861)) & np.uint64(0xFFFFFFFF))
    return (h & np.uint64(T - 1)).astype(np.int64)


def corners(u, l, scale, dense):
    pos = u.astype(np.float32) * np.float32(scale[l]) + np.float32(0.5)
    fl = np.floor(pos)
    fr = (pos - fl).astype(np.float64)
    base = fl.astype(np.int64)
    for c in range(8):
        hi = [(c >> k) & 1 for k in range(3)]
        w = np.prod([fr[:, k] if hi[k] else 1 - fr[:, k] for k in range(3)], axis=0)
        yield index(l, base[:, 0] + hi[0], base[:, 1] + hi[1], base[:, 2] + hi[2], scale, dense), w


def test_encoding_and_gradients_match_fp64():
    rng = np.random.default_rng(0)
    n = 2048
    cache = nrc.RadianceCache(n, (0, 0, 0), (1, 1, 1), seed=2)
    q = np.zeros((n, 16), np.float32)
    q[:, 0:3] = rng.uniform(0, 1, (n, 3))
    q[:, 3] = rng.uniform(0, 1, n)
    d = rng.standard_normal((n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 4:7] = d
    nn = rng.standard_normal((n, 3)); nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    q[:, 8:11] = nn
    q[:, 12:15] = rng.uniform(0, 1, (n, 3))
    target = rng.gamma(1.0, 1.0, (n, 3)).astype(np.float32)
    tq, tt = torch.from_numpy(q).cuda(), torch.from_numpy(target).cuda()
    loss_gpu = cache.train(tq, tt, lr=0.0)
    x0 = cache.get(4).reshape(n, 64).astype(np.float64)
    grid = cache.get(2).reshape(16, T, 2).astype(np.float64)
    # encoding: hash-grid features by trilinear interpolation
    scale, dense = geometry()
    feats = np.zeros((n, 32))
    for l in range(16):
        for idx, w in corners(q[:, 0:3], l, scale, dense):
            feats[:, 2 * l:2 * l + 2] += w[:, None] * grid[l, idx]
    np.testing.assert_allclose(x0[:, :32], bf(feats), rtol=1e-2, atol=1e-6)
    assert np.allclose(x0[:, 48:51], bf(nn * 0.5 + 0.5), atol=1e-2)
    assert (x0[:, 55:] == 0).all()
    # MLP forward and backward in FP64 on the BF16 weights
    W = [bf(w) for w in cache.mlp_layers(cache.get(0))]
    hidden = len(nrc.LAYERS) - 1
    h = [x0]
    for l in range(hidden):
        h.append(bf(np.maximum(h[-1] @ W[l].T, 0)))
    o = bf(h[-1] @ W[hidden].T)
    oc = o[:, :3]
    den = oc * oc + 0.01
    loss_ref = ((oc - target) ** 2 / den).mean()
    assert abs(loss_gpu - loss_ref) <= 0.02 * loss_ref
    g = np.zeros_like(o)
    g[:, :3] = 2 * (oc - target) / den
    g = bf(g)
    grads = [None] * (hidden + 1)
    grads[hidden] = g.T @ h[hidden]
    dh = g @ W[hidden]
    for l in reversed(range(hidden)):
        dz = dh * (h[l + 1] > 0)
        grads[l] = dz.T @ h[l]
        dh = dz @ W[l]
    got = cache.mlp_layers(cache.get(1))
    for l in range(hidden + 1):
        a, b = got[l].ravel().astype(np.float64), grads[l].ravel()
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert cos >= 0.98 and rel <= 0.2, (l, cos, rel)
    # hash-grid gradient: scatter of d(loss)/d(features)
    gg = np.zeros((16, T, 2))
    for l in range(16):
        for idx, w in corners(q[:, 0:3], l, scale, dense):
            np.add.at(gg[l], idx, w[:, None] * dh[:, 2 * l:2 * l + 2])
    got = cache.get(3).reshape(16, T, 2).astype(np.float64)
    a, b = got.ravel(), gg.ravel()
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    assert cos >= 0.98, cos


def test_online_training_fits_a_radiance_field():
    rng = np.random.default_rng(1)
    n = 1 << 16
    cache = nrc.RadianceCache(n, (-1, -1, -1), (1, 1, 1), seed=0)
    def batch():
        q = np.zeros((n, 16), np.float32)
        p = rng.uniform(-1, 1, (n, 3))
        q[:, 0:3] = p
        q[:, 3] = 0.5
        d = rng.standard_normal((n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
        q[:, 4:7] = d
        q[:, 8:11] = d
        q[:, 12:15] = 0.5
        t = np.stack([1 + np.sin(3 * p[:, 0]) * d[:, 1], 1 + 0.5 * p[:, 1], 2 + np.cos(2 * p[:, 2])], 1)
        return torch.from_numpy(q).cuda(), torch.from_numpy(t.astype(np.float32)).cuda()
    q, t = batch()
    first = cache.train(q, t, lr=0.0)
    for _ in range(300):
        q, t = batch()
        cache.train(q, t, lr=5e-3, want_loss=False)
    q, t = batch()
    last = cache.train(q, t, lr=0.0)
    assert last < 0.1 * first
    out = cache.infer(q)
    err = (out - t).abs().mean().item()
    assert err < 0.2
