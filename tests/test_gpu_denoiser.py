"""The U-Net denoiser: every layer's gradient against an FP64 NumPy
evaluation of the same network on the same BF16-rounded weights, training
lowers the loss, and the denoised image is closer to the converged one."""
import numpy as np
import pytest

from nectarrender_b200 import capi, denoise, scenes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ENC = [32, 48, 64, 96, 128]


def bf(a):
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def conv(x, w, b):
    """x [H,W,ci], w [9,co,ci] -> [H,W,co]"""
    H, W, ci = x.shape
    xp = np.zeros((H + 2, W + 2, ci))
    xp[1:-1, 1:-1] = x
    out = np.zeros((H, W, w.shape[1])) + b
    for t in range(9):
        out += xp[t // 3:t // 3 + H, t % 3:t % 3 + W] @ w[t].T
    return out


def conv_bwd(g, x, w):
    """grads of sum(g * conv(x, w, b)) w.r.t. w, b, x"""
    H, W, ci = x.shape
    xp = np.zeros((H + 2, W + 2, ci))
    xp[1:-1, 1:-1] = x
    dw = np.stack([g.reshape(-1, g.shape[-1]).T @ xp[t // 3:t // 3 + H, t % 3:t % 3 + W].reshape(-1, ci)
                   for t in range(9)])
    wr = np.stack([w[8 - t].T for t in range(9)])
    return dw, g.sum((0, 1)), conv(g, wr, 0.0)


def pool(x):
    return 0.25 * (x[0::2, 0::2] + x[1::2, 0::2] + x[0::2, 1::2] + x[1::2, 1::2])


def pool_bwd(g):
    return 0.25 * np.repeat(np.repeat(g, 2, 0), 2, 1)


def up(x):
    return np.repeat(np.repeat(x, 2, 0), 2, 1)


def up_bwd(g):
    return g[0::2, 0::2] + g[1::2, 0::2] + g[0::2, 1::2] + g[1::2, 1::2]


def unet_grads(params, x0, target, base, kind=1):
    """FP64 forward + backward of the network in denoiser.cuh (prediction =
    base + the first three output channels; loss kind 1 = mean |d|, 0 =
    mean 0.5 d^2); returns the loss and [(dw, db)] in parameter order."""
    P = [(w.astype(np.float64), b.astype(np.float64)) for w, b in params]
    acts = {}
    relu = lambda a: np.maximum(a, 0)
    x = x0
    skips = []
    i = 0
    for l in range(5):
        a = relu(conv(x, *P[i])); acts[i] = (x, a); i += 1
        b = relu(conv(a, *P[i])); acts[i] = (a, b); i += 1
        skips.append(b)
        x = pool(b) if l < 4 else b
    below = x
    for l in range(3, -1, -1):
        cat = np.concatenate([up(below), skips[l]], -1)
        a = relu(conv(cat, *P[i])); acts[i] = (cat, a); i += 1
        b = relu(conv(a, *P[i])); acts[i] = (a, b); i += 1
        below = b
    out = conv(below, *P[i]); acts[i] = (below, out)
    d = (base + out[..., :3]) - target
    loss = np.abs(d).mean() if kind == 1 else (0.5 * d * d).mean()
    g_out = np.zeros_like(out)
    g_out[..., :3] = np.sign(d) if kind == 1 else d
    grads = [None] * len(P)
    dskip = {}
    dw, db, dx = conv_bwd(g_out, acts[i][0], P[i][0]); grads[i] = (dw, db)
    for l in range(4):
        for j in (1, 0):
            li = 10 + 2 * (3 - l) + j
            xin, y = acts[li]
            g = dx * (y > 0)
            dw, db, dx = conv_bwd(g, xin, P[li][0]); grads[li] = (dw, db)
        c_up = ENC[l + 1]
        dskip[l] = dx[..., c_up:]
        dx = up_bwd(dx[..., :c_up])
    for l in range(4, -1, -1):
        if l < 4:
            dx = pool_bwd(dx) + dskip[l]
        for j in (1, 0):
            li = 2 * l + j
            xin, y = acts[li]
            g = dx * (y > 0)
            dw, db, dx = conv_bwd(g, xin, P[li][0]); grads[li] = (dw, db)
    return loss, grads


@pytest.mark.parametrize("kind", [denoise.LOSS_ABSOLUTE, denoise.LOSS_SQUARED])
def test_gradients_match_fp64_network(kind):
    den = denoise.Denoiser(max_pixels=32 * 32, seed=3)
    den.set_loss(kind)
    params = den.params()
    # the GPU computes with BF16 weights: give the FP64 model the same values
    params64 = [(bf(w), b.astype(np.float64)) for w, b in params]
    rng = np.random.default_rng(0)
    beauty = rng.gamma(1.0, 0.5, (1, 3, 32, 32)).astype(np.float32)
    diffuse = rng.uniform(0, 1, (1, 3, 32, 32)).astype(np.float32)
    normal = rng.uniform(-1, 1, (1, 3, 32, 32)).astype(np.float32)
    depth = rng.uniform(0.5, 8.0, (1, 1, 32, 32)).astype(np.float32)
    target = rng.gamma(1.0, 0.5, (1, 3, 32, 32)).astype(np.float32)
    t = lambda a: torch.from_numpy(a).cuda()
    loss_gpu = den.train_step(t(beauty), t(diffuse), t(normal), t(target), lr=0.0, depth=t(depth))
    grads = den.grads()
    x0 = np.zeros((32, 32, 16))
    x0[..., 0:3] = np.log1p(beauty[0].transpose(1, 2, 0))
    x0[..., 3:6] = diffuse[0].transpose(1, 2, 0)
    x0[..., 6:9] = normal[0].transpose(1, 2, 0)
    x0[..., 9] = np.log1p(depth[0, 0])
    loss_ref, ref = unet_grads(params64, bf(x0), np.log1p(target[0].transpose(1, 2, 0).astype(np.float64)),
                               np.log1p(beauty[0].transpose(1, 2, 0).astype(np.float64)), kind)
    assert abs(loss_gpu - loss_ref) <= 0.02 * loss_ref
    for k, ((gw, gb), (rw, rb)) in enumerate(zip(grads, ref)):
        rw = rw.astype(np.float64)
        cos = float((gw.ravel() @ rw.ravel()) / (np.linalg.norm(gw) * np.linalg.norm(rw) + 1e-30))
        rel = float(np.linalg.norm(gw - rw) / (np.linalg.norm(rw) + 1e-30))
        assert cos >= 0.98 and rel <= 0.2, (k, cos, rel)
        cb = float((gb @ rb) / (np.linalg.norm(gb) * np.linalg.norm(rb) + 1e-30))
        assert cb >= 0.98, (k, cb)


def test_training_reduces_loss_and_error():
    spec = scenes.mesh_stress(levels=5, res_h=128, res_w=128, spp=257, depth=8, n_spheres=24,
                              hdri_size=(256, 128), scene_seed=4)
    sc = capi.Scene(spec)
    noisy = capi.Render(sc, mode=capi.MODE_PERF, layer_mask=denoise.DENOISE_LAYERS)
    noisy.samples(1, 4)
    ref = capi.Render(sc, mode=capi.MODE_PERF, seed=99)
    ref.samples(1, 256)
    inp = denoise.render_layers(noisy)
    assert inp[3] is not None and float(inp[3].max()) > 0   # the depth layer is rendered
    target = denoise.render_layers(ref)[0]
    den = denoise.Denoiser(max_pixels=4 * 64 * 64, seed=1)
    crop = lambda a: a[:, :, :64, :64].contiguous()
    b, d, n, z = (crop(a) for a in inp)
    first = den.train_step(b, d, n, crop(target), lr=0.0, depth=z)
    steps, secs, last = denoise.train(den, [(inp, target)], steps=300, crop=64, batch=4)
    assert np.isfinite(last) and last < 0.7 * first
    out = den.infer(b, d, n, depth=z)
    assert torch.isfinite(out).all()
