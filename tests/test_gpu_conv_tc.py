"""tcgen05 3x3 convolutions (forward, backward-data through rotated weights,
backward-weights) against an FP64 NumPy evaluation of the same BF16 inputs."""
import ctypes as C

import numpy as np
import pytest

from nectarrender_b200 import capi, last_error

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def conv_ref(x, w, b=None):
    """x [B,H,W,ci] float64, w [9,co,ci] -> [B,H,W,co], zero padding 1."""
    B, H, W, ci = x.shape
    xp = np.zeros((B, H + 2, W + 2, ci))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((B, H, W, w.shape[1]))
    for t in range(9):
        dy, dx = t // 3, t % 3
        out += xp[:, dy:dy + H, dx:dx + W] @ w[t].T
    if b is not None:
        out += b
    return out


def wgrad_ref(dy, x):
    """dy [B,H,W,co], x [B,H,W,ci] -> dw [9,co,ci]"""
    B, H, W, ci = x.shape
    xp = np.zeros((B, H + 2, W + 2, ci))
    xp[:, 1:-1, 1:-1] = x
    co = dy.shape[-1]
    dw = np.zeros((9, co, ci))
    for t in range(9):
        ty, tx = t // 3, t % 3
        xs = xp[:, ty:ty + H, tx:tx + W].reshape(-1, ci)
        dw[t] = dy.reshape(-1, co).T @ xs
    return dw


def bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)


def ptr(t):
    return C.c_void_p(t.data_ptr())


# H % 16 == 0 and W % 8 == 0 take the halo-tile kernels (resident weights
# when a slice of at least 32 output channels fits with two halos, else
# streamed weights), the others the per-tap gather kernel
@pytest.mark.parametrize("B,H,W,ci,co,relu", [(2, 16, 24, 32, 48, 1), (1, 32, 32, 16, 32, 0),
                                              (1, 8, 48, 160, 96, 1), (1, 16, 16, 64, 256, 0),
                                              (2, 48, 40, 176, 80, 1), (1, 24, 20, 48, 64, 1),
                                              (4, 128, 128, 32, 32, 1),  # several tiles per CTA
                                              (4, 64, 64, 96, 96, 0)])   # two 48-channel slices
def test_forward(B, H, W, ci, co, relu):
    lib = capi.library()
    rng = np.random.default_rng(ci * 1000 + co)
    xs, xo, ys, yo = ci + 16, 8, co + 8, 8
    x = bf16(rng.standard_normal((B * H * W, xs))).cuda()
    w = bf16(rng.standard_normal((9, co, ci)) / np.sqrt(9 * ci)).cuda()
    b = torch.from_numpy(rng.standard_normal(co).astype(np.float32)).cuda()
    y = torch.full((B * H * W, ys), 7.0, dtype=torch.bfloat16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.nr_conv3x3_forward_device(ptr(x), xs, xo, ptr(w), C.cast(b.data_ptr(), C.POINTER(C.c_float)),
                                       ptr(y), ys, yo, ci, co, B, H, W, relu, C.c_uint64(s))
    assert rc == 0, last_error()
    torch.cuda.synchronize()
    xr = x.float().cpu().numpy().astype(np.float64)[:, xo:xo + ci].reshape(B, H, W, ci)
    ref = conv_ref(xr, w.float().cpu().numpy().astype(np.float64), b.cpu().numpy().astype(np.float64))
    if relu:
        ref = np.maximum(ref, 0)
    got = y.float().cpu().numpy()
    np.testing.assert_allclose(got[:, yo:yo + co].reshape(B, H, W, co), ref, rtol=1e-2, atol=2e-2)
    assert (got[:, :yo] == 7.0).all() and (got[:, yo + co:] == 7.0).all()  # untouched channels


def test_backward_data_via_rotated_weights():
    lib = capi.library()
    B, H, W, ci, co = 2, 16, 16, 32, 64
    rng = np.random.default_rng(5)
    w = rng.standard_normal((9, co, ci)) / np.sqrt(9 * ci)
    dy = rng.standard_normal((B * H * W, co))
    w_bd = np.stack([w[8 - t].T for t in range(9)])  # [9][ci][co]
    dyt, wt = bf16(dy).cuda(), bf16(w_bd).cuda()
    dx = torch.zeros((B * H * W, ci), dtype=torch.bfloat16, device="cuda")
    rc = lib.nr_conv3x3_forward_device(ptr(dyt), co, 0, ptr(wt), None, ptr(dx), ci, 0, co, ci,
                                       B, H, W, 0, C.c_uint64(0))
    assert rc == 0, last_error()
    torch.cuda.synchronize()
    # FP64 gradient of sum(g * conv(x, w)) w.r.t. x equals the correlation
    # of g with the rotated kernel
    g = dyt.float().cpu().numpy().astype(np.float64).reshape(B, H, W, co)
    wr = wt.float().cpu().numpy().astype(np.float64)
    ref = conv_ref(g, wr)
    np.testing.assert_allclose(dx.float().cpu().numpy().reshape(B, H, W, ci), ref, rtol=1e-2, atol=2e-2)
    # and that is the true adjoint: <conv(x, w), g> == <x, ref> for a random x
    x = rng.standard_normal((B, H, W, ci))
    wf = np.stack([wr[8 - t].T for t in range(9)])
    lhs = float((conv_ref(x, wf) * g).sum())
    rhs = float((x * ref).sum())
    assert abs(lhs - rhs) <= 1e-9 * max(1.0, abs(lhs))


@pytest.mark.parametrize("B,H,W,ci,co", [
    (2, 16, 24, 32, 48), (1, 64, 64, 128, 128), (1, 16, 16, 160, 16),  # halo tiles (H % 16, W % 8)
    (2, 32, 16, 96, 96),                                                # two tap groups of 5 and 4
    (1, 12, 20, 32, 16),                                                # per-tap gathers
])
def test_weight_gradient(B, H, W, ci, co):
    lib = capi.library()
    rng = np.random.default_rng(ci + co)
    dy = bf16(rng.standard_normal((B * H * W, co))).cuda()
    x = bf16(rng.standard_normal((B * H * W, ci))).cuda()
    dw = torch.zeros((9, co, ci), dtype=torch.float32, device="cuda")
    rc = lib.nr_conv3x3_wgrad_device(ptr(dy), co, 0, ptr(x), ci, 0,
                                     C.cast(dw.data_ptr(), C.POINTER(C.c_float)), ci, co, B, H, W,
                                     C.c_uint64(0))
    assert rc == 0, last_error()
    torch.cuda.synchronize()
    ref = wgrad_ref(dy.float().cpu().numpy().astype(np.float64).reshape(B, H, W, co),
                    x.float().cpu().numpy().astype(np.float64).reshape(B, H, W, ci))
    scale = np.sqrt(B * H * W)
    np.testing.assert_allclose(dw.cpu().numpy(), ref, rtol=1e-4, atol=1e-4 * scale)


def test_rejects_bad_channel_counts():
    lib = capi.library()
    x = torch.zeros(128 * 24, dtype=torch.bfloat16, device="cuda")
    rc = lib.nr_conv3x3_forward_device(ptr(x), 24, 0, ptr(x), None, ptr(x), 24, 0, 24, 16, 1, 8, 16,
                                       0, C.c_uint64(0))
    assert rc == -1 and "multiples of 16" in last_error()
