"""The corrector's tcgen05 convolution kernels against the CPU oracle
(oracle/conv_oracle.py) on the same BF16-rounded inputs: forward with and
without GELU (output BF16: relative 1e-2 of the largest value), the input
gradient through the flipped weights, the weight and bias gradients (FP32
accumulation: relative 1e-3), zero halos, and the bounded-wait error word."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from multicellular_phase_field_active_gel_organoids_b200 import capi  # noqa: E402
from oracle import conv_oracle as co  # noqa: E402

pytestmark = pytest.mark.gpu


def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def P(t):
    return ctypes.c_void_p(t.data_ptr())


def run_fwd(x, w, b, gelu_on, B, H, W, cin, cout):
    L = capi.lib()
    xd = dev(x, torch.float32).to(torch.bfloat16)
    wd = dev(w, torch.float32).to(torch.bfloat16)
    bd = dev(b, torch.float32)
    y = torch.zeros((B, H + 2, W + 2, cout), dtype=torch.bfloat16, device="cuda")
    pre = torch.zeros_like(y)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    capi.check(L.pfag_conv3x3(P(xd), P(wd), P(bd), P(y), P(pre), B, H, W, cin, cout, int(gelu_on), P(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return y.float().cpu().numpy(), pre.float().cpu().numpy()


@pytest.mark.parametrize("B,H,W,cin,cout,gelu_on", [(2, 12, 20, 16, 32, True), (1, 128, 128, 32, 32, True),
                                                  (3, 7, 9, 32, 16, False), (2, 33, 70, 16, 16, True),
                                                  (16, 128, 128, 32, 32, True)])
def test_forward_matches_oracle(B, H, W, cin, cout, gelu_on):
    rng = np.random.default_rng(B * 1000 + H)
    x = co.pad(co.bf16(rng.normal(size=(B, H, W, cin))))
    w = co.bf16(rng.normal(size=(cout, 9, cin)) / np.sqrt(9 * cin))
    b = rng.normal(size=cout).astype(np.float32).astype(np.float64)
    y, pre = run_fwd(x, w, b, gelu_on, B, H, W, cin, cout)
    z = co.conv_fwd(x, w, b)
    ref = co.gelu(z) if gelu_on else z
    scale = np.abs(ref).max()
    assert np.max(np.abs(y[:, 1:-1, 1:-1, :] - ref)) <= 1e-2 * scale
    assert np.max(np.abs(pre[:, 1:-1, 1:-1, :] - z)) <= 1e-2 * np.abs(z).max()
    for halo in (y[:, 0], y[:, -1], y[:, :, 0], y[:, :, -1]):
        assert not np.any(halo)


def test_input_gradient_through_flipped_weights():
    B, H, W, cin, cout = 2, 10, 15, 16, 32
    rng = np.random.default_rng(7)
    w = co.bf16(rng.normal(size=(cout, 9, cin)) / 12.0)
    dz = co.bf16(rng.normal(size=(B, H, W, cout)))
    L = capi.lib()
    wd = dev(w, torch.float32).to(torch.bfloat16)
    wt = torch.zeros((cin, 9, cout), dtype=torch.bfloat16, device="cuda")
    capi.check(L.pfag_conv_flip(P(wd), P(wt), cin, cout, None))
    torch.cuda.synchronize()
    assert np.array_equal(wt.float().cpu().numpy(), np.transpose(w[:, ::-1, :], (2, 1, 0)))
    dx, _ = run_fwd(co.pad(dz), wt.float().cpu().numpy(), np.zeros(cin), False, B, H, W, cout, cin)
    ref = co.conv_dgrad(dz, w)
    assert np.max(np.abs(dx[:, 1:-1, 1:-1, :] - ref)) <= 1e-2 * np.abs(ref).max()


@pytest.mark.parametrize("B,H,W,cin,cout", [(2, 9, 13, 16, 32), (1, 128, 128, 32, 32), (3, 20, 31, 32, 16),
                                            (16, 128, 128, 32, 32)])
def test_weight_gradient_matches_oracle(B, H, W, cin, cout):
    rng = np.random.default_rng(H * 31 + W)
    x = co.pad(co.bf16(rng.normal(size=(B, H, W, cin))))
    dz = co.bf16(rng.normal(size=(B, H, W, cout)))
    L = capi.lib()
    xd = dev(x, torch.float32).to(torch.bfloat16)
    dzd = dev(co.pad(dz), torch.float32).to(torch.bfloat16)
    dw = torch.zeros((cout, 9, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    capi.check(L.pfag_conv3x3_wgrad(P(xd), P(dzd), P(dw), P(db), B, H, W, cin, cout, P(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rdw, rdb = co.conv_wgrad(x, dz)
    assert np.max(np.abs(dw.cpu().numpy() - rdw)) <= 1e-3 * np.abs(rdw).max()
    assert np.max(np.abs(db.cpu().numpy() - rdb)) <= 1e-3 * np.abs(rdb).max()


def test_activation_gradient_and_loss():
    B, H, W, C = 2, 6, 7, 16
    rng = np.random.default_rng(11)
    pre = co.pad(co.bf16(rng.normal(size=(B, H, W, C))))
    dy = co.pad(co.bf16(rng.normal(size=(B, H, W, C))))
    L = capi.lib()
    pd, dyd = (dev(a, torch.float32).to(torch.bfloat16) for a in (pre, dy))
    dz = torch.ones_like(pd)
    capi.check(L.pfag_conv_act_bwd(P(dyd), P(pd), P(dz), B, H, W, C, 1, None))
    torch.cuda.synchronize()
    ref = dy * co.gelu_grad(pre)
    assert np.max(np.abs(dz.float().cpu().numpy() - ref)) <= 1e-2 * np.abs(ref).max()
    out = co.pad(co.bf16(rng.normal(size=(B, H, W, C))))
    tgt = rng.normal(size=(B, H, W, 2)).astype(np.float32)
    od, td = dev(out, torch.float32).to(torch.bfloat16), dev(tgt, torch.float32)
    dout = torch.ones_like(od)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    capi.check(L.pfag_conv_mse(P(od), P(td), P(dout), P(loss), B, H, W, C, 2, 0.5, None))
    torch.cuda.synchronize()
    d = out[:, 1:-1, 1:-1, :2] - tgt
    assert abs(float(loss.item()) - float((d * d).sum())) <= 1e-4 * float((d * d).sum())
    g = dout.float().cpu().numpy()
    assert np.max(np.abs(g[:, 1:-1, 1:-1, :2] - d)) <= 1e-2 * np.abs(d).max()
    assert not np.any(g[:, 1:-1, 1:-1, 2:]) and not np.any(g[:, 0])
