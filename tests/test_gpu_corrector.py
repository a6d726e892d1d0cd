"""The learned coarse-grid corrector on the GPU: the network's gradients
(all five layers, through the tcgen05 kernels) against the CPU oracle on the
same BF16 roundings; training on coarse/fine pairs of the plain method and
what the trained network gains on held-out organoids; the fine-grid
fallback.  Small organoids (256^2 fine, 128^2 coarse) keep it to a minute."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from multicellular_phase_field_active_gel_organoids_b200 import corrector as C  # noqa: E402
from oracle import conv_oracle as co  # noqa: E402

pytestmark = pytest.mark.gpu


def test_network_gradients_match_oracle():
    """One training step's weight gradients of every layer against a float64
    restatement of the network that rounds to BF16 where the kernels store
    BF16 (activations, pre-activations, gradients between layers)."""
    B, H, W = 2, 8, 11
    net = C.ConvNet(seed=1)
    rng = np.random.default_rng(5)
    x = np.zeros((B, H + 2, W + 2, 16))
    x[:, 1:-1, 1:-1, :4] = co.bf16(rng.normal(size=(B, H, W, 4)))
    tgt = rng.normal(size=(B, H, W, 2)).astype(np.float32)
    Ws = [co.bf16(w.cpu().numpy()) for w in net.W]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.b]
    xd = torch.as_tensor(x, dtype=torch.float32, device="cuda").to(torch.bfloat16)
    td = torch.as_tensor(tgt, device="cuda")
    # gradients: a step with lr = 0 leaves the weights; capture them through Adam's first moment
    net.train_step(xd, td, B, H, W, lr=0.0)
    torch.cuda.synchronize()
    net.check_err()
    gW = [m.cpu().numpy() / 0.1 for m in net.mW]          # m = (1 - b1) g after one step
    # host restatement
    acts, pres = [x], []
    a = x
    for k, (cin, cout, act) in enumerate(C.LAYERS):
        z = co.conv_fwd(a, Ws[k], bs[k])
        pres.append(co.pad(co.bf16(z)))
        y = co.bf16(co.gelu(z) if act else z)
        a = co.pad(y)
        acts.append(a)
    out = acts[-1][:, 1:-1, 1:-1, :2]
    n = B * H * W * 2
    dz = np.zeros((B, H, W, 16))
    dz[..., :2] = co.bf16(2.0 * (out - tgt) / n)
    for k in range(len(C.LAYERS) - 1, -1, -1):
        dw, _ = co.conv_wgrad(acts[k], dz)
        err = np.abs(gW[k] - dw).max() / max(np.abs(dw).max(), 1e-30)
        assert err <= 3e-2, (k, err)
        if k == 0:
            break
        da = co.bf16(co.conv_dgrad(dz, Ws[k]))
        dz = co.bf16(da * co.gelu_grad(pres[k - 1][:, 1:-1, 1:-1, :]))


@pytest.fixture(scope="module")
def trained():
    feats, targs = C.make_pairs(range(6), ncells_range=(5, 8), checkpoints=3, N=256, zone_size=65, warm=20)
    sc = C.fit_scales(feats, targs)
    X, T = C.scaled(feats, targs, sc)
    net = C.ConvNet(seed=0)
    hist = C.train(net, X, T, iters=300, batch=16, lr=2e-3)
    return net, sc, hist


def test_training_reduces_loss(trained):
    net, sc, hist = trained
    assert all(math.isfinite(h) for h in hist)
    assert hist[-1] < 0.8 * hist[0], hist


def test_trained_network_gains_on_held_out_organoids(trained):
    """On organoids the network never saw, the corrected coarse interval is
    closer to the restricted fine one than the uncorrected coarse interval:
    the network's correction removes part of the coarse method's error."""
    net, sc, _ = trained
    feats, targs = C.make_pairs([100, 101], ncells_range=(5, 8), checkpoints=2, N=256, zone_size=65, warm=20)
    X, T = C.scaled(feats, targs, sc)
    pred = C.predict(net, X)
    mse_none = float((T ** 2).mean().item())
    mse_net = float(((pred - T) ** 2).mean().item())
    print("held-out scaled mse: uncorrected", mse_none, "corrected", mse_net)
    assert mse_net < 0.9 * mse_none


def test_corrected_run_and_fallback(trained):
    net, sc, _ = trained
    fcfg = C.fine_config(6, 200, N=256, zone_size=65)
    import multicellular_phase_field_active_gel_organoids_b200.capi as capi
    with capi.Simulation(fcfg.params(), 32, capi.PATH_FUSED) as fs:
        fs.set_relax_cap(100000)
        fs.upload(*fcfg.initial_state(np.float32))
        fs.step(0, 20)
        F0 = C.state_tensors(fs)
        fs.step(20, 4 * 10 * 3)
        ref = C.restrict(C.state_tensors(fs)[0])
    errs = {}
    for name, corrected in (("uncorrected", False), ("corrected", True)):
        run = C.CorrectedRun(net, sc, fcfg)
        try:
            run.start_from_fine(F0)
            run.run(3, corrected=corrected)
            errs[name] = C.shape_errors(run.state_on_coarse()[0], ref)
        finally:
            run.close()
    print("area / perimeter errors after 3 intervals:", errs)
    assert all(math.isfinite(v) for e in errs.values() for v in e)
    # an error budget of zero makes the first fine-grid check fall back to the fine method
    run = C.CorrectedRun(net, sc, fcfg, check_every=1, budget=0.0)
    try:
        run.start_from_fine(F0)
        run.run(2)
        assert run.on_fine and run.fallbacks == 1
        assert math.isfinite(run.last_check)
    finally:
        run.close()
    run = C.CorrectedRun(net, sc, fcfg, check_every=1, budget=10.0)
    try:
        run.start_from_fine(F0)
        run.run(2)
        assert not run.on_fine and run.corrections == 2
    finally:
        run.close()
