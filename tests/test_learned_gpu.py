"""GPU tests of the learned repose proposal's tensor-core kernels.

The CPU oracle (oracle/learned.py, float64) is the checker:
* forward convolutions (the nine-tap kernel and the rotating-accumulator
  kernel, SOILB200_CONV_ROT=1): f32 outputs within 1e-4 of the largest |value|
  (FP32 accumulation of exact BF16 products), BF16 outputs within BF16 rounding;
* the one-kernel inference of the whole network equals the four layer
  launches bit for bit, and the float64 oracle network within 2e-2 of the
  largest |value| (BF16 activations between layers);
* weight gradients within 1e-4 (relative to the largest |value|);
* full back-propagation of the training loss: the GPU keeps activations in
  BF16, so each layer's gradient is compared by relative L2 error <= 5e-2;
* the fixed-point flux application conserves sum(b_eff) in exact quanta, and
  proposal + plain sweep reaches the repose tolerance.
"""

import numpy as np
import pytest

import soilb200
from oracle import learned as L

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def bf16(a):
    f = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    r = (f + np.uint32(0x7FFF) + ((f >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32).astype(np.float64)


def to_dev(a, dtype):
    return torch.as_tensor(np.asarray(a, dtype=np.float32), device="cuda").to(dtype).contiguous()


def _learned():
    from soilb200 import learned
    return learned


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16), (16, 16)])
@pytest.mark.parametrize("relu", [False, True])
@pytest.mark.parametrize("rot", ["0", "1"])  # nine-tap / rotating-accumulator kernel
def test_conv_matches_oracle(cin, cout, relu, rot, monkeypatch):
    monkeypatch.setenv("SOILB200_CONV_ROT", rot)
    ln = _learned()
    rng = np.random.default_rng(cin * 100 + cout + relu)
    x = bf16(rng.normal(size=(2, 19, 300, cin)))
    w = bf16(rng.normal(scale=0.2, size=(3, 3, cin, cout)))
    ref = L.conv3x3(x, w)
    if relu:
        ref = np.maximum(ref, 0.0)
    idx = torch.as_tensor(ln.pack_index(cin, cout), device="cuda")
    wpk = to_dev(w, torch.float32).reshape(-1)[idx].to(torch.bfloat16)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = ln.conv(to_dev(x, torch.bfloat16), wpk, cin, cout, relu=relu, out_f32=True,
                  status=status)
    got = out.cpu().numpy().astype(np.float64)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-4 * scale + 1e-6
    out16 = ln.conv(to_dev(x, torch.bfloat16), wpk, cin, cout, relu=relu, status=status)
    got16 = out16.float().cpu().numpy().astype(np.float64)
    assert np.abs(got16 - ref).max() <= 8e-3 * scale + 1e-6
    assert int(status.item()) == 0


@pytest.mark.parametrize("rot", ["0", "1"])
def test_conv_mask_and_rows(rot, monkeypatch):
    monkeypatch.setenv("SOILB200_CONV_ROT", rot)
    ln = _learned()
    rng = np.random.default_rng(3)
    x = bf16(rng.normal(size=(1, 40, 130, 32)))
    w = bf16(rng.normal(scale=0.2, size=(3, 3, 32, 32)))
    m = bf16(rng.normal(size=(1, 40, 130, 32)))
    ref = L.conv3x3(x, w) * (m > 0)
    idx = torch.as_tensor(ln.pack_index(32, 32), device="cuda")
    wpk = to_dev(w, torch.float32).reshape(-1)[idx].to(torch.bfloat16)
    for rows in (1, 7, 64):
        out = ln.conv(to_dev(x, torch.bfloat16), wpk, 32, 32, relu=False, out_f32=True,
                      mask=to_dev(m, torch.bfloat16), rows=rows)
        got = out.cpu().numpy().astype(np.float64)
        assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max() + 1e-6, rows


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
def test_wgrad_matches_oracle(cin, cout):
    ln = _learned()
    rng = np.random.default_rng(cin + 7 * cout)
    x = bf16(rng.normal(size=(2, 33, 200, cin)))
    g = bf16(rng.normal(size=(2, 33, 200, cout)))
    ref = L.conv3x3_wgrad(x, g)
    for rows in (16, 5):
        dw = ln.wgrad(to_dev(x, torch.bfloat16), to_dev(g, torch.bfloat16), cin, cout, rows=rows)
        got = dw.cpu().numpy().astype(np.float64)
        assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max(), rows


def test_features_match_oracle():
    ln = _learned()
    rng = np.random.default_rng(5)
    h = rng.normal(scale=0.05, size=(2, 21, 37)).cumsum(axis=2)
    tan = np.tan(np.deg2rad(35.0))
    ref = L.features(h, 0.05, 0.05, tan)
    feat = ln.features_f64(torch.as_tensor(h, device="cuda"), 0.05, 0.05, tan)
    got = feat.float().cpu().numpy().astype(np.float64)
    assert np.abs(got[..., :4] - ref).max() <= 4e-3 * np.abs(ref).max()
    assert np.all(got[..., 4:] == 0.0)


def test_backprop_matches_oracle_gradients():
    ln = _learned()
    net = ln.ReposeNet(seed=3)
    rng = np.random.default_rng(11)
    tan = np.tan(np.deg2rad(35.0))
    pre = rng.normal(scale=0.03, size=(2, 24, 150)).cumsum(axis=1)
    tgt = rng.normal(scale=0.002, size=(2, 24, 150))
    feat = ln.features_f64(torch.as_tensor(pre, device="cuda"), 0.05, 0.05, tan)
    scale = tan * 0.05
    norm = 1.0 / (scale * scale * pre.size)
    loss, grads, flux = ln.loss_and_grads(net, feat, torch.as_tensor(tgt, device="cuda").float(),
                                          0.05, 0.05, tan, norm)
    # oracle on the same BF16 inputs and BF16-rounded weights
    x = feat.float().cpu().numpy().astype(np.float64)
    ws = [bf16(w) for w in net.numpy_weights()]
    tgt32 = tgt.astype(np.float32).astype(np.float64)
    ref_loss, ref_grads, _ = L.loss_and_grads(x, ws, tgt32, scale, norm)
    assert loss == pytest.approx(ref_loss, rel=2e-2)
    for li, (g, r) in enumerate(zip(grads, ref_grads)):
        g = g.cpu().numpy().astype(np.float64)
        err = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30)
        assert err <= 5e-2, (li, err)
    assert int(net.status.item()) == 0


def test_training_reduces_loss():
    ln = _learned()
    from soilb200 import workloads
    pre = np.stack([workloads.config3_patch(i, n=64) for i in range(8)])
    post = np.stack([soilb200.relax_critical_slope(p, (0.05, 0.05), 35.0, tolerance=1e-6)[0]
                     for p in pre])
    net = ln.ReposeNet(seed=0)
    st = ln.train(net, pre, post, dx=0.05, dy=0.05, critical_angle_deg=35.0, steps=60, batch=4,
                  lr=3e-3)
    assert np.isfinite(st.first_loss) and np.isfinite(st.last_loss)
    assert st.last_loss < st.first_loss


def test_fixed_point_proposal_conserves_volume_and_relaxes():
    ln = _learned()
    from soilb200 import workloads
    b = workloads.config3_patch(4, n=96)
    k, datum = soilb200.choose_quantization(b)
    grid = soilb200.DeviceGrid(b.shape, 0.05, 0.05, precision="fx32", height_exponent=k,
                               datum_m=datum)
    grid.upload("b_eff", b)
    grid.upload("z_base", np.zeros_like(b))
    q = 2.0 ** k
    sum0 = int(np.rint((grid.download("b_eff") - datum) * q).astype(np.int64).sum())
    net = ln.ReposeNet(seed=1)
    relax = ln.LearnedRelaxation(grid, net, 35.0)
    relax.propose(rounds=2)
    sum1 = int(np.rint((grid.download("b_eff") - datum) * q).astype(np.int64).sum())
    assert sum1 == sum0
    st = relax.relax(1e-6, rounds=0)
    assert st.converged
    out = grid.download("b_eff")
    sum2 = int(np.rint((out - datum) * q).astype(np.int64).sum())
    assert sum2 == sum0
    grid.close()


def test_scaled_proposal_schedule():
    """A vanishing scale rounds every transfer to zero quanta (nothing moves);
    a damped schedule keeps the exact volume and still reaches the tolerance."""
    ln = _learned()
    from soilb200 import workloads
    b = workloads.config3_patch(5, n=96)
    k, datum = soilb200.choose_quantization(b)
    grid = soilb200.DeviceGrid(b.shape, 0.05, 0.05, precision="fx32", height_exponent=k,
                               datum_m=datum)
    grid.upload("b_eff", b)
    grid.upload("z_base", np.zeros_like(b))
    q = 2.0 ** k
    before = grid.download("b_eff")
    net = ln.ReposeNet(seed=2)
    relax = ln.LearnedRelaxation(grid, net, 35.0)
    relax.propose(rounds=1, scale=1e-30)
    assert np.array_equal(grid.download("b_eff"), before)
    with pytest.raises(ValueError):
        relax.propose(rounds=1, scale=0.0)
    with pytest.raises(ValueError):
        relax.relax(1e-6, rounds=2, scales=[1.0])
    sum0 = int(np.rint((before - datum) * q).astype(np.int64).sum())
    st = relax.relax(1e-6, rounds=4, plain_between=3, scales=[1.0, 1.0, 0.5, 0.5])
    assert st.converged
    sum1 = int(np.rint((grid.download("b_eff") - datum) * q).astype(np.int64).sum())
    assert sum1 == sum0
    grid.close()


@pytest.mark.parametrize("b,h,w,rows", [(1, 701, 701, 0), (2, 37, 300, 0), (1, 130, 123, 5),
                                        (1, 9, 250, 1), (3, 64, 128, 0), (1, 1, 5, 0)])
def test_fused_forward_equals_layer_path(b, h, w, rows):
    """One-kernel inference (activations in shared memory, 122-pixel strips,
    two-row layer skew) equals the four layer launches bit for bit, on the
    shipped network and on a random one, with every band height."""
    ln = _learned()
    from soilb200.train_repose import DEFAULT_WEIGHTS
    rng = np.random.default_rng(b * 1000 + h + w)
    feat = to_dev(bf16(rng.normal(size=(b, h, w, 16))), torch.bfloat16)
    for net in (ln.ReposeNet.load(DEFAULT_WEIGHTS), ln.ReposeNet(seed=h + w)):
        packed = net.packed()
        _, ref = ln.network_forward(net, feat, packed)
        got = ln.network_forward_fused(net, feat, packed, rows=rows)
        torch.cuda.synchronize()
        assert int(net.status.item()) == 0
        assert got.shape == ref.shape
        assert torch.equal(got, ref), float((got - ref).abs().max())


def test_fused_forward_matches_oracle():
    """The fused forward against the float64 oracle network on BF16-rounded
    inputs and weights: within the BF16 rounding of the three hidden layers."""
    ln = _learned()
    rng = np.random.default_rng(17)
    x = bf16(rng.normal(size=(1, 40, 260, 16)))
    net = ln.ReposeNet(seed=5)
    ws = [bf16(wt) for wt in net.numpy_weights()]
    ref = L.forward(x, ws)[1][..., :4]
    got = ln.network_forward_fused(net, to_dev(x, torch.bfloat16)).cpu().numpy()
    assert int(net.status.item()) == 0
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2e-2 * scale + 1e-6
