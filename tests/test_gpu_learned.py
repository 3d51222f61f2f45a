"""Learned initial guess: device forward / backward vs a PyTorch-CPU autograd oracle of the same network.

The hand-written kernels (im2col, col2im, split-K SGEMM, bias + ReLU, pooling, upsampling, MSE, Adam)
must reproduce the oracle's output, loss and every parameter gradient (FP32 vs FP64: 1e-4 relative);
a few Adam steps must lower the loss.  Grid extents are odd on purpose (ceil pooling).
"""
import numpy as np
import pytest

from oracle import learned as olearn

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("channels", [(4, 6, 8), (4, 6, 8, 10)])
def test_forward_backward_match_autograd(cuda, channels):
    import torch
    from deep_frame_b200.learned import GuessNet
    shape = (9, 7, 5)
    n = int(np.prod(shape))
    rng = np.random.default_rng(3)
    net = GuessNet(channels=channels, seed=1)
    x = rng.normal(size=(5, n)).astype(np.float32)
    t = rng.normal(size=(3, n)).astype(np.float32)
    w = (rng.uniform(size=(3, n)) > 0.2).astype(np.float32)
    cache = {}
    y = net.forward(torch.as_tensor(x, device="cuda"), shape, cache)
    loss, dy = net.loss(y, torch.as_tensor(t, device="cuda"), torch.as_tensor(w, device="cuda"))
    net.backward(dy, shape, cache, accumulate=False)
    ref_loss, ref_y, ref_grads = olearn.loss_and_grads(net.state(), x, t, w, shape, net.channels)
    assert np.allclose(y.cpu().numpy(), ref_y, rtol=1e-4, atol=1e-4 * np.abs(ref_y).max())
    assert float(loss.item()) == pytest.approx(ref_loss, rel=1e-4)
    for (gw, gb), (rw, rb) in zip(net.grads, ref_grads):
        assert np.linalg.norm(gw.cpu().numpy() - rw) <= 2e-4 * np.linalg.norm(rw) + 1e-7
        assert np.linalg.norm(gb.cpu().numpy() - rb) <= 2e-4 * np.linalg.norm(rb) + 1e-7
    # deterministic: the same pass twice gives the same bits
    cache2 = {}
    y2 = net.forward(torch.as_tensor(x, device="cuda"), shape, cache2)
    assert torch.equal(y, y2)


def test_adam_steps_reduce_the_loss(cuda):
    import torch
    from deep_frame_b200.learned import GuessNet
    shape = (12, 10, 6)
    n = int(np.prod(shape))
    rng = np.random.default_rng(4)
    net = GuessNet(channels=(4, 8, 8), seed=2)
    x = torch.as_tensor(rng.normal(size=(5, n)).astype(np.float32), device="cuda")
    t = torch.as_tensor(np.tanh(rng.normal(size=(3, n))).astype(np.float32), device="cuda")
    losses = []
    for _ in range(30):
        cache = {}
        y = net.forward(x, shape, cache)
        loss, dy = net.loss(y, t)
        losses.append(float(loss.item()))
        net.backward(dy, shape, cache, accumulate=False)
        net.adam(lr=3e-3)
    assert losses[-1] < 0.7 * losses[0]


def test_trajectory_training_and_guess_pipeline(cuda):
    """Snapshots from a short SIMP trajectory train the network; PCG from its guess reaches the same tolerance."""
    from deep_frame_b200 import learned, problems
    shape = (24, 24, 6)
    domain, _, cov = problems.plate(shape, 0)
    settings = {"coarsest_dofs": 2000, "tolerance": 1e-8}
    snapshots, live, grid = learned.record_trajectory(domain, cov, 4, multigrid=settings)
    assert len(snapshots) == 4 and grid == shape
    net = learned.GuessNet(channels=(4, 8, 8), seed=0)
    history = learned.train(net, snapshots[:3], live, grid, epochs=2, batch=8)
    assert len(history) == 2 and all(np.isfinite(history))
    result = learned.compare(net, domain, cov, snapshots[3][0], multigrid=settings)
    assert result["zero"]["mean_iterations"] > 0 and result["network"]["mean_iterations"] > 0
    policy = learned.GuessPolicy(net)
    kept = policy.assess(result["network"]["mean_iterations"], result["zero"]["mean_iterations"])
    assert kept == (result["network"]["mean_iterations"] <= result["zero"]["mean_iterations"] - 1)


@pytest.mark.parametrize("cin,cout,shape", [(5, 16, (9, 7, 5)), (32, 48, (13, 11, 6)), (80, 64, (7, 7, 7)), (16, 3, (20, 9, 4))])
def test_tensor_core_convolution_matches_fp32(cuda, cin, cout, shape):
    """tf_nn_conv16 (tcgen05, FP16 operands, FP32 accumulation) against the FP32 im2col + SGEMM layer
    and a PyTorch FP64 convolution of the FP16-rounded operands (the tensor-core product itself is
    exact to FP32 accumulation: 1e-5); against unrounded FP32 operands the FP16 rounding bounds it
    (2e-3 relative)."""
    import torch
    import torch.nn.functional as F
    from deep_frame_b200 import _lib
    from deep_frame_b200.learned import _shape3
    lib = _lib.load()
    rng = np.random.default_rng(cin + cout)
    n = int(np.prod(shape))
    x = torch.as_tensor(rng.normal(size=(cin, n)).astype(np.float32), device="cuda")
    w = torch.as_tensor((rng.normal(size=(cout, cin * 27)) * np.sqrt(2.0 / (27 * cin))).astype(np.float32), device="cuda")
    b = torch.as_tensor(rng.normal(size=cout).astype(np.float32) * 0.1, device="cuda")
    np_, kp = 16 * ((cout + 15) // 16), 64 * ((27 * cin + 63) // 64)
    w16 = torch.empty((np_, kp), dtype=torch.float16, device="cuda")
    stream = _lib.stream_of(torch.device("cuda"))
    assert lib.tf_nn_pack16(_lib.ptr(w), cout, 27 * cin, _lib.ptr(w16), np_, kp, stream) == 0
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for relu in (0, 1):
        y = torch.empty((cout, n), dtype=torch.float32, device="cuda")
        assert lib.tf_nn_conv16(_lib.ptr(x), cin, _shape3(shape), _lib.ptr(w16), cout, np_, kp, _lib.ptr(b), relu, _lib.ptr(y),
                                _lib.ptr(err), stream) == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        xh = x.half().double().cpu().reshape(1, cin, *shape)
        wh = w16[:cout, :27 * cin].double().cpu().reshape(cout, cin, 3, 3, 3)
        exact = F.conv3d(xh, wh, b.double().cpu(), padding=1)[0].reshape(cout, n)
        full = F.conv3d(x.double().cpu().reshape(1, cin, *shape), w.double().cpu().reshape(cout, cin, 3, 3, 3), b.double().cpu(),
                        padding=1)[0].reshape(cout, n)
        if relu:
            exact, full = exact.clamp_min(0), full.clamp_min(0)
        got = y.double().cpu()
        assert float((got - exact).norm() / exact.norm()) < 1e-5
        assert float((got - full).norm() / full.norm()) < 2e-3
    # the padded weight rows and columns are zero
    assert float(w16[cout:].abs().max() if np_ > cout else 0.0) == 0.0
    assert float(w16[:, 27 * cin:].abs().max() if kp > 27 * cin else 0.0) == 0.0


def test_packed_network_matches_training_forward(cuda):
    """The four-level network on the tensor cores (pack(), no cache) against its FP32 training forward."""
    import torch
    from deep_frame_b200.learned import GuessNet
    shape = (17, 13, 9)
    n = int(np.prod(shape))
    rng = np.random.default_rng(5)
    net = GuessNet(channels=(16, 32, 48, 64), seed=3)
    x = torch.as_tensor(rng.normal(size=(5, n)).astype(np.float32), device="cuda")
    ref = net.forward(x, shape, {})
    got = net.pack().forward(x, shape)
    assert float((got - ref).norm() / ref.norm()) < 1e-2
    assert torch.equal(got, net.forward(x, shape))   # deterministic
