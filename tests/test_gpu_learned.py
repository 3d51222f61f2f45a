"""Learned initial guess: device forward / backward vs a PyTorch-CPU autograd oracle of the same network.

The hand-written kernels (im2col, col2im, split-K SGEMM, bias + ReLU, pooling, upsampling, MSE, Adam)
must reproduce the oracle's output, loss and every parameter gradient (FP32 vs FP64: 1e-4 relative);
a few Adam steps must lower the loss.  Grid extents are odd on purpose (ceil pooling).
"""
import numpy as np
import pytest

from oracle import learned as olearn

pytestmark = pytest.mark.gpu


def test_forward_backward_match_autograd(cuda):
    import torch
    from deep_frame_b200.learned import GuessNet
    shape = (9, 7, 5)
    n = int(np.prod(shape))
    rng = np.random.default_rng(3)
    net = GuessNet(channels=(4, 6, 8), seed=1)
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
    assert kept == (result["network"]["mean_iterations"] < result["zero"]["mean_iterations"])
