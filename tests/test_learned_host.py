"""Host side of the learned initial guess: the network's input features, its training target and the
policy that drops it when it stops saving PCG iterations.  No GPU (the layers are tested on the
device by test_gpu_learned.py)."""
import numpy as np
import pytest

from deep_frame_b200 import learned


def test_node_stiffness_is_the_log_mean_of_the_elements_around_each_node():
    shape = (3, 2, 2)
    moduli = np.arange(1, 13, dtype=float) * 1e-3
    s = learned.node_stiffness(moduli, shape)
    assert s.shape == (4, 3, 3)
    e = moduli.reshape(shape)
    assert np.isclose(s[0, 0, 0], np.log10(e[0, 0, 0]) / 9)                       # corner node: one element
    assert np.isclose(s[1, 1, 1], np.log10(e[0:2, 0:2, 0:2].mean()) / 9)          # interior node: eight
    assert np.isclose(learned.node_stiffness(np.full(12, 1e-20), shape)[0, 0, 0], -12 / 9)   # floored at 1e-12


def test_features_and_target_scaling():
    rng = np.random.default_rng(0)
    n = 10
    force = rng.normal(size=3 * n)
    stiffness, live = rng.uniform(-1, 0, n), (rng.uniform(size=n) > 0.3).astype(float)
    x, scale = learned.features(force, stiffness, live)
    assert x.shape == (5, n) and x.dtype == np.float32
    assert scale == np.abs(force).max() and np.isclose(np.abs(x[:3]).max(), 1.0)
    assert np.allclose(x[:3].T.ravel() * scale, force, rtol=1e-6)                  # dof = 3 node + component
    assert np.allclose(x[3], stiffness) and np.array_equal(x[4], live.astype(np.float32))
    u = rng.normal(size=3 * n) * 1e-3
    t, rms = learned.target(u)
    assert t.shape == (3, n) and np.isclose(np.sqrt(np.mean(t.astype(float) ** 2)), 1.0, rtol=1e-6)
    assert np.allclose(t.T.ravel() * rms, u, rtol=1e-6)
    assert learned.features(np.zeros(3 * n), stiffness, live)[1] == 1e-300       # a zero load is not divided by zero


def test_guess_policy_drops_the_network_once_it_stops_saving_iterations():
    policy = learned.GuessPolicy(net=None)
    assert policy.assess(12, 15) and policy.enabled
    assert not policy.assess(15, 15) and not policy.enabled                       # no saving: dropped
    assert not policy.assess(5, 15)                                               # and stays dropped
    assert policy.record == [(12, 15), (15, 15), (5, 15)]
    # a fraction of an iteration is no saving, and neither is a saving that costs time
    assert not learned.GuessPolicy(net=None).assess(165.93, 165.94)
    assert not learned.GuessPolicy(net=None).assess(20, 25, seconds_with=1.9, seconds_without=0.8)
    assert learned.GuessPolicy(net=None).assess(20, 25, seconds_with=0.6, seconds_without=0.8)


def test_network_layers_for_any_depth_match_the_oracle_network():
    """The layer list of a four-level network (two convolutions per encoder level, one per decoder
    level, a linear head) is the one the oracle's forward pass consumes, in the same order."""
    import torch
    from oracle import learned as olearn
    net = learned.GuessNet(channels=(16, 32, 48, 64), seed=0, device="cpu")
    assert net.specs == [(5, 16, 1), (16, 16, 1), (16, 32, 1), (32, 32, 1), (32, 48, 1), (48, 48, 1), (48, 64, 1), (64, 64, 1),
                         (112, 48, 1), (80, 32, 1), (48, 16, 1), (16, 3, 0)]
    shape = (9, 7, 5)
    params = [(torch.tensor(w.numpy(), dtype=torch.float64), torch.tensor(b.numpy(), dtype=torch.float64)) for w, b in net.params]
    y = olearn.forward(params, torch.zeros((5, int(np.prod(shape))), dtype=torch.float64), shape, net.channels)
    assert tuple(y.shape) == (3, int(np.prod(shape)))
    with pytest.raises(ValueError):
        learned.GuessNet(channels=(16,), device="cpu")
