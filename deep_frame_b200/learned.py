"""Learned initial guess for the covariance solves: a small 3-D convolutional encoder / decoder.

The network maps, per load column, the node fields (load f scaled by max|f|, log10 of the node
stiffness, live mask) to the shape of the displacement u (the target is u / rms(u)); the scale of
the guess is then fixed by one operator apply, x0 = alpha y with alpha = (y . f) / (y . K y), the
energy-optimal multiple of the prediction.  It is trained on (density, load, displacement) snapshots
the solver itself produces along SIMP trajectories and assessed by the iterations GMG-PCG needs from
its guess to the same tolerance; ``GuessPolicy`` drops it whenever it does not reduce them.

Layers (channel-major FP32 node grids, every kernel in libtfb200.so, deterministic):
  level 0: conv 5->c0, conv c0->c0          level 1 (pool): conv c0->c1, conv c1->c1
  level 2 (pool): conv c1->c2, conv c2->c2   up + concat(level 1): conv (c2+c1)->c1
  up + concat(level 0): conv (c1+c0)->c0, conv c0->3 (linear)
Convolutions are 3 x 3 x 3 with zero padding (im2col + SGEMM), ReLU after every hidden layer.
The reference has no counterpart: this is the learned part of the B200 design.
"""
import ctypes

import numpy as np

from . import _lib

IN_CHANNELS = 5


def _shape3(shape):
    return (ctypes.c_int32 * 3)(*[int(s) for s in shape])


def _half(shape):
    return tuple((int(s) + 1) // 2 for s in shape)


class GuessNet:
    """The encoder / decoder over len(channels) levels; the default (16, 32, 48, 64) has four."""

    def __init__(self, channels=(16, 32, 48, 64), seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.lib = _lib.load()
        if len(channels) < 2 or any(int(c) < 1 or int(c) > 64 for c in channels):
            raise ValueError("channels: at least two levels of 1 to 64 channels")
        self.channels = tuple(int(c) for c in channels)
        ch = self.channels
        # (cin, cout, relu) in execution order: two convolutions per encoder level, one per decoder
        # level (after the upsampled coarser features are concatenated with the encoder's), a linear head
        self.specs = [(IN_CHANNELS, ch[0], 1), (ch[0], ch[0], 1)]
        for lo, hi in zip(ch[:-1], ch[1:]):
            self.specs += [(lo, hi, 1), (hi, hi, 1)]
        for level in range(len(ch) - 2, -1, -1):
            self.specs.append((ch[level + 1] + ch[level], ch[level], 1))
        self.specs.append((ch[0], 3, 0))
        rng = np.random.default_rng(seed)
        self.params = []
        for cin, cout, relu in self.specs:
            scale = np.sqrt((2.0 if relu else 1.0) / (cin * 27))
            w = torch.as_tensor(rng.normal(0.0, scale, (cout, cin * 27)).astype(np.float32), device=self.device)
            b = torch.zeros(cout, dtype=torch.float32, device=self.device)
            self.params.append([w, b])
        self.grads = [[torch.zeros_like(w), torch.zeros_like(b)] for w, b in self.params]
        self.moments = [[(torch.zeros_like(w), torch.zeros_like(w)), (torch.zeros_like(b), torch.zeros_like(b))] for w, b in self.params]
        self.step_count = 0
        self.work = torch.empty(0, dtype=torch.float32, device=self.device)
        self.mse_scratch = torch.zeros(int(self.lib.tf_nn_mse_scratch_doubles()) + 1, dtype=torch.float64, device=self.device)
        self.packed = None
        self.tc_error = torch.zeros(1, dtype=torch.int32, device=self.device)

    def pack(self):
        """FP16 copies of the weights for the tensor-core inference (tf_nn_pack16); call after training."""
        torch = self.torch
        self.packed = []
        for (cin, cout, _), (w, _) in zip(self.specs, self.params):
            np_, kp = 16 * ((cout + 15) // 16), 64 * ((27 * cin + 63) // 64)
            w16 = torch.empty((np_, kp), dtype=torch.float16, device=self.device)
            self._check(self.lib.tf_nn_pack16(_lib.ptr(w), cout, 27 * cin, _lib.ptr(w16), np_, kp, self._stream()), "tf_nn_pack16")
            self.packed.append((w16, np_, kp))
        return self

    # ------------------------------------------------------------ plumbing --
    def _stream(self):
        return _lib.stream_of(self.device)

    def _check(self, status, what):
        if status:
            message = (self.lib.tf_nn_last_error() or b"").decode()
            if status == 1:
                raise ValueError(f"{what} failed: {message}")
            raise _lib.TfError(status, f"{what} failed: {message}")

    def _gemm(self, ta, tb, m, n, k, a, lda, b, ldb, c, ldc, beta=0.0):
        need = 64 * m * n
        if self.work.numel() < need:
            self.work = self.torch.empty(need, dtype=self.torch.float32, device=self.device)
        self._check(self.lib.tf_nn_gemm(ta, tb, m, n, k, 1.0, _lib.ptr(a), lda, _lib.ptr(b), ldb, float(beta), _lib.ptr(c), ldc,
                                        _lib.ptr(self.work), self.work.numel(), self._stream()), "tf_nn_gemm")

    def _conv(self, index, x, shape, cache):
        torch = self.torch
        cin, cout, relu = self.specs[index]
        w, b = self.params[index]
        n = int(np.prod(shape))
        if cache is None and self.packed is not None:
            # inference on the tensor cores: FP16 operands, FP32 accumulation
            w16, np_, kp = self.packed[index]
            y = torch.empty((cout, n), dtype=torch.float32, device=self.device)
            self._check(self.lib.tf_nn_conv16(_lib.ptr(x), cin, _shape3(shape), _lib.ptr(w16), cout, np_, kp, _lib.ptr(b), relu,
                                              _lib.ptr(y), _lib.ptr(self.tc_error), self._stream()), "tf_nn_conv16")
            return y
        col = torch.empty((cin * 27, n), dtype=torch.float32, device=self.device)
        self._check(self.lib.tf_nn_im2col(_lib.ptr(x), cin, _shape3(shape), _lib.ptr(col), self._stream()), "tf_nn_im2col")
        y = torch.empty((cout, n), dtype=torch.float32, device=self.device)
        self._gemm(0, 0, cout, n, cin * 27, w, cin * 27, col, n, y, n)
        self._check(self.lib.tf_nn_bias_act(_lib.ptr(y), _lib.ptr(b), cout, n, relu, self._stream()), "tf_nn_bias_act")
        if cache is not None:
            cache[index] = (col, y, shape)
        return y

    def _conv_back(self, index, dy, cache, accumulate):
        """dy: gradient w.r.t. this layer's output (modified in place); returns the input gradient."""
        torch = self.torch
        cin, cout, relu = self.specs[index]
        w, _ = self.params[index]
        gw, gb = self.grads[index]
        col, y, shape = cache[index]
        n = int(np.prod(shape))
        self._check(self.lib.tf_nn_act_back(_lib.ptr(dy), _lib.ptr(y), cout, n, relu, _lib.ptr(gb), 1 if accumulate else 0, self._stream()),
                    "tf_nn_act_back")
        self._gemm(0, 1, cout, cin * 27, n, dy, n, col, n, gw, cin * 27, beta=1.0 if accumulate else 0.0)
        dcol = torch.empty((cin * 27, n), dtype=torch.float32, device=self.device)
        self._gemm(1, 0, cin * 27, n, cout, w, cin * 27, dy, n, dcol, n)
        dx = torch.empty((cin, n), dtype=torch.float32, device=self.device)
        self._check(self.lib.tf_nn_col2im(_lib.ptr(dcol), cin, _shape3(shape), _lib.ptr(dx), self._stream()), "tf_nn_col2im")
        return dx

    def _pool(self, x, channels, fine):
        coarse = _half(fine)
        out = self.torch.empty((channels, int(np.prod(coarse))), dtype=self.torch.float32, device=self.device)
        self._check(self.lib.tf_nn_pool(_lib.ptr(x), channels, _shape3(fine), _shape3(coarse), _lib.ptr(out), self._stream()), "tf_nn_pool")
        return out

    def _resample(self, x, channels, fine, mode):
        coarse = _half(fine)
        n = int(np.prod(coarse if mode == 2 else fine))
        out = self.torch.empty((channels, n), dtype=self.torch.float32, device=self.device)
        self._check(self.lib.tf_nn_resample(_lib.ptr(x), channels, _shape3(fine), _shape3(coarse), mode, _lib.ptr(out), self._stream()),
                    "tf_nn_resample")
        return out

    # ------------------------------------------------------------- network --
    def forward(self, x, shape, cache=None):
        """x: [5, n] FP32 features on the node grid `shape`; returns [3, n].  With a cache (training)
        every convolution runs as im2col + FP32 SGEMM and keeps what backward needs; without one,
        after pack(), every convolution runs on the tensor cores in FP16."""
        torch = self.torch
        ch = self.channels
        shapes = [tuple(int(s) for s in shape)]
        for _ in ch[1:]:
            shapes.append(_half(shapes[-1]))
        layer = 0
        skips = []
        h = x.contiguous()
        for level, c in enumerate(ch):
            if level > 0:
                h = self._pool(h, ch[level - 1], shapes[level - 1])
            h = self._conv(layer, h, shapes[level], cache)
            h = self._conv(layer + 1, h, shapes[level], cache)
            layer += 2
            skips.append(h)
        for level in range(len(ch) - 2, -1, -1):
            up = self._resample(h, ch[level + 1], shapes[level], 0)
            h = self._conv(layer, torch.cat([up, skips[level]]).contiguous(), shapes[level], cache)
            layer += 1
        y = self._conv(layer, h, shapes[0], cache)
        if cache is None and self.packed is not None and int(self.tc_error.item()):
            raise _lib.TfError(5, "tf_nn_conv16: a tensor-core wait timed out")
        return y

    def backward(self, dy, shape, cache, accumulate):
        """Gradients of all parameters (added to the stored ones when accumulate) from dy = dL/d output."""
        ch = self.channels
        shapes = [tuple(int(s) for s in shape)]
        for _ in ch[1:]:
            shapes.append(_half(shapes[-1]))
        layer = len(self.specs) - 1
        g = self._conv_back(layer, dy.contiguous(), cache, accumulate)
        dskip = [None] * len(ch)
        for level in range(len(ch) - 1):   # decoder, finest first (reverse of the forward order)
            layer -= 1
            dcat = self._conv_back(layer, g, cache, accumulate)
            dskip[level] = dcat[ch[level + 1]:].clone()
            g = self._resample(dcat[:ch[level + 1]].contiguous(), ch[level + 1], shapes[level], 2)
        for level in range(len(ch) - 1, -1, -1):   # encoder, coarsest first
            if dskip[level] is not None:
                g = g + dskip[level]
            layer -= 2
            g = self._conv_back(layer, self._conv_back(layer + 1, g, cache, accumulate), cache, accumulate)
            if level > 0:
                g = self._resample(g, ch[level - 1], shapes[level - 1], 1)

    def loss(self, y, target, weight=None, want_grad=True):
        """Mean squared error over the weighted entries; returns (loss tensor [1] FP64, dL/dy or None)."""
        torch = self.torch
        count = float(weight.sum()) if weight is not None else float(y.numel())
        dy = torch.empty_like(y) if want_grad else None
        out = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._check(self.lib.tf_nn_mse(_lib.ptr(y), _lib.ptr(target), _lib.ptr(weight), y.numel(), max(count, 1.0), _lib.ptr(dy),
                                       _lib.ptr(self.mse_scratch), _lib.ptr(out), self._stream()), "tf_nn_mse")
        return out, dy

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, scale=1.0):
        """One Adam step on the stored gradients (multiplied by `scale`, e.g. 1 / batch size)."""
        self.step_count += 1
        for (p_w, p_b), (g_w, g_b), ((m_w, v_w), (m_b, v_b)) in zip(self.params, self.grads, self.moments):
            for p, g, m, v in ((p_w, g_w, m_w, v_w), (p_b, g_b, m_b, v_b)):
                if scale != 1.0:
                    g.mul_(scale)
                self._check(self.lib.tf_nn_adam(_lib.ptr(p), _lib.ptr(g), _lib.ptr(m), _lib.ptr(v), p.numel(), lr, beta1, beta2, eps,
                                                self.step_count, self._stream()), "tf_nn_adam")

    def state(self):
        return [(w.cpu().numpy(), b.cpu().numpy()) for w, b in self.params]


# ------------------------------------------------------------------ features --
def node_stiffness(moduli, shape):
    """log10 of the mean modulus of the (up to 8) elements around every node, scaled to about [-1, 0]."""
    e = np.asarray(moduli, dtype=float).reshape(shape)
    nodes = tuple(s + 1 for s in shape)
    total, count = np.zeros(nodes), np.zeros(nodes)
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                total[dx:dx + shape[0], dy:dy + shape[1], dz:dz + shape[2]] += e
                count[dx:dx + shape[0], dy:dy + shape[1], dz:dz + shape[2]] += 1
    return np.log10(np.maximum(total / np.maximum(count, 1), 1e-12)) / 9.0


def features(force, stiffness, live):
    """[5, n] FP32: force / max|force| (3 channels, dof = 3 node + comp), node stiffness, node live flag."""
    f = np.asarray(force, dtype=float).reshape(-1, 3)
    scale = max(np.abs(f).max(), 1e-300)
    x = np.concatenate([(f / scale).T, stiffness.reshape(1, -1), live.reshape(1, -1)], axis=0)
    return x.astype(np.float32), scale


def target(u):
    """u / rms(u) as [3, n] FP32 and the rms."""
    v = np.asarray(u, dtype=float).reshape(-1, 3)
    rms = max(float(np.sqrt(np.mean(v ** 2))), 1e-300)
    return (v / rms).T.astype(np.float32), rms


class GuessPolicy:
    """Use the network's guess only while it pays: at least one PCG iteration fewer than the
    comparison start and, when the times are given, less time with its inference included."""

    def __init__(self, net):
        self.net, self.enabled, self.record = net, True, []

    def assess(self, iterations_with, iterations_without, seconds_with=None, seconds_without=None):
        self.record.append((int(iterations_with), int(iterations_without)))
        if iterations_with > iterations_without - 1:
            self.enabled = False
        if seconds_with is not None and seconds_without is not None and seconds_with >= seconds_without:
            self.enabled = False
        return self.enabled


# ------------------------------------------------------------ training data --
def record_trajectory(domain, covariance, iterations, multigrid=None, device="cuda", stride=1):
    """Run the covariance SIMP + MMA loop and keep, per iteration, the node stiffness of the design
    and of every group every `stride`-th load column's sample on the device: the network input
    (force / max|force|, node stiffness, node live flag: [5, n] FP32) and target (u / rms(u):
    [3, n] FP32).  Returns (snapshots, live, shape) with snapshots = [(moduli, [(key, x, t)])] and
    live = {key: (node live [n], dof live [3, n] FP32 on the device)}."""
    import torch
    from .optimize import CovarianceSimp
    loop = CovarianceSimp(domain, covariance, volume_fraction=0.15, filter_radius=1.5, move=0.2,
                          multigrid={**(multigrid or {}), "device": str(device)})
    system = loop.system
    live = {}
    for key in system.groups:
        node_live, dof_live = _live_nodes(system, key)
        live[key] = (torch.as_tensor(node_live, device=device), torch.as_tensor(dof_live, device=device))
    snapshots = []
    original = loop.model.solve_all

    def solve_and_keep(initial=None):
        solved = original(initial)
        moduli = loop.moduli.cpu().numpy().copy()
        stiffness = torch.as_tensor(node_stiffness(moduli, system.shape).reshape(1, -1).astype(np.float32), device=device)
        kept = []
        for key, _, forces, u, _ in solved:
            for j in range(0, forces.shape[0], stride):
                f = forces[j].reshape(-1, 3).to(torch.float32)
                scale = f.abs().max()
                if float(scale) == 0.0:
                    continue
                v = u[j].reshape(-1, 3).to(torch.float64)
                rms = v.pow(2).mean().sqrt().clamp_min(1e-300)
                x = torch.cat([(f / scale).T, stiffness, live[key][0][None, :]]).contiguous()
                kept.append((key, x, (v / rms).to(torch.float32).T.contiguous()))
        snapshots.append((moduli, kept))
        return solved

    loop.model.solve_all = solve_and_keep
    try:
        loop.run(iterations)
    finally:
        loop.model.solve_all = original
    shape = system.shape
    loop.close()
    return snapshots, live, shape


def _live_nodes(system, key):
    """Per node: 1 where any dof is free in fixture group `key`, and the [3, n] dof mask."""
    free = np.zeros(system.ndof, dtype=np.float32)
    free[system.groups[key][0][1]["free"]] = 1.0
    dofs = free.reshape(-1, 3)
    return dofs.max(axis=1), dofs.T.copy()


def samples(snapshots, live, shape):
    """Yield (x [5, n], target [3, n], weight [3, n]) device FP32 for every kept column of every snapshot."""
    for _, kept in snapshots:
        for key, x, t in kept:
            yield x, t, live[key][1]


def train(net, snapshots, live, shape, epochs=6, batch=8, lr=2e-3, seed=0):
    """Adam on the mean squared error of u / rms(u); returns the mean loss of every epoch."""
    torch = net.torch
    data = list(samples(snapshots, live, shape))
    order = np.random.default_rng(seed).permutation(len(data))
    node_shape = tuple(s + 1 for s in shape)
    history = []
    for epoch in range(epochs):
        total, seen = 0.0, 0
        for start in range(0, len(order), batch):
            chunk = order[start:start + batch]
            losses = []
            for position, index in enumerate(chunk):
                x, t, w = data[index]
                cache = {}
                y = net.forward(x, node_shape, cache)
                loss, dy = net.loss(y, t, w)
                net.backward(dy, node_shape, cache, accumulate=position > 0)
                losses.append(loss)
            net.adam(lr=lr, scale=1.0 / len(chunk))
            total += float(torch.cat(losses).sum())
            seen += len(chunk)
        history.append(total / max(seen, 1))
        order = np.random.default_rng(seed + epoch + 1).permutation(len(data))
    return history


def predict(net, multigrid, key, fixed, forces, moduli, shape, live):
    """Initial guesses [R, ndof] FP64 for a group's force block: the network's shape, scaled per column
    to the energy-optimal multiple (one masked operator apply for all columns).  The features are
    formed on the device; with pack() done the network runs on the tensor cores."""
    torch = net.torch
    node_live, dof_live = (torch.as_tensor(a, device=forces.device) for a in live)
    stiffness = torch.as_tensor(node_stiffness(moduli, shape).reshape(1, -1).astype(np.float32), device=forces.device)
    node_shape = tuple(s + 1 for s in shape)
    shapes = torch.zeros_like(forces)
    for j in range(forces.shape[0]):
        f = forces[j].reshape(-1, 3).to(torch.float32)
        scale = f.abs().max()
        if float(scale) == 0.0:
            continue
        x = torch.cat([(f / scale).T, stiffness, node_live[None, :].to(torch.float32)]).contiguous()
        y = net.forward(x, node_shape)
        shapes[j] = (y * dof_live).T.reshape(-1).to(torch.float64)
    applied = multigrid.apply_device(shapes.contiguous(), key, fixed)
    energy = (shapes * applied).sum(1)
    work = (shapes * forces).sum(1)
    alpha = torch.where(energy > 0, work / energy.clamp_min(1e-300), torch.zeros_like(energy))
    return (alpha[:, None] * shapes).contiguous()


def compare(net, domain, covariance, design_moduli, multigrid=None, device="cuda"):
    """PCG iterations and seconds of one covariance solve (both halves) from zero and from the network's
    guess (inference included), for the element moduli `design_moduli`."""
    import time
    import torch
    from .covariance import InterfaceCovariance
    from .elasticity import HexElasticity
    system = HexElasticity(domain, multigrid={**(multigrid or {}), "device": str(device)})
    model = InterfaceCovariance(system, covariance, domain["interfaces"])
    mg = system._multigrid()
    mg.update_device(torch.as_tensor(design_moduli, device=device))
    out = {"zero": {"iterations": [], "seconds": 0.0}, "network": {"iterations": [], "seconds": 0.0}}
    for key, _, forces in model.groups():     # hierarchy set-up outside the timings
        system.solve_group_device(key, forces)
    for label in ("zero", "network"):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for key, _, forces in model.groups():
            fixed = system.groups[key][0][1]["fixed"]
            guess = None if label == "zero" else predict(net, mg, key, fixed, forces, design_moduli, system.shape, _live_nodes(system, key))
            _, report = system.solve_group_device(key, forces, initial=guess)
            out[label]["iterations"] += report["iterations"]
        torch.cuda.synchronize()
        out[label]["seconds"] = time.perf_counter() - t0
    system.close()
    for label in out:
        its = [i for i in out[label]["iterations"] if i > 0]
        out[label]["mean_iterations"] = float(np.mean(its)) if its else 0.0
        out[label]["max_iterations"] = int(max(its)) if its else 0
    return out
