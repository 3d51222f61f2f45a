"""CPU reference of the learned-guess network (oracle, test only).

The same encoder / decoder as deep_frame_b200/learned.py written with PyTorch CPU operations
(3 x 3 x 3 zero-padded convolutions, ReLU, 2 x 2 x 2 average pooling over a zero-padded even
extent, nearest upsampling cropped to the fine extent, concatenation, mean squared error), so
its autograd gradients check the hand-written device backward pass.  No reference counterpart.
"""
import numpy as np


def forward(params, x, shape, channels):
    """params: [(w [cout, cin*27], b [cout])] torch tensors; x: [5, n] tensor; returns [3, n]."""
    import torch
    import torch.nn.functional as F
    s0 = tuple(int(s) for s in shape)

    def conv(i, v, s, relu=True):
        w, b = params[i]
        cout, k = w.shape
        cin = k // 27
        y = F.conv3d(v.reshape(1, cin, *s), w.reshape(cout, cin, 3, 3, 3), b, padding=1)[0]
        return torch.relu(y) if relu else y

    def pool(v):
        c, s = v.shape[0], v.shape[1:]
        pad = [0, s[2] % 2, 0, s[1] % 2, 0, s[0] % 2]
        return F.avg_pool3d(F.pad(v[None], pad), 2)[0]

    def up(v, s):
        return v.repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3)[:, :s[0], :s[1], :s[2]]

    g = x.reshape(5, *s0)
    layer, skips, shapes = 0, [], [s0]
    h = g
    for level in range(len(channels)):
        if level > 0:
            h = pool(h)
            shapes.append(tuple(h.shape[1:]))
        h = conv(layer + 1, conv(layer, h, shapes[level]), shapes[level])
        layer += 2
        skips.append(h)
    for level in range(len(channels) - 2, -1, -1):
        h = conv(layer, torch.cat([up(h, shapes[level]), skips[level]]), shapes[level])
        layer += 1
    return conv(layer, h, s0, relu=False).reshape(3, -1)


def loss_and_grads(params_np, x, target, weight, shape, channels):
    """MSE (sum w (y - t)^2 / sum w) and its gradients w.r.t. every parameter (NumPy in, NumPy out)."""
    import torch
    params = [(torch.tensor(w, dtype=torch.float64, requires_grad=True), torch.tensor(b, dtype=torch.float64, requires_grad=True))
              for w, b in params_np]
    y = forward(params, torch.tensor(x, dtype=torch.float64), shape, channels)
    t = torch.tensor(target, dtype=torch.float64)
    w = torch.tensor(weight, dtype=torch.float64)
    loss = (w * (y - t) ** 2).sum() / w.sum()
    loss.backward()
    return float(loss.detach()), y.detach().numpy(), [(w_.grad.numpy(), b_.grad.numpy()) for w_, b_ in params]
