"""World-size-2 gloo run of the RHS-sharded covariance exchange on the CPU.

Each rank solves its slice of the 42 directions with the oracle (direct sparse
solves); the exchange (F columns + all-reduce, tr-gradient all-reduce, partial
U v all-reduce for the lambda_max gradient) must reproduce the single-process
oracle measure.  No GPU is involved.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    from deep_frame_b200 import problems
    from deep_frame_b200.covariance import InterfaceCovariance
    from deep_frame_b200.elasticity import HexElasticity
    shape = (10, 8, 3)
    domain, density, cov = problems.plate(shape, 4)
    system = HexElasticity(domain, multigrid={"device": "cpu"})
    model = InterfaceCovariance(system, cov, domain["interfaces"])
    return shape, system, model, density


class OracleOps:
    """CPU test doubles of the device kernels (direct solves, NumPy energies)."""

    def __init__(self, shape, system, moduli):
        from oracle import operator as op
        self.op, self.shape, self.system = op, shape, system
        self.matrix = op.assemble(shape, system.ke, moduli).tocsc()
        self.moduli = moduli

    def solve(self, key, forces):
        import torch
        from scipy.sparse.linalg import spsolve
        f = forces.numpy().T
        live = self.op.live_dofs(self.shape, self.moduli, self.system.groups[key][0][1]["fixed"])
        u = np.zeros_like(f)
        u[live] = spsolve(self.matrix[live][:, live].tocsc(), f[live]).reshape(u[live].shape)
        return torch.as_tensor(u.T.copy())

    def gram(self, p_all, u_local):
        return p_all @ u_local.T

    def energy(self, columns, coefficients, scale):
        import torch
        e = self.op.element_energy(self.shape, self.system.ke, columns.numpy().T)
        e = e.reshape(len(coefficients), -1) if e.ndim == 2 else e[None]
        return torch.as_tensor(scale.numpy() * (np.asarray(coefficients) @ e))


    def combine(self, columns, mixing):
        import torch
        return torch.as_tensor(np.asarray(mixing).T) @ columns


def _groups(model):
    import torch
    index = {name: k for k, name in enumerate(model.cases)}
    groups = []
    for key, members in model.system.groups.items():
        ks = np.asarray([index[case["name"]] for case, _ in members])
        forces = torch.as_tensor(np.stack([part["force"] for _, part in members]))
        groups.append((key, ks, forces))
    return groups


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from deep_frame_b200.distributed import ShardedMeasure
        shape, system, model, density = _problem()
        moduli, derivative = system.moduli(density, 3.0, 1e-9)
        measure = ShardedMeasure(_groups(model), model.rank, model.factor, OracleOps(shape, system, moduli))
        rows, flex = measure.measure(torch.as_tensor(-derivative))
        out[rank] = (rows[0]["value"], rows[1]["value"], rows[0]["gradient"].numpy(), rows[1]["gradient"].numpy(),
                     [len(g["local"]) for g in measure.groups])
    finally:
        dist.destroy_process_group()


def _oracle_reference():
    from oracle import covariance as ocov
    import torch
    shape, system, model, density = _problem()
    moduli, derivative = system.moduli(density, 3.0, 1e-9)
    ops = OracleOps(shape, system, moduli)
    parts = []
    index = {name: k for k, name in enumerate(model.cases)}
    for key, members in system.groups.items():
        forces = np.zeros((system.ndof, model.rank))
        for case, part in members:
            forces[:, index[case["name"]]] = part["force"]
        u = ops.solve(key, torch.as_tensor(forces.T.copy())).numpy().T
        parts.append((forces, u))
    return ocov.measure(parts, model.factor, shape, system.ke, derivative)


def test_unsharded_measure_matches_the_oracle():
    """One process (no process group): the exchange's all-reduces are no-ops and the measure equals
    the oracle's single-process measure."""
    import torch
    from deep_frame_b200.distributed import ShardedMeasure
    ref = _oracle_reference()
    shape, system, model, density = _problem()
    moduli, derivative = system.moduli(density, 3.0, 1e-9)
    rows, _ = ShardedMeasure(_groups(model), model.rank, model.factor, OracleOps(shape, system, moduli)).measure(torch.as_tensor(-derivative))
    assert rows[0]["value"] == pytest.approx(ref["load_mean"], rel=1e-12)
    assert rows[1]["value"] == pytest.approx(ref["load_worst"], rel=1e-12)
    assert rows[1]["info"]["ks_n_mm"] == pytest.approx(ref["ks"], rel=1e-12)
    assert np.linalg.norm(rows[1]["gradient"].numpy() - ref["grad_worst"]) < 1e-10 * np.linalg.norm(ref["grad_worst"])


def test_sharded_measure_matches_single_process_oracle():
    ref = _oracle_reference()
    world, port = 2, _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    assert out[0][4] == [21, 21] and out[1][4] == [21, 21]    # 42 directions per half, split evenly
    for rank in (0, 1):
        tr, lam, gm, gw, _ = out[rank]
        assert tr == pytest.approx(ref["load_mean"], rel=1e-12)
        assert lam == pytest.approx(ref["load_worst"], rel=1e-12)
        assert np.linalg.norm(gm - ref["grad_mean"]) < 1e-10 * np.linalg.norm(ref["grad_mean"])
        assert np.linalg.norm(gw - ref["grad_worst"]) < 1e-10 * np.linalg.norm(ref["grad_worst"])
