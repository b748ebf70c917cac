"""Porosity tracers (kernels.py:3182-3255).

Advection is pinned to the reference through the ``tracers`` kernel fixture
(every kernel case runs on the oracle and on the GPU).  Injection draws its
offsets from a counter-based hash instead of ti.random(), so it is checked by
its properties on the oracle and bit for bit between the GPU and the oracle.
"""
import numpy as np
import pytest

from cases import OracleBackend


def _oracle_inject(m, head, seed, count=50, arc=(1e-3, 2e-3, 5e-4), sigma=3e-4):
    O = OracleBackend().O
    pos = np.zeros((m, 3), np.float32)
    act = np.zeros(m, np.int32)
    h = np.array([head], np.int32)
    O.call("wo_inject_tracers", pos, act, h, m, arc[0], arc[1], arc[2], sigma, count, seed)
    return pos, act, int(h[0])


def test_inject_fills_ring_slots_within_the_footprint():
    m = 64
    pos, act, head = _oracle_inject(m, head=40, seed=7)
    assert head == 90
    slots = [(40 + t) % m for t in range(50)]
    assert np.all(act[slots] == 1) and act.sum() == 50
    assert np.all(np.abs(pos[slots, 0] - np.float32(1e-3)) <= np.float32(3e-4) * 1.0001)
    assert np.all(np.abs(pos[slots, 1] - np.float32(2e-3)) <= np.float32(3e-4) * 1.0001)
    assert np.all(pos[slots, 2] == np.float32(5e-4))
    # different seeds give different offsets, the same seed the same ones
    pos2, _, _ = _oracle_inject(m, head=40, seed=8)
    pos3, _, _ = _oracle_inject(m, head=40, seed=7)
    assert not np.array_equal(pos, pos2) and np.array_equal(pos, pos3)
    # offsets cover the square roughly uniformly
    big, _, _ = _oracle_inject(4096, head=0, seed=3, count=4096)
    dxs = (big[:, 0] - np.float32(1e-3)) / np.float32(3e-4)
    assert abs(float(dxs.mean())) < 0.05 and 0.30 < float(dxs.var()) < 0.37


@pytest.mark.gpu
@pytest.mark.parametrize("head,count,m", [(0, 50, 64), (40, 50, 64), (1000, 300, 512)])
def test_gpu_inject_matches_oracle(head, count, m):
    import torch
    from waam_solver_b200 import kernels
    want_pos, want_act, want_head = _oracle_inject(m, head=head, seed=11, count=count)
    pos = torch.zeros((m, 3), dtype=torch.float32, device="cuda")
    act = torch.zeros(m, dtype=torch.int32, device="cuda")
    h = torch.full((), head, dtype=torch.int32, device="cuda")
    kernels.inject_tracers(pos, act, h, m, 1e-3, 2e-3, 5e-4, 3e-4, count, seed=11)
    torch.cuda.synchronize()
    assert int(h.item()) == want_head
    assert np.array_equal(act.cpu().numpy(), want_act)
    assert np.array_equal(pos.cpu().numpy(), want_pos)
