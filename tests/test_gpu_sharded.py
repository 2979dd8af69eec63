"""Hash-owner sharding on the GPU: one sum spread over two ranks (ppvm_b200.sharded), each a
process on this box's GPU, exchanging rows through gloo on the host.  The ranks run the
CUDA partition (k_shard_hist / k_shard_scan / k_shard_scatter) and append (k_shard_append)
kernels of ppvm_sum_shard_export / ppvm_sum_shard_append; their kernels never wait on each
other.  Their terms together must equal the single-GPU engine's term set, every coefficient
bit for bit, with <O> within 1e-10.  The NCCL path differs only in moving device tensors and
needs one GPU per rank."""

import hashlib
import json
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _cases():
    from ppvm_b200 import circuits as C
    from ppvm_b200 import gates as G

    ki = C.kicked_ising_2d(L=12, layers=4, theta_h=0.6, thr=1e-5, max_weight=10)
    rng = np.random.default_rng(9)
    hot = [0, 1, 2, 3, 4, 5, 64, 65, 66, 67, 68, 69]
    mixed = []
    for i in range(80):
        a = int(rng.integers(len(hot)))
        q, p = hot[a], hot[(a + 1 + int(rng.integers(len(hot) - 1))) % len(hot)]
        k = i % 6
        if k == 0:
            mixed.append(G.r1(G.RX, q, 0.3))
        elif k == 1:
            mixed.append(G.r2(G.RZZ, q, p, 0.5))
        elif k == 2:
            mixed.append(G.r1(G.RY, q, -0.4))
        elif k == 3:
            mixed.append(G.g2(G.CNOT, q, p))
        elif k == 4:
            mixed.append(G.amplitude_damping(q, 0.05))
        else:
            mixed.append(G.r2(G.RXX, q, p, 0.2))
        if i % 4 == 3:
            mixed.append(G.truncate())
    obs = "".join("XYZ"[int(rng.integers(3))] if j in hot[::2] else "I" for j in range(70))
    return [("kicked_ising_12x12_4_layers", ki.n_qubits, ki.observable[0][0], ki.ops, ki.min_abs_coeff,
             ki.max_weight, True),
            ("mixed_70", 70, obs, mixed, 1e-6, None, False)]


def _digest(x, z, c):
    """Hash of the term set: rows (x, z, coefficient bits) in sorted order."""
    rows = np.concatenate([x, z, c.view(np.uint64)[:, None]], axis=1)
    rows = rows[np.lexsort(rows.T[::-1])]
    return hashlib.sha256(rows.tobytes()).hexdigest()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from ppvm_b200.sharded import sharded_sum

        out = {}
        for name, n, word, ops, thr, maxw, ca in _cases():
            s = sharded_sum([word], n, [1.0], min_abs_coeff=thr, max_pauli_weight=maxw, clifford_angles=ca, device=0)
            s.run(ops)
            x, z, c = s.gather_terms()
            out[name] = {"digest": _digest(x, z, c), "len": len(s), "owz": s.overlap_with_zero(),
                         "exchanges": s.exchanges, "moved": s.rows_moved, "mine": len(s.share)}
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_hold_the_single_gpu_term_set(tmp_path):
    import torch.multiprocessing as mp

    from ppvm_b200.paulisum import PauliSum

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for name, n, word, ops, thr, maxw, ca in _cases():
        one = PauliSum([word], n, [1.0], min_abs_coeff=thr, max_pauli_weight=maxw, clifford_angles=ca)
        one.run(ops)
        want = _digest(*one.export())
        for r in res:
            got = r[name]
            assert got["digest"] == want, name
            assert got["len"] == len(one), name
            assert abs(got["owz"] - one.overlap_with_zero()) < 1e-10, name
            assert got["exchanges"] > 0
        assert all(r[name]["mine"] > 0 for r in res), name
        assert sum(r[name]["moved"] for r in res) > 0, name
        assert sum(r[name]["mine"] for r in res) == len(one)


def test_export_and_append_round_trip_on_one_rank():
    # one part: every row comes back in the sum's own order; the sum is empty in between
    import ctypes

    import torch

    from ppvm_b200 import circuits as C
    from ppvm_b200.sharded import DeviceShare
    from ppvm_b200.paulisum import PauliSum

    wl = C.kicked_ising_2d(L=6, layers=2, thr=1e-6, max_weight=8)
    s = PauliSum([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=wl.min_abs_coeff,
                 max_pauli_weight=wl.max_weight, clifford_angles=True)
    s.run(wl.ops)
    before = s.export()
    share = DeviceShare(s)
    W = share.W
    rows, counts = share.export(np.zeros(W, np.uint64), np.zeros(W, np.uint64), 1)
    assert len(s) == 0 and counts.tolist() == [len(before[2])]
    share.append(rows)
    after = s.export()
    for u, v in zip(before, after):
        assert np.array_equal(np.asarray(u).view(np.uint64), np.asarray(v).view(np.uint64))
    # four parts: counts add up, and each part's rows are a contiguous slice
    rows, counts = share.export(np.zeros(W, np.uint64), np.zeros(W, np.uint64), 4)
    assert int(counts.sum()) == len(before[2]) and (counts > 0).all()
    share.append(rows)
    assert _digest(*s.export()) == _digest(*before)
    from ppvm_b200._lib import lib
    with pytest.raises(ValueError):
        share._check(lib().ppvm_sum_shard_export(s.handle, None, None, 33, ctypes.c_void_p(rows.data_ptr()),
                                                 len(s), None))
    torch.cuda.synchronize()
