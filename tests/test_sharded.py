"""Hash-owner sharding of one sum (ppvm_b200.sharded) on CPU ranks (gloo), no GPU.

The step plan is checked directly.  The exchange protocol runs on two ranks with the oracle
as each rank's engine (a test-side share with the same export / append / run methods as the
device share): the ranks' terms together must equal the unsharded oracle's term for term,
coefficients bit for bit, and <O> to 1e-12.  That holds only if every pair of keys a step
can merge sits on one rank when the step runs.  The device share (the CUDA partition and
append kernels) is exercised by tests/test_gpu_sharded.py."""

import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from ppvm_b200 import gates as G  # noqa: E402
from ppvm_b200.sharded import plan  # noqa: E402


def test_plan_cuts_at_merging_steps_with_their_flip_bits():
    ops = [G.g1(G.H, 0), G.r1(G.RX, 1, 0.3), G.r1(G.RX, 2, 0.3), G.r1(G.RX, 1, 0.2), G.truncate(),
           G.r2(G.RZZ, 0, 3, -np.pi / 2), G.r2(G.RZZ, 0, 3, 0.4), G.amplitude_damping(70, 0.1),
           G.r1(G.RY, 65, 0.1), G.pauli_error(2, (0.1, 0.0, 0.0))]
    steps = plan(ops, 80, clifford_angles=True)
    assert [len(s.ops) for s in steps] == [1, 2, 3, 1, 1, 2]
    assert steps[0].mask_x is None                        # H alone: nothing to merge yet
    assert steps[1].mask_x.tolist() == [0b110, 0] and steps[1].mask_z.tolist() == [0, 0]  # RX run on 1, 2
    assert steps[2].mask_x.tolist() == [0b10, 0]          # RX(1) again starts a new run
    assert steps[3].mask_z.tolist() == [0b1001, 0]        # RZZ(0.4): Z bits of both qubits
    assert steps[4].mask_z.tolist() == [0, 1 << 6]        # damping on 70: its Z bit
    assert steps[5].mask_x.tolist() == [0, 2] and steps[5].mask_z.tolist() == [0, 2]  # RY on 65
    with pytest.raises(ValueError):
        plan([G.loss_channel(0, 0.1)], 4)


class OracleShare:
    """A rank's share held by the oracle; owner = a hash of the masked key."""

    def __init__(self, n, thr, maxw, clifford_angles, terms=None):
        from oracle.pyoracle import OracleSum

        self.args = (n, thr, maxw, clifford_angles)
        self.W = G.words(n)
        self.o = OracleSum(*self.args)
        if terms is not None:
            self.o.add_terms(*terms)

    def export(self, mask_x, mask_z, nparts):
        import torch
        from oracle.pyoracle import OracleSum

        x, z, c = self.o.export()
        kx, kz = x & ~mask_x, z & ~mask_z
        h = np.zeros(len(c), dtype=np.uint64)
        for w in range(self.W):
            h = (h ^ kx[:, w]) * np.uint64(0x9E3779B97F4A7C15)
            h = (h ^ kz[:, w]) * np.uint64(0xC2B2AE3D27D4EB4F)
        owner = ((h >> np.uint64(40)) % np.uint64(nparts)).astype(np.int64)
        order = np.argsort(owner, kind="stable")
        rows = np.concatenate([x, z, c.view(np.uint64)[:, None]], axis=1)[order]
        self.o = OracleSum(*self.args)
        return torch.from_numpy(rows.view(np.int64).reshape(-1).copy()), np.bincount(owner, minlength=nparts)

    def append(self, rows):
        r = rows.numpy().view(np.uint64).reshape(-1, 2 * self.W + 1)
        if len(r):
            self.o.add_terms(r[:, :self.W].copy(), r[:, self.W:2 * self.W].copy(), r[:, 2 * self.W].view(np.float64).copy())

    def run(self, ops):
        self.o.run_ops(ops)

    def overlap_with_zero(self):
        return self.o.overlap_with_zero()

    def __len__(self):
        return len(self.o)

    def export_terms(self):
        return self.o.export()


def _circuits():
    from ppvm_b200 import circuits as C

    ki = C.kicked_ising_2d(L=4, layers=3, thr=1e-6, max_weight=8)
    rng = np.random.default_rng(5)
    hot = [0, 1, 2, 3, 4, 5, 64, 65, 66, 67, 68, 69]  # both words of the 70-qubit planes
    mixed = []
    for i in range(60):
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
    return [("kicked", ki.n_qubits, ki.observable[0][0], ki.ops, ki.min_abs_coeff, ki.max_weight, True),
            ("mixed", 70, obs, mixed, 1e-5, None, False)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from ppvm_b200.sharded import ShardedPauliSum

        out = {}
        for name, n, word, ops, thr, maxw, ca in _circuits():
            x, z = G.parse_word(word, n)
            terms = (x[None], z[None], np.array([1.0])) if rank == 0 else None
            s = ShardedPauliSum(OracleShare(n, thr, maxw, ca, terms), n, ca)
            s.run(ops)
            gx, gz, gc = s.gather_terms()
            out[name] = {"owz": s.overlap_with_zero(), "len": len(s), "exchanges": s.exchanges,
                         "moved": s.rows_moved, "mine": len(s.share),
                         "terms": sorted(zip(map(lambda r: r.tobytes().hex(), np.concatenate([gx, gz], 1)),
                                             gc.view(np.uint64).tolist()))}
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_hold_the_unsharded_term_set(tmp_path, world):
    import torch.multiprocessing as mp

    from oracle.pyoracle import OracleSum

    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for name, n, word, ops, thr, maxw, ca in _circuits():
        o = OracleSum(n, thr, maxw, ca)
        x, z = G.parse_word(word, n)
        o.add_terms(x[None], z[None], np.array([1.0]))
        o.run_ops(ops)
        ox, oz, oc = o.export()
        want = sorted(zip(map(lambda r: r.tobytes().hex(), np.concatenate([ox, oz], 1)), oc.view(np.uint64).tolist()))
        for r in res:
            got = r[name]
            assert [tuple(t) for t in got["terms"]] == want, name
            assert got["len"] == len(want)
            assert abs(got["owz"] - o.overlap_with_zero()) < 1e-12
            assert got["exchanges"] > 0
        # both ranks hold terms, and terms really moved between them
        assert all(r[name]["mine"] > 0 for r in res), name
        assert sum(r[name]["moved"] for r in res) > 0, name
        assert sum(r[name]["mine"] for r in res) == len(want)
