"""``ShardedPauliSum``: one PauliSum spread over the ranks of a ``torch.distributed`` group.

Every key lives on exactly one rank.  A gate list is cut into steps.  A step starts with the
ops that merge keys (a run of RX or of RZ rotations on distinct qubits, any other rotation,
amplitude damping) and goes on with the ops that do not (Cliffords, Clifford-angle rotations,
Pauli-error and depolarising channels, TRUNCATE).  The keys a step merges differ only in its
flip bits: the X bits of an RX run's qubits, the Z bits of an RZ run's, a rotation's
generator bits, the Z bit of a damped qubit.  So before each step the ranks send every term
to the owner of its key with those bits cleared, which puts every pair of keys the step can
merge on one rank.  Each rank then runs the step with the single-sum engine
(``ppvm_sum_shard_export`` / all-to-all / ``ppvm_sum_shard_append`` in include/ppvm_cuda.h).

A merge adds at most two contributions, and a fused run's group sits on one rank, so every
coefficient is the same IEEE value as on one GPU: the ranks together hold the single-GPU
engine's term set (term order aside).  ``overlap_with_zero`` adds the ranks' partial sums, so
it agrees to rounding (1e-10 in the tests), not bit for bit.

The reference keeps a sum in one process and has no counterpart.  Lossy sums and loss
channels are not sharded here.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import gates as G
from ._lib import EINVAL, OK, PPVMError, lib

_HALF_PI = 1.5707963267948966

# generator flip bits of a rotation: (x bits, z bits) on each of its qubits
_ROT_FLIPS = {G.RX: (1, 0), G.RY: (1, 1), G.RZ: (0, 1), G.RXX: (1, 0), G.RYY: (1, 1), G.RZZ: (0, 1)}
_TWO = {G.RXX, G.RYY, G.RZZ}


@dataclass
class Step:
    """Ops run on every rank alone after the terms moved to their owners under the mask
    (mask None: no exchange needed, the step merges nothing)."""
    mask_x: np.ndarray | None
    mask_z: np.ndarray | None
    ops: list = field(default_factory=list)


def _merging(op, clifford_angles: bool) -> bool:
    code = op[0]
    if code in _ROT_FLIPS:
        return not (clifford_angles and abs(op[3]) == _HALF_PI)
    return code == G.AMPLITUDE_DAMPING


def plan(ops, n_qubits: int, clifford_angles: bool = False) -> list[Step]:
    """The steps of a gate list (``ppvm_b200.gates`` tuples) for a sharded sum."""
    W = G.words(n_qubits)

    def setbit(m, q):
        m[q // 64] |= np.uint64(1) << np.uint64(q % 64)

    steps: list[Step] = []
    i = 0
    while i < len(ops):
        op = ops[i]
        if op[0] in (G.LOSS_CHANNEL, G.RESET_LOSS_CHANNEL, G.CORRELATED_LOSS_CHANNEL):
            raise ValueError("loss channels need a lossy sum, which is not sharded")
        if not _merging(op, clifford_angles):
            if not steps:
                steps.append(Step(None, None))
            steps[-1].ops.append(op)
            i += 1
            continue
        mx = np.zeros(W, dtype=np.uint64)
        mz = np.zeros(W, dtype=np.uint64)
        if op[0] in (G.RX, G.RZ):  # a run of RX (or RZ) rotations on distinct qubits
            seen = set()
            j = i
            while (j < len(ops) and ops[j][0] == op[0] and ops[j][1] not in seen
                   and _merging(ops[j], clifford_angles)):
                seen.add(ops[j][1])
                setbit(mx if op[0] == G.RX else mz, ops[j][1])
                j += 1
            steps.append(Step(mx, mz, list(ops[i:j])))
            i = j
            continue
        if op[0] == G.AMPLITUDE_DAMPING:
            setbit(mz, op[1])
        else:
            fx, fz = _ROT_FLIPS[op[0]]
            for q in ((op[1], op[2]) if op[0] in _TWO else (op[1],)):
                if fx:
                    setbit(mx, q)
                if fz:
                    setbit(mz, q)
        steps.append(Step(mx, mz, [op]))
        i += 1
    return steps


class DeviceShare:
    """A rank's share of the sum: a ``PauliSum`` on its GPU, with the row exchange of the C
    ABI.  Rows are 2W+1 signed 64-bit words (x[W], z[W], the coefficient's bits)."""

    def __init__(self, local, device: int = 0):
        import torch

        self.s = local
        self.W = local.W
        self.device = torch.device("cuda", device)

    def _check(self, st):
        if st != OK:
            msg = lib().ppvm_last_error_string().decode(errors="replace")
            raise ValueError(msg) if st == EINVAL else PPVMError(st, msg)

    def export(self, mask_x, mask_z, nparts: int):
        """Every term as a row, grouped by owner; the share is left empty.  Returns (rows as a
        flat int64 device tensor, counts per owner)."""
        import torch

        n = len(self.s)
        R = 2 * self.W + 1
        rows = torch.empty(max(n, 1) * R, dtype=torch.int64, device=self.device)
        counts = np.zeros(nparts, dtype=np.uint64)
        mx = np.ascontiguousarray(mask_x, dtype=np.uint64)
        mz = np.ascontiguousarray(mask_z, dtype=np.uint64)
        p64 = ctypes.POINTER(ctypes.c_uint64)
        self._check(lib().ppvm_sum_shard_export(self.s.handle, mx.ctypes.data_as(p64), mz.ctypes.data_as(p64),
                                                nparts, ctypes.c_void_p(rows.data_ptr()), n,
                                                counts.ctypes.data_as(p64)))
        return rows[: n * R], counts.astype(np.int64)

    def append(self, rows) -> None:
        import torch

        k = rows.numel() // (2 * self.W + 1)
        if k == 0:
            return
        rows = rows.to(self.device).contiguous()
        torch.cuda.current_stream(self.device).synchronize()  # the rows are complete
        self._check(lib().ppvm_sum_shard_append(self.s.handle, ctypes.c_void_p(rows.data_ptr()), k))

    def run(self, ops) -> None:
        self.s.run(ops)

    def overlap_with_zero(self) -> float:
        return self.s.overlap_with_zero()

    def __len__(self) -> int:
        return len(self.s)

    def export_terms(self):
        return self.s.export()


class ShardedPauliSum:
    """One sum spread over the ranks of ``group``.  ``share`` is this rank's part: a
    ``DeviceShare`` (or any object with the same export / append / run / overlap_with_zero /
    len / export_terms methods).  Rank 0's share starts with the initial terms, the other
    ranks' start empty, and the first step moves every term to its owner."""

    def __init__(self, share, n_qubits: int, clifford_angles: bool = False, group=None):
        import torch.distributed as dist

        self.share = share
        self.n_qubits = int(n_qubits)
        self.clifford_angles = clifford_angles
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.host_staging = dist.get_backend(group) != "nccl"  # gloo moves host tensors
        self.exchanges = 0
        self.rows_moved = 0  # rows this rank sent to other ranks

    def _all_to_all(self, rows, counts):
        """Sends owner p's rows (counts[p] of them, in order) to rank p; returns the rows
        this rank receives (flat int64 tensor, on the host with gloo, else on the device)."""
        import torch
        import torch.distributed as dist

        R = 2 * self.share.W + 1
        dev = rows.device if not self.host_staging else torch.device("cpu")
        send_counts = torch.tensor(counts, dtype=torch.int64, device=dev)
        recv_counts = torch.empty_like(send_counts)
        dist.all_to_all_single(recv_counts, send_counts, group=self.group)
        recv_n = recv_counts.tolist()
        send = rows.to(dev) if self.host_staging else rows
        recv = torch.empty(int(sum(recv_n)) * R, dtype=torch.int64, device=dev)
        dist.all_to_all_single(recv, send, output_split_sizes=[c * R for c in recv_n],
                               input_split_sizes=[int(c) * R for c in counts], group=self.group)
        self.exchanges += 1
        self.rows_moved += int(sum(counts)) - int(counts[self.rank])
        return recv

    def redistribute(self, mask_x, mask_z) -> None:
        """Every term to the owner of its key with the mask bits cleared."""
        rows, counts = self.share.export(mask_x, mask_z, self.world)
        self.share.append(self._all_to_all(rows, counts))

    def run(self, ops) -> None:
        """Applies a gate list (Heisenberg order, ``ppvm_b200.gates`` tuples)."""
        for step in plan(list(ops), self.n_qubits, self.clifford_angles):
            if step.mask_x is not None and self.world > 1:
                self.redistribute(step.mask_x, step.mask_z)
            self.share.run(step.ops)

    def _allreduce(self, v: float, dtype) -> float:
        import torch
        import torch.distributed as dist

        dev = "cpu" if self.host_staging else self.share.device
        t = torch.tensor([v], dtype=dtype, device=dev)
        dist.all_reduce(t, group=self.group)
        return t.item()

    def overlap_with_zero(self) -> float:
        """The ranks' partial sums added (agrees with one GPU to rounding)."""
        import torch

        return self._allreduce(self.share.overlap_with_zero(), torch.float64)

    def __len__(self) -> int:
        import torch

        return int(self._allreduce(float(len(self.share)), torch.float64))

    def gather_terms(self):
        """Every rank's terms on every rank, as (x, z, c) arrays (for checks on small sums)."""
        import torch.distributed as dist

        mine = [np.asarray(a) for a in self.share.export_terms()]
        parts = [None] * self.world
        dist.all_gather_object(parts, mine, group=self.group)
        return tuple(np.concatenate([p[k] for p in parts]) for k in range(3))


def sharded_sum(initial_terms, n_qubits: int, coefficients=(), min_abs_coeff: float = 1e-10,
                max_pauli_weight: int | None = None, *, clifford_angles: bool = False, group=None,
                device: int = 0) -> ShardedPauliSum:
    """A sum over the ranks of ``group`` on this rank's GPU ``device``: every rank calls it
    with the same arguments."""
    import torch.distributed as dist

    from .paulisum import PauliSum

    local = PauliSum(list(initial_terms), n_qubits, list(coefficients), min_abs_coeff=min_abs_coeff,
                     max_pauli_weight=max_pauli_weight, clifford_angles=clifford_angles, device=device)
    share = DeviceShare(local, device)
    if dist.get_rank(group) != 0:  # the initial terms live on rank 0 only
        W = share.W
        share.export(np.zeros(W, dtype=np.uint64), np.zeros(W, dtype=np.uint64), 1)
    return ShardedPauliSum(share, n_qubits, clifford_angles, group)


__all__ = ["DeviceShare", "ShardedPauliSum", "Step", "plan", "sharded_sum"]
