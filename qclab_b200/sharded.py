"""One state vector split over the ranks of a process group.

A state of n qubits on W = 2^g ranks: rank r holds the 2^(n-g) amplitudes
whose global index has r in its top g bits (QCLAB++ numbering: qubit 0 is
the most significant bit, so physical slots 0..g-1 are the rank's bits and
slots g..n-1 are the local state's qubits 0..n-g-1).  The reference keeps
the whole vector in one address space (``QCircuit::simulate``,
include/qclab/QCircuit.hpp:130-166, index bits of ``masks`` in
src/qgates/apply.hpp:227-256); this splits it on its top qubits.

Gates whose qubits all sit in local slots run on the local state through the
library (consecutive ones as one ``qsv_apply`` / ``qsv_apply_fused`` call).
A gate on a qubit in a global slot first brings that qubit into the local
state: the qubit in global slot p and the one in the local state's top slot
change places by one pairwise exchange -- every rank sends the half of its
local state whose top bit differs from its own bit p to the rank that
differs from it in bit p, and receives that rank's matching half (a
contiguous half either way).  The logical-qubit -> slot map records the
moves; ``download`` returns the state in logical order.

Transport: over NCCL the halves move device to device (each rank's own
buffers, no peer memory in any kernel); over gloo they are staged through
host memory.  Every rank takes the same exchanges in the same order (the
plan depends only on the gate list), so collectives always match.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .state import StateVector, to_records

_TORCH_DTYPE = {np.dtype(np.complex64): "complex64", np.dtype(np.complex128): "complex128"}


def _log2_exact(w: int) -> int:
    g = int(w).bit_length() - 1
    if w < 1 or (1 << g) != w:
        raise ValueError(f"the group size {w} is not a power of two")
    return g


class CudaEngine:
    """The local state as a torch device buffer wrapped by the library
    (``qsv_wrap``), its kernels on the current torch stream (the stream NCCL
    orders against)."""

    def __init__(self, buf, nbQubits: int, dtype):
        import torch
        self.buf = buf
        self.sv = StateVector.wrap(buf.data_ptr(), nbQubits, dtype)
        self.sv.set_stream(torch.cuda.current_stream(buf.device).cuda_stream)

    def apply(self, records, op: str, fused: bool) -> None:
        self.sv.apply(records, op, 0, fused=fused)

    def norm2(self) -> float:
        return self.sv.norm2()

    def expectation(self, paulis, coefs) -> float:
        from .observable import Observable
        return self.sv.expectation(Observable(self.sv.nbQubits, zip(coefs, paulis)))

    def synchronize(self) -> None:
        self.sv.synchronize()

    def close(self) -> None:
        self.sv.close()


class ShardedStateVector:
    """An n-qubit state split over the ranks of ``group`` (default: the
    world group; its size must be a power of two, W = 2^g, with n - g >= 3).
    Created as |0...0>.

    ``engine`` makes the local engine from (buffer, local qubits, dtype):
    by default a ``CudaEngine`` on ``device`` (default cuda:LOCAL_RANK)."""

    def __init__(self, nbQubits: int, dtype=np.complex128, *, group=None, device=None,
                 engine=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.numpy_dtype = np.dtype(dtype)
        if self.numpy_dtype not in _TORCH_DTYPE:
            raise TypeError("sharded states are complex64 or complex128")
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.g = _log2_exact(self.world)
        self.n = int(nbQubits)
        self.nl = self.n - self.g
        if self.nl < 3:
            raise ValueError(f"{self.n} qubits on {self.world} ranks leave fewer than 3 local qubits")
        self.backend = dist.get_backend(group)
        tdt = getattr(torch, _TORCH_DTYPE[self.numpy_dtype])
        if device is None:
            import os
            device = (torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
                      if engine is None else torch.device("cpu"))
        self.device = torch.device(device)
        if self.device.type == "cuda":  # NCCL's point-to-point calls need the device current
            torch.cuda.set_device(self.device)
        self.buf = torch.zeros(1 << self.nl, dtype=tdt, device=self.device)
        self.stage = torch.empty(1 << (self.nl - 1), dtype=tdt, device=self.device)
        if self.rank == 0:
            self.buf[0] = 1
        self.engine = (engine or CudaEngine)(self.buf, self.nl, self.numpy_dtype)
        self.slot_of = list(range(self.n))   # logical qubit -> physical slot
        self.exchanges = 0

    # ---- the map ---------------------------------------------------------------
    def _qubit_at(self, slot: int) -> int:
        return self.slot_of.index(slot)

    def _swap_slots(self, a: int, b: int) -> None:
        qa, qb = self._qubit_at(a), self._qubit_at(b)
        self.slot_of[qa], self.slot_of[qb] = b, a

    # ---- data movement -----------------------------------------------------------
    def _exchange(self, p: int) -> None:
        """Global slot p <-> local slot g (the local state's top qubit): swap
        the half of the local state whose top bit differs from this rank's
        bit p with the rank that differs in bit p."""
        import torch
        dist = self.dist
        bit = self.g - 1 - p                      # rank bit of slot p
        partner = self.rank ^ (1 << bit)
        mine = (self.rank >> bit) & 1
        half = 1 << (self.nl - 1)
        part = self.buf[half:] if mine == 0 else self.buf[:half]
        self.engine.synchronize()
        if self.backend == "nccl":
            send, recv = torch.view_as_real(part), torch.view_as_real(self.stage)
        else:  # host staging
            send = torch.view_as_real(part).cpu()
            recv = torch.empty_like(send)
        peer = dist.get_global_rank(self.group, partner) if self.group is not None else partner
        ops = [dist.P2POp(dist.isend, send, peer, self.group),
               dist.P2POp(dist.irecv, recv, peer, self.group)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        if self.backend == "nccl":
            part.copy_(self.stage)
        else:
            part.copy_(torch.view_as_complex(recv).to(self.device))
        self._swap_slots(p, self.g)
        self.exchanges += 1

    def _local_swap(self, a: int, b: int) -> None:
        """Local slots a and b change qubits (a SWAP gate on the local state)."""
        rec = np.zeros(1, dtype=L.GATE_DTYPE)
        rec["kind"] = L.SWAP
        rec["qubit0"], rec["qubit1"], rec["control_state"] = a - self.g, b - self.g, 1
        self.engine.apply(rec, "N", False)
        self._swap_slots(a, b)

    # ---- gates -------------------------------------------------------------------
    def apply(self, records, op: str = "N", fused: bool = False) -> None:
        """``QCircuit::apply(op, n, vector)`` on the split state: gate order
        (reversed for 'T' and 'C', every gate transposed or adjoined by the
        library), logical qubits as in ``records``."""
        if op not in ("N", "T", "C"):
            raise ValueError("op is 'N', 'T' or 'C'")
        recs = to_records(records)
        for r in recs:
            for f in ("qubit0", "qubit1"):
                if r[f] >= self.n:
                    raise ValueError(f"gate on qubit {int(r[f])} of a {self.n}-qubit state")
        order = range(len(recs)) if op == "N" else range(len(recs) - 1, -1, -1)
        pending: list[np.ndarray] = []

        def flush():
            if pending:
                seg = np.concatenate(pending if op == "N" else pending[::-1])
                self.engine.apply(seg, op, fused)
                pending.clear()

        for i in order:
            r = recs[i:i + 1].copy()
            qs = [int(r[f][0]) for f in ("qubit0", "qubit1") if r[f][0] >= 0]
            for q in qs:
                p = self.slot_of[q]
                if p >= self.g:
                    continue
                flush()
                used = {self.slot_of[x] for x in qs}
                if self.g in used:  # the top local slot holds another qubit of this gate
                    t = next(s for s in range(self.g + 1, self.n) if s not in used)
                    self._local_swap(self.g, t)
                self._exchange(p)
            for f in ("qubit0", "qubit1"):
                if r[f][0] >= 0:
                    r[f] = self.slot_of[int(r[f][0])] - self.g
            pending.append(r)
        flush()

    # ---- reductions and host copies ----------------------------------------------------
    def expectation(self, obs) -> float:
        """<psi|H|psi> in FP64 for a Pauli sum (``observable.Observable`` on
        the logical qubits; a term may hold at most n - g X/Y factors).  A
        term's X and Y factors on qubits in global slots are first moved into
        the local state (the gates' exchanges); a Z on a global slot is this
        rank's sign.  Terms between two exchanges
        are evaluated by one library call on the local state; the ranks' sums
        are all-reduced."""
        import torch
        if obs.nbQubits != self.n:
            raise ValueError("observable and state sizes differ")
        total = 0.0
        loc_p: list[str] = []
        loc_c: list[float] = []

        def flush():
            nonlocal total
            if loc_p:
                total += self.engine.expectation(list(loc_p), list(loc_c))
                loc_p.clear()
                loc_c.clear()

        for coef, pstr in zip(obs.coefs, obs.paulis):
            support = [q for q, c in enumerate(pstr) if c != "I"]
            flips = [q for q in support if pstr[q] in "XY"]
            if len(flips) > self.nl:
                raise ValueError(f"a term with {len(flips)} X/Y factors does not fit "
                                 f"{self.nl} local qubits")
            for q in flips:
                p = self.slot_of[q]
                if p >= self.g:
                    continue
                flush()
                # the top local slot must not hold another X/Y qubit of the
                # term (a Z qubit may go to a rank's slot: it becomes a sign)
                used = {self.slot_of[x] for x in flips}
                if self.g in used:
                    t = next(s for s in range(self.g + 1, self.n) if s not in used)
                    self._local_swap(self.g, t)
                self._exchange(p)
            local = ["I"] * self.nl
            sign = 1.0
            for q in support:
                s = self.slot_of[q]
                if s >= self.g:
                    local[s - self.g] = pstr[q]
                elif (self.rank >> (self.g - 1 - s)) & 1:  # a Z on this rank's bit 1
                    sign = -sign
            loc_p.append("".join(local))
            loc_c.append(sign * coef)
        flush()
        t = torch.tensor([total], dtype=torch.float64,
                         device=self.device if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def norm2(self) -> float:
        """<psi|psi> in FP64: the local sums, then one all-reduce."""
        import torch
        t = torch.tensor([self.engine.norm2()], dtype=torch.float64,
                         device=self.device if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def download(self) -> np.ndarray | None:
        """The whole state in logical qubit order on rank 0 (None on the
        others); every rank must call it."""
        import torch
        self.engine.synchronize()
        local = torch.view_as_real(self.buf if self.backend == "nccl" else self.buf.cpu())
        parts = [torch.empty_like(local) for _ in range(self.world)] if self.rank == 0 else None
        self.dist.gather(local, parts, dst=self._global(0), group=self.group)
        if self.rank != 0:
            return None
        phys = torch.view_as_complex(torch.cat(parts)).cpu().numpy().astype(self.numpy_dtype)
        # axis k of the reshaped array is physical slot k (slot 0 = top bit);
        # logical qubit q sits on axis slot_of[q]
        t = phys.reshape((2,) * self.n).transpose(self.slot_of)
        return np.ascontiguousarray(t).reshape(-1)

    def upload(self, host: np.ndarray) -> None:
        """Every rank passes the whole state (logical order); each keeps its
        part, and the qubit map is reset."""
        import torch
        x = np.ascontiguousarray(host, dtype=self.numpy_dtype)
        if x.size != 1 << self.n:
            raise ValueError("host vector size does not match the state")
        self.engine.synchronize()
        lo = self.rank << self.nl
        self.buf.copy_(torch.from_numpy(x[lo:lo + (1 << self.nl)].copy()).to(self.device))
        self.slot_of = list(range(self.n))

    def _global(self, r: int) -> int:
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def close(self) -> None:
        if getattr(self, "engine", None) is not None:
            self.engine.close()
            self.engine = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
