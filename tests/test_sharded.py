"""One state split over 2, 4 and 8 ranks (``qclab_b200.sharded``): the gate
list runs on the local states with pairwise half-state exchanges for gates
on the ranks' qubits, and the state downloaded in logical order must equal
the oracle applied to the whole vector.  On CPU the ranks are gloo
processes whose local engine is the C oracle (this tests the qubit map,
the exchanges and the gate rewriting); the GPU test runs the same on two
gloo processes sharing cuda:0 with the library as the local engine (the
ranks meet only on the host, no kernel waits for another process).
Tolerance 1e-13 for the reference-exact path: an exchange only moves
amplitudes, but a two-qubit gate whose qubits swap order under the map forms
its sums in the other order (measured differences about 1e-16)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from qclab_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleEngine:
    """Local engine for the CPU test: the C oracle on the rank's buffer."""

    def __init__(self, buf, n, dtype):
        self.x = buf.numpy()   # shares the tensor's memory

    def apply(self, recs, op, fused):
        oracle.apply(self.x, recs, op)

    def norm2(self):
        return float(np.vdot(self.x, self.x).real)

    def expectation(self, paulis, coefs):
        return oracle.expectation(self.x, list(zip(coefs, paulis)))

    def synchronize(self):
        pass

    def close(self):
        pass


def _circuit(n, seed):
    c = W.random_mixed(n, 90, seed=seed)
    return c.gate_records(np.complex128)


def _observable(n):
    """Ising chain plus strings with X, Y and Z on the ranks' top qubits."""
    from qclab_b200.observable import ising
    H = ising(n)
    rng = np.random.default_rng(9)
    for _ in range(8):
        t = ["I"] * n
        for q in rng.choice(n, size=4, replace=False):
            t[q] = "XYZ"[rng.integers(3)]
        H.add(float(rng.normal()), "".join(t))
    H.add(0.7, "XY" + "Z" * (n - 2))
    H.add(-0.3, "ZZZ" + "X" * (n - 3))
    return H


def _rank_main(rank, world, port, out, n, use_gpu):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from qclab_b200.sharded import ShardedStateVector
        res = {}
        rng = np.random.default_rng(3)
        x0 = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        x0 /= np.linalg.norm(x0)
        recs = _circuit(n, 11)
        kw = {} if use_gpu else {"engine": OracleEngine, "device": "cpu"}
        for op in ("N", "T", "C"):
            for fused in ((False, True) if use_gpu else (False,)):
                with ShardedStateVector(n, np.complex128, **kw) as s:
                    s.upload(x0)
                    s.apply(recs, op, fused=fused)
                    n2 = s.norm2()
                    e = s.expectation(_observable(n))
                    y = s.download()
                    if rank == 0:
                        res[(op, fused)] = (y, n2, s.exchanges, e)
        with ShardedStateVector(n, np.complex128, **kw) as s:   # |0...0> start
            s.apply(recs[:30], "N")
            y = s.download()
            if rank == 0:
                res["zero"] = y
            # a term with more X/Y factors than local qubits is refused on
            # every rank alike (before any exchange for it)
            from qclab_b200.observable import Observable
            try:
                s.expectation(Observable(n).add(1.0, "X" * n))
                res["wide"] = "accepted"
            except ValueError:
                res["wide"] = "refused"
            try:
                ShardedStateVector(world.bit_length() + 1, np.complex128, **kw)
                res["small"] = "accepted"
            except ValueError:
                res["small"] = "refused"
        if rank == 0:
            out.update({str(k): v for k, v in res.items()})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world, n, use_gpu):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out, n, use_gpu), nprocs=world,
                           join=True, start_method="spawn")
        return dict(out)


def _expected(n, op, x0=None):
    if x0 is None:
        rng = np.random.default_rng(3)
        x0 = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        x0 /= np.linalg.norm(x0)
    return oracle.apply(x0.copy(), _circuit(n, 11), op)


@pytest.mark.parametrize("world, n", [(2, 7), (4, 7), (8, 8)])
def test_sharded_state_matches_whole_vector(world, n):
    res = _run(world, n, use_gpu=False)
    for op in ("N", "T", "C"):
        y, n2, ex, e = res[str((op, False))]
        want = _expected(n, op)
        assert np.max(np.abs(y - want)) <= 1e-13, op
        assert ex > 0                      # the circuit touches the ranks' qubits
        assert abs(n2 - float(np.vdot(want, want).real)) < 1e-12
        e_want = oracle.expectation(want, _observable(n).matrix_free_terms())
        assert abs(e - e_want) <= 1e-12 * max(1.0, abs(e_want)), (op, e, e_want)
    z = np.zeros(1 << n, dtype=np.complex128)
    z[0] = 1
    assert np.max(np.abs(res["zero"] - oracle.apply(z, _circuit(n, 11)[:30], "N"))) <= 1e-13
    assert res["wide"] == "refused"     # n X factors, n - g local qubits
    assert res["small"] == "refused"    # fewer than 3 local qubits


def test_sharded_rejects_bad_sizes():
    import torch.distributed as dist
    from qclab_b200.sharded import _log2_exact
    assert _log2_exact(4) == 2
    with pytest.raises(ValueError):
        _log2_exact(6)
    assert not dist.is_initialized()


@pytest.mark.gpu
def test_sharded_state_on_the_gpu(cuda):
    n = 12
    res = _run(2, n, use_gpu=True)
    for op in ("N", "T", "C"):
        want = _expected(n, op)
        y, n2, ex, e = res[str((op, False))]
        assert np.max(np.abs(y - want)) <= 1e-13, op
        assert ex > 0
        e_want = oracle.expectation(want, _observable(n).matrix_free_terms())
        assert abs(e - e_want) <= 1e-12 * max(1.0, abs(e_want)), (op, e, e_want)
        yf, _, _, _ = res[str((op, True))]
        assert np.max(np.abs(yf - want)) <= 1e-12, op
