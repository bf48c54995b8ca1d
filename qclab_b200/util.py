"""Enumerations of ``include/qclab/util.hpp:15-30``."""
from __future__ import annotations

import enum


class Op(str, enum.Enum):
    """Operation applied to each gate: NoTrans, Trans or ConjTrans."""
    NoTrans = "N"
    Trans = "T"
    ConjTrans = "C"


class Side(str, enum.Enum):
    Left = "L"
    Right = "R"


def as_op(op) -> "Op":
    if isinstance(op, Op):
        return op
    if isinstance(op, str) and op in ("N", "T", "C"):
        return Op(op)
    raise ValueError(f"op must be Op.NoTrans/Trans/ConjTrans or 'N'/'T'/'C', got {op!r}")


def state_summary(chunks, n: int, idx, blocks: int = 256) -> dict:
    """A state's SHA-256 digest (of its bytes in index order), FP64 norm^2,
    the amplitudes at the sorted indices ``idx`` and the FP64 sum of
    |a_i|^2 over each of ``blocks`` equal contiguous blocks, from the state
    given as consecutive chunks (numpy arrays covering 2^n elements in order,
    each a whole number of blocks).  The same numpy reductions run on the
    same block data wherever the chunks come from, so two summaries of
    equal states are equal bit for bit."""
    import hashlib

    import numpy as np
    h = hashlib.sha256()
    bs = (1 << n) // blocks
    idx = np.asarray(idx, dtype=np.int64)
    amps = []
    block_p = []
    start = 0
    for c in chunks:
        if c.size % bs:
            raise ValueError("chunks must hold whole blocks")
        h.update(memoryview(np.ascontiguousarray(c)).cast("B"))
        for b in range(0, c.size, bs):
            seg = c[b:b + bs]
            block_p.append(float(np.sum(seg.real.astype(np.float64) ** 2 +
                                        seg.imag.astype(np.float64) ** 2)))
        sel = idx[(idx >= start) & (idx < start + c.size)]
        amps.append(c[sel - start].copy())
        start += c.size
    if start != 1 << n:
        raise ValueError("chunks do not cover the state")
    p = np.array(block_p)
    return {"sha256": h.hexdigest(), "norm2": float(p.sum()), "idx": idx,
            "amp": np.concatenate(amps) if amps else np.zeros(0), "block_p": p}
