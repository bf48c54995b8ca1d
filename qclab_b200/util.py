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
