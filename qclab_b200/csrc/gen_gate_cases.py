"""Writes gate_cases.inc: the two-level switch of the gate-specialised
stage kernel (apply_gates.cu) -- on the op kind, then on its register
position(s) -- for register passes of R = 3, 4 and 5 bits.

The kind and position indices are those of device_word (gate_plan.hpp):
one-qubit kinds, controlled kinds, two-qubit kinds, the scale, and the
gradient terms of two-vector sweeps.  Each case calls GX1(op<...>) (the op
on psi, and on lambda in two-vector sweeps) or GXR(kind, p) (a gradient
term); apply_gates.cu defines both.  Run after changing the op kinds:

    python qclab_b200/csrc/gen_gate_cases.py
"""
from pathlib import Path

KIND1 = ["G_H", "G_SHEAR", "G_SHEARO", "G_ISHEAR", "G_ISHEARO", "G_PHASE", "G_GEN2", "G_REAL2",
         "G_X", "G_Z"]
KIND2 = ["G_CX", "G_CGEN2", "G_CNEG", "G_CPH"]
KIND4 = ["G_SWAP", "G_ISWAP", "G_GEN4"]
KINDR = ["G_RDX", "G_RDY", "G_RDZ", "G_RDG"]


def nested(R: int) -> list[str]:
    out = ["switch (kind) {"]
    k0 = 0
    for k, name in enumerate(KIND1):
        out.append(f"case {k0 + k}: switch (sub) {{")
        for p in range(R):
            out.append(f"  case {p}: GX1((op1<{name}, {p}>)); break;")
        out.append("  default: __builtin_unreachable(); } break;")
    k0 += len(KIND1)
    for k, name in enumerate(KIND2):
        out.append(f"case {k0 + k}: switch (sub) {{")
        for t in range(R):
            for c in range(R):
                if t == c:
                    continue
                for cv in range(2):
                    out.append(f"  case {(t * R + c) * 2 + cv}: GX1((op2<{name}, {t}, {c}, {cv}>)); "
                               f"break;")
        out.append("  default: __builtin_unreachable(); } break;")
    k0 += len(KIND2)
    for k, name in enumerate(KIND4):
        out.append(f"case {k0 + k}: switch (sub) {{")
        for p0 in range(R):
            for p1 in range(p0):
                out.append(f"  case {p0 * R + p1}: GX1((op4<{name}, {p0}, {p1}>)); break;")
        out.append("  default: __builtin_unreachable(); } break;")
    k0 += len(KIND4)
    out.append(f"case {k0}: GX1(op_scale); break;")
    k0 += 1
    for k, name in enumerate(KINDR):
        if name == "G_RDG":  # any generator: masks in its coefficients, position 0
            out.append(f"case {k0 + k}: GXR({name}, 0); break;")
            continue
        out.append(f"case {k0 + k}: switch (sub) {{")
        for p in range(R):
            out.append(f"  case {p}: GXR({name}, {p}); break;")
        out.append("  default: __builtin_unreachable(); } break;")
    out.append("default: __builtin_unreachable();")
    out.append("}")
    return out


def main() -> None:
    lines = ["// Generated by gen_gate_cases.py -- do not edit.",
             "// Two-level op dispatch of apply_word (apply_gates.cu) for R = 3, 4, 5."]
    for R in (3, 4, 5):
        lines.append(f"#define QSV_GX_NESTED_{R} \\")
        body = nested(R)
        for i, c in enumerate(body):
            lines.append("  " + c + (" \\" if i + 1 < len(body) else ""))
        lines.append("")
    path = Path(__file__).resolve().parent / "gate_cases.inc"
    path.write_text("\n".join(lines) + "\n")
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
