"""Writes gate_cases.inc: the switch cases of the gate-specialised stage
kernel (apply_gates.cu), one per op kind and register position(s), for
register passes of R = 3, 4 and 5 bits.

Every case label carries a static_assert against the host's code formula
(gate_plan.hpp: code1 / code2 / code4 / code_scale), so the two cannot drift
apart.  Run after changing the op kinds:

    python qclab_b200/csrc/gen_gate_cases.py
"""
from pathlib import Path

KIND1 = ["G_H", "G_SHEAR", "G_SHEARO", "G_ISHEAR", "G_ISHEARO", "G_PHASE", "G_GEN2", "G_REAL2",
         "G_X", "G_Z"]
KIND2 = ["G_CX", "G_CGEN2", "G_CNEG", "G_CPH"]
KIND4 = ["G_SWAP", "G_ISWAP", "G_GEN4"]


def cases(R: int) -> list[str]:
    out = []
    n1, n2, n4 = len(KIND1), len(KIND2), len(KIND4)
    for k, name in enumerate(KIND1):
        for p in range(R):
            code = k * R + p
            out.append(f"case {code}: static_assert({code} == code1({R}, {name}, {p}), \"\"); "
                       f"op1<{name}, {p}>(x, c); break;")
    base2 = n1 * R
    for k, name in enumerate(KIND2):
        for t in range(R):
            for c in range(R):
                if t == c:
                    continue
                for cv in range(2):
                    code = base2 + ((k * R + t) * R + c) * 2 + cv
                    out.append(f"case {code}: static_assert({code} == code2({R}, {name}, {t}, {c}, "
                               f"{cv}), \"\"); op2<{name}, {t}, {c}, {cv}>(x, c); break;")
    base4 = base2 + n2 * R * R * 2
    for k, name in enumerate(KIND4):
        for p0 in range(R):
            for p1 in range(p0):
                code = base4 + (k * R + p0) * R + p1
                out.append(f"case {code}: static_assert({code} == code4({R}, {name}, {p0}, {p1}), "
                           f"\"\"); op4<{name}, {p0}, {p1}>(x, c); break;")
    code = base4 + n4 * R * R
    out.append(f"case {code}: static_assert({code} == code_scale({R}), \"\"); "
               f"op_scale(x, c); break;")
    return out


def nested(R: int) -> list[str]:
    """The same cases as a two-level switch: on the op kind (code / block
    size), then on the register position(s) within the kind's block, so an
    op costs two short compare trees instead of one over every code."""
    out = ["switch (kind) {"]
    n1, n2 = len(KIND1), len(KIND2)
    for k, name in enumerate(KIND1):
        out.append(f"case {k}: switch (sub) {{")
        for p in range(R):
            out.append(f"  case {p}: op1<{name}, {p}>(x, c); break;")
        out.append("  default: __builtin_unreachable(); } break;")
    for k, name in enumerate(KIND2):
        out.append(f"case {n1 + k}: switch (sub) {{")
        for t in range(R):
            for c in range(R):
                if t == c:
                    continue
                for cv in range(2):
                    out.append(f"  case {(t * R + c) * 2 + cv}: op2<{name}, {t}, {c}, {cv}>(x, c); "
                               f"break;")
        out.append("  default: __builtin_unreachable(); } break;")
    for k, name in enumerate(KIND4):
        out.append(f"case {n1 + n2 + k}: switch (sub) {{")
        for p0 in range(R):
            for p1 in range(p0):
                out.append(f"  case {p0 * R + p1}: op4<{name}, {p0}, {p1}>(x, c); break;")
        out.append("  default: __builtin_unreachable(); } break;")
    out.append(f"case {n1 + n2 + len(KIND4)}: op_scale(x, c); break;")
    out.append("default: __builtin_unreachable();")
    out.append("}")
    return out


def main() -> None:
    lines = ["// Generated by gen_gate_cases.py -- do not edit.",
             "// Switch cases of apply_word (apply_gates.cu) for R = 4 and R = 5 register bits."]
    for R in (3, 4, 5):
        lines.append(f"#define QSV_GX_CASES_{R} \\")
        body = cases(R)
        for i, c in enumerate(body):
            lines.append("  " + c + (" \\" if i + 1 < len(body) else ""))
        lines.append("")
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
