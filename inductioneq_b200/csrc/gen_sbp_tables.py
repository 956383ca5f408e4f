"""Build step: regenerate ``sbp_tables.inc`` and ``sbp_tables.json`` from operator headers.

The summation-by-parts coefficients are published mathematical constants that the GPU
kernels must use bit for bit to agree with the reference.  InductionEq ships them as
padded ``(2*NUM_BOUNDS+1) x STENCIL_WIDTH`` row tables in its operator headers
(include/{2,4,6}thOrder[Extended].h).  This script reads those headers (an operator-header
path list, as the reference host passes them to the OpenCL compiler) and stores each table
in this project's compact form:

* only the left-boundary rows and the interior row are stored;
* the right-boundary rows follow by mirror symmetry -- antisymmetric for first-derivative
  rows (D, its adjoint), symmetric for the norm M^-1 and the -Laplacians, and reversed with
  sign (-1)^(W-1) for the dissipation factor D_HO.  The symmetry is checked exactly here;
  a table that is not an exact mirror is stored with all rows.
* values are written as exact binary64 hex literals (a/b entries evaluated the way a C
  compiler folds ``a.0/b.0``).

Usage: python gen_sbp_tables.py <reference include dir>
"""
from __future__ import annotations

import json
import os
import re
import sys

OPERATORS = [(2, False), (4, False), (6, False), (2, True), (4, True), (6, True)]
LAPLACE = [("WS_D0", "SBP_minus_laplace_WS_D0"), ("NS_D0", "SBP_minus_laplace_NS_D0"),
           ("WS_LN", "SBP_minus_laplace_WS_LN")]


def header_name(order: int, ext: bool) -> str:
    return f"{order}{'th' if order > 2 else 'nd'}Order{'Extended' if ext else ''}.h"


def op_key(order: int, ext: bool) -> str:
    return f"{order}{'e' if ext else 'c'}"


def _value(tok: str) -> float:
    tok = tok.strip()
    if "/" in tok:
        a, b = tok.split("/")
        return float(a) / float(b)
    return float(tok)


def parse_header(text: str) -> tuple[dict, dict]:
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(\w+)\s+(\d+)", text)}
    tables = {}
    for m in re.finditer(r"REAL\s+constant\s+(\w+)\s*((?:\[[^\]]*\])+)\s*=\s*\{(.*?)\};", text, re.S):
        name, body = m.group(1), m.group(3)
        rows = re.findall(r"\{([^{}]*)\}", body)
        if rows:
            tables[name] = [[_value(t) for t in r.split(",") if t.strip()] for r in rows]
        else:
            tables[name] = [_value(t) for t in body.split(",") if t.strip()]
    return defines, tables


def mirror_ok(rows: list[list[float]], sign: float, reverse_only: bool) -> bool:
    n = len(rows)
    nb = (n - 1) // 2
    for j in range(nb):
        left, right = rows[j], rows[n - 1 - j]
        w = len(left)
        for i in range(w):
            if right[i] != sign * left[w - 1 - i] and not (right[i] == 0 and left[w - 1 - i] == 0):
                return False
    return True


def compact(rows: list[list[float]], sign: float) -> dict:
    n = len(rows)
    nb = (n - 1) // 2
    if mirror_ok(rows, sign, False):
        keep = rows[: nb + 1]
        explicit = False
    else:
        keep = rows
        explicit = True
    return {"nb": nb, "width": len(rows[0]), "sign": int(sign), "explicit": explicit,
            "rows": [[float(x).hex() for x in r] for r in keep]}


def build(include_dir: str) -> dict:
    out = {}
    for order, ext in OPERATORS:
        with open(os.path.join(include_dir, header_name(order, ext))) as f:
            defs, tabs = parse_header(f.read())
        nb, sw, whod = defs["NUM_BOUNDS"], defs["STENCIL_WIDTH"], defs["STENCIL_WIDTH_HOD"]
        assert defs["ORDER"] == order
        minv = tabs["M_INV"]
        assert all(minv[i] == minv[len(minv) - 1 - i] for i in range(len(minv)))
        entry = {
            "order": order, "extended": ext, "nb": nb, "sw": sw, "w_hod": whod,
            "D": compact(tabs["SBP_diff"], -1.0),
            "Dadj": compact(tabs["SBP_diff_adjoint"], -1.0),
            "DHO": compact(tabs["D_HO"], -1.0 if (whod - 1) % 2 else 1.0),
            "Minv": [float(x).hex() for x in minv[: nb + 1]],
            "laplace": {},
        }
        for short, name in LAPLACE:
            if name in tabs:
                entry["laplace"][short] = compact(tabs[name], 1.0)
        out[op_key(order, ext)] = entry
    return out


def expand(tab: dict) -> list[list[float]]:
    """Full (2*nb+1) x width table from the compact form (used to self-check here)."""
    rows = [[float.fromhex(x) for x in r] for r in tab["rows"]]
    if tab["explicit"]:
        return rows
    nb, s = tab["nb"], tab["sign"]
    full = rows + [[0.0] * tab["width"] for _ in range(nb)]
    for j in range(nb):
        full[2 * nb - j] = [s * v if v != 0 else 0.0 for v in rows[j][::-1]]
    return full


def emit_inc(data: dict) -> str:
    lines = ["// Generated by gen_sbp_tables.py -- do not edit by hand.",
             "// Compact SBP coefficient tables: left-boundary rows then the interior row;",
             "// right-boundary rows follow by the stated mirror sign unless `explicit`.",
             "// Columns are stencil offsets -(width-1)/2 .. +(width-1)/2 (D_HO: start index).",
             ""]
    for key, e in data.items():
        def arr(name, tab):
            vals = ", ".join(x for r in tab["rows"] for x in r)
            lines.append(f"static const double k{key}_{name}[] = {{{vals}}};")
        arr("D", e["D"])
        arr("Dadj", e["Dadj"])
        arr("DHO", e["DHO"])
        lines.append(f"static const double k{key}_Minv[] = {{{', '.join(e['Minv'])}}};")
        for short in ("WS_D0", "NS_D0", "WS_LN"):
            if short in e["laplace"]:
                arr("L" + short, e["laplace"][short])
    lines.append("")
    lines.append("static const SbpOperatorSource kSbpOperators[] = {")
    for key, e in data.items():
        def tab(name, t):
            if t is None:
                return "{0, 0, 0, 0, nullptr}"
            return f"{{{t['nb']}, {t['width']}, {t['sign']}, {1 if t['explicit'] else 0}, k{key}_{name}}}"
        lap = [tab("L" + s, e["laplace"].get(s)) for s in ("WS_D0", "NS_D0", "WS_LN")]
        lines.append(f"  {{{e['order']}, {1 if e['extended'] else 0}, {e['nb']}, {e['sw']}, {e['w_hod']},")
        lines.append(f"   {tab('D', e['D'])}, {tab('Dadj', e['Dadj'])}, {tab('DHO', e['DHO'])},")
        lines.append(f"   k{key}_Minv, {{{', '.join(lap)}}}}},")
    lines.append("};")
    return "\n".join(lines) + "\n"


def main() -> None:
    # the reference's include directory: the first argument, else $IEQ_REFERENCE_DIR/include
    if len(sys.argv) > 1:
        inc_dir = sys.argv[1]
    elif os.environ.get("IEQ_REFERENCE_DIR"):
        inc_dir = os.path.join(os.environ["IEQ_REFERENCE_DIR"], "include")
    else:
        sys.exit("usage: gen_sbp_tables.py <reference include directory> (or set IEQ_REFERENCE_DIR)")
    data = build(inc_dir)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "sbp_tables.inc"), "w") as f:
        f.write(emit_inc(data))
    with open(os.path.join(os.path.dirname(here), "sbp_tables.json"), "w") as f:
        json.dump(data, f, indent=0)
    # self-check: the compact form expands back to the header tables exactly
    for order, ext in OPERATORS:
        with open(os.path.join(inc_dir, header_name(order, ext))) as f:
            _, tabs = parse_header(f.read())
        e = data[op_key(order, ext)]
        assert expand(e["D"]) == tabs["SBP_diff"]
        assert expand(e["Dadj"]) == tabs["SBP_diff_adjoint"]
        assert expand(e["DHO"]) == tabs["D_HO"]
    print("ok:", ", ".join(f"{k}: D {'explicit' if v['D']['explicit'] else 'mirrored'}, "
                           f"Dadj {'explicit' if v['Dadj']['explicit'] else 'mirrored'}, "
                           f"DHO {'explicit' if v['DHO']['explicit'] else 'mirrored'}, "
                           f"lap {[(s, 'x' if t['explicit'] else 'm') for s, t in v['laplace'].items()]}"
                           for k, v in data.items()))


if __name__ == "__main__":
    main()
