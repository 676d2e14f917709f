#!/usr/bin/env python3
"""Generates spec_tables_gen.h: the normative AV1 constant tables the sm_100a
kernels and the host helpers read (subpel filters, transform geometry, scan
orders, intra/CDEF/loop-restoration constants, quantizer lookups).

The values are fixed by the AV1 specification, so they must equal the
reference encoder's copy bit for bit. This script reads the reference's
table header (spec_tables.h and spec_enums.h of neolite/mav1-encoder) and
writes every table as a plain integer initializer macro,
``MAV1T_<Name>`` with dimensions ``MAV1T_<Name>_DIMS``; symbolic entries
(BLOCK_*, TX_*, DCT_DCT ...) are resolved to integers. It runs once on a
machine that has the reference checkout; the output file is committed.

usage: gen_spec_tables.py <reference src dir> <output header>
"""
import hashlib
import re
import sys

TABLES = [
    # inter prediction
    "Subpel_Filters",
    # transforms
    "Cos128_Lookup", "Transform_Row_Shift", "Tx_Width", "Tx_Height", "Tx_Width_Log2",
    "Tx_Height_Log2", "Tx_Size_Sqr", "Tx_Size_Sqr_Up", "Split_Tx_Size", "Mode_To_Txfm",
    "Tx_Type_In_Set_Intra", "Tx_Type_In_Set_Inter",
    # block geometry
    "Max_Tx_Size_Rect", "Max_Tx_Depth", "Num_4x4_Blocks_Wide", "Num_4x4_Blocks_High",
    "Mi_Width_Log2", "Mi_Height_Log2", "Subsampled_Size", "Partition_Subsize",
    # intra
    "Mode_To_Angle", "Dr_Intra_Derivative", "Intra_Edge_Kernel", "Sm_Weights_Tx_4x4",
    "Sm_Weights_Tx_8x8", "Sm_Weights_Tx_16x16", "Sm_Weights_Tx_32x32", "Sm_Weights_Tx_64x64",
    # scans
    "Default_Scan_4x4", "Mcol_Scan_4x4", "Mrow_Scan_4x4", "Default_Scan_4x8", "Mcol_Scan_4x8",
    "Mrow_Scan_4x8", "Default_Scan_8x4", "Mcol_Scan_8x4", "Mrow_Scan_8x4", "Default_Scan_8x8",
    "Mcol_Scan_8x8", "Mrow_Scan_8x8", "Default_Scan_8x16", "Mcol_Scan_8x16", "Mrow_Scan_8x16",
    "Default_Scan_16x8", "Mcol_Scan_16x8", "Mrow_Scan_16x8", "Default_Scan_16x16",
    "Mcol_Scan_16x16", "Mrow_Scan_16x16", "Default_Scan_16x32", "Default_Scan_32x16",
    "Default_Scan_32x32", "Default_Scan_4x16", "Mcol_Scan_4x16", "Mrow_Scan_4x16",
    "Default_Scan_16x4", "Mcol_Scan_16x4", "Mrow_Scan_16x4", "Default_Scan_8x32",
    "Default_Scan_32x8",
    # quantizer
    "Dc_Qlookup", "Ac_Qlookup",
    # CDEF
    "Div_Table", "Cdef_Uv_Dir", "Cdef_Pri_Taps", "Cdef_Sec_Taps", "Cdef_Directions",
    # loop restoration
    "Sgr_Params", "Wiener_Taps_Min", "Wiener_Taps_Max", "Wiener_Taps_K", "Wiener_Taps_Mid",
    "Sgrproj_Xqd_Min", "Sgrproj_Xqd_Max", "Sgrproj_Xqd_Mid",
]


def symbols(src):
    sym = {}
    enums = open(f"{src}/spec_enums.h").read()
    for body in re.findall(r"enum\s*\{(.*?)\};", enums, re.S):
        val = -1
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            if "=" in item:
                name, expr = [s.strip() for s in item.split("=")]
                val = evaluate(expr, sym)
            else:
                name = item
                val += 1
            sym[name] = val
    text = open(f"{src}/spec_tables.h").read()
    for name, expr in re.findall(r"^#define\s+(\w+)\s+(.+)$", text, re.M):
        try:
            sym[name] = evaluate(expr, sym)
        except Exception:
            pass
    return sym, text


def evaluate(expr, sym):
    expr = expr.strip()
    py = re.sub(r"\b([A-Za-z_]\w*)\b", lambda m: str(sym[m.group(1)]), expr)
    return int(eval(py, {"__builtins__": {}}))


def parse_table(text, name, sym):
    m = re.search(r"SPEC_CONST\s+(\w+)\s+" + name + r"\s*((?:\[[^\]]*\]\s*)+)=\s*\{", text)
    if not m:
        raise KeyError(name)
    ctype = m.group(1)
    dims = [evaluate(d, sym) for d in re.findall(r"\[([^\]]*)\]", m.group(2))]
    i = m.end() - 1
    depth, j = 0, i
    while True:
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                break
        j += 1
    body = re.sub(r"/\*.*?\*/", "", text[i:j + 1], flags=re.S)
    body = re.sub(r"//[^\n]*", "", body)
    items = [t for t in re.split(r"[{},\s]+", body) if t]
    vals = [evaluate(t, sym) for t in items]
    n = 1
    for d in dims:
        n *= d
    if len(vals) != n:
        raise ValueError(f"{name}: {len(vals)} values for dims {dims}")
    return ctype, dims, vals


def main():
    src, out = sys.argv[1], sys.argv[2]
    sym, text = symbols(src)
    lines = [
        "/* Generated by gen_spec_tables.py: normative AV1 constant tables as",
        " * integer initializer macros (values fixed by the AV1 specification).",
        " * Do not edit. */",
        "#ifndef MAV1T_SPEC_TABLES_GEN_H",
        "#define MAV1T_SPEC_TABLES_GEN_H",
        "",
    ]
    digest = hashlib.sha256()
    for name in TABLES:
        ctype, dims, vals = parse_table(text, name, sym)
        digest.update(name.encode())
        digest.update(",".join(map(str, vals)).encode())
        lines.append(f"#define MAV1T_{name}_DIMS " + "".join(f"[{d}]" for d in dims))
        rows = [", ".join(map(str, vals[k:k + 16])) for k in range(0, len(vals), 16)]
        lines.append(f"#define MAV1T_{name} {{ \\")
        for r in rows[:-1]:
            lines.append(f"  {r}, \\")
        lines.append(f"  {rows[-1]} }}")
    lines.append(f'#define MAV1T_DIGEST "{digest.hexdigest()}"')
    lines.append("")
    lines.append("#endif")
    open(out, "w").write("\n".join(lines) + "\n")
    print(out, digest.hexdigest())


if __name__ == "__main__":
    main()
