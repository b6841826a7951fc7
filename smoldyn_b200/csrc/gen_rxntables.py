"""Generate the binding-radius and surface-adsorption lookup table headers
from the reference source.

The per-step reaction-rate tables used by Smoldyn's binding/unbinding radius
solver (``yi``, ``yr``, ``yb`` in ``numrxnrate`` and ``kirr``, ``krev``, ``kb`` in
``numrxnrateprob``; source/libSteve/rxnparam.c:57-391) are numerical data that
the exact FP64 solver needs verbatim.  rxnparam.c is in the public domain
(rxnparam.c:1-3).  Rather than carrying a copy of that data in this repository,
this script reads it from a reference checkout at build time and writes
``_gen/rxntables.h`` (git-ignored).

Usage: python gen_rxntables.py [REFERENCE_ROOT] [OUTPUT_HEADER]
REFERENCE_ROOT defaults to $SMOLDYN_REF, then /root/reference.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "_gen", "rxntables.h")

# name in rxnparam.c -> (name in the generated header, expected length)
TABLES = {
    "yi": ("SMOLB_TAB_YI", 31),
    "yr": ("SMOLB_TAB_YR", 16 * 31),
    "yb": ("SMOLB_TAB_YB", 11 * 31),
    "kirr": ("SMOLB_TAB_KIRR", 8 * 31),
    "krev": ("SMOLB_TAB_KREV", 16 * 8 * 31),
    "kb": ("SMOLB_TAB_KB", 11 * 8 * 31),
}


def extract(text, name):
    m = re.search(r"const\s+double\s+" + name + r"\s*\[\s*\]\s*=\s*\{", text)
    if not m:
        raise RuntimeError("table %s not found in rxnparam.c" % name)
    end = text.index("};", m.end())
    body = text[m.end():end]
    body = re.sub(r"//[^\n]*", "", body)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    vals = [v.strip() for v in body.split(",") if v.strip()]
    for v in vals:
        float(v)
    return vals


# SurfaceParam.c (public domain, SurfaceParam.c:1-2): the adsorption lookup
# tables that surfaceprob interpolates (lookupirrevadsorb :504, lookuprevads
# :566), named by (function, array) -> (generated name, expected length).
SURF_TABLES = {
    ("lookupirrevadsorb", "ponlist"): ("SMOLB_SRF_PON", 21),
    ("lookupirrevadsorb", "kappalist"): ("SMOLB_SRF_KAPPA", 21),
    ("lookuprevads", "xlist"): ("SMOLB_SRF_REVX", 21),
    ("lookuprevads", "adsprobtable"): ("SMOLB_SRF_REVADS", 21 * 21),
}


def extract_local(text, func, name):
    m = re.search(r"double\s+" + func + r"\s*\(", text)
    if not m:
        raise RuntimeError("function %s not found in SurfaceParam.c" % func)
    m2 = re.compile(r"double\s+" + name + r"\s*\[\s*\]\s*=\s*\{").search(text, m.end())
    if not m2:
        raise RuntimeError("table %s not found in %s" % (name, func))
    end = text.index("};", m2.end())
    body = re.sub(r"/\*.*?\*/", "", text[m2.end():end], flags=re.S)
    vals = [v.strip() for v in body.split(",") if v.strip()]
    for v in vals:
        float(v)
    return vals


def generate_surface(ref_root, out_path):
    src = os.path.join(ref_root, "source", "libSteve", "SurfaceParam.c")
    with open(src) as f:
        text = f.read()
    lines = [
        "/* Generated by gen_rxntables.py from source/libSteve/SurfaceParam.c of the",
        " * reference (public domain).  Do not edit; not committed. */",
        "#pragma once",
    ]
    for (func, name), (cname, n) in SURF_TABLES.items():
        vals = extract_local(text, func, name)
        if len(vals) != n:
            raise RuntimeError("table %s: expected %d values, got %d" % (name, n, len(vals)))
        lines.append("#define %s_LEN %d" % (cname, n))
        lines.append("#define %s_INIT { \\" % cname)
        for i in range(0, n, 8):
            lines.append("  " + ",".join(vals[i:i + 8]) + ", \\")
        lines.append("}")
    tmp = out_path + ".tmp"
    os.makedirs(os.path.dirname(out_path), exist_ok=True)
    with open(tmp, "w") as f:
        f.write("\n".join(lines) + "\n")
    os.replace(tmp, out_path)
    return out_path


def generate(ref_root, out_path):
    src = os.path.join(ref_root, "source", "libSteve", "rxnparam.c")
    with open(src) as f:
        text = f.read()
    lines = [
        "/* Generated by gen_rxntables.py from source/libSteve/rxnparam.c of the",
        " * reference (public domain).  Do not edit; not committed. */",
        "#pragma once",
    ]
    for name, (cname, n) in TABLES.items():
        vals = extract(text, name)
        if len(vals) != n:
            raise RuntimeError("table %s: expected %d values, got %d" % (name, n, len(vals)))
        lines.append("#define %s_LEN %d" % (cname, n))
        lines.append("#define %s_INIT { \\" % cname)
        for i in range(0, n, 8):
            lines.append("  " + ",".join(vals[i:i + 8]) + ", \\")
        lines.append("}")
    tmp = out_path + ".tmp"
    os.makedirs(os.path.dirname(out_path), exist_ok=True)
    with open(tmp, "w") as f:
        f.write("\n".join(lines) + "\n")
    os.replace(tmp, out_path)
    return out_path


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("SMOLDYN_REF", "/root/reference")
    out = argv[2] if len(argv) > 2 else DEFAULT_OUT
    if not os.path.exists(os.path.join(ref, "source", "libSteve", "rxnparam.c")):
        if os.path.exists(out) and os.path.exists(os.path.join(os.path.dirname(out), "srftables.h")):
            print("reference not found at %s; keeping existing generated headers" % ref)
            return 0
        sys.stderr.write("rxnparam tables: reference checkout not found at %s and no "
                         "generated header present; set SMOLDYN_REF\n" % ref)
        return 1
    print("wrote", generate(ref, out))
    print("wrote", generate_surface(ref, os.path.join(os.path.dirname(out), "srftables.h")))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
