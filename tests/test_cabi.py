"""The C-ABI library loads, exports every symbol include/smoldyn_b200.h
declares, and its host-side API (no engine launch) behaves like libsmoldyn's
(source/Smoldyn/libsmoldyn.cpp) on a machine without a GPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import smoldyn_b200 as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "smoldyn_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(smol\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    sb.load()
    out = subprocess.check_output(["nm", "-D", "--defined-only", sb.LIB_PATH]).decode()
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    declared = header_functions()
    assert len(declared) >= 50
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    # and every declared function has a ctypes prototype
    assert not [f for f in declared if f not in sb.PROTOTYPES]


def test_errors_follow_libsmoldyn_convention():
    lib = sb.load()
    lib.smolClearError()
    s = sb.Sim(3, (0, 0, 0), (10, 10, 10))
    s.add_species("A", 1.0)
    rc = lib.smolAddSpecies(s.ptr, b"A", None)
    assert rc == sb.ECsame
    code, fn, msg = sb.last_error()
    assert code == sb.ECsame and fn == "smolAddSpecies" and "exists" in msg
    assert lib.smolGetSpeciesIndexNT(s.ptr, b"nope") == sb.ECnonexist
    assert lib.smolGetSpeciesIndex(s.ptr, b"A") == 1
    buf = C.create_string_buffer(64)
    lib.smolGetSpeciesName(s.ptr, 1, buf)
    assert buf.value == b"A"
    lo = np.array([1.0, 0, 0])
    hi = np.array([0.0, 1, 1])
    assert not lib.smolNewSim(3, sb.dptr(lo), sb.dptr(hi))
    assert sb.last_error()[0] == sb.ECbounds


def test_pending_molecules_and_counts_without_engine():
    s = sb.Sim(3, (0, 0, 0), (100, 100, 100))
    s.add_species("A", 1.0)
    s.add_species("B", 1.0)
    s.add_molecules("A", 1000)
    s.add_molecules("B", 500, (10, 10, 10), (20, 20, 20))
    assert s.count("A") == 1000 and s.count("B") == 500 and s.count("all") == 1500
    pos, sp, sn = s.molecules()
    b = pos[sp == 2]
    assert (b >= 10).all() and (b <= 20).all()
    a = pos[sp == 1]
    assert (a >= 0).all() and (a <= 100).all()


def test_reaction_parameters_match_reference_known_answer():
    """Config 1 of the workload (A+B<->C, kf=0.05, kr=0.1, D=1,1,0.5, dt=0.01):
    the reference prints binding radius 0.049234 and unbinding radius 0 with
    the default pgemmaxw 0.2 placement (smoldyn output, 'ORDER 2 REACTION
    PARAMETERS'), and probability 1-exp(-0.1*0.01) for the reverse."""
    s = sb.Sim(3, (0, 0, 0), (100, 100, 100))
    for nm, d in (("A", 1), ("B", 1), ("C", 0.5)):
        s.add_species(nm, d)
    s.set_times(0, 10, 0.01)
    s.add_reaction("fwd", "A", "B", ["C"], 0.05)
    s.add_reaction("rev", "C", None, ["A", "B"], 0.1)
    b, u, p = s.reaction_params("fwd")
    assert abs(b - 0.049234) < 5e-7
    assert p == 1.0
    b2, u2, p2 = s.reaction_params("rev")
    assert u2 == 0.0
    assert abs(p2 - (1 - np.exp(-0.1 * 0.01))) < 1e-15


def test_config_reader_statements(tmp_path):
    cfg = tmp_path / "c.txt"
    cfg.write_text("""
# comment
dim 3
species A B
difc A 2
difc B 1
boundaries 0 0 50 p
boundaries 1 0 50 p
boundaries 2 0 50 p
time_start 0
time_stop 1
time_step 0.01
random_seed 7
reaction r1 A + B -> 0 0.5
define NMOL 300
mol NMOL A u u u
mol 200 B 25 25 25
ifdefine NOPE
mol 5 A u u u
endif
end_file
""")
    lib = sb.load()
    simp = C.c_void_p()
    rc = lib.smolLoadSimFromFile(str(tmp_path).encode(), b"c.txt", C.byref(simp), b"")
    assert rc == 0, sb.last_error()
    s = sb.Sim(ptr=simp.value)
    assert s.count("A") == 300 and s.count("B") == 200
    b, u, p = s.reaction_params("r1")
    assert b > 0


def test_unsupported_statement_reports_syntax_error():
    s = sb.Sim(3, (0, 0, 0), (1, 1, 1))
    with pytest.raises(RuntimeError):
        s.statement("surface_drift", "A all 1 1")
