"""Compartments on the host (smolcomparts.c): volumes, logic and placement.
No GPU needed: the volume enters the zeroth-order reaction probability
(rxnsetrate, smolreact.c:1327: prob = rate * dt * compartment volume), which
smolgpuGetReactionParams reports after the parameter derivation."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import smoldyn_b200 as sb

CFG = """dim 3
species A
difc A 0
boundaries 0 0 20
boundaries 1 0 20
boundaries 2 0 20
time_start 0
time_stop 1
time_step 0.01
random_seed 4
start_surface walls
action both all reflect
panel rect +0 0 0 0 20 20
panel rect -0 20 0 0 20 20
panel rect +1 0 0 0 20 20
panel rect -1 0 20 0 20 20
panel rect +2 0 0 0 20 20
panel rect -2 0 0 20 20 20
end_surface
start_surface outer
action both all transmit
panel sph 10 10 10 6 20 20
end_surface
start_surface inner
action both all transmit
panel sph 10 10 10 3 20 20
end_surface
start_compartment big
surface outer
point 10 10 10
end_compartment
start_compartment small
surface inner
point 10 10 10
end_compartment
start_compartment shell
compartment equal big
compartment andnot small
end_compartment
start_compartment outside
compartment equalnot big
end_compartment
reaction cmpt=big bb 0 -> A 1
reaction compartment=shell bs 0 -> A 1
reaction_cmpt outside bo 0 -> A 1
compartment_mol 3000 A shell
end_file
"""


def load(text):
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text)
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    return sb.Sim(ptr=simp.value)


def test_compartment_volumes_and_logic():
    s = load(CFG)
    dt = 0.01
    vol = {}
    for rx in ("bb", "bs", "bo"):
        _, _, prob = s.reaction_params(rx)
        vol[rx] = prob / (1.0 * dt)
    big = 4 / 3 * np.pi * 6 ** 3
    small = 4 / 3 * np.pi * 3 ** 3
    assert abs(vol["bb"] / big - 1) < 0.03, vol
    assert abs(vol["bs"] / (big - small) - 1) < 0.03, vol
    assert abs(vol["bo"] / (8000 - big) - 1) < 0.02, vol
    s.close()


def test_compartment_molecules_are_placed_inside():
    s = load(CFG)
    lib = s.lib
    assert lib.smolGetCompartmentIndex(s.ptr, b"shell") == 2
    buf = C.create_string_buffer(64)
    assert lib.smolGetCompartmentName(s.ptr, 3, buf) == b"outside"
    n = C.c_longlong(0)
    assert lib.smolgpuGetMolecules(s.ptr, C.byref(n), None, None, None) == 0
    pos = np.zeros((n.value, 3))
    sp = np.zeros(n.value, dtype=np.int32)
    sn = np.zeros(n.value, dtype=np.uint64)
    assert lib.smolgpuGetMolecules(s.ptr, C.byref(n), sb.dptr(pos), sp.ctypes.data_as(C.POINTER(C.c_int)),
                                   sn.ctypes.data_as(C.POINTER(C.c_uint64))) == 0
    r = np.linalg.norm(pos - 10.0, axis=1)
    assert n.value == 3000 and r.min() >= 3 and r.max() <= 6
    s.close()


def test_api_builds_the_same_compartment():
    s = sb.Sim(3, (0, 0, 0), (20, 20, 20))
    s.add_species("A", 0.0)
    s.set_times(0, 1, 0.01)
    lib = s.lib
    assert lib.smolAddSurface(s.ptr, b"ball") == 0
    prm = np.array([10, 10, 10, 6, 20, 20], dtype=float)
    assert lib.smolAddPanel(s.ptr, b"ball", sb.PSsph, None, None, sb.dptr(prm)) == 0
    assert lib.smolAddCompartment(s.ptr, b"in") == 0
    assert lib.smolAddCompartmentSurface(s.ptr, b"in", b"ball") == 0
    pt = np.array([10.0, 10.0, 10.0])
    assert lib.smolAddCompartmentPoint(s.ptr, b"in", sb.dptr(pt)) == 0
    assert lib.smolAddCompartment(s.ptr, b"out") == 0
    assert lib.smolAddCompartmentLogic(s.ptr, b"out", sb.CLequalnot, b"in") == 0
    assert lib.smolAddCompartmentLogic(s.ptr, b"out", 9, b"in") < 0
    assert lib.smolAddCompartmentMolecules(s.ptr, b"A", 500, b"in") == 0
    s.add_reaction("birth", None, None, ["A"], 2.0)
    assert lib.smolSetReactionRegion(s.ptr, b"birth", b"out", None) == 0
    # a surface too: the compartment takes precedence for births (zeroreact
    # smolreact.c:2949-2992); a surface restriction of a solution reaction of
    # order 1 is refused
    assert lib.smolSetReactionRegion(s.ptr, b"birth", b"out", b"ball") == 0
    s.add_reaction("decay", "A", None, [], 1.0)
    assert lib.smolSetReactionRegion(s.ptr, b"decay", None, b"ball") < 0
    _, _, prob = s.reaction_params("birth")
    assert abs(prob / (2.0 * 0.01) / (8000 - 4 / 3 * np.pi * 216) - 1) < 0.02
    s.close()
