"""Surface-bound states through the libsmoldyn C entry points (no GPU).

The same configuration is built twice: from a text configuration, and by the
C API calls a libsmoldyn client would make (smolAddSurface, smolAddPanel with
panel names, smolSetSurfaceAction, smolSetSurfaceRate, smolAddPanelNeighbor,
smolSetSpeciesMobility for the front state, smolAddSurfaceMolecules); the
derived surface rules (smolgpuGetSurfaceRule) must be identical, and the
surface-bound molecules (smolgpuGetSurfaceMolecules) must sit on their panel
on the requested side.  Second-order reactions of a bound and a solution
reactant: binding radii and effective rates against the values the
reference binary prints for the same configurations (golden fixture).
Jump statements parse and their malformed forms are refused.
Error paths: an unknown panel, a state the engine does not build, bound
reactants with more products than built,
solution reactants with bound products, and bound-reactant reactions with a
bounce placement.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import smoldyn_b200 as sb

TEXT = """dim 3
species A B
difc A 1
difc A(front) 0.3
time_step 0.01
boundaries 0 0 10
boundaries 1 0 10
boundaries 2 0 10
random_seed 7
start_surface membrane
action both all reflect
rate A fsoln front 1.5
rate A front fsoln 2
rate A front back 0.5 B
panel rect +0 5 0 0 10 10 m1
panel rect +0 5 0 10 10 10 m2
neighbors m1 m2
end_surface
surface_mol 100 A(front) membrane rect m1
end_file
"""


def from_text():
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "c.txt"), "w") as f:
        f.write(TEXT)
    return sb.Sim.load_file(os.path.join(d, "c.txt"))


def from_api():
    lib = sb.load()
    s = sb.Sim(3, (0, 0, 0), (10, 10, 10))
    s.add_species("A", 1.0)
    s.add_species("B")
    assert lib.smolSetSpeciesMobility(s.ptr, b"A", sb.MSfront, 0.3, None, None) == 0
    s.set_times(0, 1, 0.01)
    s.seed(7)
    assert lib.smolAddSurface(s.ptr, b"membrane") == 0
    assert lib.smolSetSurfaceAction(s.ptr, b"membrane", sb.PFboth, b"all", sb.MSsoln, sb.SAreflect, None) == 0
    assert lib.smolSetSurfaceRate(s.ptr, b"membrane", b"A", sb.MSsoln, sb.MSsoln, sb.MSfront, 1.5, None, 0) == 0
    assert lib.smolSetSurfaceRate(s.ptr, b"membrane", b"A", sb.MSfront, sb.MSfront, sb.MSsoln, 2.0, None, 0) == 0
    assert lib.smolSetSurfaceRate(s.ptr, b"membrane", b"A", sb.MSfront, sb.MSfront, sb.MSback, 0.5, b"B", 0) == 0
    for name, y in ((b"m1", 0.0), (b"m2", 10.0)):
        prm = np.array([5.0, 0.0, y, 10.0, 10.0])
        assert lib.smolAddPanel(s.ptr, b"membrane", sb.PSrect, name, b"+0", sb.dptr(prm)) == 0
    assert lib.smolAddPanelNeighbor(s.ptr, b"membrane", b"m1", b"membrane", b"m2", 0) == 0
    assert lib.smolAddSurfaceMolecules(s.ptr, b"A", sb.MSfront, 100, b"membrane", sb.PSrect, b"m1", None) == 0
    return s


@pytest.mark.parametrize("make", [from_text, from_api])
def test_bound_molecules_on_their_panel(make):
    s = make()
    pos, sp, st, srf, pnl, sn = s.surface_molecules()
    assert len(pos) == 100 and np.all(sp == 1) and np.all(st == sb.MSfront) and np.all(pnl == 0)
    assert np.all(pos[:, 0] > 5.0) and np.all(pos[:, 0] - 5.0 < 1e-12)  # just on the front (+x) side
    assert np.all((pos[:, 1] >= 0) & (pos[:, 1] <= 10) & (pos[:, 2] >= 0) & (pos[:, 2] <= 10))
    assert s.count("A", sb.MSfront) == 100 and s.count("A", sb.MSsoln) == 0
    s.close()


def test_api_and_text_derive_the_same_rules():
    a, b = from_text(), from_api()
    for sp in ("A", "B"):
        for ms in (sb.MSsoln, sb.MSfront, sb.MSback):
            for face in (sb.PFfront, sb.PFback, sb.PFnone):
                ra, rb = a.surface_rule("membrane", sp, ms, face), b.surface_rule("membrane", sp, ms, face)
                assert ra[0] == rb[0], (sp, ms, face, ra[0], rb[0])
                for x, y in zip(ra[1:], rb[1:]):
                    assert np.array_equal(x, y), (sp, ms, face, x, y)
    # adsorption from the front, desorption and the flip are rate-based (SAmult = 5)
    assert a.surface_rule("membrane", "A", sb.MSsoln, sb.PFfront)[0] == 5
    act, pr, cu, rv = a.surface_rule("membrane", "A", sb.MSfront, sb.PFnone)
    assert act == 5 and pr[sb.MSsoln] > 0 and pr[sb.MSback] > 0 and abs(cu[-1] - 1.0) < 1e-12
    a.close()
    b.close()


def test_errors():
    lib = sb.load()
    s = from_api()
    assert lib.smolAddPanelNeighbor(s.ptr, b"membrane", b"m1", b"membrane", b"nope", 0) != 0
    assert lib.smolAddSurfaceMolecules(s.ptr, b"A", sb.MSup, 5, b"membrane", sb.PSrect, b"m1", None) != 0
    assert lib.smolSetSurfaceRate(s.ptr, b"membrane", b"A", sb.MSup, sb.MSup, sb.MSsoln, 1.0, None, 0) != 0
    s.close()
    for stmt in ("reaction r A(front) + A(back) -> A(front) + B 1", "reaction r A(front) -> B(front) + B(front) + B 1",
                 "reaction r A -> B(front) 1", "reaction r A(front) + B -> A(front) 1\nproduct_placement r bounce -2",
                 "reaction r A(front) + B -> A(front) + B 1"):
        d = tempfile.mkdtemp()
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(TEXT.replace("end_file", stmt + "\nend_file"))
        with pytest.raises(RuntimeError):
            sb.Sim.load_file(os.path.join(d, "c.txt"))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bound_pair_params.npz")


def test_bound_reaction_parameters_match_reference():
    """Reactions of surface-bound reactants: A(front) + B style reactions
    (the rate doubles for one surface and one solution reactant and the bound
    state's diffusion coefficient counts, smolreact.c:1371-1377), reversible
    surface binding (the reverse found with states, the default pgemmaxw
    placement, the unbinding radius from the products' state diffusion
    coefficients) and emission from a bound molecule: actual rate, binding
    radius and unbinding radius as the reference prints them (six digits)."""
    z = np.load(GOLDEN)
    d = tempfile.mkdtemp()
    nchecked = 0
    for text, names, rates, radii, uradii in zip(z["texts"], z["names"], z["rates"], z["radii"], z["uradii"]):
        path = os.path.join(d, "c.txt")
        with open(path, "w") as f:
            f.write(str(text))
        s = sb.Sim.load_file(path)
        for k, nm in enumerate(str(names).split(",")):
            b, u, _ = s.reaction_params(nm)
            rate, _ = s.effective_rate(nm)
            for got, want in ((rate, rates[k]), (b, radii[k]), (u, uradii[k])):
                if np.isnan(want):
                    continue
                assert abs(got - want) <= 2e-5 * abs(want) + 1e-9, (nm, got, want, str(text))
                nchecked += 1
        s.close()
    assert nchecked > 150


def test_add_reaction_with_states_through_the_c_api():
    """smolAddReaction takes reactant and product states as the text form
    does (libsmoldyn.cpp smolAddReaction): the same derived parameters, and
    the same refusals."""
    lib = sb.load()
    text = TEXT.replace("end_file", "difc B 0.7\nreaction r A(front) + B -> A(front) 1.2\nend_file")
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "c.txt"), "w") as f:
        f.write(text)
    a = sb.Sim.load_file(os.path.join(d, "c.txt"))
    b = from_api()
    assert lib.smolSetSpeciesMobility(b.ptr, b"B", sb.MSsoln, 0.7, None, None) == 0
    prods = (C.c_char_p * 1)(b"A")
    states = (C.c_int * 1)(sb.MSfront)
    assert lib.smolAddReaction(b.ptr, b"r", b"A", sb.MSfront, b"B", sb.MSsoln, 1, prods,
                               C.cast(states, C.POINTER(C.c_int)), 1.2) == 0
    assert a.reaction_params("r") == b.reaction_params("r")
    assert a.effective_rate("r") == b.effective_rate("r")
    # two bound reactants react on one panel; with two products they are
    # refused, as is a bound product of solution reactants
    assert lib.smolAddReaction(b.ptr, b"r2", b"A", sb.MSfront, b"A", sb.MSback, 1, prods,
                               C.cast(states, C.POINTER(C.c_int)), 1.0) == 0
    prods2 = (C.c_char_p * 2)(b"A", b"B")
    states2 = (C.c_int * 2)(sb.MSfront, sb.MSsoln)
    assert lib.smolAddReaction(b.ptr, b"r4", b"A", sb.MSfront, b"A", sb.MSback, 2, prods2,
                               C.cast(states2, C.POINTER(C.c_int)), 1.0) != 0
    assert lib.smolAddReaction(b.ptr, b"r3", b"B", sb.MSsoln, None, sb.MSsoln, 1, prods,
                               C.cast(states, C.POINTER(C.c_int)), 1.0) != 0
    a.close()
    b.close()


def test_surface_restricted_reactions_parse_and_refuse():
    """srf= / reaction_surface / smolSetReactionRegion(surface): built for
    reactions of bound reactants, refused for solution reactions and unknown
    surfaces."""
    lib = sb.load()
    ok = TEXT.replace("end_file", "reaction srf=membrane r1 A(front) -> B(front) 1\n"
                                  "reaction_surface membrane r2 A(front) + B -> A(front) 1\nend_file")
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "c.txt"), "w") as f:
        f.write(ok)
    s = sb.Sim.load_file(os.path.join(d, "c.txt"))
    assert lib.smolSetReactionRegion(s.ptr, b"r1", None, b"membrane") == 0
    assert lib.smolSetReactionRegion(s.ptr, b"r1", None, b"nope") != 0
    s.close()
    for stmt in ("reaction srf=membrane r A -> B 1", "reaction srf=nope r A(front) -> B(front) 1",
                 "reaction_surface membrane r A + B -> A 1"):
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(TEXT.replace("end_file", stmt + "\nend_file"))
        with pytest.raises(RuntimeError):
            sb.Sim.load_file(os.path.join(d, "c.txt"))
    b = from_api()
    assert lib.smolAddReaction(b.ptr, b"rs", b"B", sb.MSsoln, None, sb.MSsoln, 0, None, None, 1.0) == 0
    assert lib.smolSetReactionRegion(b.ptr, b"rs", None, b"membrane") != 0
    b.close()


def test_births_on_a_surface_parse():
    """Order-0 reactions on a surface: births per step are rate x dt x the
    surface's area (smolreact.c:1328); bound products need the surface."""
    ok = TEXT.replace("end_file", "reaction srf=membrane b0 0 -> A(front) 0.5\nend_file")
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "c.txt"), "w") as f:
        f.write(ok)
    s = sb.Sim.load_file(os.path.join(d, "c.txt"))
    assert abs(s.reaction_params("b0")[2] - 0.5 * 0.01 * 200.0) < 1e-12  # two 10 x 10 panels
    assert abs(s.effective_rate("b0")[0] - 0.5) < 1e-12
    s.close()
    with open(os.path.join(d, "c.txt"), "w") as f:
        f.write(TEXT.replace("end_file", "reaction b0 0 -> A(front) 0.5\nend_file"))
    with pytest.raises(RuntimeError):
        sb.Sim.load_file(os.path.join(d, "c.txt"))


def test_jump_statements_parse_and_refuse():
    """jump panel1 face1 -> / <-> panel2 face2 (smolsurface.c:3574-3600): panels
    of one surface with the same shape, faces front or back; the jump action
    applies to solution molecules."""
    base = """dim 3
species A
difc A 1
time_step 0.01
boundaries 0 0 10
boundaries 1 0 10
boundaries 2 0 10
start_surface ends
action both all jump
panel rect +0 0 0 0 10 10 left
panel rect -0 10 0 0 10 10 right
panel sph 5 5 5 1 10 10 ball
%s
end_surface
end_file
"""
    d = tempfile.mkdtemp()
    path = os.path.join(d, "c.txt")
    with open(path, "w") as f:
        f.write(base % "jump left front <-> right front")
    sb.Sim.load_file(path).close()
    for stmt in ("jump left front <-> nope front", "jump left front <-> ball front", "jump left up -> right front",
                 "jump left front => right front", "jump left front -> left back"):
        with open(path, "w") as f:
            f.write(base % stmt)
        with pytest.raises(RuntimeError):
            sb.Sim.load_file(path)
    with open(path, "w") as f:
        f.write((base % "jump left front <-> right front").replace("action both all jump",
                                                                   "action both A(front) jump"))
    with pytest.raises(RuntimeError):
        sb.Sim.load_file(path)
