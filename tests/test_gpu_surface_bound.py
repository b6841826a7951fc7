"""Surface-bound states on the GPU against the reference binary.

Each configuration is run by the engine (its text configuration through the
libsmoldyn C API) and by the reference Smoldyn binary compiled from the
reference's sources (oracle/_ref/smoldyn), 32 seeds each; the mean counts at
every output time must agree within 3.5 combined standard errors (plus one
molecule).  `molcountspecies A(front)` counts a state, `molcountonsurf` the bound
molecules of one surface, `molcount` all states (conservation); transmission
changes the species, so `molcount` separates the two sides.
  1. reversible adsorption / desorption on a plane, bound molecules mobile
     (rates in both directions: the reversible adsorption tables);
  2. molecules placed on a sphere (surface_mol) diffusing on it and
     desorbing irreversibly to the outside;
  3. molecules placed on one face of a cube of six rectangles, each its own
     surface, with neighbour lists: bound diffusion carries them across the
     edges onto the other faces (counts per face);
  4. flips between the front and back states of a plane;
  5. one-way transmission through a membrane at a given rate;
  6. first-order reactions of bound molecules: A(front) -> B(front),
     B(front) -> C(soln) (released into solution), A(front) -> 0;
  7. a capsule: a cylinder with hemisphere caps, neighbours across the rims
     (counts on the body and on the caps);
  9. reversible surface binding A(front) + B <-> C(front) (the reverse is a
     first-order bound reaction with a bound and a solution product, placed
     at the geminate unbinding radius) and emission A(front) -> A(front) + D;
  10. reactions restricted to a surface (`srf=`, `reaction_surface`): a
     first-order and a bound-solution reaction, each on one of two planes;
  11. the same in two dimensions: adsorption and desorption on a circle,
     diffusion along it, reversible binding (products offset in the plane);
  12. births on a surface (order 0 restricted to a surface): bound products
     placed by area on a sphere, solution products on its back (inner) side;
  13. reactions of two bound molecules on one panel: reversible dimerization
     (the reverse with two bound products) and mutual removal (no reactant
     shared between the two, so the reference's list order decides no
     contest between them);
  14. jump surfaces: two end panels that send solution molecules to each
     other (a periodic box made of panels), counts in the left half;
  8. second-order reactions of a bound and a solution reactant, with a
     bound product, a solution product and none; solution molecules behind
     the panel do not react.  The bound molecules sit within one binding
     radius of each other, so bound molecules contest solution molecules; the
     reference settles a contest by its molecule-list order, and with one
     list for all states it favours products of earlier steps (they fill the
     list slots of reacted molecules, ahead of the solution molecules).  The
     configuration keeps bound and solution molecules in separate lists, the
     layout in which the reference's order carries no such preference (its
     C(front) count then agrees with the engine's random-priority contests).
Engine-side geometric checks: bound molecules stay on their panel's surface
(sphere radius; cube faces) to 1e-6.
"""
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

pytestmark = pytest.mark.gpu

REF_EXE = os.path.join(oracle_lib.REF_DIR, "smoldyn")
NSEED = 32

WALLS = """start_surface walls
action both all reflect
panel rect +0 0 0 0 {L} {L}
panel rect -0 {L} 0 0 {L} {L}
panel rect +1 0 0 0 {L} {L}
panel rect -1 0 {L} 0 {L} {L}
panel rect +2 0 0 0 {L} {L}
panel rect -2 0 0 {L} {L} {L}
end_surface
"""

HEAD = """dim 3
boundaries 0 0 {L}
boundaries 1 0 {L}
boundaries 2 0 {L}
time_start 0
time_stop {T}
time_step {dt}
random_seed {seed}
"""

ADSORB = HEAD + """species A
difc A 1
difc A(front) 0.3
""" + WALLS + """start_surface membrane
action both all reflect
rate A fsoln front 1.5
rate A front fsoln 2
panel rect +0 5 0 0 10 10 m1
end_surface
mol 3000 A 5-10 u u
output_files out.txt outf.txt
cmd N 20 molcount out.txt
cmd N 20 molcountspecies A(front) outf.txt
end_file
"""

SPHERE = HEAD + """species A
difc A 1
difc A(front) 1
""" + WALLS + """start_surface cell
action both all reflect
rate A front fsoln 0.8
panel sph 10 10 10 4 30 30 s1
end_surface
surface_mol 2000 A(front) cell sph all
output_files out.txt outf.txt
cmd N 20 molcount out.txt
cmd N 20 molcountspecies A(front) outf.txt
end_file
"""

FACES = [("xlo", "-0 5 5 5 10 10"), ("xhi", "+0 15 5 5 10 10"), ("ylo", "-1 5 5 5 10 10"),
         ("yhi", "+1 5 15 5 10 10"), ("zlo", "-2 5 5 5 10 10"), ("zhi", "+2 5 5 15 10 10")]
ADJ = {"xlo": "ylo yhi zlo zhi", "xhi": "ylo yhi zlo zhi", "ylo": "xlo xhi zlo zhi",
       "yhi": "xlo xhi zlo zhi", "zlo": "xlo xhi ylo yhi", "zhi": "xlo xhi ylo yhi"}


def cube_config():
    txt = HEAD + "species B\ndifc B(front) 1\n" + WALLS
    for nm, prm in FACES:
        txt += "start_surface %s\npanel rect %s p\nend_surface\n" % (nm, prm)
    for nm, _ in FACES:
        txt += "start_surface %s\nneighbors p %s\nend_surface\n" % (
            nm, " ".join("%s:p" % o for o in ADJ[nm].split()))
    txt += "surface_mol 2000 B(front) xlo rect p\noutput_files out.txt\n"
    for nm, _ in FACES:
        txt += "cmd N 25 molcountonsurf %s out_%s.txt\n" % (nm, nm)
    txt = txt.replace("output_files out.txt", "output_files " + " ".join("out_%s.txt" % nm for nm, _ in FACES))
    return txt + "end_file\n"


FLIP = HEAD + """species B
""" + WALLS + """start_surface plane
rate B front back 2
rate B back front 1
panel rect +0 10 0 0 20 20 p1
end_surface
surface_mol 2000 B(front) plane rect p1
output_files out.txt outb.txt
cmd N 10 molcount out.txt
cmd N 10 molcountspecies B(back) outb.txt
end_file
"""

CAPSULE = HEAD + """species B
difc B(front) 1
""" + WALLS + """start_surface body
panel cyl 8 10 10 12 10 10 2 20 20 c1
end_surface
start_surface caps
panel hemi 8 10 10 2 1 0 0 20 20 h1
panel hemi 12 10 10 2 -1 0 0 20 20 h2
end_surface
start_surface body
neighbors c1 caps:h1 caps:h2
end_surface
start_surface caps
neighbors h1 body:c1
neighbors h2 body:c1
end_surface
surface_mol 2000 B(front) body cyl c1
output_files out_body.txt out_caps.txt
cmd N 20 molcountonsurf body out_body.txt
cmd N 20 molcountonsurf caps out_caps.txt
end_file
"""

BOUNDRXN = HEAD + """species A B C
difc A(front) 0.5
difc B(front) 0.5
difc C 1
""" + WALLS + """start_surface plane
action both all reflect
panel rect +0 10 0 0 20 20 p1
end_surface
reaction r1 A(front) -> B(front) 1
reaction r2 B(front) -> C(soln) 0.5
reaction r3 A(front) -> 0 0.2
surface_mol 2000 A(front) plane rect p1
output_files out.txt outa.txt outb.txt
cmd N 10 molcount out.txt
cmd N 10 molcountspecies A(front) outa.txt
cmd N 10 molcountspecies B(front) outb.txt
end_file
"""

BIRXN = HEAD + """species A B C D
difc A(front) 0.2
difc B 1
difc C(front) 0.2
difc D 1
""" + WALLS + """start_surface plane
action both all reflect
panel rect +0 10 0 0 20 20 p1
end_surface
reaction r1 A(front) + B -> C(front) 4
reaction r2 B + C(front) -> D 4
reaction r3 A(front) + D -> 0 1
start_compartment behind
surface plane
point 5 10 10
end_compartment
molecule_lists blist bndlist
mol_list B blist
mol_list D blist
mol_list A(front) bndlist
mol_list C(front) bndlist
surface_mol 2000 A(front) plane rect p1
mol 4000 B u u u
output_files out.txt outb.txt
cmd N 10 molcount out.txt
cmd N 10 molcountincmpt behind outb.txt
end_file
"""

BIRXN_BACK = HEAD + """species A B C
difc A(back) 0.2
difc B 1
difc C 1
""" + WALLS + """start_surface plane
action both all reflect
panel rect +0 10 0 0 20 20 p1
end_surface
reaction r1 A(back) + B -> C(bsoln) 4
start_compartment behind
surface plane
point 5 10 10
end_compartment
molecule_lists blist bndlist
mol_list B blist
mol_list C blist
mol_list A(back) bndlist
surface_mol 1000 A(back) plane rect p1
mol 4000 B u u u
output_files out.txt outb.txt
cmd N 10 molcount out.txt
cmd N 10 molcountincmpt behind outb.txt
end_file
"""

REVBIND = HEAD + """species A B C D
difc A(front) 0.2
difc B 1
difc C(front) 0.1
difc D 1
""" + WALLS + """start_surface plane
action both all reflect
panel rect +0 10 0 0 20 20 p1
end_surface
reaction r1 A(front) + B <-> C(front) 2 1
reaction e1 A(front) -> A(front) + D 0.2
start_compartment behind
surface plane
point 5 10 10
end_compartment
molecule_lists blist bndlist
mol_list B blist
mol_list D blist
mol_list A(front) bndlist
mol_list C(front) bndlist
surface_mol 1000 A(front) plane rect p1
mol 4000 B u u u
output_files out.txt outb.txt
cmd N 10 molcount out.txt
cmd N 10 molcountincmpt behind outb.txt
end_file
"""

SRFRXN = HEAD + """species A B C
difc A(front) 0.1
difc B(front) 0.1
difc C 1
""" + WALLS + """start_surface s1
action both all reflect
panel rect +0 6 0 0 20 20 p1
end_surface
start_surface s2
action both all reflect
panel rect +0 14 0 0 20 20 p2
end_surface
reaction srf=s1 r1 A(front) -> B(front) 1
reaction_surface s2 r2 A(front) + C -> A(front) 2
molecule_lists blist bndlist
mol_list C blist
mol_list A(front) bndlist
mol_list B(front) bndlist
surface_mol 1000 A(front) s1 rect p1
surface_mol 1000 A(front) s2 rect p2
mol 3000 C u u u
output_files out.txt out1.txt
cmd N 10 molcount out.txt
cmd N 10 molcountonsurf s1 out1.txt
end_file
"""

PLANAR = """dim 2
boundaries 0 0 100
boundaries 1 0 100
time_start 0
time_stop {T}
time_step {dt}
random_seed {seed}
species A B C
difc A 3
difc A(front) 0.5
difc B 1
difc C(front) 0.2
start_surface walls
action both all reflect
panel rect +0 0 0 100
panel rect -0 100 0 100
panel rect +1 0 0 100
panel rect -1 0 100 100
end_surface
start_surface stick
action both all reflect
rate A fsoln front 1
rate A front fsoln 0.2
panel sph 50 50 20 40
end_surface
reaction r1 A(front) + B <-> C(front) 20 0.5
molecule_lists blist bndlist
mol_list A blist
mol_list B blist
mol_list A(front) bndlist
mol_list C(front) bndlist
mol 1000 A u u
mol 1000 B u u
surface_mol 300 A(front) stick all all
output_files out.txt outs.txt
cmd N 20 molcount out.txt
cmd N 20 molcountonsurf stick outs.txt
end_file
"""

SRFBIRTH = HEAD + """species A B
difc A(front) 0.2
difc B 1
""" + WALLS + """start_surface ball
action both all reflect
panel sph 10 10 10 4 20 20 s1
end_surface
start_compartment inside
surface ball
point 10 10 10
end_compartment
reaction srf=ball g 0 -> A(front) 2
reaction_surface ball h 0 -> B(bsoln) 1
reaction decay A(front) -> 0 0.5
output_files out.txt outi.txt
cmd N 10 molcount out.txt
cmd N 10 molcountincmpt inside outi.txt
end_file
"""

BBRXN = HEAD + """species A C D E
difc A(front) 0.5
difc C(front) 0.2
difc D(front) 0.3
difc E(front) 0.3
""" + WALLS + """start_surface plane
action both all reflect
panel rect +0 10 0 0 20 20 p1
end_surface
reaction d A(front) + A(front) <-> C(front) 0.5 0.5
reaction h D(front) + E(front) -> 0 1
surface_mol 1000 A(front) plane rect p1
surface_mol 500 D(front) plane rect p1
surface_mol 500 E(front) plane rect p1
output_files out.txt
cmd N 10 molcount out.txt
end_file
"""

JUMP = HEAD + """species A
difc A 1
start_surface sides
action both all reflect
panel rect +1 0 0 0 20 20
panel rect -1 0 20 0 20 20
panel rect +2 0 0 0 20 20
panel rect -2 0 0 20 20 20
end_surface
start_surface ends
action both all jump
panel rect +0 0 0 0 20 20 left
panel rect -0 20 0 0 20 20 right
jump left front <-> right front
end_surface
start_surface mid
action both all transmit
panel rect +0 10 0 0 20 20 m
end_surface
start_compartment lefthalf
surface mid
point 5 10 10
end_compartment
mol 2000 A 1 u u
output_files out.txt outl.txt
cmd N 10 molcount out.txt
cmd N 10 molcountincmpt lefthalf outl.txt
end_file
"""

TRANSMIT = HEAD + """species A B
difc A 1
difc B 1
""" + WALLS + """start_surface membrane
rate A fsoln bsoln 0.5 B
panel rect +0 10 0 0 20 20 m1
end_surface
mol 3000 A 10-20 u u
output_files out.txt
cmd N 20 molcount out.txt
end_file
"""


def read_rows(path):
    with open(path) as f:
        return np.array([[float(x) for x in ln.split()] for ln in f if ln.strip()])


def run_ref(text, seed, outs):
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text.replace("{seed}", str(seed)))
        subprocess.run([REF_EXE, "c.txt", "-qt"], cwd=d, check=True, stdin=subprocess.DEVNULL,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, SMOLDYN_NO_PROMPT="1"), timeout=600)
        return [read_rows(os.path.join(d, o)) for o in outs]


def run_gpu(text, seed, outs, check=None):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "c.txt"), "w") as f:
        f.write(text.replace("{seed}", str(seed)))
    s = sb.Sim.load_file(os.path.join(d, "c.txt"))
    s.run()
    res = [np.array(s.output_data(o)) for o in outs]
    if check:
        check(s)
    s.close()
    return res


def fill(text, **kw):
    for k, v in kw.items():
        text = text.replace("{%s}" % k, str(v))
    return text


def compare(text, outs, cols, what, check=None):
    """Mean counts over seeds, engine against reference, at every output row."""
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        ref = list(ex.map(lambda sd: run_ref(text, sd, outs), range(1, NSEED + 1)))
    gpu = [run_gpu(text, 1000 + sd, outs, check if sd == 0 else None) for sd in range(NSEED)]
    for k, o in enumerate(outs):
        R = np.stack([r[k] for r in ref])   # [seed, row, col]
        G = np.stack([g[k] for g in gpu])
        n = min(R.shape[1], G.shape[1])
        assert abs(R.shape[1] - G.shape[1]) <= 1, (o, R.shape, G.shape)
        R, G = R[:, :n], G[:, :n]
        assert np.allclose(R[0, :, 0], G[0, :, 0]), (R[0, :, 0], G[0, :, 0])
        for c in cols:
            mr, mg = R[:, :, c].mean(0), G[:, :, c].mean(0)
            se = np.sqrt(R[:, :, c].var(0, ddof=1) / NSEED + G[:, :, c].var(0, ddof=1) / NSEED)
            z = np.abs(mr - mg) / (se + 1e-9)
            print("%s %s col %d: ref %s gpu %s max z %.2f" % (what, o, c, np.round(mr[-3:], 1), np.round(mg[-3:], 1),
                                                             z.max()))
            assert np.all(np.abs(mr - mg) <= 3.5 * se + 1.0), (what, o, c, mr, mg, se)
    return ref, gpu


def test_reversible_adsorption_on_plane():
    text = fill(ADSORB, L=10, T=1.0, dt=0.005)
    _, gpu = compare(text, ["out.txt", "outf.txt"], [1], "adsorb")
    assert all(np.all(g[0][:, 1] == 3000) for g in gpu)  # conserved
    B = np.stack([g[1][:, 1] for g in gpu])
    assert B[:, -1].mean() > 100  # a sizable bound population forms


def test_sphere_bound_diffusion_and_desorption():
    def on_sphere(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert len(pos) > 100
        r = np.linalg.norm(pos - 10.0, axis=1)
        assert np.all(np.abs(r - 4.0) < 1e-6), np.abs(r - 4.0).max()
        # the bound molecules have spread over the sphere
        assert np.abs((pos - 10.0).mean(0)).max() < 1.0
    text = fill(SPHERE, L=20, T=1.0, dt=0.005)
    ref, gpu = compare(text, ["out.txt", "outf.txt"], [1], "sphere", check=on_sphere)
    G = np.stack([g[1] for g in gpu])
    t, b = G[0, :, 0], G[:, :, 1].mean(0)
    # irreversible desorption at 0.8/s from a start of 2000
    assert np.all(np.abs(b - 2000 * np.exp(-0.8 * t)) < 60), (b, 2000 * np.exp(-0.8 * t))


def test_cube_faces_neighbour_hopping():
    def on_cube(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert len(pos) == 2000
        on_face = np.min(np.stack([np.abs(pos - 5.0), np.abs(pos - 15.0)]), axis=0)  # distance per axis
        assert np.all(on_face.min(1) < 1e-6), on_face.min(1).max()
        assert np.all((pos > 5.0 - 1e-6) & (pos < 15.0 + 1e-6))
        # the four adjacent faces have been reached (the opposite one is too far
        # for this time; the reference reaches it as rarely)
        assert {1, 3, 4, 5, 6} <= set(srf.tolist())
    text = fill(cube_config(), L=20, T=4.0, dt=0.01)
    outs = ["out_%s.txt" % nm for nm, _ in FACES]
    compare(text, outs, [1], "cube", check=on_cube)


def test_flip_front_back():
    text = fill(FLIP, L=20, T=2.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outb.txt"], [1], "flip")
    G = np.stack([g[1] for g in gpu])
    t, c = G[0, :, 0], G[:, :, 1].mean(0)
    # two-state kinetics: back -> 2000 * 2/3 (1 - exp(-3 t)) (rates 2 and 1)
    assert np.all(np.abs(c - 2000 * 2 / 3 * (1 - np.exp(-3 * t))) < 40)


def test_one_way_transmission_rate():
    text = fill(TRANSMIT, L=20, T=1.0, dt=0.005)
    _, gpu = compare(text, ["out.txt"], [1, 2], "transmit")
    B = np.stack([g[0][:, 2] for g in gpu])
    assert B[:, -1].mean() > 50


def test_first_order_reactions_of_bound_molecules():
    text = fill(BOUNDRXN, L=20, T=2.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outa.txt", "outb.txt"], [1], "boundrxn")
    A = np.stack([g[1] for g in gpu])
    t, a = A[0, :, 0], A[:, :, 1].mean(0)
    # A(front) leaves by two first-order reactions, 1 + 0.2 per unit time
    assert np.all(np.abs(a - 2000 * np.exp(-1.2 * t)) < 40), (a, 2000 * np.exp(-1.2 * t))
    C = np.stack([g[0][:, 3] for g in gpu]).mean(0)
    assert C[-1] > 300  # B(front) -> C(soln) released molecules into solution


def test_capsule_cylinder_and_hemisphere_caps():
    def on_capsule(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert len(pos) == 2000
        x = pos[:, 0]
        c = np.where(x < 8, 8.0, np.where(x > 12, 12.0, x))  # nearest point of the axis segment
        r = np.sqrt((x - c) ** 2 + (pos[:, 1] - 10) ** 2 + (pos[:, 2] - 10) ** 2)
        assert np.all(np.abs(r - 2.0) < 1e-6), np.abs(r - 2.0).max()
        assert set(srf.tolist()) == {1, 2}
    text = fill(CAPSULE, L=20, T=2.0, dt=0.01)
    _, gpu = compare(text, ["out_body.txt", "out_caps.txt"], [1], "capsule", check=on_capsule)
    caps = np.stack([g[1][:, 1] for g in gpu]).mean(0)
    assert caps[-1] > 500  # the caps (half the area) fill from the cylinder



def test_bound_solution_pair_reactions():
    def on_plane(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert len(pos) > 100
        assert np.all(np.abs(pos[:, 0] - 10.0) < 1e-6) and np.all(pos[:, 0] > 10.0)  # the front side
        assert set(sp.tolist()) <= {1, 3}  # A and C
    text = fill(BIRXN, L=20, T=3.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outb.txt"], [1, 2, 3, 4], "birxn", check=on_plane)
    G = np.stack([g[0] for g in gpu]).mean(0)
    assert G[-1, 1] < 1800 and G[-1, 3] > 200 and G[:, 4].max() > 3  # A reacted; C formed; D released
    Bk = np.stack([g[1] for g in gpu]).mean(0)
    assert np.all(Bk[:, 2] > 1800)  # B behind the panel (x < 10) does not react


def test_bound_solution_pair_reaction_back_state():
    """A(back) + B -> C(bsoln): the solution reactant is read against the
    panel's front side (morebireact), the product starts behind the panel."""
    def on_back(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert len(pos) > 100 and np.all(st == sb.MSback) and np.all(pos[:, 0] < 10.0)
    text = fill(BIRXN_BACK, L=20, T=2.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outb.txt"], [1, 2, 3], "birxn_back", check=on_back)
    G = np.stack([g[0] for g in gpu]).mean(0)
    Bk = np.stack([g[1] for g in gpu]).mean(0)
    assert G[-1, 3] > 50  # C formed
    assert np.all(np.abs(Bk[:, 3] - G[:, 3]) < 1e-9)  # every C starts (and, reflected, stays) behind


def test_reversible_surface_binding_and_emission():
    def on_plane(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert np.all(np.abs(pos[:, 0] - 10.0) < 1e-6) and np.all(pos[:, 0] > 10.0)
        assert set(sp.tolist()) <= {1, 3} and len(pos) == 1000  # A and C: bound molecules are conserved
    text = fill(REVBIND, L=20, T=3.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outb.txt"], [1, 2, 3, 4], "revbind", check=on_plane)
    G = np.stack([g[0] for g in gpu]).mean(0)
    assert G[-1, 3] > 50 and G[-1, 4] > 300  # complexes formed; D emitted
    Bk = np.stack([g[1] for g in gpu]).mean(0)
    assert np.all(Bk[:, 4] < 1e-9)  # D starts in front of the panel and stays there


def test_surface_restricted_reactions():
    def per_surface(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert np.all(sp[srf == 2] == 1)  # A(front) on s2 does not convert (r1 is restricted to s1)
    text = fill(SRFRXN, L=20, T=2.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "out1.txt"], [1, 2, 3], "srfrxn", check=per_surface)
    G = np.stack([g[0] for g in gpu]).mean(0)
    t, b = G[:, 0], np.stack([g[1][:, 2] for g in gpu]).mean(0)  # B(front) on s1
    assert np.all(np.abs(b - 1000 * (1 - np.exp(-t))) < 40)  # only the 1000 molecules on s1 convert
    assert G[-1, 3] < 2950  # C reacts at s2


def test_planar_bound_states():
    def on_circle(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        r = np.hypot(pos[:, 0] - 50.0, pos[:, 1] - 50.0)
        assert len(pos) > 100 and np.all(np.abs(r - 20.0) < 1e-6) and np.all(pos[:, 2] == 0)
    text = fill(PLANAR, T=4.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outs.txt"], [1, 2, 3], "planar", check=on_circle)
    G = np.stack([g[1] for g in gpu]).mean(0)
    assert G[-1, 3] > 20  # complexes on the circle


def test_births_on_a_surface():
    def on_sphere(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        r = np.linalg.norm(pos - 10.0, axis=1)
        assert len(pos) > 100 and np.all(np.abs(r - 4.0) < 1e-6)
        assert np.abs((pos - 10.0).mean(0)).max() < 1.0  # spread over the sphere
    text = fill(SRFBIRTH, L=20, T=3.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outi.txt"], [1, 2], "srfbirth", check=on_sphere)
    G = np.stack([g[0] for g in gpu]).mean(0)
    t, a = G[:, 0], G[:, 1]
    area = 4 * np.pi * 16
    # births at 2 per unit area and time, decay at 0.5: A(t) = 4 area (1 - exp(-t/2))
    assert np.all(np.abs(a - 4 * area * (1 - np.exp(-0.5 * t))) < 30), (a, 4 * area * (1 - np.exp(-0.5 * t)))


def test_bound_bound_reactions():
    def on_plane(s):
        pos, sp, st, srf, pnl, sn = s.surface_molecules()
        assert np.all(np.abs(pos[:, 0] - 10.0) < 1e-6) and np.all(pos[:, 0] > 10.0)
    text = fill(BBRXN, L=20, T=3.0, dt=0.01)
    _, gpu = compare(text, ["out.txt"], [1, 2, 3, 4], "bbrxn", check=on_plane)
    G = np.stack([g[0] for g in gpu]).mean(0)
    assert G[-1, 2] > 50 and G[-1, 3] < 450  # dimers formed; D and E removed each other


def test_jump_surfaces():
    text = fill(JUMP, L=20, T=3.0, dt=0.01)
    _, gpu = compare(text, ["out.txt", "outl.txt"], [1], "jump")
    L = np.stack([g[1][:, 1] for g in gpu]).mean(0)
    assert np.all(np.stack([g[0][:, 1] for g in gpu]) == 2000)  # nothing lost at the ends
    assert L[-1] < 1900  # molecules crossed the left end into the right half
