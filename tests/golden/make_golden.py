"""Generate the one-step golden fixtures from the reference engine itself.

Runs oracle/_ref/ref_harness (the reference's libsmoldyn compiled from its
sources, with its diffuse and unireact wrapped to record displacements and
first-order outcomes) on the configurations below and writes
tests/golden/<name>.npz with:
  pos0, sp0, serno0   state at the start of the step (reference's own initial
                      placement from its config, seed fixed)
  disp                the reference's displacement of each molecule this step
  uni                 1 where the reference's first-order reaction fired
  bind2               squared binding radius of A + B -> C (reference value)
  pos1, sp1, serno1   the reference's state after the step
  L, wall, kf, kr     cube side, boundary type ("t": walls transparent, the
                      case's surfaces close the box), rate constants
  ub                  unbinding radius of the unbind case (-1 elsewhere)
  config              the configuration text the reference ran
Usage: python tests/golden/make_golden.py   (needs `make -C oracle ref`)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

# A + B <-> C with the reverse products at the reaction site (irrev placement:
# zero unbinding radius), so a step has no random product orientation.
CONFIG = """dim 3
species A B C
difc A 1
difc B 1
difc C 0.5
time_start 0
time_stop 1
time_step 0.01
boundaries 0 0 {L} {w}
boundaries 1 0 {L} {w}
boundaries 2 0 {L} {w}
random_seed {seed}
reaction fwd A + B -> C {kf}
reaction rev C -> A + B {kr}
product_placement rev irrev
mol {nA} A u u u
mol {nB} B u u u
mol {nC} C u u u
end_file
"""

# Bimolecular product placement: confspread (products take the reactants'
# places and serial numbers) and bounce (reactants pushed apart to the
# unbinding distance); probability 1 so every in-radius pair is decided by
# geometry alone.
PLACEMENT_CONFIG = """dim 3
species A B C
difc A 1
difc B 1
difc C 0.5
time_start 0
time_stop 1
time_step 0.01
boundaries 0 0 {L} p
boundaries 1 0 {L} p
boundaries 2 0 {L} p
random_seed {seed}
{reactions}
mol {nA} A u u u
mol {nB} B u u u
end_file
"""
PLACEMENT_CASES = {
    "onestep_confspread": dict(L=20, seed=21, nA=1500, nB=1500,
                               reactions="reaction fwd A + B -> A + C 1e6\nconfspread_radius fwd 0.4"),
    "onestep_bounce": dict(L=20, seed=22, nA=1500, nB=1500,
                           reactions="reaction fwd A + B -> A + B\nbinding_radius fwd 0.4\n"
                                     "product_placement fwd bounce 0.6"),
}

# Surface reflection by every panel shape: a cube closed by reflective
# rectangles holds a tilted triangle, a cylinder, a hemisphere and a disk,
# all reflective; no reactions, and a large diffusion coefficient so that many
# molecules meet a panel in the one recorded step.
SURFACE_CONFIG = """dim 3
species A
difc A 4
time_start 0
time_stop 1
time_step 0.01
boundaries 0 0 {L}
boundaries 1 0 {L}
boundaries 2 0 {L}
random_seed {seed}
start_surface walls
action both all reflect
panel rect +0 0 0 0 {L} {L}
panel rect -0 {L} 0 0 {L} {L}
panel rect +1 0 0 0 {L} {L}
panel rect -1 0 {L} 0 {L} {L}
panel rect +2 0 0 0 {L} {L}
panel rect -2 0 0 {L} {L} {L}
end_surface
start_surface shapes
{actions}
panel tri 1 1 5 9 2 4.5 4 9 5.5
panel disk 4 7 3 1.5 0.6 0.8 0 20
end_surface
start_surface tube
{tube_action}
panel cyl 3 5 2 7 5 8 2 20 20
end_surface
start_surface cap
{cap_action}
panel hemi 7 3 7 2 0.3 -0.5 0.8 20 20
end_surface
mol {nA} A u u u
end_file
"""
SURFACE_CASES = {
    "onestep_panels": dict(L=10, seed=31, nA=4000, actions="action both all reflect",
                           tube_action="action both all reflect", cap_action="action both all reflect"),
    # mixed actions: the triangle absorbs on its front face and reflects on
    # its back, the cylinder transmits, the hemisphere absorbs
    "onestep_panels_actions": dict(L=10, seed=32, nA=4000,
                                   actions="action both all reflect\naction front all absorb",
                                   tube_action="action both all transmit", cap_action="action both all absorb"),
}

# Product placement at the unbinding radius: every C splits into A + B in the
# recorded step (rate 1000, so the first-order probability 1 - e^-10) with
# product_placement unbindrad, so each pair of products sits at distance 0.6
# along one random direction, split by the products' diffusion coefficients
# (rxnsetproduct, smolreact.c:1545-1548; random orientation in doreact,
# smolreact.c:2840-2850).  C does not diffuse, so the reaction sites are the
# start positions.
UNBIND_CONFIG = """dim 3
species A B C
difc A 1
difc B 0.5
difc C 0
time_start 0
time_stop 1
time_step 0.01
boundaries 0 0 {L} p
boundaries 1 0 {L} p
boundaries 2 0 {L} p
random_seed {seed}
reaction split C -> A + B 1000
product_placement split unbindrad {ub}
mol {nC} C u u u
end_file
"""
UNBIND_CASES = {"onestep_unbind": dict(L=100, seed=41, nC=3000, ub=0.6)}

CASES = {
    "onestep_reflect": dict(L=20, w="r", seed=11, kf=20, kr=1, nA=1600, nB=1600, nC=800),
    "onestep_periodic": dict(L=20, w="p", seed=12, kf=20, kr=1, nA=1600, nB=1600, nC=800),
    "onestep_sparse": dict(L=20, w="p", seed=13, kf=1, kr=1, nA=1600, nB=1600, nC=800),
}
SPECIES = {1: "A", 2: "B", 3: "C"}


def run_case(name, cfg, template=CONFIG):
    text = template.format(**cfg)
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "cfg.txt"), "w") as f:
            f.write(text)
        out = os.path.join(tmp, "out.txt")
        subprocess.run([HARNESS, tmp + "/", "cfg.txt", out], check=True, stdin=subprocess.DEVNULL,
                       stdout=subprocess.DEVNULL)
        D, U, F, B = [], [], [], {}
        for line in open(out):
            t = line.split()
            if t[0] == "D":
                D.append((int(t[1]), int(t[2]), *map(float, t[3:9])))
            elif t[0] == "U":
                U.append(int(t[1]))
            elif t[0] == "F":
                F.append((int(t[1]), int(t[2]), *map(float, t[3:6])))
            elif t[0] == "B":
                B[int(t[1])] = float(t[2])
    D.sort()
    F.sort()
    serno0 = np.array([d[0] for d in D], dtype=np.uint64)
    uset = set(U)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        pos0=np.array([d[2:5] for d in D]), sp0=np.array([d[1] for d in D], dtype=np.int32), serno0=serno0,
        disp=np.array([d[5:8] for d in D]),
        uni=np.array([1 if int(s) in uset else 0 for s in serno0], dtype=np.int32),
        bind2=np.float64(B.get(0, 0.0)),
        pos1=np.array([f[2:5] for f in F]), sp1=np.array([f[1] for f in F], dtype=np.int32),
        serno1=np.array([f[0] for f in F], dtype=np.uint64),
        L=np.float64(cfg["L"]), wall=np.array(cfg.get("w", "t")), kf=np.float64(cfg.get("kf", -1)),
        kr=np.float64(cfg.get("kr", -1)), ub=np.float64(cfg.get("ub", -1)), config=np.array(text))
    print(name, "molecules", len(D), "->", len(F), "first-order", len(U))


if __name__ == "__main__":
    if not os.path.exists(HARNESS):
        sys.exit("build the reference first: make -C oracle ref")
    for k, v in CASES.items():
        run_case(k, v)
    for k, v in PLACEMENT_CASES.items():
        run_case(k, v, PLACEMENT_CONFIG)
    for k, v in SURFACE_CASES.items():
        run_case(k, v, SURFACE_CONFIG)
    for k, v in UNBIND_CASES.items():
        run_case(k, v, UNBIND_CONFIG)
