"""Generate tests/golden/bound_pair_params.npz from the reference binary.

Seeded random configurations with second-order reactions between a
surface-bound reactant (front or back state, first or second reactant) and a
solution reactant are loaded by oracle/_ref/smoldyn with `-t` (text output,
no simulation past the start); its "Reaction details" block prints, per
reaction, the requested and actual rate constants and the binding radius
(rxnsetrate smolreact.c:1364-1410, rxncalcrate :1592-1680).  Stored: the
configuration texts, the reaction names and the printed actual rates and
binding radii.
Usage: python tests/golden/make_bound_pair_golden.py   (needs `make -C oracle ref`)
"""
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "smoldyn")
NCASE = 24


def make_config(rng):
    dt = 10 ** rng.uniform(-4, -2)
    dsol = 10 ** rng.uniform(-1, 1, 2)
    dfront, dback = 10 ** rng.uniform(-2, 0, 2)
    lines = ["dim 3", "species A B C", "difc B %.6g" % dsol[0], "difc C %.6g" % dsol[1],
             "difc A(front) %.6g" % dfront, "difc A(back) %.6g" % dback,
             "difc C(front) %.6g" % (0.5 * dfront),
             "time_start 0", "time_stop %.6g" % dt, "time_step %.6g" % dt]
    lines += ["boundaries %d 0 10 r" % d for d in range(3)]
    lines += ["random_seed 1", "start_surface s1", "action both all reflect",
              "panel rect +0 5 0 0 10 10 r1", "end_surface"]
    names = []
    forms = ["A(front) + B -> C(front)", "B + A(back) -> C", "A(front) + C -> 0", "C + A(front) -> A(front)",
             "A(back) + B -> C(bsoln)", "A(front) + A -> A(front)"]
    pick = rng.choice(len(forms), size=3, replace=False)
    for q, f in enumerate(pick):
        nm = "r%d" % q
        names.append(nm)
        lines.append("reaction %s %s %.6g" % (nm, forms[f], 10 ** rng.uniform(-1.5, 0.5)))
    lines.append("end_file")
    return "\n".join(lines) + "\n", names


def run_ref(text):
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text)
        out = subprocess.run([REF, "c.txt", "-t"], cwd=d, capture_output=True, text=True, timeout=120,
                             stdin=subprocess.DEVNULL, env=dict(os.environ, SMOLDYN_NO_PROMPT="1")).stdout
    res = {}
    for m in re.finditer(r"Reaction (\w+):[^\n]*\n\s*requested and actual rate constants : ([^,]+), (\S+)\n"
                         r"\s*binding radius: (\S+)", out):
        res[m.group(1)] = (float(m.group(3)), float(m.group(4)))
    return res


def main():
    rng = np.random.default_rng(20260611)
    texts, names, rates, radii = [], [], [], []
    for _ in range(NCASE):
        text, nms = make_config(rng)
        res = run_ref(text)
        assert set(res) == set(nms), (res, nms, text)
        texts.append(text)
        names.append(",".join(nms))
        rates.append([res[n][0] for n in nms])
        radii.append([res[n][1] for n in nms])
    np.savez(os.path.join(HERE, "bound_pair_params.npz"), texts=np.array(texts), names=np.array(names),
             rates=np.array(rates), radii=np.array(radii))
    print("wrote", NCASE, "cases")


if __name__ == "__main__":
    main()
