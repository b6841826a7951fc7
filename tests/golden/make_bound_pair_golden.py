"""Generate tests/golden/bound_pair_params.npz from the reference binary.

Seeded random configurations with reactions of surface-bound reactants are
loaded by oracle/_ref/smoldyn with `-t` (text output, no simulation past the
start): second-order reactions between a bound reactant (front or back
state, first or second reactant) and a solution reactant, reversible surface
binding (`A(front) + B <-> C(front)`, whose reverse is a first-order bound
reaction with a bound and a solution product), emission from a bound
molecule (`A(front) -> A(front) + B`) and reactions of two bound molecules
(`A(front) + C(front) -> A(front)`, reversible dimerization).  Its "Reaction details" block prints,
per reaction, the requested and actual rate constants, the binding radius
(second order) and the unbinding radius (two products) (rxnsetrate
smolreact.c:1307-1410, rxnsetproduct :1431-1577, rxncalcrate :1592-1680).
Stored: the configuration texts, the reaction names and the printed actual
rates, binding radii and unbinding radii (NaN where not printed).
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
NCASE = 40


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
             "A(back) + B -> C(bsoln)", "A(front) + A -> A(front)", "A(front) + B <-> C(front)",
             "C(front) -> A(front) + B", "A(front) -> A(front) + B", "A(back) -> C(front) + B(bsoln)",
             "A(front) + C(front) -> A(front)", "A(front) + A(front) -> C(front)", "A(back) + A(front) -> 0",
             "A(front) + A(front) <-> C(front)"]
    pick = rng.choice(len(forms), size=3, replace=False)
    for q, f in enumerate(pick):
        nm = "r%d" % q
        if "<->" in forms[f]:
            names += [nm + "fwd", nm + "rev"]
            lines.append("reaction %s %s %.6g %.6g" % (nm, forms[f], 10 ** rng.uniform(-1.5, 0.5),
                                                       10 ** rng.uniform(-1.5, 0.5)))
        else:
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
    blocks = re.split(r"\n\s*Reaction (?=\w+:)", out)
    for blk in blocks[1:]:
        name = blk.split(":", 1)[0]
        m = re.search(r"requested and actual rate constants : [^,]+, (\S+)", blk)
        if not m:
            continue
        b = re.search(r"\n\s*binding radius: (\S+)", blk)
        u = re.search(r"\n\s*unbinding radius: (\S+)", blk)
        res[name] = (float(m.group(1)), float(b.group(1)) if b else float("nan"),
                     float(u.group(1)) if u else float("nan"))
    return res


def main():
    rng = np.random.default_rng(20260611)
    texts, names, rates, radii, uradii = [], [], [], [], []
    for _ in range(NCASE):
        text, nms = make_config(rng)
        res = run_ref(text)
        assert set(nms) <= set(res), (res, nms, text)
        texts.append(text)
        names.append(",".join(nms))
        rates.append([res[n][0] for n in nms] + [np.nan] * (6 - len(nms)))
        radii.append([res[n][1] for n in nms] + [np.nan] * (6 - len(nms)))
        uradii.append([res[n][2] for n in nms] + [np.nan] * (6 - len(nms)))
    np.savez(os.path.join(HERE, "bound_pair_params.npz"), texts=np.array(texts), names=np.array(names),
             rates=np.array(rates), radii=np.array(radii), uradii=np.array(uradii))
    print("wrote", NCASE, "cases")


if __name__ == "__main__":
    main()
