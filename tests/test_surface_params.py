"""Surface interaction probabilities derived from rates, against the reference.

tests/golden/surface_probs.npz holds, for 48 seeded random configurations of
adsorption, desorption, flip and one- and two-way transmission rates (two
species, one rectangle), the action of every (species, state, face) and the
probabilities, cumulative probabilities and reverse probabilities that the
reference's own surfupdateparams derived (written by
tests/golden/make_surface_golden.py through oracle/_ref/ref_harness).  The
host restatement (smoldyn_b200/csrc/surface.cpp, surfparam.h) must give the
same actions and the same numbers to 1e-9.  The adsorption probabilities
interpolate the reference's published tables, so this also pins the
interpolation; rates of -1 ("every time") and rate_internal probabilities
are among the cases.  One exception to 1e-9: one-way transmission (a
fsoln -> bsoln rate) with the back face left transmitting is reversible
transmission with the reverse "always"; the reference finds the unknown
coefficient by a random walk that stops at 0.1% steps and reports its last
trial, the restatement solves for it exactly, so those rules (and the rules
of that species whose reverse probability is that one) agree to 2e-3 in
absolute terms.
The CPU suite needs no GPU: the derivation is host code, read back through
smolgpuGetSurfaceRule.
"""
import os
import tempfile

import numpy as np
import smoldyn_b200 as sb

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "surface_probs.npz")


def load_case(text):
    d = tempfile.mkdtemp()
    path = os.path.join(d, "c.txt")
    with open(path, "w") as f:
        f.write(text)
    return sb.Sim.load_file(path)


def transmission_walk(text, name):
    """Whether the reference's random walk decides a transmission probability
    of species `name`: one direction given, the other the default "always"
    (no rate) or -1, but not both."""
    rates = {}
    for ln in text.splitlines():
        w = ln.split()
        if len(w) >= 5 and w[0] == "rate" and w[1] == name and {w[2], w[3]} == {"fsoln", "bsoln"}:
            rates[w[2]] = float(w[4])
    if not rates:
        return False
    fwd, back = rates.get("fsoln"), rates.get("bsoln")
    if fwd is None or back is None:
        return True
    return (fwd == -1) != (back == -1)


def test_derived_probabilities_match_reference():
    g = np.load(GOLD)
    configs, acts, probs = g["configs"], g["acts"], g["probs"]
    names = {1: "A", 2: "B"}
    nrule = 0
    worst = 0.0
    for c, text in enumerate(configs):
        s = load_case(str(text))
        ref_rows = {tuple(int(v) for v in r[1:5]): r[5:] for r in probs[probs[:, 0] == c]}
        for row in acts[acts[:, 0] == c]:
            _, srf, sp, ms, face, act = (int(v) for v in row)
            a, pr, cu, rv = s.surface_rule("s1", names[sp], ms, face)
            assert a == act, (c, srf, sp, ms, face, a, act)
            key = (srf, sp, ms, face)
            if key in ref_rows:
                ref = ref_rows[key]
                got = np.concatenate([pr, cu, rv])
                err = np.abs(got - ref) / np.maximum(1e-300, np.maximum(np.abs(ref), 1e-3))
                # the walk's result, and the rules whose reverse probability is it
                walk = transmission_walk(str(text), names[sp])
                if walk:
                    ok = np.all(np.abs(got - ref) <= 2e-3)
                else:
                    worst = max(worst, float(err.max()))
                    ok = np.all(err <= 1e-9)
                assert ok, (c, key, got, ref, str(text))
                nrule += 1
        s.close()
    print("%d rate-based rules matched; worst relative difference %.3g" % (nrule, worst))
    assert nrule > 100
