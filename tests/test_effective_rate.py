"""Effective rate constants (rxncalcrate, smolreact.c:1592-1680) against the
reference.

The same configuration goes through this library's config reader and
parameter derivation (smolgpuGetEffectiveRate, host FP64, no GPU needed) and
through the reference engine compiled from its sources (oracle/_ref/
ref_harness in "rates" mode calls the reference's own rxncalcrate after
smolUpdateSim).  Rates and geminate probabilities agree to 1e-9 relative;
the rate implied by the derived parameters reproduces the requested rate to
the bisection tolerance of the radius solve.
"""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

HARNESS = os.path.join(oracle_lib.REF_DIR, "ref_harness")

BASE = """dim 3
species A B C D
difc A 1
difc B 0.7
difc C 0.5
difc D 2
boundaries 0 0 50 r
boundaries 1 0 50 r
boundaries 2 0 50 r
time_start 0
time_stop 1
time_step 0.01
random_seed 3
"""

CASES = {
    "default_placement": (["fwd A + B -> C 0.05", "rev C -> A + B 0.1"], []),
    "ratio": (["fwd A + B -> C 2", "rev C -> A + B 1"], ["product_placement rev ratio 0.2"]),
    "unbindrad": (["fwd A + B -> C 5", "rev C -> A + B 3"], ["product_placement rev unbindrad 0.4"]),
    "pgem": (["fwd A + B -> C 1", "rev C -> A + B 0.5"], ["product_placement rev pgem 0.05"]),
    "same_species_and_lists": (["dimer A + A -> D 0.3", "split D -> A + A 0.2", "decay D -> 0 0.05",
                                "birth 0 -> B 0.001"], []),
    "irreversible": (["fwd A + D -> C 10"], []),
    "confspread": (["fwd A + B -> A + C 5"], ["confspread_radius fwd 0.3"]),
    "bounce": (["fwd A + B -> A + B 2"], ["product_placement fwd bounce 0.6"]),
    "anisotropic": (["fwd A + B -> C 1"], ["difm A 1 0.5 0 0 2 0 0 0 0.5"]),
    # reaction probability p < 1: bindingradiusprob's 1-D search (rxnparam.c:612-636)
    "probability": (["fwd A + B -> C 0.05"], ["reaction_probability fwd 0.3"]),
    "probability_reversible": (["fwd A + B -> C 2", "rev C -> A + B 1"],
                               ["reaction_probability fwd 0.5", "product_placement rev ratio 1.5"]),
    "probability_unbindrad": (["fwd A + B -> C 5", "rev C -> A + B 3"],
                              ["reaction_probability fwd 0.2", "product_placement rev unbindrad 0.4"]),
    # requested chi: the 2-D search over (radius, probability) (rxnparam.c:638-676)
    "chi": (["fwd A + B -> C 0.05"], ["reaction_chi fwd 0.01"]),
    "chi_reversible": (["fwd A + B -> C 2", "rev C -> A + B 1"],
                       ["reaction_chi fwd 0.05", "product_placement rev ratio 1.5"]),
}
NAMES = {
    "default_placement": [(2, "fwd"), (1, "rev")],
    "ratio": [(2, "fwd"), (1, "rev")],
    "unbindrad": [(2, "fwd"), (1, "rev")],
    "pgem": [(2, "fwd"), (1, "rev")],
    "same_species_and_lists": [(2, "dimer"), (1, "split"), (1, "decay"), (0, "birth")],
    "irreversible": [(2, "fwd")],
    "confspread": [(2, "fwd")],
    "bounce": [(2, "fwd")],
    "anisotropic": [(2, "fwd")],
    "probability": [(2, "fwd")],
    "probability_reversible": [(2, "fwd"), (1, "rev")],
    "probability_unbindrad": [(2, "fwd"), (1, "rev")],
    "chi": [(2, "fwd")],
    "chi_reversible": [(2, "fwd"), (1, "rev")],
}


def config(rxns, extra):
    txt = BASE
    for r in rxns:
        txt += "reaction %s\n" % r
    for e in extra:
        txt += e + "\n"
    return txt + "mol 100 A u u u\nmol 100 B u u u\nend_file\n"


def reference_rates(d, name):
    out = os.path.join(d, "rates.txt")
    subprocess.run([HARNESS, d + "/", name, out, "rates"], check=True, stdin=subprocess.DEVNULL,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   env=dict(os.environ, SMOLDYN_NO_PROMPT="1"), timeout=120)
    res = {}
    for ln in open(out):
        t = ln.split()
        if t and t[0] == "R":
            res[(int(t[1]), int(t[2]))] = (float(t[3]), float(t[4]))
        if t and t[0] == "P":  # second-order binding radius squared and probability
            res[("P", int(t[1]))] = (float(t[2]), float(t[3]))
    return res


@pytest.mark.parametrize("case", sorted(CASES))
def test_effective_rate_matches_reference(case):
    if not os.path.exists(HARNESS):
        pytest.skip("reference harness not built")
    rxns, extra = CASES[case]
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(config(rxns, extra))
        ref = reference_rates(d, "c.txt")
        lib = sb.load()
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
        s = sb.Sim(ptr=simp.value)
        counters = {0: 0, 1: 0, 2: 0}
        for order, nm in NAMES[case]:
            r = counters[order]
            counters[order] += 1
            rate, pgem = s.effective_rate(nm)
            rr, rp = ref[(order, r)]
            assert abs(rate - rr) <= 1e-9 * abs(rr) + 1e-300, (nm, rate, rr)
            assert abs(pgem - rp) <= 1e-9 * max(abs(rp), 1e-12), (nm, pgem, rp)
            if order == 2 and ("P", r) in ref:
                # binding radius and reaction probability as derived (rxnsetrate, smolreact.c:1396-1408)
                b2_ref, p_ref = ref[("P", r)]
                b, _, p = s.reaction_params(nm)
                assert abs(b * b - b2_ref) <= 1e-9 * b2_ref + 1e-300, (nm, b * b, b2_ref)
                assert abs(p - p_ref) <= 1e-9 * max(p_ref, 1e-12), (nm, p, p_ref)
        s.close()


def test_effective_rate_reproduces_requested_rate():
    """rate -> binding radius (doubling + 15 bisections) -> rate: the round
    trip is within the bisection tolerance for an irreversible reaction."""
    s = sb.Sim(3, (0, 0, 0), (50, 50, 50))
    s.add_species("A", 1.0)
    s.add_species("B", 1.0)
    s.add_species("C", 0.5)
    s.set_times(0, 1, 0.01)
    for k in (0.01, 0.1, 1.0, 10.0):
        s.add_reaction("r%g" % k, "A", "B", ["C"], k)
    for k in (0.01, 0.1, 1.0, 10.0):
        rate, _ = s.effective_rate("r%g" % k)
        assert abs(rate / k - 1) < 2e-4, (k, rate)
