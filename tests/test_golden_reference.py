"""The engine oracle against one step recorded from the reference itself.

The fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
reference engine compiled in oracle/_ref) hold the reference's start state,
its displacements and first-order outcomes for one step, and its state after
the step.  ora_step (oracle/engine_oracle.c) given the same displacements and
outcomes must reproduce that state: survivors and their positions to 1e-9 of
the box side, products at the same places, pair events identical away from
ties and ambiguous groups.  This pins the oracle the GPU parity tests use.
"""
import numpy as np
import pytest

from tests import golden_cases as gd
from tests import gpu_cases as gc
from tests import oracle_lib


@pytest.mark.parametrize("name", gd.CASES)
def test_oracle_reproduces_reference_step(name):
    g = gd.load(name)
    force = np.where(g["uni"] == 1, 0, -1).astype(np.int32)
    net = gc.oracle_net(None, g["L"], g["wall"], gd.DIFC, g["bind2"], (0.0, 0.0))
    o = oracle_lib.ora_step(net, g["pos0"], g["sp0"], g["serno0"], g["disp"], force)
    act = dict(pos=o["pos"], sp=o["sp"], serno=o["serno"], orig=o["parent"] == 0)
    ncommon, nprod, nties = gd.compare(g, gd.reference_state(g), act, 1e-9)
    assert ncommon > 2500 and nprod >= 10, (ncommon, nprod, nties)


@pytest.mark.parametrize("name", gd.CASES)
def test_fixture_binding_radius_matches_host_solver(name):
    """The reference's bindrad2 equals the radius this library derives
    (smolgpuGetReactionParams, CPU only) to 1e-9."""
    import smoldyn_b200 as sb
    g = gd.load(name)
    s = gc.make_sim(L=g["L"], wall=g["wall"], kf=g["kf"], kr=g["kr"], difc=gd.DIFC, dt=gd.DT,
                    rev_placement=(sb.RPirrev, 0.0))
    bind, _, _ = s.reaction_params("fwd")
    assert abs(bind * bind - g["bind2"]) <= 1e-9 * g["bind2"]
