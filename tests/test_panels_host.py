"""Panel definitions on the host (surfaddpanel, smolsurface.c:2432): bad
parameters are rejected when the panel is added, before any engine exists;
the config reader accepts every shape.  No GPU needed."""
import ctypes as C
import os
import tempfile

import numpy as np

import smoldyn_b200 as sb


def test_panel_parameters_are_checked():
    lib = sb.load()
    s = sb.Sim(3, (0, 0, 0), (20, 20, 20))
    s.add_species("A", 1.0)
    assert lib.smolAddSurface(s.ptr, b"s") == 0
    bad = {
        sb.PScyl: [1, 1, 1, 1, 1, 1, 2],          # coincident end points
        sb.PSdisk: [5, 5, 5, 2, 0, 0, 0],         # zero normal
        sb.PStri: [0, 0, 0, 1, 1, 1, 2, 2, 2],    # collinear vertices
        sb.PShemi: [5, 5, 5, 2, 0, 0, 0],         # zero outward vector
    }
    for shape, prm in bad.items():
        arr = np.array(prm, dtype=float)
        assert lib.smolAddPanel(s.ptr, b"s", shape, None, None, sb.dptr(arr)) < 0
    ok = np.array([1, 1, 1, 1, 1, 5, 2], dtype=float)
    assert lib.smolAddPanel(s.ptr, b"s", sb.PScyl, None, None, sb.dptr(ok)) == 0


def test_config_reader_accepts_all_shapes():
    text = """dim 3
species A
difc A 1
boundaries 0 0 20
boundaries 1 0 20
boundaries 2 0 20
time_start 0
time_stop 1
time_step 0.01
start_surface s
action both all reflect
panel rect +0 0 0 0 20 20 r1
panel sph 10 10 10 -3 20 20
panel tri 4 4 10 16 5 9 9 16 11 t1
panel cyl 10 10 4 10 12 16 4 20 20
panel hemi 10 10 10 5 0 0.6 0.8 20 20
panel disk 10 10 10 5 1 0.5 0 20
end_surface
end_file
"""
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text)
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    sb.Sim(ptr=simp.value).close()
