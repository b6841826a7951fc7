"""Compiled C clients of the drop-in boundary.

1. The C example of INTEGRATION.md, compiled from the document as it stands
   with warnings for implicit declarations turned into errors (gcc >= 14
   rejects those by default), linked against libsmoldyn_b200.so; on the GPU
   it runs the plain small reaction and prints a C count.
2. The reference's own libsmoldyn client,
   examples/S97_libsmoldyn/testcode/testcode.c (a Lotka-Volterra system of
   rabbits and foxes in a periodic slab, with molecule lists and display
   calls), compiled unchanged against include/libsmoldyn.h and this library
   (oracle/_ref/testcode_b200), and against the reference library
   (oracle/_ref/testcode_ref); `make -C oracle client` builds both where the
   reference sources are present.  On the GPU both builds must run to
   completion and print the same 19 report lines.  The client fixes its
   random seed, so one run of either build is one realisation of a
   Lotka-Volterra system started at its fixed point (R = F = 1000), which
   oscillates with a growing random amplitude; the b200 run's counts are
   therefore compared with the envelope (widened by a factor of two) of 24
   seeds of the same model written as a configuration file and run by the
   reference binary.
"""
import os
import re
import shutil
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
B200_CLIENT = os.path.join(oracle_lib.REF_DIR, "testcode_b200")
REF_CLIENT = os.path.join(oracle_lib.REF_DIR, "testcode_ref")
LINE = re.compile(r"t= ([0-9.eE+-]+), rabbit = (\d+), fox=(\d+)")


def integration_example():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```c\n(.*?)```", text, flags=re.S)
    assert m, "no C example in INTEGRATION.md"
    return m.group(1)


def build_example(workdir):
    src = os.path.join(workdir, "demo.c")
    with open(src, "w") as f:
        f.write(integration_example())
    exe = os.path.join(workdir, "demo")
    sb.load()
    libdir = os.path.dirname(sb.LIB_PATH)
    subprocess.check_call(["gcc", "-Wall", "-Werror=implicit-function-declaration", src,
                           "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lsmoldyn_b200",
                           "-Wl,-rpath," + libdir, "-o", exe])
    return exe


def parse_report(text):
    rows = [(float(a), int(b), int(c)) for a, b, c in LINE.findall(text)]
    return np.array(rows)


def test_integration_example_compiles():
    with tempfile.TemporaryDirectory() as d:
        exe = build_example(d)
        assert os.path.exists(exe)


def test_reference_client_links_against_b200():
    if not os.path.exists(B200_CLIENT):
        pytest.skip("oracle/_ref/testcode_b200 not built (needs the reference sources: make -C oracle client)")
    out = subprocess.check_output(["ldd", B200_CLIENT]).decode()
    assert "libsmoldyn_b200.so" in out and "not found" not in out
    # every libsmoldyn call the client makes resolves in this library
    und = subprocess.check_output(["nm", "-u", B200_CLIENT]).decode()
    calls = sorted({ln.split()[-1] for ln in und.splitlines() if ln.split()[-1].startswith("smol")})
    exported = subprocess.check_output(["nm", "-D", "--defined-only", sb.LIB_PATH]).decode()
    missing = [c for c in calls if (" T " + c) not in exported]
    assert len(calls) >= 15 and not missing, missing


@pytest.mark.gpu
def test_integration_example_runs():
    with tempfile.TemporaryDirectory() as d:
        exe = build_example(d)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=600, cwd=d)
        assert out.returncode == 0, out.stderr[-2000:]
        m = re.search(r"C: (-?\d+)", out.stdout)
        assert m and int(m.group(1)) > 0, out.stdout[-2000:]


LV_CONFIG = """dim 3
species rabbit fox
difc rabbit 100
difc fox 100
boundaries 0 -100 100 p
boundaries 1 -100 100 p
boundaries 2 -10 10 p
time_start 0
time_stop 2
time_step 0.001
random_seed %d
reaction r1 rabbit -> rabbit + rabbit 10
reaction r2 rabbit + fox -> fox + fox 8000
reaction r3 fox -> 0 10
mol 1000 rabbit u u u
mol 1000 fox u u u
output_files o.txt
cmd N 100 molcount o.txt
end_file
"""


@pytest.mark.gpu
def test_reference_client_runs_on_b200():
    if not (os.path.exists(B200_CLIENT) and os.path.exists(REF_CLIENT)):
        pytest.skip("reference client builds absent (make -C oracle client)")
    run = subprocess.run([B200_CLIENT], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr[-2000:]
    gpu = parse_report(run.stdout)
    assert gpu.shape == (19, 3), run.stdout[-2000:]

    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([REF_CLIENT], capture_output=True, text=True, timeout=600, cwd=d,
                           env=dict(os.environ, SMOLDYN_NO_PROMPT="1"))
    assert r.returncode == 0
    assert parse_report(r.stdout).shape == (19, 3)
    ref_exe = os.path.join(oracle_lib.REF_DIR, "smoldyn")

    def ref_seed(seed):
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "lv.txt"), "w") as f:
                f.write(LV_CONFIG % seed)
            subprocess.run([ref_exe, "lv.txt", "-qt"], cwd=d, check=True, stdin=subprocess.DEVNULL,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                           env=dict(os.environ, SMOLDYN_NO_PROMPT="1"), timeout=1200)
            rows = np.array([[float(x) for x in ln.split()] for ln in open(os.path.join(d, "o.txt")) if ln.strip()])
        return rows[1:20]  # t = 0.1 .. 1.9, the client's report times

    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        R = np.stack(list(ex.map(ref_seed, range(1, 25))))  # [seed, time, (t, rabbit, fox)]
    assert np.allclose(gpu[:, 0], R[0, :, 0])
    for col in (1, 2):
        lo = R[:, :, col].min(axis=0) * 0.5
        hi = R[:, :, col].max(axis=0) * 2.0 + 10
        bad = np.nonzero((gpu[:, col] < lo) | (gpu[:, col] > hi))[0]
        assert not len(bad), (col, gpu[bad, col], lo[bad], hi[bad])
