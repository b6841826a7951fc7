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
   reference sources are present.  On the GPU the b200 build must run to
   completion and print the same 19 report lines; its counts are compared
   with 24 runs of the reference build at every report time (the system sits
   at the Lotka-Volterra fixed point R = F = 1000 and drifts, so the check is
   the reference's envelope widened by a factor of two).
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


@pytest.mark.gpu
def test_reference_client_runs_on_b200():
    if not (os.path.exists(B200_CLIENT) and os.path.exists(REF_CLIENT)):
        pytest.skip("reference client builds absent (make -C oracle client)")
    run = subprocess.run([B200_CLIENT], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr[-2000:]
    gpu = parse_report(run.stdout)
    assert gpu.shape == (19, 3), run.stdout[-2000:]

    def ref_once(k):
        with tempfile.TemporaryDirectory() as d:
            r = subprocess.run([REF_CLIENT], capture_output=True, text=True, timeout=600, cwd=d,
                               env=dict(os.environ, SMOLDYN_NO_PROMPT="1"))
            assert r.returncode == 0
            return parse_report(r.stdout)

    with ThreadPoolExecutor(max_workers=max(1, min(24, os.cpu_count() or 1))) as ex:
        refs = [r for r in ex.map(ref_once, range(24))]
    refs = [r for r in refs if r.shape == (19, 3)]
    assert len(refs) >= 20
    R = np.stack(refs)  # [run, time, (t, rabbit, fox)]
    assert np.allclose(gpu[:, 0], R[0, :, 0])
    for col in (1, 2):
        lo = R[:, :, col].min(axis=0) * 0.5
        hi = R[:, :, col].max(axis=0) * 2.0 + 10
        bad = np.nonzero((gpu[:, col] < lo) | (gpu[:, col] > hi))[0]
        assert not len(bad), (col, gpu[bad, col], lo[bad], hi[bad])
