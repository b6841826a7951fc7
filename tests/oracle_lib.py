"""ctypes access to the CPU oracle (oracle/_ref/*.so) for the tests.

Test infrastructure only: the oracle is the checker, never the thing tested.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
REFERENCE = os.environ.get("SMOLDYN_REF", "/root/reference")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u64p = C.POINTER(C.c_uint64)


def ensure_built():
    """Build the oracle restatement (needs the generated tables header)."""
    so = os.path.join(REF_DIR, "liboracle.so")
    if not os.path.exists(so):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"])
    return so


def oracle():
    lib = C.CDLL(ensure_built())
    for nm in ("ora_numrxnrate",):
        getattr(lib, nm).restype = C.c_double
        getattr(lib, nm).argtypes = [C.c_double] * 3
    lib.ora_numrxnrateprob.restype = C.c_double
    lib.ora_numrxnrateprob.argtypes = [C.c_double] * 4
    lib.ora_bindingradius.restype = C.c_double
    lib.ora_bindingradius.argtypes = [C.c_double] * 4 + [C.c_int]
    lib.ora_bindingradiusprob.restype = C.c_double
    lib.ora_bindingradiusprob.argtypes = [C.c_double] * 4 + [C.c_int, C.c_double, _dp]
    lib.ora_unbindingradius.restype = C.c_double
    lib.ora_unbindingradius.argtypes = [C.c_double] * 4
    return lib


def reference_rxnparam():
    """The reference's own rxnparam.c compiled by oracle/Makefile, or None."""
    so = os.path.join(REF_DIR, "librxnparam_ref.so")
    if not os.path.exists(so):
        return None
    lib = C.CDLL(so)
    lib.numrxnrate.restype = C.c_double
    lib.numrxnrate.argtypes = [C.c_double] * 3
    lib.numrxnrateprob.restype = C.c_double
    lib.numrxnrateprob.argtypes = [C.c_double] * 4
    lib.bindingradius.restype = C.c_double
    lib.bindingradius.argtypes = [C.c_double] * 4 + [C.c_int]
    lib.bindingradiusprob.restype = C.c_double
    lib.bindingradiusprob.argtypes = [C.c_double] * 4 + [C.c_int, C.c_double, _dp]
    lib.unbindingradius.restype = C.c_double
    lib.unbindingradius.argtypes = [C.c_double] * 4
    return lib


class OraNet(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("wall", (C.c_char * 2) * 3),
        ("nsp", C.c_int), ("difc", C.c_double * 32),
        ("nr1", C.c_int), ("r1_rct", C.c_int * 16), ("r1_nprod", C.c_int * 16), ("r1_prd", (C.c_int * 4) * 16),
        ("r1_prdpos", ((C.c_double * 3) * 4) * 16),
        ("nr2", C.c_int), ("r2_rct", (C.c_int * 2) * 16), ("r2_bind2", C.c_double * 16),
        ("r2_nprod", C.c_int * 16), ("r2_prd", (C.c_int * 4) * 16), ("r2_prdpos", ((C.c_double * 3) * 4) * 16),
    ]


def ora_step(net, pos, sp, serno, disp, force1):
    lib = C.CDLL(ensure_built())
    n = len(sp)
    cap = 5 * n + 16
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    sp = np.ascontiguousarray(sp, dtype=np.int32)
    serno = np.ascontiguousarray(serno, dtype=np.uint64)
    disp = np.ascontiguousarray(disp, dtype=np.float64)
    force1 = np.ascontiguousarray(force1, dtype=np.int32)
    opos = np.zeros((cap, 3))
    osp = np.zeros(cap, dtype=np.int32)
    osn = np.zeros(cap, dtype=np.uint64)
    opar = np.zeros(cap, dtype=np.uint64)
    fate = np.zeros(max(n, 1), dtype=np.int32)
    partner = np.zeros(max(n, 1), dtype=np.uint64)
    on = C.c_int()
    namb = C.c_int()
    rc = lib.ora_step(C.byref(net), n, pos.ctypes.data_as(_dp), sp.ctypes.data_as(_ip),
                      serno.ctypes.data_as(_u64p), disp.ctypes.data_as(_dp), force1.ctypes.data_as(_ip), cap,
                      opos.ctypes.data_as(_dp), osp.ctypes.data_as(_ip), osn.ctypes.data_as(_u64p),
                      opar.ctypes.data_as(_u64p), C.byref(on), fate.ctypes.data_as(_ip),
                      partner.ctypes.data_as(_u64p), C.byref(namb))
    assert rc == 0
    k = on.value
    return dict(pos=opos[:k], sp=osp[:k], serno=osn[:k], parent=opar[:k], fate=fate[:n], partner=partner[:n],
                nambig=namb.value)
