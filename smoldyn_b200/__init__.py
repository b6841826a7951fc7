"""Python access to libsmoldyn_b200.so, the B200 particle engine behind a
libsmoldyn-compatible C API (Smoldyn source/Smoldyn/libsmoldyn.h).

This module only loads the in-tree shared library and declares the C
prototypes for ctypes; every computation happens in the library.  Importing
fails loudly if the library has not been built (run
``python -m smoldyn_b200.build``).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsmoldyn_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "smoldyn_b200.h")

# enum values (libsmoldyn.h:13-26, smoldyn.h:251-512)
ECok, ECnotify, ECwarning, ECnonexist, ECall, ECmissing, ECbounds, ECsyntax, ECerror, ECmemory, \
    ECbug, ECsame, ECwildcard = 0, -1, -2, -3, -4, -5, -6, -7, -8, -9, -10, -11, -12
MSsoln, MSfront, MSback, MSup, MSdown, MSbsoln, MSall, MSnone, MSsome = range(9)
(RPnone, RPirrev, RPconfspread, RPbounce, RPpgem, RPpgemmax, RPpgemmaxw, RPratio, RPunbindrad,
 RPpgem2, RPpgemmax2, RPratio2, RPoffset, RPfixed) = range(14)
PFfront, PFback, PFnone, PFboth = range(4)
PSrect, PStri, PSsph, PScyl, PShemi, PSdisk, PSall, PSnone = range(8)
CLequal, CLequalnot, CLand, CLor, CLxor, CLandnot, CLornot, CLnone = range(8)
SAreflect, SAtrans, SAabsorb = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p
_sim = C.c_void_p

# name -> (restype, argtypes); every function declared in include/smoldyn_b200.h
PROTOTYPES = {
    "smolGetVersion": (C.c_double, []),
    "smolGetError": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int]),
    "smolClearError": (None, []),
    "smolSetDebugMode": (None, [C.c_int]),
    "smolErrorCodeToString": (C.c_char_p, [C.c_int, C.c_char_p]),
    "smolNewSim": (_sim, [C.c_int, _dp, _dp]),
    "smolUpdateSim": (C.c_int, [_sim]),
    "smolRunTimeStep": (C.c_int, [_sim]),
    "smolRunSim": (C.c_int, [_sim]),
    "smolRunSimUntil": (C.c_int, [_sim, C.c_double]),
    "smolFreeSim": (C.c_int, [_sim]),
    "smolPrepareSimFromFile": (_sim, [C.c_char_p, C.c_char_p, C.c_char_p]),
    "smolLoadSimFromFile": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_sim), C.c_char_p]),
    "smolReadConfigString": (C.c_int, [_sim, C.c_char_p, C.c_char_p]),
    "smolSetSimTimes": (C.c_int, [_sim, C.c_double, C.c_double, C.c_double]),
    "smolSetTimeStart": (C.c_int, [_sim, C.c_double]),
    "smolSetTimeStop": (C.c_int, [_sim, C.c_double]),
    "smolSetTimeNow": (C.c_int, [_sim, C.c_double]),
    "smolSetTimeStep": (C.c_int, [_sim, C.c_double]),
    "smolSetRandomSeed": (C.c_int, [_sim, C.c_long]),
    "smolSetPartitions": (C.c_int, [_sim, C.c_char_p, C.c_double]),
    "smolAddOutputData": (C.c_int, [_sim, C.c_char_p]),
    "smolAddCommandFromString": (C.c_int, [_sim, C.c_char_p]),
    "smolGetOutputData": (C.c_int, [_sim, C.c_char_p, _ip, _ip, C.POINTER(_dp), C.c_int]),
    "smolAddSpecies": (C.c_int, [_sim, C.c_char_p, C.c_char_p]),
    "smolGetSpeciesIndex": (C.c_int, [_sim, C.c_char_p]),
    "smolGetSpeciesIndexNT": (C.c_int, [_sim, C.c_char_p]),
    "smolGetSpeciesName": (None, [_sim, C.c_int, C.c_char_p]),
    "smolSetSpeciesMobility": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_double, _dp, _dp]),
    "smolSetMaxMolecules": (C.c_int, [_sim, C.c_int]),
    "smolAddMolList": (C.c_int, [_sim, C.c_char_p]),
    "smolGetMolListIndex": (C.c_int, [_sim, C.c_char_p]),
    "smolGetMolListIndexNT": (C.c_int, [_sim, C.c_char_p]),
    "smolGetMolListName": (C.c_char_p, [_sim, C.c_int, C.c_char_p]),
    "smolSetMolList": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_char_p]),
    "smolDisplaySim": (C.c_int, [_sim]),
    "smolSetGraphicsParams": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_int]),
    "smolSetMoleculeColor": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_void_p]),
    "smolSetMoleculeSize": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_double]),
    "smolSetMoleculeStyle": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_double, C.c_void_p]),
    "smolAddSolutionMolecules": (C.c_int, [_sim, C.c_char_p, C.c_int, _dp, _dp]),
    "smolGetMoleculeCount": (C.c_int, [_sim, C.c_char_p, C.c_int]),
    "smolSetBoundaryType": (C.c_int, [_sim, C.c_int, C.c_int, C.c_char]),
    "smolAddSurface": (C.c_int, [_sim, C.c_char_p]),
    "smolAddCompartment": (C.c_int, [_sim, C.c_char_p]),
    "smolGetCompartmentIndex": (C.c_int, [_sim, C.c_char_p]),
    "smolGetCompartmentIndexNT": (C.c_int, [_sim, C.c_char_p]),
    "smolGetCompartmentName": (C.c_char_p, [_sim, C.c_int, C.c_char_p]),
    "smolAddCompartmentSurface": (C.c_int, [_sim, C.c_char_p, C.c_char_p]),
    "smolAddCompartmentPoint": (C.c_int, [_sim, C.c_char_p, _dp]),
    "smolAddCompartmentLogic": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_char_p]),
    "smolAddCompartmentMolecules": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_char_p]),
    "smolSetReactionRegion": (C.c_int, [_sim, C.c_char_p, C.c_char_p, C.c_char_p]),
    "smolSetSurfaceAction": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_char_p]),
    "smolAddPanel": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_char_p, C.c_char_p, _dp]),
    "smolSetSurfaceRate": (C.c_int, [_sim, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_char_p, C.c_int]),
    "smolAddSurfaceMolecules": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_char_p, _dp]),
    "smolAddPanelNeighbor": (C.c_int, [_sim, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]),
    "smolSetSurfaceSimParams": (C.c_int, [_sim, C.c_char_p, C.c_double]),
    "smolgpuGetSurfaceRule": (C.c_int, [_sim, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int), _dp, _dp,
                                        _dp]),
    "smolgpuGetSurfaceMolecules": (C.c_int, [_sim, C.POINTER(C.c_longlong), _dp, C.POINTER(C.c_int),
                                             C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.c_uint64)]),
    "smolAddReaction": (C.c_int, [_sim, C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int,
                                  C.POINTER(C.c_char_p), _ip, C.c_double]),
    "smolGetReactionIndex": (C.c_int, [_sim, _ip, C.c_char_p]),
    "smolSetReactionRate": (C.c_int, [_sim, C.c_char_p, C.c_double, C.c_int]),
    "smolSetReactionProducts": (C.c_int, [_sim, C.c_char_p, C.c_int, C.c_double, C.c_char_p, _dp]),
    "smolAddBimolecularReaction": (C.c_int, [_sim, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int,
                                             C.POINTER(C.c_char_p), C.c_double]),
    "smolgpuGetReactionParams": (C.c_int, [_sim, C.c_char_p, _dp, _dp, _dp]),
    "smolgpuGetEffectiveRate": (C.c_int, [_sim, C.c_char_p, _dp, _dp]),
    "smolgpuGetTime": (C.c_double, [_sim]),
    "smolgpuGetStepCount": (C.c_longlong, [_sim]),
    "smolgpuGetTotalMolecules": (C.c_longlong, [_sim]),
    "smolgpuGetMolecules": (C.c_int, [_sim, C.POINTER(C.c_longlong), _dp, _ip, _u64p]),
    "smolgpuSetMolecules": (C.c_int, [_sim, C.c_longlong, _dp, _ip, _u64p]),
    "smolgpuGetEventCounts": (C.c_int, [_sim, C.POINTER(C.c_longlong)]),
    "smolgpuSetInjectedDisplacements": (C.c_int, [_sim, C.c_longlong, _u64p, _dp]),
    "smolgpuSetStream": (C.c_int, [_sim, _vp]),
    "smolgpuGetLaunchCount": (C.c_longlong, [_sim]),
    "smolgpuSynchronize": (C.c_int, [_sim]),
    "smolgpuAutotune": (C.c_int, [_sim, C.c_int, _dp]),
    "smolgpuGetTuning": (C.c_int, [_sim, _dp, _ip, _ip, _ip]),
    "smolgpuRunSteps": (C.c_int, [_sim, C.c_longlong]),
    "smolgpuProfileSteps": (C.c_int, [_sim, C.c_longlong, _ip, C.c_char_p, _dp, C.POINTER(C.c_longlong)]),
    "smolgpuSolveRadii": (C.c_int, [C.c_int, C.c_longlong, _dp, C.c_double, _dp, _dp, C.c_int, _dp]),
    "smolgpuSolveRadiiNoAlloc": (C.c_int, [C.c_int, C.c_longlong, _dp, C.c_double, _dp, _dp, C.c_int, _dp]),
    "smolgpuBindingRadiusHost": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]),
    "smolgpuNumRxnRateProbHost": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double]),
    "smolgpuBindingRadiusProbHost": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                                  C.c_double, _dp]),
    "smolgpuSolveRadiiProb": (C.c_int, [C.c_longlong, _dp, C.c_double, _dp, _dp, C.c_int, _dp, _dp, _dp]),
    "smolgpuUnbindingRadiusHost": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double]),
    "smolgpuRdfTable": (C.c_int, [C.c_char, C.c_int, C.c_double, C.c_char, C.c_int, _dp, _dp, _ip, _ip]),
    "smolgpuRdfSteadyState": (C.c_int, [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp,
                                        _ip]),
    "smolgpuRxnTable": (C.c_int, [C.c_char_p, _dp, C.c_int]),
    "smolgpuNewEnsemble": (_vp, [_sim, C.c_int]),
    "smolgpuEnsembleSetBoxes": (C.c_int, [_vp, _dp, _dp]),
    "smolgpuEnsembleSetRates": (C.c_int, [_vp, C.c_char_p, _dp]),
    "smolgpuEnsembleAddMolecules": (C.c_int, [_vp, C.c_char_p, _ip]),
    "smolgpuEnsembleSetRadiusMode": (C.c_int, [_vp, C.c_int]),
    "smolgpuEnsembleAttachSurrogate": (C.c_int, [_vp, _vp]),
    "smolgpuEnsembleUpdate": (C.c_int, [_vp]),
    "smolgpuEnsembleSetEngine": (C.c_int, [_vp, C.c_int]),
    "smolgpuEnsembleGetEngine": (C.c_int, [_vp]),
    "smolgpuEnsembleGetEventCounts": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "smolgpuEnsembleGetMolecules": (C.c_int, [_vp, C.POINTER(C.c_longlong), _dp, _ip, _ip, _u64p]),
    "smolgpuEnsembleRunSteps": (C.c_int, [_vp, C.c_longlong]),
    "smolgpuEnsembleGetCounts": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "smolgpuEnsembleGetReactionParams": (C.c_int, [_vp, C.c_char_p, _dp, _dp]),
    "smolgpuEnsembleGetFallbackCount": (C.c_longlong, [_vp]),
    "smolgpuEnsembleSetStream": (C.c_int, [_vp, _vp]),
    "smolgpuEnsembleGetLaunchCount": (C.c_longlong, [_vp]),
    "smolgpuEnsembleSynchronize": (C.c_int, [_vp]),
    "smolgpuEnsembleAutotune": (C.c_int, [_vp, C.c_int, _dp]),
    "smolgpuEnsembleGetTuning": (C.c_int, [_vp, _dp, _ip, _ip, _ip]),
    "smolgpuEnsembleFree": (C.c_int, [_vp]),
    "smolgpuSurrogateNew": (_vp, []),
    "smolgpuSurrogateFree": (C.c_int, [_vp]),
    "smolgpuSurrogateTrain": (C.c_int, [_vp, C.c_longlong, C.c_int, C.c_int, C.c_double, C.c_ulonglong, _dp,
                                        _dp]),
    "smolgpuSurrogateSamples": (C.c_int, [_vp, C.c_longlong, C.c_ulonglong, _dp, _dp]),
    "smolgpuSurrogateForward": (C.c_int, [_vp, C.c_longlong, _dp, _dp]),
    "smolgpuSurrogateLossGrad": (C.c_int, [_vp, C.c_longlong, _dp, _dp, _dp, C.POINTER(C.c_float)]),
    "smolgpuSurrogateParamCount": (C.c_int, []),
    "smolgpuSurrogateGetParams": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "smolgpuSurrogateSetParams": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "smolgpuSurrogateSetTolerance": (C.c_int, [_vp, C.c_double]),
    "smolgpuSurrogatePairRadii": (C.c_int, [_vp, C.c_longlong, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_int,
                                            C.c_double, _dp, _dp, C.POINTER(C.c_longlong)]),
}

_lib = None


def load():
    """Load libsmoldyn_b200.so and declare its prototypes (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libsmoldyn_b200.so is not built; run python -m smoldyn_b200.build")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def dptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def last_error():
    lib = load()
    fn = C.create_string_buffer(256)
    msg = C.create_string_buffer(256)
    code = lib.smolGetError(fn, msg, 0)
    return code, fn.value.decode(), msg.value.decode()


def check(code):
    if code < ECwarning:
        c, fn, msg = last_error()
        raise RuntimeError("libsmoldyn_b200 error %d in %s: %s" % (code, fn, msg))
    return code


def _get_tuning(fn, ptr):
    mpb = C.c_double()
    tile, tb, mb = C.c_int(), C.c_int(), C.c_int()
    check(fn(ptr, C.byref(mpb), C.byref(tile), C.byref(tb), C.byref(mb)))
    return {"molperbox": mpb.value, "pair_tile": tile.value, "tile_blocks_per_sm": tb.value,
            "mol_blocks_per_sm": mb.value}


class Sim:
    """Thin owner of a simptr with helpers; all methods call the C ABI."""

    def __init__(self, dim=3, low=(0, 0, 0), high=(1, 1, 1), ptr=None):
        self.lib = load()
        if ptr is None:
            lo = np.asarray(low[:dim], dtype=np.float64)
            hi = np.asarray(high[:dim], dtype=np.float64)
            ptr = self.lib.smolNewSim(dim, dptr(lo), dptr(hi))
            if not ptr:
                check(ECerror)
        self.ptr = ptr
        self.dim = dim

    @classmethod
    def from_file(cls, path, flags=""):
        lib = load()
        d, f = os.path.split(os.path.abspath(path))
        ptr = lib.smolPrepareSimFromFile(d.encode(), f.encode(), flags.encode())
        if not ptr:
            check(ECerror)
        return cls(ptr=ptr)

    @classmethod
    def load_file(cls, path, flags=""):
        """Read a configuration file without building the engine (no GPU needed)."""
        lib = load()
        d, f = os.path.split(os.path.abspath(path))
        ptr = _sim()
        check(lib.smolLoadSimFromFile((d + "/").encode(), f.encode(), C.byref(ptr), flags.encode()))
        return cls(ptr=ptr.value)

    def close(self):
        if self.ptr:
            self.lib.smolFreeSim(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- configuration
    def statement(self, word, params=""):
        return check(self.lib.smolReadConfigString(self.ptr, word.encode(), params.encode()))

    def set_times(self, t0, t1, dt):
        return check(self.lib.smolSetSimTimes(self.ptr, t0, t1, dt))

    def seed(self, s):
        return check(self.lib.smolSetRandomSeed(self.ptr, s))

    def add_species(self, name, difc=None):
        check(self.lib.smolAddSpecies(self.ptr, name.encode(), None))
        if difc is not None:
            check(self.lib.smolSetSpeciesMobility(self.ptr, name.encode(), MSsoln, float(difc), None, None))

    def boundary(self, dim, high, t):
        return check(self.lib.smolSetBoundaryType(self.ptr, dim, high, t.encode()))

    def add_molecules(self, species, n, low=None, high=None):
        lo = None if low is None else dptr(np.asarray(low, dtype=np.float64))
        hi = None if high is None else dptr(np.asarray(high, dtype=np.float64))
        return check(self.lib.smolAddSolutionMolecules(self.ptr, species.encode(), int(n), lo, hi))

    def add_reaction(self, name, r1, r2, products, rate):
        arr = (C.c_char_p * max(1, len(products)))(*[p.encode() for p in products])
        return check(self.lib.smolAddReaction(self.ptr, name.encode(), r1.encode() if r1 else None, MSsoln,
                                              r2.encode() if r2 else None, MSsoln, len(products), arr, None,
                                              float(rate)))

    def set_products(self, rxn, method, param):
        return check(self.lib.smolSetReactionProducts(self.ptr, rxn.encode(), method, float(param), None, None))

    def update(self):
        return check(self.lib.smolUpdateSim(self.ptr))

    def run_step(self):
        return check(self.lib.smolRunTimeStep(self.ptr))

    def run(self):
        return check(self.lib.smolRunSim(self.ptr))

    def run_until(self, t):
        return check(self.lib.smolRunSimUntil(self.ptr, float(t)))

    def run_steps(self, n):
        return check(self.lib.smolgpuRunSteps(self.ptr, int(n)))

    def profile_steps(self, n):
        cap = 64
        nk = C.c_int(cap)
        names = C.create_string_buffer(32 * cap)
        ms = np.zeros(cap)
        launches = np.zeros(cap, dtype=np.int64)
        check(self.lib.smolgpuProfileSteps(self.ptr, int(n), C.byref(nk), names, dptr(ms),
                                           launches.ctypes.data_as(C.POINTER(C.c_longlong))))
        out = {}
        for k in range(min(nk.value, cap)):
            nm = names.raw[32 * k:32 * k + 32].split(b"\0")[0].decode()
            out[nm] = (float(ms[k]), int(launches[k]))
        return out

    def set_stream(self, stream_ptr):
        return check(self.lib.smolgpuSetStream(self.ptr, C.c_void_p(stream_ptr)))

    def synchronize(self):
        return check(self.lib.smolgpuSynchronize(self.ptr))

    def autotune(self, trial_steps=20):
        """Pick box width and kernel launch shape by timed trials (before the
        first step); returns the best trial's ms per step."""
        ms = C.c_double()
        check(self.lib.smolgpuAutotune(self.ptr, int(trial_steps), C.byref(ms)))
        return ms.value

    def tuning(self):
        return _get_tuning(self.lib.smolgpuGetTuning, self.ptr)

    def launches(self):
        return self.lib.smolgpuGetLaunchCount(self.ptr)

    # ---- state
    def count(self, species="all", state=MSall):
        n = self.lib.smolGetMoleculeCount(self.ptr, species.encode(), state)
        check(n if n < 0 else 0)
        return n

    def surface_rule(self, surface, species, state, face):
        """(action, prob, cumprob, revprob) of a surface interaction."""
        a = C.c_int(0)
        pr, cu, rv = np.zeros(6), np.zeros(6), np.zeros(6)
        check(self.lib.smolgpuGetSurfaceRule(self.ptr, surface.encode(), species.encode(), state, face, C.byref(a),
                                             dptr(pr), dptr(cu), dptr(rv)))
        return a.value, pr, cu, rv

    def surface_molecules(self):
        """Surface-bound molecules: positions (n, 3), species, state (MSfront /
        MSback), surface index, panel index and serial number, by serial."""
        n = C.c_longlong(0)
        check(self.lib.smolgpuGetSurfaceMolecules(self.ptr, C.byref(n), None, None, None, None, None, None))
        cnt = max(n.value, 1)
        pos = np.zeros((cnt, 3))
        ints = [np.zeros(cnt, dtype=np.int32) for _ in range(4)]
        sn = np.zeros(cnt, dtype=np.uint64)
        n = C.c_longlong(cnt)
        ip = [a.ctypes.data_as(C.POINTER(C.c_int)) for a in ints]
        check(self.lib.smolgpuGetSurfaceMolecules(self.ptr, C.byref(n), dptr(pos), ip[0], ip[1], ip[2], ip[3],
                                                  sn.ctypes.data_as(C.POINTER(C.c_uint64))))
        k = n.value
        return pos[:k], ints[0][:k], ints[1][:k], ints[2][:k], ints[3][:k], sn[:k]

    def total(self):
        return self.lib.smolgpuGetTotalMolecules(self.ptr)

    def time(self):
        return self.lib.smolgpuGetTime(self.ptr)

    def molecules(self):
        n = C.c_longlong(0)
        check(self.lib.smolgpuGetMolecules(self.ptr, C.byref(n), None, None, None))
        cnt = n.value
        pos = np.zeros((max(cnt, 1), 3), dtype=np.float64)
        sp = np.zeros(max(cnt, 1), dtype=np.int32)
        sn = np.zeros(max(cnt, 1), dtype=np.uint64)
        n = C.c_longlong(max(cnt, 1))
        check(self.lib.smolgpuGetMolecules(self.ptr, C.byref(n), dptr(pos), sp.ctypes.data_as(_ip),
                                           sn.ctypes.data_as(_u64p)))
        k = n.value
        return pos[:k], sp[:k], sn[:k]

    def set_molecules(self, pos, species, serno=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        species = np.ascontiguousarray(species, dtype=np.int32)
        sp = serno
        if serno is not None:
            sp = np.ascontiguousarray(serno, dtype=np.uint64).ctypes.data_as(_u64p)
        return check(self.lib.smolgpuSetMolecules(self.ptr, len(species), dptr(pos),
                                                  species.ctypes.data_as(_ip), sp))

    def inject(self, sernos, disp4):
        sernos = np.ascontiguousarray(sernos, dtype=np.uint64)
        disp4 = np.ascontiguousarray(disp4, dtype=np.float64)
        return check(self.lib.smolgpuSetInjectedDisplacements(self.ptr, len(sernos),
                                                              sernos.ctypes.data_as(_u64p), dptr(disp4)))

    def events(self):
        a = (C.c_longlong * 8)()
        check(self.lib.smolgpuGetEventCounts(self.ptr, a))
        return list(a)

    def effective_rate(self, rxn):
        """(rate, pgem) implied by the derived parameters (rxncalcrate)."""
        rate, pgem = C.c_double(), C.c_double()
        check(self.lib.smolgpuGetEffectiveRate(self.ptr, rxn.encode(), C.byref(rate), C.byref(pgem)))
        return rate.value, pgem.value

    def reaction_params(self, rxn):
        b, u, p = C.c_double(), C.c_double(), C.c_double()
        check(self.lib.smolgpuGetReactionParams(self.ptr, rxn.encode(), C.byref(b), C.byref(u), C.byref(p)))
        return b.value, u.value, p.value

    def output_data(self, name, erase=False):
        nr, nc = C.c_int(), C.c_int()
        arr = _dp()
        check(self.lib.smolGetOutputData(self.ptr, name.encode(), C.byref(nr), C.byref(nc), C.byref(arr),
                                         int(erase)))
        out = np.ctypeslib.as_array(arr, shape=(nr.value * nc.value,)).copy().reshape(nr.value, nc.value) \
            if nr.value * nc.value else np.zeros((0, nc.value))
        C.CDLL(None).free(arr)
        return out


class Ensemble:
    """Independent replicates of a template Sim in one engine (C ABI owner)."""

    def __init__(self, template, nrep):
        self.lib = load()
        self.nrep = nrep
        self.dim = template.dim
        self.template = template
        self.ptr = self.lib.smolgpuNewEnsemble(template.ptr, nrep)
        if not self.ptr:
            check(ECerror)

    def close(self):
        if self.ptr:
            self.lib.smolgpuEnsembleFree(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_boxes(self, low, high):
        low = np.ascontiguousarray(low, dtype=np.float64).reshape(-1)
        high = np.ascontiguousarray(high, dtype=np.float64).reshape(-1)
        return check(self.lib.smolgpuEnsembleSetBoxes(self.ptr, dptr(low), dptr(high)))

    def set_rates(self, rxn, rates):
        rates = np.ascontiguousarray(rates, dtype=np.float64)
        return check(self.lib.smolgpuEnsembleSetRates(self.ptr, rxn.encode(), dptr(rates)))

    def add_molecules(self, species, counts):
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        return check(self.lib.smolgpuEnsembleAddMolecules(self.ptr, species.encode(), counts.ctypes.data_as(_ip)))

    def engine(self, mode=None):
        """Set the stepping engine (0 automatic, 1 step pipeline, 2
        persistent kernel) when mode is given; return the engine in use
        (1 or 2)."""
        if mode is not None:
            check(self.lib.smolgpuEnsembleSetEngine(self.ptr, mode))
        return self.lib.smolgpuEnsembleGetEngine(self.ptr)

    def radius_mode(self, mode):
        return check(self.lib.smolgpuEnsembleSetRadiusMode(self.ptr, mode))

    def attach(self, sur):
        return check(self.lib.smolgpuEnsembleAttachSurrogate(self.ptr, sur.ptr))

    def update(self):
        return check(self.lib.smolgpuEnsembleUpdate(self.ptr))

    def run_steps(self, n):
        return check(self.lib.smolgpuEnsembleRunSteps(self.ptr, int(n)))

    def events(self):
        a = (C.c_longlong * 8)()
        check(self.lib.smolgpuEnsembleGetEventCounts(self.ptr, a))
        return list(a)

    def molecules(self):
        """(positions [n,3], species, replicate, serial) of every molecule."""
        n = C.c_longlong(0)
        check(self.lib.smolgpuEnsembleGetMolecules(self.ptr, C.byref(n), None, None, None, None))
        cnt = max(n.value, 1)
        pos = np.zeros((cnt, 3), dtype=np.float64)
        sp = np.zeros(cnt, dtype=np.int32)
        rp = np.zeros(cnt, dtype=np.int32)
        sn = np.zeros(cnt, dtype=np.uint64)
        n = C.c_longlong(cnt)
        check(self.lib.smolgpuEnsembleGetMolecules(self.ptr, C.byref(n), dptr(pos), sp.ctypes.data_as(_ip),
                                                   rp.ctypes.data_as(_ip), sn.ctypes.data_as(_u64p)))
        k = n.value
        return pos[:k], sp[:k], rp[:k], sn[:k]

    def counts(self, nspecies):
        out = np.zeros(self.nrep * nspecies, dtype=np.int64)
        check(self.lib.smolgpuEnsembleGetCounts(self.ptr, out.ctypes.data_as(C.POINTER(C.c_longlong))))
        return out.reshape(self.nrep, nspecies)

    def reaction_params(self, rxn):
        b = np.zeros(self.nrep)
        u = np.zeros(self.nrep)
        check(self.lib.smolgpuEnsembleGetReactionParams(self.ptr, rxn.encode(), dptr(b), dptr(u)))
        return b, u

    def fallbacks(self):
        return self.lib.smolgpuEnsembleGetFallbackCount(self.ptr)

    def set_stream(self, stream_ptr):
        return check(self.lib.smolgpuEnsembleSetStream(self.ptr, C.c_void_p(stream_ptr)))

    def synchronize(self):
        return check(self.lib.smolgpuEnsembleSynchronize(self.ptr))

    def autotune(self, trial_steps=20):
        ms = C.c_double()
        check(self.lib.smolgpuEnsembleAutotune(self.ptr, int(trial_steps), C.byref(ms)))
        return ms.value

    def tuning(self):
        return _get_tuning(self.lib.smolgpuEnsembleGetTuning, self.ptr)

    def launches(self):
        return self.lib.smolgpuEnsembleGetLaunchCount(self.ptr)


class Surrogate:
    """MLP surrogate of the radius solve (C ABI owner)."""

    def __init__(self):
        self.lib = load()
        self.ptr = self.lib.smolgpuSurrogateNew()

    def close(self):
        if self.ptr:
            self.lib.smolgpuSurrogateFree(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train(self, nsamples=1_000_000, epochs=20, batch=1024, lr=2e-3, seed=12345):
        loss, secs = C.c_double(), C.c_double()
        check(self.lib.smolgpuSurrogateTrain(self.ptr, int(nsamples), int(epochs), int(batch), float(lr), int(seed),
                                             C.byref(loss), C.byref(secs)))
        return loss.value, secs.value

    def samples(self, n, seed=1):
        x = np.zeros((n, 3))
        y = np.zeros((n, 2))
        check(self.lib.smolgpuSurrogateSamples(self.ptr, int(n), int(seed), dptr(x), dptr(y)))
        return x, y

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros((len(x), 2))
        check(self.lib.smolgpuSurrogateForward(self.ptr, len(x), dptr(x), dptr(y)))
        return y

    def loss_grad(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        loss = C.c_double()
        g = np.zeros(self.lib.smolgpuSurrogateParamCount(), dtype=np.float32)
        check(self.lib.smolgpuSurrogateLossGrad(self.ptr, len(x), dptr(x), dptr(y), C.byref(loss),
                                                g.ctypes.data_as(C.POINTER(C.c_float))))
        return loss.value, g

    def params(self):
        p = np.zeros(self.lib.smolgpuSurrogateParamCount(), dtype=np.float32)
        check(self.lib.smolgpuSurrogateGetParams(self.ptr, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        return check(self.lib.smolgpuSurrogateSetParams(self.ptr, p.ctypes.data_as(C.POINTER(C.c_float))))

    def tolerance(self, tol):
        return check(self.lib.smolgpuSurrogateSetTolerance(self.ptr, float(tol)))

    def pair_radii(self, kf, dsum, dt, same=0, rev=1, rparamt=RPratio, rparam=0.2):
        kf = np.ascontiguousarray(kf, dtype=np.float64)
        dsum = np.ascontiguousarray(dsum, dtype=np.float64)
        b = np.zeros(len(kf))
        u = np.zeros(len(kf))
        nfb = C.c_longlong()
        check(self.lib.smolgpuSurrogatePairRadii(self.ptr, len(kf), dptr(kf), dptr(dsum), float(dt), same, rev,
                                                 rparamt, float(rparam), dptr(b), dptr(u), C.byref(nfb)))
        return b, u, nfb.value


def solve_radii_device(mode, rate, dt, difc, b, rel=0):
    lib = load()
    rate = np.ascontiguousarray(rate, dtype=np.float64)
    difc = np.ascontiguousarray(difc, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros_like(rate)
    check(lib.smolgpuSolveRadii(mode, len(rate), dptr(rate), dt, dptr(difc), dptr(b), rel, dptr(out)))
    return out


def solve_radii_prob_device(rate, dt, difc, b, rel, chi, prob):
    """smolgpuSolveRadiiProb: bindingradiusprob on the device; returns
    (radii, probabilities)."""
    lib = load()
    rate = np.ascontiguousarray(rate, dtype=np.float64)
    difc = np.ascontiguousarray(difc, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    chi = np.ascontiguousarray(chi, dtype=np.float64)
    prob = np.array(prob, dtype=np.float64, copy=True)
    out = np.zeros_like(rate)
    check(lib.smolgpuSolveRadiiProb(len(rate), dptr(rate), dt, dptr(difc), dptr(b), rel, dptr(chi), dptr(prob),
                                    dptr(out)))
    return out, prob


RDF_ROWS = {"i": 1, "r": 16, "b": 11}
RDF_STEPS = 31


def rdf_table(mode, n, eps, direction, probs=None):
    """smolgpuRdfTable: steady-state reaction fluxes over the table sweep of
    rdfmaketable / rdfmaketableprob (rxnparam.c:920, 1008) on the device.
    Returns (flux, iters), each [rows, nprob, 31]."""
    lib = load()
    pr = None if probs is None else np.ascontiguousarray(probs, dtype=np.float64)
    nprob = 1 if pr is None else len(pr)
    rows = RDF_ROWS[mode]
    flux = np.zeros(rows * nprob * RDF_STEPS)
    iters = np.zeros(rows * nprob * RDF_STEPS, dtype=np.int32)
    nrows = C.c_int()
    check(lib.smolgpuRdfTable(mode.encode(), n, eps, direction.encode(), nprob, None if pr is None else dptr(pr),
                              dptr(flux), iptr(iters), C.byref(nrows)))
    assert nrows.value == rows
    return flux.reshape(rows, nprob, RDF_STEPS), iters.reshape(rows, nprob, RDF_STEPS)


def rdf_steady_state(r, rdfa, step, a, b, prob, eps):
    """smolgpuRdfSteadyState: batched rdfsteadystate (rxnparam.c:898).
    r, rdfa: [nsolve, n]; step, a, b, prob: [nsolve].  Returns
    (flux, rdfa_out, rdfd_out, iters)."""
    lib = load()
    r = np.ascontiguousarray(np.atleast_2d(r), dtype=np.float64)
    ra = np.array(np.atleast_2d(rdfa), dtype=np.float64, order="C")
    nsolve, n = r.shape
    vec = lambda v: np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (nsolve,)))
    step, a, b, prob = vec(step), vec(a), vec(b), vec(prob)
    rd = np.zeros_like(ra)
    flux = np.zeros(nsolve)
    iters = np.zeros(nsolve, dtype=np.int32)
    check(lib.smolgpuRdfSteadyState(nsolve, n, dptr(r), dptr(ra), dptr(rd), dptr(step), dptr(a), dptr(b), dptr(prob),
                                    eps, dptr(flux), iptr(iters)))
    return flux, ra, rd, iters


def rxn_table(name):
    """smolgpuRxnTable: a rate table compiled into the library."""
    lib = load()
    n = lib.smolgpuRxnTable(name.encode(), None, 0)
    if n < 0:
        raise KeyError(name)
    out = np.zeros(n)
    lib.smolgpuRxnTable(name.encode(), dptr(out), n)
    return out


def solve_radii_device_noalloc(mode, rate, dt, difc, b, rel=0):
    """smolgpuSolveRadiiNoAlloc: the same solve for callers that cannot
    allocate device memory, through a fixed device scratch (at most 65536
    problems per call; calls must not overlap on the GPU)."""
    lib = load()
    rate = np.ascontiguousarray(rate, dtype=np.float64)
    difc = np.ascontiguousarray(difc, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros_like(rate)
    check(lib.smolgpuSolveRadiiNoAlloc(mode, len(rate), dptr(rate), dt, dptr(difc), dptr(b), rel, dptr(out)))
    return out
