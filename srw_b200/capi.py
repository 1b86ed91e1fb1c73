"""ctypes view of the C-ABI declared in include/srwl_b200.h.

Loading is strict: if the in-tree CUDA library (srw_b200/_lib/libsrwl_b200.so) is missing this
module raises; there is no CPU fallback on the product path.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_lib', 'libsrwl_b200.so')


class SRWLParticle(C.Structure):
    _fields_ = [('x', C.c_double), ('y', C.c_double), ('z', C.c_double), ('xp', C.c_double), ('yp', C.c_double),
                ('gamma', C.c_double), ('relE0', C.c_double), ('nq', C.c_int)]


class SRWLPartBeam(C.Structure):
    _fields_ = [('Iavg', C.c_double), ('nPart', C.c_double), ('partStatMom1', SRWLParticle),
                ('arStatMom2', C.c_double * 21)]


class SRWLRadMesh(C.Structure):
    _fields_ = [('eStart', C.c_double), ('eFin', C.c_double), ('xStart', C.c_double), ('xFin', C.c_double),
                ('yStart', C.c_double), ('yFin', C.c_double), ('zStart', C.c_double),
                ('ne', C.c_long), ('nx', C.c_long), ('ny', C.c_long),
                ('nvx', C.c_double), ('nvy', C.c_double), ('nvz', C.c_double),
                ('hvx', C.c_double), ('hvy', C.c_double), ('hvz', C.c_double),
                ('arSurf', C.POINTER(C.c_double)), ('type', C.c_char), ('itStart', C.c_longlong),
                ('itFin', C.c_longlong)]


class SRWLGsnBm(C.Structure):
    _fields_ = [('x', C.c_double), ('y', C.c_double), ('z', C.c_double), ('xp', C.c_double), ('yp', C.c_double),
                ('avgPhotEn', C.c_double), ('pulseEn', C.c_double), ('repRate', C.c_double), ('polar', C.c_char),
                ('sigX', C.c_double), ('sigY', C.c_double), ('sigT', C.c_double), ('mx', C.c_char), ('my', C.c_char)]


class SRWLWfr(C.Structure):
    _fields_ = [('arEx', C.c_void_p), ('arEy', C.c_void_p), ('arExAux', C.c_void_p), ('arEyAux', C.c_void_p),
                ('mesh', SRWLRadMesh), ('Rx', C.c_double), ('Ry', C.c_double), ('dRx', C.c_double),
                ('dRy', C.c_double), ('xc', C.c_double), ('yc', C.c_double), ('avgPhotEn', C.c_double),
                ('presCA', C.c_char), ('presFT', C.c_char), ('numTypeElFld', C.c_char), ('unitElFld', C.c_char),
                ('unitElFldAng', C.c_char), ('partBeam', SRWLPartBeam), ('arElecPropMatr', C.c_void_p),
                ('arMomX', C.c_void_p), ('arMomY', C.c_void_p), ('arWfrAuxData', C.c_void_p)]


class SRWLOptD(C.Structure):
    _fields_ = [('L', C.c_double), ('treat', C.c_char)]


class SRWLOptA(C.Structure):
    _fields_ = [('shape', C.c_char), ('ap_or_ob', C.c_char), ('Dx', C.c_double), ('Dy', C.c_double),
                ('x', C.c_double), ('y', C.c_double)]


class SRWLOptL(C.Structure):
    _fields_ = [('Fx', C.c_double), ('Fy', C.c_double), ('x', C.c_double), ('y', C.c_double)]


class SRWLOptT(C.Structure):
    _fields_ = [('arTr', C.POINTER(C.c_double)), ('mesh', SRWLRadMesh), ('extTr', C.c_char), ('Fx', C.c_double),
                ('Fy', C.c_double)]


class SRWLOptC(C.Structure):
    _fields_ = [('arOpt', C.POINTER(C.c_void_p)), ('arOptTypes', C.POINTER(C.c_char_p)), ('nElem', C.c_int),
                ('arProp', C.POINTER(C.POINTER(C.c_double))), ('arPropN', C.c_char_p), ('nProp', C.c_int)]


MODIF_FUNC = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(SRWLWfr), C.c_char)
ALLOC_FUNC = C.CFUNCTYPE(C.c_void_p, C.c_char, C.c_longlong)

# symbol -> (restype, argtypes); the complete exported surface of include/srwl_b200.h
SYMBOLS = {
    'srwlCalcElecFieldGaussian': (C.c_int, [C.POINTER(SRWLWfr), C.POINTER(SRWLGsnBm), C.c_void_p]),
    'srwlCalcIntFromElecField': (C.c_int, [C.c_void_p, C.POINTER(SRWLWfr), C.c_char, C.c_char, C.c_char, C.c_double,
                                           C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    'srwlPropagElecField': (C.c_int, [C.POINTER(SRWLWfr), C.POINTER(SRWLOptC), C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.POINTER(C.c_double)]),
    'srwlUtiSetWfrModifFunc': (None, [MODIF_FUNC]),
    'srwlUtiSetAllocArrayFunc': (None, [ALLOC_FUNC]),
    'srwlUtiGetErrText': (C.c_int, [C.c_char_p, C.c_int]),
    'srwgPlanCreate': (C.c_int, [C.POINTER(SRWLWfr), C.POINTER(SRWLOptC), C.c_int, C.POINTER(C.c_void_p)]),
    'srwgPlanGetOutput': (C.c_int, [C.c_void_p, C.POINTER(SRWLWfr)]),
    'srwgPlanGetMoments': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    'srwgPlanInfo': (C.c_int, [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long),
                               C.POINTER(C.c_long), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    'srwgPlanExecute': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    'srwgPlanExecuteBatch': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p,
                                       C.c_void_p, C.c_longlong, C.c_void_p]),
    'srwgPlanExecuteTimed': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    'srwgPlanDestroy': (C.c_int, [C.c_void_p]),
    'srwgMultiECreate': (C.c_int, [C.POINTER(SRWLWfr), C.POINTER(SRWLOptC), C.POINTER(SRWLRadMesh), C.c_int, C.c_int,
                                   C.c_int, C.POINTER(C.c_void_p)]),
    'srwgMultiEAdd': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    'srwgMultiEAddE': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    'srwgMultiEInfo': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]),
    'srwgMultiEAddTimed': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_void_p]),
    'srwgMultiEGetMean': (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong), C.c_void_p]),
    'srwgMultiEAccumulator': (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_longlong)]),
    'srwgMultiESetAccumulator': (C.c_int, [C.c_void_p, C.c_void_p]),
    'srwgMultiEReset': (C.c_int, [C.c_void_p, C.c_void_p]),
    'srwgMultiEDestroy': (C.c_int, [C.c_void_p]),
    'srwgMlpGemm': (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                              C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_void_p]),
    'srwgMlpBiasAct': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    'srwgMlpActBackward': (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p]),
    'srwgMlpColSum': (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    'srwgMlpMse': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    'srwgMlpAdam': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_float,
                              C.c_float, C.c_float, C.c_int, C.c_void_p]),
    'srwgWfrFeatures': (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    'srwgPropagElecFieldStatic': (C.c_int, [C.POINTER(SRWLWfr), C.POINTER(SRWLOptC), C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.POINTER(SRWLWfr)]),
    'srwgPlanDescribe': (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    'srwgTuneSetFamily': (C.c_int, [C.c_int, C.c_int, C.c_int]),
    'srwgTuneSetLines': (C.c_int, [C.c_int, C.c_int, C.c_int]),
    'srwgTuneGetFamily': (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
    'srwgTuneGetLines': (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
    'srwgTuneLoad': (C.c_int, [C.c_char_p, C.POINTER(C.c_int)]),
    'srwgNextFftNumber': (C.c_long, [C.c_long]),
    'srwgSetWaitLimit': (C.c_int, [C.c_longlong]),
    'srwgGetWaitStatus': (C.c_int, [C.c_int, C.POINTER(C.c_int), C.c_int]),
}

_lib = None


def lib():
    """The loaded library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError('srw_b200 CUDA library not built: %s (run python -m srw_b200.build)' % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SYMBOLS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def err_text(code):
    buf = C.create_string_buffer(2048)
    lib().srwlUtiGetErrText(buf, int(code))
    return buf.value.decode(errors='replace')


def check(code, what=''):
    if code > 0:
        raise RuntimeError('%s%s (SRW error %d)' % ((what + ': ') if what else '', err_text(code), code))
    return code
