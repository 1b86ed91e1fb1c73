"""Drop-in for the reference's ``srwlpy.PropagElecField`` (cpp/src/clients/python/srwlpy.cpp:5214)
on the GPU path:

    from srw_b200 import srwlpy as srwl
    srwl.PropagElecField(wfr, optBL)          # wfr, optBL: SRWLWfr / SRWLOptC objects

Arguments, return value and error behaviour follow the reference: elements of ``optC.arOpt`` are
dispatched by class name (SRWLOptD -> "drift", SRWLOptA -> "aperture", SRWLOptL -> "lens",
SRWLOptT -> "transmission", SRWLOptC -> "container", srwlpy.cpp:2678-2700); ``optC.arProp`` is a list of propagation
parameter lists; field arrays must expose a float32 buffer (numpy or ``array('f')``); when the
mesh size changes the wavefront is re-allocated through ``wfr.allocate(ne, nx, ny, EXNeeded,
EYNeeded, typeE, backupNeeded)`` (srwlpy.cpp:4141); after the call the mesh, radii, centres and
representation flags are written back to the Python object (UpdatePyWfr, srwlpy.cpp:3599); errors
raise RuntimeError with the library's error text.  ``dev`` is the 1-based GPU index (default 1).
"""
import ctypes as C
from array import array

import numpy as np

from . import capi

_ELEM_TYPES = {'SRWLOptD': 'drift', 'SRWLOptA': 'aperture', 'SRWLOptL': 'lens', 'SRWLOptT': 'transmission',
               'SRWLOptC': 'container'}


def _buf_ptr(a, keep, dtype):
    """Address of a contiguous buffer of the given numpy dtype (numpy array or array.array)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype != dtype or not a.flags['C_CONTIGUOUS']:
            raise RuntimeError('field/moment arrays must be contiguous %s' % np.dtype(dtype).name)
        keep.append(a)
        return a.ctypes.data
    if isinstance(a, array):
        if np.dtype(a.typecode) != np.dtype(dtype):
            raise RuntimeError("array type '%s' where %s is required" % (a.typecode, np.dtype(dtype).name))
        keep.append(a)
        return a.buffer_info()[0] if len(a) > 0 else None
    m = memoryview(a)
    keep.append(m)
    npv = np.frombuffer(m, dtype=dtype)
    keep.append(npv)
    return npv.ctypes.data


def _chr(v, default):
    if v is None:
        return default
    if isinstance(v, (bytes, bytearray)):
        return bytes(v[:1])
    if isinstance(v, str):
        return v[:1].encode()
    return bytes([int(v) & 0xff])


def make_c_wfr(wfr, keep):
    """SRWLWfr (C) view of a Python wavefront object (ParseSructSRWLWfr, srwlpy.cpp:3058)."""
    w = capi.SRWLWfr()
    w.arEx = _buf_ptr(getattr(wfr, 'arEx', None), keep, np.float32)
    w.arEy = _buf_ptr(getattr(wfr, 'arEy', None), keep, np.float32)
    m = wfr.mesh
    w.mesh.eStart, w.mesh.eFin = float(m.eStart), float(m.eFin)
    w.mesh.xStart, w.mesh.xFin = float(m.xStart), float(m.xFin)
    w.mesh.yStart, w.mesh.yFin = float(m.yStart), float(m.yFin)
    w.mesh.zStart = float(getattr(m, 'zStart', 0.))
    w.mesh.ne, w.mesh.nx, w.mesh.ny = int(m.ne), int(m.nx), int(m.ny)
    w.Rx, w.Ry = float(wfr.Rx), float(wfr.Ry)
    w.dRx, w.dRy = float(wfr.dRx), float(wfr.dRy)
    w.xc, w.yc = float(wfr.xc), float(wfr.yc)
    w.avgPhotEn = float(getattr(wfr, 'avgPhotEn', 0.))
    w.presCA = _chr(int(getattr(wfr, 'presCA', 0)), b'\0')
    w.presFT = _chr(int(getattr(wfr, 'presFT', 0)), b'\0')
    w.numTypeElFld = _chr(getattr(wfr, 'numTypeElFld', 'f'), b'f')
    w.unitElFld = _chr(int(getattr(wfr, 'unitElFld', 1)), b'\1')
    w.unitElFldAng = _chr(int(getattr(wfr, 'unitElFldAng', 0)), b'\0')
    w.arMomX = _buf_ptr(getattr(wfr, 'arMomX', None), keep, np.float64) if len(getattr(wfr, 'arMomX', [])) >= 11 else None
    w.arMomY = _buf_ptr(getattr(wfr, 'arMomY', None), keep, np.float64) if len(getattr(wfr, 'arMomY', [])) >= 11 else None
    pm = getattr(wfr, 'arElecPropMatr', None)
    w.arElecPropMatr = _buf_ptr(pm, keep, np.float64) if pm is not None and len(pm) >= 20 else None
    pb = getattr(wfr, 'partBeam', None)
    if pb is not None and getattr(pb, 'partStatMom1', None) is not None:
        w.partBeam.partStatMom1.z = float(getattr(pb.partStatMom1, 'z', 0.))
    return w


def make_c_optc(opt, keep):
    """SRWLOptC (C) view of a Python container (ParseSructSRWLOptC, srwlpy.cpp:2618)."""
    els = list(opt.arOpt)
    props = list(getattr(opt, 'arProp', []) or [])
    n = len(els)
    if n <= 0:
        raise RuntimeError('No objects in optical container')
    c = capi.SRWLOptC()
    arOpt = (C.c_void_p * n)()
    arTypes = (C.c_char_p * n)()
    for i, e in enumerate(els):
        cls = type(e).__name__
        kind = _ELEM_TYPES.get(cls)
        if kind is None:
            raise RuntimeError('optical element %s is not supported on the GPU path' % cls)
        if kind == 'drift':
            s = capi.SRWLOptD(float(e.L), _chr(int(getattr(e, 'treat', 0)), b'\0'))
        elif kind == 'aperture':
            s = capi.SRWLOptA(_chr(e.shape, b'r'), _chr(e.ap_or_ob, b'a'), float(e.Dx), float(e.Dy), float(e.x), float(e.y))
        elif kind == 'lens':
            s = capi.SRWLOptL(float(e.Fx), float(e.Fy), float(e.x), float(e.y))
        elif kind == 'transmission':
            # ParseSructSRWLOptT (srwlpy.cpp:1940): the table buffer, its mesh, extTr, Fx, Fy
            s = capi.SRWLOptT()
            tr = _buf_ptr(e.arTr, keep, np.float64)
            if tr is None:
                raise RuntimeError('Incorrect Transmission structure')
            s.arTr = C.cast(tr, C.POINTER(C.c_double))
            m = e.mesh
            s.mesh.eStart, s.mesh.eFin = float(m.eStart), float(m.eFin)
            s.mesh.xStart, s.mesh.xFin = float(m.xStart), float(m.xFin)
            s.mesh.yStart, s.mesh.yFin = float(m.yStart), float(m.yFin)
            s.mesh.ne, s.mesh.nx, s.mesh.ny = int(m.ne), int(m.nx), int(m.ny)
            if len(e.arTr) < 2 * int(m.ne) * int(m.nx) * int(m.ny):
                raise RuntimeError('Incorrect Transmission structure')
            s.extTr = bytes([int(e.extTr) & 0xff])
            s.Fx, s.Fy = float(e.Fx), float(e.Fy)
        else:
            s = make_c_optc(e, keep)
        keep.append(s)
        arOpt[i] = C.cast(C.pointer(s), C.c_void_p)
        tb = C.create_string_buffer(kind.encode())
        keep.append(tb)
        arTypes[i] = C.cast(tb, C.c_char_p)
    keep += [arOpt, arTypes]
    c.arOpt = C.cast(arOpt, C.POINTER(C.c_void_p))
    c.arOptTypes = C.cast(arTypes, C.POINTER(C.c_char_p))
    c.nElem = n
    npr = len(props)
    if npr > 0:
        arProp = (C.POINTER(C.c_double) * npr)()
        arPropN = C.create_string_buffer(npr)
        for i, p in enumerate(props):
            vals = [float(v) for v in p] if isinstance(p, (list, tuple, array, np.ndarray)) else []
            buf = (C.c_double * max(1, len(vals)))(*vals)
            keep.append(buf)
            arProp[i] = C.cast(buf, C.POINTER(C.c_double))
            arPropN[i] = bytes([len(vals)])
        keep += [arProp, arPropN]
        c.arProp = C.cast(arProp, C.POINTER(C.POINTER(C.c_double)))
        c.arPropN = C.cast(arPropN, C.c_char_p)
    c.nProp = npr
    return c


def _update_py_wfr(wfr, w):
    """UpdatePyWfr (srwlpy.cpp:3599)."""
    m = wfr.mesh
    m.eStart, m.eFin = w.mesh.eStart, w.mesh.eFin
    m.xStart, m.xFin = w.mesh.xStart, w.mesh.xFin
    m.yStart, m.yFin = w.mesh.yStart, w.mesh.yFin
    m.zStart = w.mesh.zStart
    m.ne, m.nx, m.ny = int(w.mesh.ne), int(w.mesh.nx), int(w.mesh.ny)
    wfr.Rx, wfr.Ry, wfr.dRx, wfr.dRy = w.Rx, w.Ry, w.dRx, w.dRy
    wfr.xc, wfr.yc = w.xc, w.yc
    wfr.avgPhotEn = w.avgPhotEn
    wfr.presCA = ord(w.presCA) if w.presCA else 0
    wfr.presFT = ord(w.presFT) if w.presFT else 0


_state = {'wfr': None, 'keep': None, 'arrays': {}}


@capi.MODIF_FUNC
def _modif(action, pw, pol):
    """Re-allocation callback (ModifySRWLWfr, srwlpy.cpp:4141)."""
    try:
        wfr = _state['wfr']
        if wfr is None or action < 0:
            return -1
        p = pol if isinstance(pol, int) else (pol[0] if pol else 0)
        ex_needed = 1 if p in (0, ord('x'), ord('X')) else 0
        ey_needed = 1 if p in (0, ord('y'), ord('Y'), ord('z'), ord('Z')) else 0
        w = pw.contents
        if action in (2, 12):
            wfr.allocate(int(w.mesh.ne), int(w.mesh.nx), int(w.mesh.ny), ex_needed, ey_needed,
                         getattr(wfr, 'numTypeElFld', 'f'), 1 if action == 12 else 0)
        elif action == 0:
            wfr.allocate(0, 0, 0, 1, 1, getattr(wfr, 'numTypeElFld', 'f'))
        else:
            return -1
        keep = _state['keep']
        w.arEx = _buf_ptr(wfr.arEx, keep, np.float32)
        w.arEy = _buf_ptr(wfr.arEy, keep, np.float32)
        w.arMomX = _buf_ptr(wfr.arMomX, keep, np.float64) if len(wfr.arMomX) >= 11 else None
        w.arMomY = _buf_ptr(wfr.arMomY, keep, np.float64) if len(wfr.arMomY) >= 11 else None
        pm = getattr(wfr, 'arElecPropMatr', None)
        w.arElecPropMatr = _buf_ptr(pm, keep, np.float64) if pm is not None and len(pm) >= 20 else None
        return 0
    except Exception:
        return -1


@capi.ALLOC_FUNC
def _alloc_array(typ, n):
    """Client array for an extracted intensity (the reference's AllocPyArrayGetBuf, srwlpy.cpp:4424:
    srwl_uti_array_alloc(type, n), zero-filled); kept until the call returns."""
    t = typ.decode() if isinstance(typ, bytes) else chr(typ)
    if t not in ('d', 'f', 'i') or n <= 0:
        return None
    a = array(t, bytes(int(n) * array(t).itemsize))
    addr = a.buffer_info()[0]
    _state['arrays'][addr] = a
    return addr


def _is_mesh(o):
    return type(o).__name__ == 'SRWLRadMesh'


def _parse_int_list(intList):
    """ParseSructSRWLPropIntDef (srwlpy.cpp:2784): (requests [el, pol, type, dep, pres], meshes, flat).
    Flat format: [[el, pol, type, dep, pres, SRWLRadMesh], ...]; column format: [els, pols, types, deps,
    press, meshes], each a list or one value for all (later entries then take the first one's)."""
    if not isinstance(intList, list) or len(intList) <= 0:
        raise RuntimeError('Incorrect list of parameters for intensity extraction at propagation')
    o = intList[0]
    if isinstance(o, list) and len(o) == 6 and _is_mesh(o[5]):
        return [list(map(int, it[:5])) for it in intList], [it[5] for it in intList], True
    n = len(o) if isinstance(o, list) else 1
    cols = []
    for j in range(6):
        v = intList[j]
        if isinstance(v, list) and isinstance(o, list):
            cols.append(list(v))
        elif j == 0 and isinstance(o, list):
            raise RuntimeError('Incorrect list of parameters for intensity extraction at propagation')
        else:
            cols.append([v] + [None] * (n - 1))
    reqs = [[(-1 if cols[j][i] is None else int(cols[j][i])) for j in range(5)] for i in range(n)]
    return reqs, cols[5], False


def _mesh_to_c(m, cm):
    if m is None:
        cm.ne = -1
        return
    cm.eStart, cm.eFin = float(m.eStart), float(m.eFin)
    cm.xStart, cm.xFin = float(m.xStart), float(m.xFin)
    cm.yStart, cm.yFin = float(m.yStart), float(m.yFin)
    cm.zStart = float(getattr(m, 'zStart', 0.))
    cm.ne, cm.nx, cm.ny = int(m.ne), int(m.nx), int(m.ny)


def _mesh_from_c(cm, m):
    """UpdatePyRadMesh (srwlpy.cpp): the mesh object takes the extraction's mesh."""
    m.eStart, m.eFin = cm.eStart, cm.eFin
    m.xStart, m.xFin = cm.xStart, cm.xFin
    m.yStart, m.yFin = cm.yStart, cm.yFin
    m.ne, m.nx, m.ny = int(cm.ne), int(cm.nx), int(cm.ny)


def _copy_mesh(m):
    f = getattr(m, 'copy', None)
    if callable(f):
        return f()
    import copy
    return copy.copy(m)


def _update_int_list(intList, flat, meshes, cms, arrays):
    """UpdatePyPropInt (srwlpy.cpp:3809): meshes updated in place and the intensity arrays added
    (flat format: as the 7th item of each request; column format: as item 6, a list when there are
    several requests)."""
    if flat:
        for i, it in enumerate(intList):
            _mesh_from_c(cms[i], it[5])
            if len(it) > 6:
                it[6] = arrays[i]
            else:
                it.append(arrays[i])
        return
    n = len(arrays)
    oMesh = intList[5]
    lists = n > 1 or isinstance(oMesh, list)
    if n > 1 and not isinstance(oMesh, list):
        oMesh = [oMesh] + [_copy_mesh(oMesh) for _ in range(n - 1)]
        intList[5] = oMesh
    elif lists:
        seen = set()
        for i in range(n):              # the same mesh object twice: the later ones get copies
            if id(oMesh[i]) in seen:
                oMesh[i] = _copy_mesh(oMesh[i])
            seen.add(id(oMesh[i]))
    for i in range(n):
        _mesh_from_c(cms[i], oMesh[i] if lists else oMesh)
    res = list(arrays) if lists else arrays[0]
    if len(intList) > 6:
        intList[6] = res
    else:
        intList.append(res)


def PropagElecField(wfr, optC, intList=None, dev=None):
    """Propagates ``wfr`` in place through ``optC`` on the GPU; returns ``wfr``.  ``intList``: intensities
    to extract after elements (vs x and y; the reference's list formats), completed in place with the
    extracted arrays and their meshes."""
    if wfr is None or optC is None:
        raise RuntimeError('Incorrect arguments for PropagElecField')
    L = capi.lib()
    keep = []
    w = make_c_wfr(wfr, keep)
    o = make_c_optc(optC, keep)
    par = None
    if dev is not None:
        par = (C.c_double * 2)(1., float(dev))
    nInt, arID, arIM, arI = 0, None, None, None
    if intList is not None:
        reqs, meshes, flat = _parse_int_list(intList)
        nInt = len(reqs)
        cols = [(C.c_byte * nInt)(*[max(-128, min(127, r[j])) for r in reqs]) for j in range(5)]
        arID = (C.c_void_p * 5)(*[C.cast(c, C.c_void_p) for c in cols])
        arIM = (capi.SRWLRadMesh * nInt)()
        for i in range(nInt):
            _mesh_to_c(meshes[i] if i < len(meshes) else None, arIM[i])
        arI = (C.c_void_p * nInt)()
        keep += cols + [arID, arIM, arI]
    _state['wfr'] = wfr
    _state['keep'] = keep
    _state['arrays'] = {}
    try:
        L.srwlUtiSetWfrModifFunc(_modif)
        L.srwlUtiSetAllocArrayFunc(_alloc_array)
        r = L.srwlPropagElecField(C.byref(w), C.byref(o), nInt, C.cast(arID, C.c_void_p) if arID else None,
                                  C.cast(arIM, C.c_void_p) if arIM else None,
                                  C.cast(arI, C.c_void_p) if arI else None, par)
        arrays = [_state['arrays'].get(arI[i]) for i in range(nInt)] if nInt else []
    finally:
        _state['wfr'] = None
        _state['keep'] = None
        _state['arrays'] = {}
    if r > 0:
        raise RuntimeError(capi.err_text(r))
    _update_py_wfr(wfr, w)
    if nInt:
        _update_int_list(intList, flat, meshes, arIM, arrays)
    return wfr


def CalcIntFromElecField(arI, wfr, pol, intType, depType, e, x, y, meth=None, fldTrj=None, dev=None):
    """srwlpy.CalcIntFromElecField (cpp/src/clients/python/srwlpy.cpp:4873): fills ``arI`` (array('f')
    or a float32 numpy array; float64 for the phase, intType 4) with the intensity of ``wfr`` vs x and
    y (depType 3), vs x at y (1), vs y at x (2) or at the point (x, y) (0), on the GPU.  ``meth`` (vs x
    and y): [1, n] averages into arI over n earlier iterations, [2] adds to it."""
    if fldTrj is not None:
        raise RuntimeError('intensity with the central electron field/trajectory is not supported on the GPU path')
    keep = []
    w = make_c_wfr(wfr, keep)
    pI = _buf_ptr(arI, keep, np.float64 if int(intType) == 4 else np.float32)
    pm = None
    if meth is not None:
        m = np.zeros(20)
        m[:min(20, len(meth))] = np.asarray(meth, np.float64)[:20]
        keep.append(m)
        pm = m.ctypes.data
    par = None
    if dev is not None:
        par = (C.c_double * 2)(1., float(dev))
    c = lambda v: C.c_char(int(v) & 0xff)  # noqa: E731
    r = capi.lib().srwlCalcIntFromElecField(pI, C.byref(w), c(pol), c(intType), c(depType), float(e), float(x),
                                            float(y), pm, None, par)
    if r > 0:
        raise RuntimeError(capi.err_text(r))
    return arI


def CalcElecFieldGaussian(wfr, gsnBm, precPar=None):
    """srwlpy.CalcElecFieldGaussian: the field of a Gaussian beam on ``wfr``'s mesh, computed on the GPU
    (single photon energy, no automatic sampling); sets the radius, centre, moments and 4x4 matrix."""
    keep = []
    w = make_c_wfr(wfr, keep)
    g = capi.SRWLGsnBm()
    for k in ('x', 'y', 'z', 'xp', 'yp', 'avgPhotEn', 'pulseEn', 'repRate', 'sigX', 'sigY', 'sigT'):
        setattr(g, k, float(getattr(gsnBm, k)))
    g.polar = C.c_char(int(gsnBm.polar))
    g.mx = C.c_char(int(gsnBm.mx))
    g.my = C.c_char(int(gsnBm.my))
    pp = None
    if precPar is not None:
        a = np.zeros(max(1, len(precPar)))
        a[:len(precPar)] = np.asarray(precPar, np.float64)
        keep.append(a)
        pp = a.ctypes.data
    r = capi.lib().srwlCalcElecFieldGaussian(C.byref(w), C.byref(g), pp)
    if r > 0:
        raise RuntimeError(capi.err_text(r))
    _update_py_wfr(wfr, w)
    return wfr
