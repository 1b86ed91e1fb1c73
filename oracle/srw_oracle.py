"""FP64 CPU restatement of SRW's wavefront-propagation path (drift / thin lens / aperture /
transmission).

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``srw_b200``) imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may use it, and
only as the checker.

This module restates, in double precision with numpy, the algorithm of the reference
``srwlPropagElecField`` (cpp/src/lib/srwlib.cpp:1023) for SRWLOptC chains of drifts, thin
lenses, rectangular/circular apertures/obstacles and generic transmission tables, with the per-element propagation
parameter lists.  Each function cites the reference file:line it follows.  Mesh/integer logic
follows the reference operation order exactly (so meshes are bit-exact in IEEE double); field
arithmetic is FP64 (numpy.fft / pocketfft) instead of the reference's FP32 FFTW, so the field
agrees with the reference to FP32 round-off (rel. L2 ~1e-6) and serves as the FP64 oracle.

Parity pin: the restatement is checked against the reference itself (built from source by
``oracle/Makefile`` into ``oracle/_ref/``) through the golden fixtures in ``tests/golden/``
made by ``tests/golden/make_golden.py``.

Statistical moments: propagated with the reference's analytic matrices, and recomputed from the
field (ComputeRadMoments, sroptelm.cpp:1608) where an aperture or obstacle asks for it.

Not restated (documented gaps): the auto-resize Meth_1/Meth_2 machinery (pp[0], pp[1] != 0);
drift modes pp[3] >= 100; ne > 1.
"""
from __future__ import annotations

import bisect
import math
from dataclasses import dataclass, field

import numpy as np

# ----------------------------------------------------------------------------------------
# FFT "good numbers" (cpp/src/ext/genmath/gmfft.cpp:26-154, NextCorrectNumberForFFT :156-228)
# ----------------------------------------------------------------------------------------


def _good_numbers():
    """Even n <= 100000 of the form 2^a 3^b 5^c 7^d 11^e 13^f with e, f <= 1 (the reference's
    table at gmfft.cpp:26 is exactly this set; pinned by tests/golden/good_numbers.txt)."""
    out = []
    for n in range(2, 100001, 2):
        m = n
        for p, lim in ((2, 64), (3, 64), (5, 64), (7, 64), (11, 1), (13, 1)):
            c = 0
            while m % p == 0:
                m //= p
                c += 1
            if c > lim:
                break
        else:
            if m == 1:
                out.append(n)
    return out


GOOD_NUMBERS = _good_numbers()


def next_correct_number_for_fft(n: int) -> int:
    """gmfft.cpp:156-228."""
    if n < 4:
        return 4
    if n < 100001:
        return GOOD_NUMBERS[bisect.bisect_left(GOOD_NUMBERS, n)]
    mults = (10. / 9., 9. / 8., 6. / 5., 5. / 4., 4. / 3., 3. / 2., 8. / 5., 5. / 3., 16. / 9., 15. / 8.)
    k = 99000
    for _ in range(100):
        for m in mults:
            dk = k * m
            kt = int(dk)
            if (dk - float(kt)) >= 0.5:
                kt += 1
            if n <= kt:
                return kt
        k <<= 1
        if n <= k:
            return k
    return n


# ----------------------------------------------------------------------------------------
# Wavefront state (srTSRWRadStructAccessData, cpp/src/core/srradstr.h:67)
# ----------------------------------------------------------------------------------------


@dataclass
class Wfr:
    ex: np.ndarray            # complex128 [nz, nx]
    ey: np.ndarray
    eStart: float
    xStart: float
    xStep: float
    zStart: float
    zStep: float
    nx: int
    nz: int
    RobsX: float = 0.
    RobsZ: float = 0.
    RobsXAbsErr: float = 0.
    RobsZAbsErr: float = 0.
    xc: float = 0.
    zc: float = 0.
    xWfrMin: float = 0.
    xWfrMax: float = 0.
    zWfrMin: float = 0.
    zWfrMax: float = 0.
    Pres: int = 0
    yStart: float = 0.     # longitudinal position (mesh.zStart)
    avgPhotEn: float = 0.
    momX: np.ndarray = field(default_factory=lambda: np.zeros(11))
    momZ: np.ndarray = field(default_factory=lambda: np.zeros(11))
    propM: np.ndarray = field(default_factory=lambda: np.zeros(20))     # arElecPropMatr
    xStartTr: float = 0.
    zStartTr: float = 0.
    UseStartTrToShiftAtChangingRepresToCoord: bool = False
    AuxLong1: int = 0
    AuxLong2: int = 0
    AuxLong3: int = 0
    AuxLong4: int = 0
    xLinOnly: bool = False      # m_xLinOnlyPhaseTermWasSubtracted
    zLinOnly: bool = False
    dxcSub: float = 0.
    dzcSub: float = 0.
    QuadX: bool = False         # WfrQuadTermCanBeTreatedAtResizeX
    QuadZ: bool = False

    # --- SRWLWfr <-> internal mesh (srradstr.cpp:501-634, 687-758)
    @staticmethod
    def from_srwl(ex, ey, mesh, Rx, Ry, dRx, dRy, xc, yc, presCA=0, momX=None, momY=None, avgPhotEn=0., propM=None):
        """InSRWRadPtrs (srradstr.cpp:501).  ``mesh`` is a dict of SRWLRadMesh fields."""
        nx, ny = int(mesh['nx']), int(mesh['ny'])
        if nx <= 1:
            xStart, xStep = 0.5 * (mesh['xStart'] + mesh['xFin']), 0.
        else:
            xStart, xStep = mesh['xStart'], (mesh['xFin'] - mesh['xStart']) / (nx - 1)
        if ny <= 1:
            zStart, zStep = 0.5 * (mesh['yStart'] + mesh['yFin']), 0.
        else:
            zStart, zStep = mesh['yStart'], (mesh['yFin'] - mesh['yStart']) / (ny - 1)
        w = Wfr(ex=np.asarray(ex, np.complex128).reshape(ny, nx).copy(),
                ey=np.asarray(ey, np.complex128).reshape(ny, nx).copy(),
                eStart=mesh['eStart'], xStart=xStart, xStep=xStep, zStart=zStart, zStep=zStep,
                nx=nx, nz=ny, RobsX=Rx, RobsZ=Ry, RobsXAbsErr=dRx, RobsZAbsErr=dRy, xc=xc, zc=yc,
                xWfrMin=mesh['xStart'], xWfrMax=mesh['xFin'], zWfrMin=mesh['yStart'], zWfrMax=mesh['yFin'],
                Pres=int(presCA), yStart=mesh.get('zStart', 0.), avgPhotEn=avgPhotEn)
        if momX is not None:
            w.momX = np.array(momX, np.float64)[:11].copy()
        if momY is not None:
            w.momZ = np.array(momY, np.float64)[:11].copy()
        if propM is not None:
            w.propM = np.array(propM, np.float64)[:20].copy()
        return w

    def out_mesh(self):
        """OutSRWRadPtrs (srradstr.cpp:687): SRWLRadMesh values."""
        return dict(nx=self.nx, ny=self.nz, xStart=self.xStart, xFin=self.xStart + self.xStep * (self.nx - 1),
                    yStart=self.zStart, yFin=self.zStart + self.zStep * (self.nz - 1), eStart=self.eStart,
                    eFin=self.eStart, zStart=self.yStart)

    def srwl_roundtrip(self):
        """ModifyWfrNeNxNz (srradstr.cpp:760-797): OutSRWRadPtrs then InSRWRadPtrs on the same
        SRWLWfr after the client re-allocates.  Only the mesh round trip matters here: the step is
        re-derived from xFin and the non-zero limits reset to the mesh ends."""
        m = self.out_mesh()
        nx, nz = self.nx, self.nz
        if nx <= 1:
            self.xStart, self.xStep = 0.5 * (m['xStart'] + m['xFin']), 0.
        else:
            self.xStart, self.xStep = m['xStart'], (m['xFin'] - m['xStart']) / (nx - 1)
        if nz <= 1:
            self.zStart, self.zStep = 0.5 * (m['yStart'] + m['yFin']), 0.
        else:
            self.zStart, self.zStep = m['yStart'], (m['yFin'] - m['yStart']) / (nz - 1)
        self.xWfrMin, self.xWfrMax = m['xStart'], m['xFin']
        self.zWfrMin, self.zWfrMax = m['yStart'], m['yFin']

    def set_full_range(self):
        """SetNonZeroWavefrontLimitsToFullRange (srradstr.h:339)."""
        self.xWfrMin = self.xStart
        self.xWfrMax = self.xStart + self.nx * self.xStep
        self.zWfrMin = self.zStart
        self.zWfrMax = self.zStart + self.nz * self.zStep

    def coords(self):
        x = self.xStart + np.arange(self.nx) * self.xStep
        z = self.zStart + np.arange(self.nz) * self.zStep
        return x[None, :], z[:, None]

    def mult(self, factor):
        self.ex = self.ex * factor
        self.ey = self.ey * factor


# ----------------------------------------------------------------------------------------
# Centred physical 2D FFT (CGenMathFFT2D::Make2DFFT, gmfft.cpp:295-897; helpers gmfft.h:232-480)
# ----------------------------------------------------------------------------------------


def _shift_table(N, t0, tStep):
    """FillArrayShift (gmfft.h:250): exp(i 2 pi t0 (k - N/2) tStep) per index k."""
    k = np.arange(N) - (N >> 1)
    return np.exp(1j * 2. * math.pi * t0 * (k * tStep))


def make_2d_fft(data, Nx, Ny, xStep, yStep, xStart, yStart, Dir, use_given=False, xStartTrIn=0., yStartTrIn=0.):
    """Returns (transformed data, xStepTr, yStepTr, xStartTr, yStartTr)."""
    RelShiftTol = 1.e-06
    HalfNx, HalfNy = Nx >> 1, Ny >> 1
    xStartTr = -0.5 / xStep                         # SetupLimitsTr (gmfft.h:232)
    xStepTr = -xStartTr / HalfNx
    yStartTr = -0.5 / yStep
    yStepTr = -yStartTr / HalfNy
    if use_given:
        xStartTrOut, yStartTrOut = xStartTrIn, yStartTrIn
    else:
        xStartTrOut, yStartTrOut = xStartTr, yStartTr
    xStepNx = Nx * xStep
    yStepNy = Ny * yStep
    x0_After = xStart + 0.5 * xStepNx
    y0_After = yStart + 0.5 * yStepNy
    needAfterX = abs(x0_After) > RelShiftTol * xStepNx
    needAfterY = abs(y0_After) > RelShiftTol * yStepNy
    needBefX = needBefY = False
    x0_Before = y0_Before = 0.
    if use_given:
        x0_Before = xStartTrIn - xStartTr
        y0_Before = yStartTrIn - yStartTr
        needBefX = abs(x0_Before) > RelShiftTol * abs(xStartTr)
        needBefY = abs(y0_Before) > RelShiftTol * abs(yStartTr)
    sgn = -1. if Dir > 0 else 1.
    d = np.array(data, np.complex128, copy=True)
    if needBefX:
        d = d * _shift_table(Nx, sgn * x0_Before, xStep)[None, :]
    if needBefY:
        d = d * _shift_table(Ny, sgn * y0_Before, yStep)[:, None]
    Mult = xStep * yStep
    iy = np.arange(Ny)[:, None]
    ix = np.arange(Nx)[None, :]
    sign = np.where(((ix + iy) & 1) == 1, -1., 1.)
    if Dir > 0:
        d = np.fft.fft2(d)
        d = d * sign                                # RepairSignAfter2DFFT (gmfft.h:334)
        d = np.roll(d, (HalfNy, HalfNx), axis=(0, 1))   # RotateDataAfter2DFFT (gmfft.h:279), even N
    else:
        d = np.roll(d, (HalfNy, HalfNx), axis=(0, 1))
        d = d * sign
        d = np.fft.ifft2(d) * (Nx * Ny)             # FFTW_BACKWARD is unnormalised
    d = d * Mult
    if needAfterX:
        d = d * _shift_table(Nx, sgn * x0_After, xStepTr)[None, :]
    if needAfterY:
        d = d * _shift_table(Ny, sgn * y0_After, yStepTr)[:, None]
    return d, xStepTr, yStepTr, xStartTrOut, yStartTrOut


def set_rad_repres(w: Wfr, coord_or_ang: int):
    """srTGenOptElem::SetRadRepres (sroptelm.cpp:1243-1528), ne == 1; the edge correction is never
    enabled (WfrEdgeCorrShouldBeDone is 0 from Initialize, srradstr.cpp:1532)."""
    if w.Pres == coord_or_ang:
        return
    Dir = -1 if coord_or_ang == 0 else 1
    use_given = (w.AuxLong4 == 7777777) or ((coord_or_ang == 0) and w.UseStartTrToShiftAtChangingRepresToCoord)
    res = None
    for comp in ('ex', 'ey'):
        d, xs, ys, x0, y0 = make_2d_fft(getattr(w, comp), w.nx, w.nz, w.xStep, w.zStep, w.xStart, w.zStart,
                                        Dir, use_given, w.xStartTr, w.zStartTr)
        setattr(w, comp, d)
        res = (xs, ys, x0, y0)
    w.xStep, w.zStep, w.xStart, w.zStart = res
    w.Pres = coord_or_ang
    w.set_full_range()


def _apply_phase(w: Wfr, phase):
    w.mult(np.exp(1j * phase))


# ----------------------------------------------------------------------------------------
# Drift space (cpp/src/core/sroptdrf.h, sroptdrf.cpp)
# ----------------------------------------------------------------------------------------

PI_D_LAMBDA_PER_EV = 2.53384080189E+06      # sroptdrf.h:479 (pi/lambda[m] per eV)
INV_LAMBDA_PER_EV = 806546.577258           # sroptdrf.h:481
LAMBDA_EV_M = 1.239842e-06                  # sroptdrf.h:617


def _diff_lim_spot(w: Wfr, x_or_z, L):
    """DiffractionLimitedPropagatedSpotSize (sroptdrf.h:1020)."""
    lam = LAMBDA_EV_M / w.eStart
    if x_or_z == 'x':
        dLim = (w.nx - 1) * w.xStep
        dWfr = w.xWfrMax - w.xWfrMin
    else:
        dLim = (w.nz - 1) * w.zStep
        dWfr = w.zWfrMax - w.zWfrMin
    d = dWfr if ((dWfr > 0.) and (dWfr < dLim)) else dLim
    return lam * L / d


def _mom_apply(mom, ax, az):
    """MultSquareMatrByVect steps of AuxPropagateRadMoments (sroptdrf.cpp:22) / GenAuxPropagateRadMoments
    (sroptelm.cpp:2095) on one 11-moment record [Tot, x, x', z, z', xx, xx', x'x', zz, zz', z'z']."""
    bx = [[ax[0][0] * ax[0][0], 2. * ax[0][0] * ax[0][1], ax[0][1] * ax[0][1]],
          [ax[0][0] * ax[1][0], ax[0][1] * ax[1][0] + ax[0][0] * ax[1][1], ax[0][1] * ax[1][1]],
          [ax[1][0] * ax[1][0], 2. * ax[1][0] * ax[1][1], ax[1][1] * ax[1][1]]]
    bz = [[az[0][0] * az[0][0], 2. * az[0][0] * az[0][1], az[0][1] * az[0][1]],
          [az[0][0] * az[1][0], az[0][1] * az[1][0] + az[0][0] * az[1][1], az[0][1] * az[1][1]],
          [az[1][0] * az[1][0], 2. * az[1][0] * az[1][1], az[1][1] * az[1][1]]]

    def mv(a, v):
        return [sum(a[i][j] * v[j] for j in range(len(v))) for i in range(len(v))]
    m = mom
    m[1], m[2] = mv(ax, [m[1], m[2]])
    m[3], m[4] = mv(az, [m[3], m[4]])
    m[5], m[6], m[7] = mv(bx, [m[5], m[6], m[7]])
    m[8], m[9], m[10] = mv(bz, [m[8], m[9], m[10]])


def drift_propagate_moments(w: Wfr, L):
    """srTDriftSpace::PropagateRadMoments -> AuxPropagateRadMoments (sroptdrf.h:967, sroptdrf.cpp:22)."""
    a = [[1., L], [0., 1.]]
    for mom in (w.momX, w.momZ):
        if mom[0] != 0.:
            _mom_apply(mom, a, a)
            sx = _diff_lim_spot(w, 'x', L)
            if mom[5] - mom[1] * mom[1] < sx * sx:
                mom[5] = sx * sx + mom[1] * mom[1]
            sz = _diff_lim_spot(w, 'z', L)
            if mom[8] - mom[3] * mom[3] < sz * sz:
                mom[8] = sz * sz + mom[3] * mom[3]


def drift_ang_repres(w: Wfr, L, treat):
    """PropagateRadiationSimple_AngRepres (sroptdrf.h:348-411) + RadPointModifier_AngRepres (:615)."""
    xStartOld, zStartOld = w.xStart, w.zStart
    w.xStart = -(w.nx >> 1) * w.xStep
    w.zStart = -(w.nz >> 1) * w.zStep
    xShift, zShift = w.xStart - xStartOld, w.zStart - zStartOld
    w.xWfrMin += xShift; w.xWfrMax += xShift
    w.zWfrMin += zShift; w.zWfrMax += zShift
    if w.Pres != 1:
        set_rad_repres(w, 1)
    qx, qz = w.coords()
    lam = LAMBDA_EV_M / w.eStart
    c0 = -3.1415926536 * L * lam
    c1 = 0.25 * lam * lam
    q2 = qx * qx + qz * qz
    c1q2 = c1 * q2
    ph = c0 * q2 * (1. + c1q2 + 2. * c1q2 * c1q2)
    if treat == 1:
        ph = ph + 5.067730652e+06 * L * w.eStart
    _apply_phase(w, ph)
    if w.UseStartTrToShiftAtChangingRepresToCoord:
        w.xStartTr += xShift
        w.zStartTr += zShift
    set_rad_repres(w, 0)
    w.xStart, w.zStart = xStartOld, zStartOld
    if w.UseStartTrToShiftAtChangingRepresToCoord:
        w.xStart = w.xStartTr - xShift
        w.zStart = w.zStartTr - zShift
    w.set_full_range()


def drift_to_waist(w: Wfr, L, treat):
    """PropagateRadiationSimple_PropToWaist (sroptdrf.cpp:356-489), SetupPropBufVars_PropToWaist
    (sroptdrf.h:476-502), RadPointModifier_PropToWaist (sroptdrf.h:649-710)."""
    w.set_full_range()
    InvLength = 1. / L
    Pi_d_LambdaM = w.eStart * PI_D_LAMBDA_PER_EV
    Pi_d_LambdaM_d_Length = Pi_d_LambdaM * InvLength
    InvLength_d_Lambda = InvLength * w.eStart * INV_LAMBDA_PER_EV
    TwoPi_d_LambdaM = 2. * Pi_d_LambdaM
    TwoPiXc_d_LambdaMRx = TwoPi_d_LambdaM * w.xc / w.RobsX
    TwoPiZc_d_LambdaMRz = TwoPi_d_LambdaM * w.zc / w.RobsZ
    if w.Pres != 0:
        set_rad_repres(w, 0)
    x, z = w.coords()
    ph = Pi_d_LambdaM_d_Length * (x * x + z * z) + TwoPiXc_d_LambdaMRx * x + TwoPiZc_d_LambdaMRz * z
    if treat == 1:
        ph = ph + 5.067730652e+06 * L * w.eStart
    _apply_phase(w, ph)
    InvLambda_m = w.eStart * INV_LAMBDA_PER_EV
    InvLambda_m_d_Length = InvLambda_m / L
    LambdaM_Length = 1. / InvLambda_m_d_Length
    r = None
    for comp in ('ex', 'ey'):
        d, xs, ys, x0, y0 = make_2d_fft(getattr(w, comp), w.nx, w.nz, w.xStep, w.zStep, w.xStart, w.zStart, 1)
        setattr(w, comp, d)
        r = (xs, ys, x0, y0)
    xStepTr, yStepTr, xStartTr, yStartTr = r
    qxCen = -w.xc * InvLambda_m / w.RobsX
    qzCen = -w.zc * InvLambda_m / w.RobsZ
    w.xStart = (xStartTr + qxCen) * LambdaM_Length
    w.zStart = (yStartTr + qzCen) * LambdaM_Length
    w.xStep = xStepTr * LambdaM_Length
    w.zStep = yStepTr * LambdaM_Length
    x, z = w.coords()
    ph = Pi_d_LambdaM_d_Length * (x * x + z * z)
    w.mult(np.exp(1j * ph) * (-1j * InvLength_d_Lambda))
    if LambdaM_Length < 0:
        mirror_field(w, -1, -1)
        xEnd = w.xStart + w.xStep * (w.nx - 1)
        w.xStart = xEnd
        w.xStep *= -1.
        zEnd = w.zStart + w.zStep * (w.nz - 1)
        w.zStart = zEnd
        w.zStep *= -1.


def drift_from_waist(w: Wfr, L, treat):
    """PropagateRadiationSimple_PropFromWaist (sroptdrf.cpp:614-724), SetupPropBufVars_PropFromWaist
    (sroptdrf.h:522-535), RadPointModifier_PropFromWaist (sroptdrf.h:756-804): quadratic phase,
    forward FFT, mesh scaled by lambda L, quadratic phase again with the 1/(lambda L) factor and the
    -i; no centre terms and no mirror."""
    InvLength = 1. / L
    Pi_d_LambdaM = w.eStart * PI_D_LAMBDA_PER_EV
    Pi_d_LambdaM_d_Length = Pi_d_LambdaM * InvLength
    InvLength_d_Lambda = InvLength * w.eStart * INV_LAMBDA_PER_EV
    if w.Pres != 0:
        set_rad_repres(w, 0)
    x, z = w.coords()
    _apply_phase(w, Pi_d_LambdaM_d_Length * (x * x + z * z))
    InvLambda_m = w.eStart * INV_LAMBDA_PER_EV
    LambdaM_Length = 1. / (InvLambda_m / L)
    r = None
    for comp in ('ex', 'ey'):
        d, xs, ys, x0, y0 = make_2d_fft(getattr(w, comp), w.nx, w.nz, w.xStep, w.zStep, w.xStart, w.zStart, 1)
        setattr(w, comp, d)
        r = (xs, ys, x0, y0)
    xStepTr, yStepTr, xStartTr, yStartTr = r
    w.xStart = xStartTr * LambdaM_Length
    w.zStart = yStartTr * LambdaM_Length
    w.xStep = xStepTr * LambdaM_Length
    w.zStep = yStepTr * LambdaM_Length
    x, z = w.coords()
    ph = Pi_d_LambdaM_d_Length * (x * x + z * z)
    if treat == 1:
        ph = ph + 5.067730652e+06 * L * w.eStart
    w.mult(np.exp(1j * ph) * (-1j * InvLength_d_Lambda))


def _radical(x, plus_one):
    """sqrt(1 + x) (plus_one) or sqrt(1 + x) - 1 as sroptdrf.h:731-735 evaluates them: the square
    root for |x| > 0.01, else the 8-term binomial series of sqrt(1 + x) - 1 (plus 1)."""
    x = np.asarray(x, np.float64)
    ser = x * (0.5 + x * (-0.125 + x * (0.0625 + x * (-0.0390625 + x * (0.02734375 + x * (-0.0205078125 +
                                                                                      x * 0.01611328125))))))
    root = np.sqrt(np.maximum(1. + x, 0.))
    if plus_one:
        return np.where(np.abs(x) > 0.01, root, 1. + ser)
    return np.where(np.abs(x) > 0.01, root - 1., ser)


def drift_to_waist_beyond_parax(w: Wfr, L, treat):
    """PropagateRadiationSimple_PropToWaistBeyondParax (sroptdrf.cpp:491-612), its buffer set-up
    (sroptdrf.h:492-520) and RadPointModifier_PropToWaistBeyondParax (sroptdrf.h:712-754): the
    quadratic phase off (TreatQuadPhaseTerm 'r' with the wavefront's current treatment flags), the
    mesh mapped to angular frequencies (x - xc)/(lambda R), the exact propagator
    exp(i k L (sqrt(1 - lambda^2 q^2) - 1)) with the curvature and Gouy terms, an inverse FFT, and a
    mirror where the transformed steps are negative."""
    w.set_full_range()
    sqrtAbsRxRz = math.sqrt(abs(w.RobsX * w.RobsZ))
    sgnRx = 1 if w.RobsX >= 0 else -1
    sgnRz = 1 if w.RobsZ >= 0 else -1
    dPhaseSignR = 0.7853981633974483 * (sgnRx + sgnRz)
    Pi_MultLambdaM = 3.141592653589793 * 1.239842e-06
    Pi_MultLambdaM_Rx = Pi_MultLambdaM * w.RobsX
    Pi_MultLambdaM_Rz = Pi_MultLambdaM * w.RobsZ
    MultEn_TwoPi_L_d_LambdaM = 2. * 2.53384080189E+06 * L
    if w.Pres != 0:
        set_rad_repres(w, 0)
    _treat_strongly_oscillating(w, 'r')       # srradstr.h:841, with the flags as they stand
    xcOrig, zcOrig = w.xc, w.zc
    InvLambdaM = w.eStart * 806546.577258
    InvLambdaM_d_Rx = InvLambdaM / w.RobsX
    InvLambdaM_d_Rz = InvLambdaM / w.RobsZ
    w.xStep *= InvLambdaM_d_Rx
    w.zStep *= InvLambdaM_d_Rz
    w.xStart = (w.xStart - xcOrig) * InvLambdaM_d_Rx
    w.zStart = (w.zStart - zcOrig) * InvLambdaM_d_Rz
    x, z = w.coords()
    e = w.eStart
    ph = -(Pi_MultLambdaM_Rx * x * x + Pi_MultLambdaM_Rz * z * z) / e
    kL = MultEn_TwoPi_L_d_LambdaM * e
    LambdaM = 1.239842e-06 / e
    lx, lz = LambdaM * x, LambdaM * z
    X = -(lx * lx + lz * lz)
    ph = ph + kL * _radical(X, treat == 1) + dPhaseSignR
    w.mult(np.exp(1j * ph) * (LambdaM * sqrtAbsRxRz))
    res = None
    for comp in ('ex', 'ey'):
        d, xs, ys, x0, y0 = make_2d_fft(getattr(w, comp), w.nx, w.nz, w.xStep, w.zStep, w.xStart, w.zStart, -1)
        setattr(w, comp, d)
        res = (xs, ys, x0, y0)
    xStepTr, yStepTr, xStartTr, yStartTr = res
    sx = sz = 1
    xStartNew, xStepNew = xStartTr + xcOrig, xStepTr
    zStartNew, zStepNew = yStartTr + zcOrig, yStepTr
    if xStepTr < 0:
        sx = -1
        xStartNew, xStepNew = -xStartTr + xcOrig, -xStepTr
    if yStepTr < 0:
        sz = -1
        zStartNew, zStepNew = -yStartTr + zcOrig, -yStepTr
    if sx < 0 or sz < 0:
        mirror_field(w, sx, sz)
    w.xStart, w.zStart, w.xStep, w.zStep = xStartNew, zStartNew, xStepNew, zStepNew


def _sign(v):
    return 1. if v > 0 else (-1. if v < 0 else 0.)


def drift_quad(w: Wfr, L, treat, subtype):
    """PropagateRadiationSimple_AnalytTreatQuadPhaseTerm (sroptdrf.cpp:726-887) with
    SetupPropBufVars_AnalytTreatQuadPhaseTerm (:889-1083) and the pp[3]=2 radius estimate
    EstimateWfrRadToSub2_AnalytTreatQuadPhaseTerm (:1085-1120); modifier sroptdrf.h:806-880."""
    infLarge = 1E+23
    xc, zc = w.xc, w.zc
    invRx = invRz = 0.
    Lx = Lz = 0.
    invRxL = invRzL = 1. / L
    kx = kxc = kz = kzc = infLarge
    trueRx, trueRz = w.RobsX, w.RobsZ
    if subtype == 2:
        factRadEr = 3.
        minAbsEffRx = factRadEr * w.RobsXAbsErr
        minAbsEffRz = factRadEr * w.RobsZAbsErr
        effRx_p_L = trueRx + L
        if abs(trueRx) < minAbsEffRx:
            trueRx = minAbsEffRx * (1. if trueRx >= 0 else -1.)
        elif abs(effRx_p_L) < minAbsEffRx:
            trueRx = minAbsEffRx * (1. if effRx_p_L >= 0 else -1.) - L
        effRz_p_L = trueRz + L
        if abs(trueRz) < minAbsEffRz:
            trueRz = minAbsEffRz * (1. if trueRz >= 0 else -1.)
        elif abs(effRz_p_L) < minAbsEffRz:
            trueRz = minAbsEffRz * (1. if effRz_p_L >= 0 else -1.) - L
    elif subtype == 1:
        trueRx, trueRz = estimate_rad_to_sub(w, L)
    if trueRx != 0:
        invRx = 1. / trueRx
        kx = (trueRx + L) * invRx
        kxc = L / trueRx
        if -L != trueRx:
            Lx = L / (1. + L * invRx)
            invRxL = 1. / (L + trueRx)
        else:
            Lx = infLarge
            invRxL = infLarge
    if trueRz != 0:
        invRz = 1. / trueRz
        kz = (trueRz + L) * invRz
        kzc = L / trueRz
        if -L != trueRz:
            Lz = L / (1. + L * invRz)
            invRzL = 1. / (L + trueRz)
        else:
            Lz = infLarge
            invRzL = infLarge
    sqrt_LxLz_d_L = math.sqrt(abs(Lx * Lz)) / L
    phase_term_signLxLz = 0.25 * 3.141592653589793 * (2. - _sign(Lx) - _sign(Lz))

    if w.Pres != 0:
        set_rad_repres(w, 0)
    lam = LAMBDA_EV_M / w.eStart
    x, z = w.coords()
    rx, rz = x - xc, z - zc
    Pi_d_Lambda_m = 3.1415926536 / lam
    _apply_phase(w, -Pi_d_Lambda_m * (invRx * rx * rx + invRz * rz * rz))
    xStartOld, zStartOld = w.xStart, w.zStart
    w.xStart = -(w.nx >> 1) * w.xStep
    w.zStart = -(w.nz >> 1) * w.zStep
    xShift, zShift = w.xStart - xStartOld, w.zStart - zStartOld
    w.xWfrMin += xShift; w.xWfrMax += xShift
    w.zWfrMin += zShift; w.zWfrMax += zShift
    set_rad_repres(w, 1)
    qx, qz = w.coords()
    Pi_Lambda_m = 3.1415926536 * lam
    c0x, c0z = -Pi_Lambda_m * Lx, -Pi_Lambda_m * Lz
    w.mult(np.exp(1j * (c0x * qx * qx + c0z * qz * qz + phase_term_signLxLz)) * sqrt_LxLz_d_L)
    if w.UseStartTrToShiftAtChangingRepresToCoord:
        w.xStartTr += xShift
        w.zStartTr += zShift
    set_rad_repres(w, 0)
    w.xStart, w.zStart = xStartOld, zStartOld
    if w.UseStartTrToShiftAtChangingRepresToCoord:
        w.xStart = w.xStartTr - xShift
        w.zStart = w.zStartTr - zShift
    w.xStart = kx * w.xStart - kxc * w.xc
    w.xStep *= kx
    w.zStart = kz * w.zStart - kzc * w.zc
    w.zStep *= kz
    x, z = w.coords()
    rx, rz = x - xc, z - zc
    ph = Pi_d_Lambda_m * (invRxL * rx * rx + invRzL * rz * rz)
    if treat == 1:
        ph = ph + 2 * Pi_d_Lambda_m * L
    _apply_phase(w, ph)
    mirror_field(w, int(_sign(kx)), int(_sign(kz)))
    if kx < 0:
        xEnd = w.xStart + (w.nx - 1) * w.xStep
        w.xStart = xEnd
        w.xStep *= -1
    if kz < 0:
        zEnd = w.zStart + (w.nz - 1) * w.zStep
        w.zStart = zEnd
        w.zStep *= -1
    w.set_full_range()


def mirror_field(w: Wfr, sx, sz):
    """MirrorFieldData (srradstr.cpp:2707)."""
    if sx < 0:
        w.ex = w.ex[:, ::-1].copy(); w.ey = w.ey[:, ::-1].copy()
    if sz < 0:
        w.ex = w.ex[::-1, :].copy(); w.ey = w.ey[::-1, :].copy()


def drift(w: Wfr, L, treat, anal_treatment):
    """srTDriftSpace::PropagateRadiation (sroptdrf.h:116) -> ChooseLocalPropMode (:223) ->
    PropagateRadiationSingleE_Meth_0 (:158): Simple, moments, radius, 4x4 matrix."""
    if anal_treatment in (1, 2):
        drift_quad(w, L, treat, anal_treatment)
    elif anal_treatment == 4:
        drift_to_waist(w, L, treat)
    elif anal_treatment == 3:
        drift_from_waist(w, L, treat)
    elif anal_treatment == 5:
        drift_to_waist_beyond_parax(w, L, treat)
    elif anal_treatment == 0:
        drift_ang_repres(w, L, treat)
    else:
        raise NotImplementedError("drift mode pp[3]=%d is not restated" % anal_treatment)
    drift_propagate_moments(w, L)
    w.RobsX += L                             # PropagateWaveFrontRadius (sroptdrf.h:981)
    w.RobsZ += L
    w.set_full_range()
    # Propagate4x4PropMatr of the drift (sroptdrf.h:1002)
    _prop_4x4(w, np.array([[1., L, 0., 0.], [0., 1., 0., 0.], [0., 0., 1., L], [0., 0., 0., 1.]]), np.zeros(4))


def _prop_4x4(w: Wfr, E, e):
    """GenAuxPropagate4x4PropMatr (sroptelm.cpp:5594): M <- E M, V <- E V + e on arElecPropMatr."""
    M = np.asarray(w.propM[:16], np.float64).reshape(4, 4)
    V = np.asarray(w.propM[16:20], np.float64)
    R = np.zeros((4, 4))
    RV = np.zeros(4)
    for i in range(4):
        for j in range(4):
            r = 0.
            for k in range(4):
                r += E[i, k] * M[k, j]
            R[i, j] = r
            RV[i] += E[i, j] * V[j]
    w.propM = np.concatenate([R.ravel(), RV + e])


# ----------------------------------------------------------------------------------------
# Linear phase terms (srradstr.cpp:2610-2705)
# ----------------------------------------------------------------------------------------


def _mult_phase_lin(w: Wfr, xMult, zMult):
    """MultiplyElFieldByPhaseLin (srradstr.h:509): exp(i(xMult x + zMult z))."""
    x, z = w.coords()
    _apply_phase(w, xMult * x + zMult * z)


def check_and_subtract_phase_lin(w: Wfr, newXc, newZc):
    ratAllowSubtract = 0.2
    minNumOptCycles = 10
    lambda_m = 3.1415926535898 / (w.eStart * 2.53384080189E+06)
    twoPi = 2. * 3.1415926535898
    xOK = False
    dxcSubNew = newXc - w.xc
    if w.RobsX != 0:
        rng = w.xStep * (w.nx - 1)
        ncyc = 0.25 * rng * rng / (lambda_m * w.RobsX)
        xOK = (abs(w.RobsX) > abs(w.RobsXAbsErr)) and (ncyc > minNumOptCycles) and (abs(dxcSubNew) / rng > ratAllowSubtract)
    if not xOK:
        dxcSubNew = 0
    zOK = False
    dzcSubNew = newZc - w.zc
    if w.RobsZ != 0:
        rng = w.zStep * (w.nz - 1)
        ncyc = 0.25 * rng * rng / (lambda_m * w.RobsZ)
        zOK = (abs(w.RobsZ) > abs(w.RobsZAbsErr)) and (ncyc > minNumOptCycles) and (abs(dzcSubNew) / rng > ratAllowSubtract)
    if not zOK:
        dzcSubNew = 0
    if (not xOK) and (not zOK):
        return
    dxc = dxcSubNew
    if w.xLinOnly:
        dxc -= w.dxcSub
        if abs(dxc) / abs(w.dxcSub) < ratAllowSubtract:
            dxc = 0; dxcSubNew = w.dxcSub
    w.dxcSub = dxcSubNew
    w.xLinOnly = (dxcSubNew != 0)
    xMult = -twoPi * dxc / (lambda_m * w.RobsX)
    dzc = dzcSubNew
    if zOK and w.zLinOnly:
        dzc -= w.dzcSub
        if abs(dzc) / abs(w.dzcSub) < ratAllowSubtract:
            dzc = 0; dzcSubNew = w.dzcSub
    w.dzcSub = dzcSubNew
    w.zLinOnly = (dzcSubNew != 0)
    zMult = -twoPi * dzc / (lambda_m * w.RobsZ)
    if xMult == 0 and zMult == 0:
        return
    _mult_phase_lin(w, xMult, zMult)


def check_and_reset_phase_lin(w: Wfr):
    if (not w.xLinOnly) and (not w.zLinOnly):
        return
    lambda_m = 3.1415926535898 / (w.eStart * 2.53384080189E+06)
    twoPi = 2. * 3.1415926535898
    xMult = zMult = 0.
    if w.xLinOnly and w.dxcSub != 0 and w.RobsX != 0:
        xMult = twoPi * w.dxcSub / (lambda_m * w.RobsX)
    if w.zLinOnly and w.dzcSub != 0 and w.RobsZ != 0:
        zMult = twoPi * w.dzcSub / (lambda_m * w.RobsZ)
    w.xLinOnly = w.zLinOnly = False
    w.dxcSub = w.dzcSub = 0
    if xMult == 0 and zMult == 0:
        return
    _mult_phase_lin(w, xMult, zMult)


# ----------------------------------------------------------------------------------------
# Thin lens (cpp/src/core/sroptfoc.h:18-276)
# ----------------------------------------------------------------------------------------


def _fix_abs_err(w: Wfr):
    """Tail of srTGenOptElem::PropagateRadiationMeth_0 (sroptel2.cpp:151-152, non-OpenMP build)."""
    if w.RobsX != 0 and w.RobsXAbsErr == 0:
        w.RobsXAbsErr = abs(0.1 * w.RobsX)
    if w.RobsZ != 0 and w.RobsZAbsErr == 0:
        w.RobsZAbsErr = abs(0.1 * w.RobsZ)


def lens(w: Wfr, Fx, Fz, cx, cz):
    check_and_subtract_phase_lin(w, cx, cz)
    if w.Pres != 0:
        set_rad_repres(w, 0)
    x, z = w.coords()
    Pi_d_Lambda_m = w.eStart * 2.533865612E+06
    xr, zr = x - cx, z - cz
    _apply_phase(w, -Pi_d_Lambda_m * (xr * xr / Fx + zr * zr / Fz))
    ax = [[1., 0.], [-1. / Fx, 1.]]
    az = [[1., 0.], [-1. / Fz, 1.]]
    for mom in (w.momX, w.momZ):
        _mom_apply(mom, ax, az)
    dSmall = 1E-23                                # PropagateWaveFrontRadius (sroptfoc.h:37)
    difX = dSmall if Fx == w.RobsX else Fx - w.RobsX
    difZ = dSmall if Fz == w.RobsZ else Fz - w.RobsZ
    MagnX, MagnZ = Fx / difX, Fz / difZ
    w.RobsX *= MagnX
    w.RobsZ *= MagnZ
    w.RobsXAbsErr *= MagnX * MagnX
    w.RobsZAbsErr *= MagnZ * MagnZ
    w.xc = cx - (cx - w.xc) * MagnX
    w.zc = cz - (cz - w.zc) * MagnZ
    # Propagate4x4PropMatr of the focusing element (sroptfoc.h:101)
    _prop_4x4(w, np.array([[1., 0., 0., 0.], [-1. / Fx, 1., 0., 0.], [0., 0., 1., 0.], [0., 0., -1. / Fz, 1.]]),
              np.array([0., cx / Fx, 0., cz / Fz]))
    _fix_abs_err(w)
    check_and_reset_phase_lin(w)


# ----------------------------------------------------------------------------------------
# Generic transmission (cpp/src/core/sroptgtr.h:86-140, point modifier sroptgtr.h:168-333,
# constructor from SRWLOptT sroptgtr.cpp:139-180)
# ----------------------------------------------------------------------------------------


def _tr_axis(v, start, step, n):
    """Cell index and fraction of a table axis (sroptgtr.h:205-225): index by truncation toward zero,
    snapped up within 1e-5 of a step from the next node, the first cell below the table (fraction 0
    when more than one step below, linear extrapolation within the step), the last cell with
    fraction 1 above it."""
    i = np.trunc((v - start) / step).astype(np.int64)
    i = np.where(np.abs(v - ((i + 1) * step + start)) < 1.E-05 * step, i + 1, i)
    frac = (v - (i * step + start)) / step
    frac = np.where(i < 0, 0., np.where(i > n - 2, 1., frac))
    i = np.clip(i, 0, n - 2)
    return i, frac


def transmission(w: Wfr, arTr, nx, nz, rx, rz, x, z, extTr, Fx, Fz, ne=1, eStart=0., eFin=0.):
    """srTGenTransmission: amplitude transmission T and optical path difference OPD tabulated over
    [nz][nx] (pairs, ne == 1) on the mesh of ranges rx, rz centred on (x, z) (the SRWLOptT
    constructor, srwlib.py:3071-3082), interpolated bilinearly at the wavefront's absolute
    coordinates; E *= T exp(i k OPD); zero outside the table when extTr == 0.  The bookkeeping
    (moments, radius, centre, 4x4 matrix) is the focusing element's with the estimated focal
    lengths Fx, Fz about the table's centre."""
    xStart, xFin = x - 0.5 * rx, x + 0.5 * rx
    zStart, zFin = z - 0.5 * rz, z + 0.5 * rz
    cx, cz = 0.5 * (xStart + xFin), 0.5 * (zStart + zFin)
    check_and_subtract_phase_lin(w, cx, cz)
    if w.Pres != 0:
        set_rad_repres(w, 0)
    x, z = w.coords()
    x = np.broadcast_to(x, (w.nz, w.nx))
    z = np.broadcast_to(z, (w.nz, w.nx))
    xStep, zStep = (xFin - xStart) / (nx - 1), (zFin - zStart) / (nz - 1)
    ix, xr = _tr_axis(x, xStart, xStep, nx)
    iz, zr = _tr_axis(z, zStart, zStep, nz)
    if ne == 1:
        tab = np.asarray(arTr, dtype=np.float64).reshape(nz, nx, 2)
        p00, p10, p01, p11 = tab[iz, ix], tab[iz, ix + 1], tab[iz + 1, ix], tab[iz + 1, ix + 1]
        a_xz = p00 - p01 - p10 + p11
        a_x, a_z = p10 - p00, p01 - p00
        v = a_xz * (xr * zr)[..., None] + a_x * xr[..., None] + a_z * zr[..., None] + p00
    else:
        # trilinear in (e, x, z) over [nz][nx][ne] pairs (sroptgtr.h:275-300)
        tab = np.asarray(arTr, dtype=np.float64).reshape(nz, nx, ne, 2)
        eStep = (eFin - eStart) / (ne - 1)
        ie = min(max(int((w.eStart - eStart) / eStep + 1.e-10), 0), ne - 2)
        er = (w.eStart - (ie * eStep + eStart)) / eStep
        c = lambda a, b, k: tab[iz + b, ix + a, ie + k]      # noqa: E731  (x offset a, z offset b, e offset k)
        xr_, zr_ = xr[..., None], zr[..., None]
        v = ((c(0, 0, 0) * ((1. - er) * (1. - xr_)) + c(0, 0, 1) * (er * (1. - xr_)) + c(1, 0, 0) * ((1. - er) * xr_)
              + c(1, 0, 1) * (er * xr_)) * (1. - zr_)
             + (c(0, 1, 0) * ((1. - er) * (1. - xr_)) + c(0, 1, 1) * (er * (1. - xr_)) + c(1, 1, 0) * ((1. - er) * xr_)
                + c(1, 1, 1) * (er * xr_)) * zr_)
    T, Ph = v[..., 0], v[..., 1] * (w.eStart * 5.0676816042E+06)
    fac = T * np.exp(1j * Ph)
    if extTr == 0:
        xEnd, zEnd = xStart + (nx - 1) * xStep, zStart + (nz - 1) * zStep
        tx, tz = xStep * 0.001, zStep * 0.001
        outside = (x < xStart - tx) | (x > xEnd + tx) | (z < zStart - tz) | (z > zEnd + tz)
        fac = np.where(outside, 0., fac)
    w.mult(fac)
    ax = [[1., 0.], [-1. / Fx, 1.]]
    az = [[1., 0.], [-1. / Fz, 1.]]
    for mom in (w.momX, w.momZ):
        _mom_apply(mom, ax, az)
    dSmall = 1E-23
    difX = dSmall if Fx == w.RobsX else Fx - w.RobsX
    difZ = dSmall if Fz == w.RobsZ else Fz - w.RobsZ
    MagnX, MagnZ = Fx / difX, Fz / difZ
    w.RobsX *= MagnX
    w.RobsZ *= MagnZ
    w.RobsXAbsErr *= MagnX * MagnX
    w.RobsZAbsErr *= MagnZ * MagnZ
    w.xc = cx - (cx - w.xc) * MagnX
    w.zc = cz - (cz - w.zc) * MagnZ
    _prop_4x4(w, np.array([[1., 0., 0., 0.], [-1. / Fx, 1., 0., 0.], [0., 0., 1., 0.], [0., 0., -1. / Fz, 1.]]),
              np.array([0., cx / Fx, 0., cz / Fz]))
    _fix_abs_err(w)
    check_and_reset_phase_lin(w)


# ----------------------------------------------------------------------------------------
# Apertures / obstacles (cpp/src/core/sroptapt.h)
# ----------------------------------------------------------------------------------------


def aperture(w: Wfr, shape, ap_or_ob, Dx, Dy, cx, cy):
    if w.Pres != 0:
        set_rad_repres(w, 0)
    x, z = w.coords()
    xr, zr = x - cx, z - cy
    if shape == 'r':
        hx, hz = 0.5 * Dx + 1.E-10, 0.5 * Dy + 1.E-10
        inside = (xr >= -hx) & (xr <= hx) & (zr >= -hz) & (zr <= hz)
    else:
        R = 0.5 * Dx
        inside = ~(xr * xr + zr * zr > R * R)
        if ap_or_ob in 'oO':
            inside = (xr * xr + zr * zr > R * R)
    if shape == 'r' and ap_or_ob in 'oO':
        inside = ~inside
    w.ex = np.where(inside, w.ex, 0.)
    w.ey = np.where(inside, w.ey, 0.)
    # srTAperture::PropagateRadMoments (sroptapt.cpp:248-350): recompute the moments numerically
    # when 1.7 sigma of the beam is not inside the opening (obstacles: always, sroptapt.h:294)
    if ap_or_ob in 'oO' or _moments_outside_opening(w, shape, Dx, Dy, cx, cy):
        compute_rad_moments(w)
    # SetNewNonZeroWfrLimits (apertures only; obstacles keep the limits in the cases used here)
    if ap_or_ob in 'aA':
        if shape == 'r':
            hx, hz = 0.5 * Dx, 0.5 * Dy
        else:
            hx = hz = 0.5 * Dx
        w.xWfrMin = max(w.xWfrMin, cx - hx)
        w.xWfrMax = min(w.xWfrMax, cx + hx)
        w.zWfrMin = max(w.zWfrMin, cy - hz)
        w.zWfrMax = min(w.zWfrMax, cy + hz)
    _fix_abs_err(w)


# ----------------------------------------------------------------------------------------
# Resizing (srTGenOptElem::RadResizeGen sroptelm.cpp:2242-3036, RadResizeCore :3038-3337)
# ----------------------------------------------------------------------------------------


def _int_offset_coord(xStart, xStep, xVal):
    """IntegerOffsetCoord (sroptelm.h:995)."""
    i = int((xVal - xStart) / xStep)
    if abs(xVal - ((i + 1) * xStep + xStart)) < 1.E-05 * xStep:
        i += 1
    return i


def _wavefront_term_can_be_treated(w: Wfr):
    """WaveFrontTermCanBeTreated (sroptelm.cpp:4692), checkBenefit=false."""
    w.QuadX = abs(w.RobsXAbsErr) < 0.4 * abs(w.RobsX)
    w.QuadZ = abs(w.RobsZAbsErr) < 0.4 * abs(w.RobsZ)
    return w.QuadX or w.QuadZ


def _treat_strongly_oscillating(w: Wfr, add_or_rem):
    """TreatStronglyOscillatingTerm (sroptelm.cpp:4774-5014), coordinate representation."""
    Const = 3.14159265358979 * 1.E+06 / 1.23984186
    if w.Pres == 0:
        cRx = Const / w.RobsX if w.QuadX else 0.
        cRz = Const / w.RobsZ if w.QuadZ else 0.
    else:
        lam = LAMBDA_EV_M / w.eStart
        cRx = -Const * w.RobsX * lam * lam if w.QuadX else 0.
        cRz = -Const * w.RobsZ * lam * lam if w.QuadZ else 0.
    if add_or_rem == 'r':
        cRx, cRz = -cRx, -cRz
    x, z = w.coords()
    x = x - w.xc
    z = z - w.zc
    ph = np.zeros((w.nz, w.nx))
    if w.QuadZ:
        ph = ph + cRz * w.eStart * z * z
    if w.QuadX:
        ph = ph + cRx * w.eStart * x * x
    _apply_phase(w, ph)


def _central_full(m):
    """srTMomentsPtrs::ComputeCentralMoments (srstraux.h:357): (precCenMomIsOK, SqrtMxpxp,
    SqrtMzpzp) of one component's 11 moments."""
    Mxx = m[5] - m[1] * m[1]
    Mxpxp = m[7] - m[2] * m[2]
    Mzz = m[8] - m[3] * m[3]
    Mzpzp = m[10] - m[4] * m[4]
    ok = not (Mxx < 0 or Mxpxp < 0 or Mzz < 0 or Mzpzp < 0)
    if Mxpxp < 0.1 * m[7]:
        Mxpxp = 0.1 * m[7]
    if Mzpzp < 0.1 * m[10]:
        Mzpzp = 0.1 * m[10]
    return ok, math.sqrt(abs(Mxpxp)), math.sqrt(abs(Mzpzp))


def estimate_rad_to_sub(w: Wfr, L):
    """srTDriftSpace::EstimateWfrRadToSub_AnalytTreatQuadPhaseTerm (sroptdrf.cpp:1123-1365), the
    pp[3]=1 radius estimate from the rms divergence: the moments are recomputed from the field when
    both norms are zero, or when the chosen component's central moments (as they stood before any
    recomputation) are unusable."""
    infLarge = 1E+23
    coefAngRange = 0.2
    fourPi = 4. * 3.14159265359
    cX, cZ = _central_full(w.momX), _central_full(w.momZ)
    s1X, s1Z = w.RobsX, w.RobsZ
    s2X, s2Z = s1X + L, s1Z + L
    if w.momX[0] == 0 and w.momZ[0] == 0:
        compute_rad_moments(w)
    use_x = w.momX[0] >= w.momZ[0]
    c = cX if use_x else cZ
    if (not c[0]) or c[1] == 0 or c[2] == 0:
        compute_rad_moments(w)
        c = _central_full(w.momX if use_x else w.momZ)
    SigXp, SigZp = c[1], c[2]
    if SigXp == 0 or SigZp == 0:
        return (w.RobsX if w.RobsX != 0 else infLarge), (w.RobsZ if w.RobsZ != 0 else infLarge)
    lambM = 1.239842E-06 / w.eStart

    def one(s1, s2, sig):
        ap = coefAngRange * sig
        smin = lambM / (fourPi * ap * ap)
        Rmin = 2 * smin
        if abs(s1) < smin:
            if abs(s2) < smin:
                if abs(s1) < abs(s2):
                    return Rmin if L > 0 else -Rmin
                return (-Rmin - L) if L > 0 else (Rmin - L)
            return Rmin if L > 0 else -Rmin
        eff = s1 + smin * smin / s1
        eff_p_L = eff + L
        minRmin = 0.007 * abs(eff)
        if Rmin < minRmin:
            Rmin = minRmin
        if abs(eff_p_L) < Rmin:
            eff = (-Rmin - L) if eff_p_L < 0 else (Rmin - L)
        return eff
    return one(s1X, s2X, SigXp), one(s1Z, s2Z, SigZp)


def central_moments(m):
    """srTMomentsPtrs::ComputeCentralMoments (srstraux.h:357): (sqrt Mxx, sqrt Mzz) with the 0.1
    safety floor on the central second moments."""
    Mxx = m[5] - m[1] * m[1]
    Mzz = m[8] - m[3] * m[3]
    if Mxx < 0.1 * m[5]:
        Mxx = 0.1 * m[5]
    if Mzz < 0.1 * m[8]:
        Mzz = 0.1 * m[8]
    return math.sqrt(abs(Mxx)), math.sqrt(abs(Mzz))


def _moments_outside_opening(w: Wfr, shape, Dx, Dy, cx, cy):
    """CheckIfMomentsShouldBeRecomputed of the rectangular (sroptapt.h:206) and circular
    (sroptapt.h:384) apertures, applied to the Ex and Ez moments with the 1.7 sigma margin."""
    hx, hz = (0.5 * Dx, 0.5 * Dy) if shape == 'r' else (0.5 * Dx, 0.5 * Dx)
    for m in (w.momX, w.momZ):
        sx, sz = central_moments(m)
        sx, sz = 1.7 * sx, 1.7 * sz
        if (m[1] - sx) < (cx - hx) or (m[1] + sx) > (cx + hx) or (m[3] - sz) < (cy - hz) or (m[3] + sz) > (cy + hz):
            return True
    return False


def _find_limit_left(a, stop):
    """srTAuxMatStat::FindLimit1DLeft (srmatsta.cpp:400): first index where the running sum
    exceeds `stop` (0 when it never does)."""
    s = 0.
    for i in range(len(a)):
        s += a[i]
        if s > stop:
            return i
    return 0


def _find_limit_right(a, stop):
    """FindLimit1DRight (srmatsta.cpp:426): the same from the right end (n - 1 when never)."""
    n = len(a)
    s = 0.
    for i in range(n):
        s += a[n - 1 - i]
        if s > stop:
            return n - 1 - i
    return n - 1


def _sum_up(a):
    """SumUpArray (srmatsta.h:437) over a whole line: 0 for fewer than two points."""
    return float(np.sum(a, dtype=np.float64)) if len(a) >= 2 else 0.


def find_intensity_limits_inds(I, w: Wfr, rel_pow=0.9):
    """srTAuxMatStat::FindIntensityLimitsInds (srmatsta.cpp:572) with FindIntensityLimits2D (:452):
    the index box holding `rel_pow` of the power of the FP32 intensity I [nz, nx], trimmed by
    (1 - rel_pow)/4 of the total at each edge, first along z (rows summed over x) then along x
    within the z limits.  Returns [ix0, ix1, iz0, iz1]; the whole mesh when the search fails."""
    nx, nz = w.nx, w.nz
    full = [0, nx - 1, 0, nz - 1]
    I = np.asarray(I, np.float32)
    tot = float(np.float32(float(np.sum(I, dtype=np.float64)) * w.xStep * w.zStep))   # IntegrateSimple
    stop = tot * (1. - rel_pow) * 0.25
    if nx < 2 or nz < 2:                                   # IntegrateOverX: ixStart >= ixEnd
        return full
    rows = np.array([w.xStep * _sum_up(I[iz, :]) for iz in range(nz)])
    iy0 = _find_limit_left(rows, stop / w.zStep)
    iy1 = _find_limit_right(rows, stop / w.zStep)
    if iy1 <= iy0:
        return full
    cols = np.array([w.zStep * (float(np.sum(I[iy0:iy1 + 1, ix], dtype=np.float64))) for ix in range(nx)])
    ix0 = _find_limit_left(cols, stop / w.xStep)
    ix1 = _find_limit_right(cols, stop / w.xStep)
    f = [np.float32(w.xStart + w.xStep * ix0), np.float32(w.xStart + w.xStep * ix1),
         np.float32(w.zStart + w.zStep * iy0), np.float32(w.zStart + w.zStep * iy1)]
    lims = [int((float(f[0]) - w.xStart) * 1.0000001 / w.xStep), int((float(f[1]) - w.xStart) * 1.0000001 / w.xStep),
            int((float(f[2]) - w.zStart) * 1.0000001 / w.zStep), int((float(f[3]) - w.zStart) * 1.0000001 / w.zStep)]
    lims[0] = max(lims[0], 0)
    lims[1] = min(lims[1], nx - 1)
    lims[2] = max(lims[2], 0)
    lims[3] = min(lims[3], nz - 1)
    return lims


def moment_sums(ex, ey, w: Wfr, lims):
    """The 22 weighted sums of srTGenOptElem::ComputeRadMoments (sroptelm.cpp:1745-1935) for the
    coordinate representation: per component norm, first moments, and (inside the power limits)
    second moments; the angular moments from finite differences of the field along x and z plus
    the wavefront-curvature term 2 pi/(lambda R) * step * coordinate.  Trapezoid weights: 1/2 at
    the mesh edges, and 1/2 again on the angular terms of the second row / column."""
    nx, nz = w.nx, w.nz
    lam = 1.239842E-06 / w.eStart
    R_x = w.RobsX if w.RobsX != 0. else 100. * lam
    R_z = w.RobsZ if w.RobsZ != 0. else 100. * lam
    four_pi = 3.141592653590 * 2. * 2.
    lam_d_4pi = 1.239842E-06 / (four_pi * w.eStart)
    ax = 0.5 * (w.xStep * ((1. / lam_d_4pi) / R_x))         # TwoPi_d_Lamb_d_Rx_xStep
    az = 0.5 * (w.zStep * ((1. / lam_d_4pi) / R_z))
    x = (w.xStart + np.arange(nx) * w.xStep)[None, :]
    z = (w.zStart + np.arange(nz) * w.zStep)[:, None]
    ix = np.arange(nx)[None, :]
    iz = np.arange(nz)[:, None]
    inside = (ix >= lims[0]) & (ix <= lims[1]) & (iz >= lims[2]) & (iz <= lims[3])
    S = np.zeros(22)
    for base, E in ((0, ex), (11, ey)):
        re, im = np.real(E).astype(np.float64), np.imag(E).astype(np.float64)
        f = [None] * 11
        n = re * re + im * im
        f[0] = n
        f[1] = x * n
        f[3] = z * n
        f[5] = np.where(inside, x * f[1], 0.)
        f[8] = np.where(inside, z * f[3], 0.)
        # along x (ix > 0)
        dr = np.zeros_like(re); di = np.zeros_like(im)
        dr[:, 1:] = re[:, 1:] - re[:, :-1]
        di[:, 1:] = im[:, 1:] - im[:, :-1]
        cr = di * re - dr * im
        hasx = np.broadcast_to(ix > 0, re.shape)
        f[2] = np.where(hasx, cr + ax * x * n, 0.)
        f[6] = np.where(hasx & inside, x * f[2], 0.)
        f[7] = np.where(hasx & inside, (dr * dr + di * di) + cr * ax * x + ax * ax * x * x * n, 0.)
        # along z (iz > 0)
        dr = np.zeros_like(re); di = np.zeros_like(im)
        dr[1:, :] = re[1:, :] - re[:-1, :]
        di[1:, :] = im[1:, :] - im[:-1, :]
        cr = di * re - dr * im
        hasz = np.broadcast_to(iz > 0, re.shape)
        f[4] = np.where(hasz, cr + az * z * n, 0.)
        f[9] = np.where(hasz & inside, z * f[4], 0.)
        f[10] = np.where(hasz & inside, (dr * dr + di * di) + cr * az * z + az * az * z * z * n, 0.)
        wx = np.ones(nx); wx[0] *= 0.5; wx[-1] *= 0.5
        wz = np.ones(nz); wz[0] *= 0.5; wz[-1] *= 0.5
        wx1 = wx.copy()
        if nx > 1:
            wx1[1] *= 0.5
        wz1 = wz.copy()
        if nz > 1:
            wz1[1] *= 0.5
        for k in range(11):
            cx = wx1 if k in (2, 6, 7) else wx
            cz = wz1 if k in (4, 9, 10) else wz
            S[base + k] = float(np.sum(f[k] * cx[None, :] * cz[:, None]))
    return S, ax, az


def moments_from_sums(S, w: Wfr):
    """Normalisation of the sums into the 11 moments of Ex and of Ez, each rounded to FP32 as the
    reference stores it (sroptelm.cpp:1937-2080, coordinate representation)."""
    lam_d_4pi = 1.239842E-06 / (3.141592653590 * 2. * 2. * w.eStart)
    lam_d_2pi = 2. * lam_d_4pi
    lam_d_2pi_e2 = lam_d_2pi * lam_d_2pi
    inv_sx, inv_sz = 1. / w.xStep, 1. / w.zStep
    scan_x, scan_z = w.nx > 1, w.nz > 1
    out = []
    for b in (0, 11):
        if S[b] == 0.:
            out.append(np.zeros(11))
            continue
        inv_n = 1. / S[b]
        a = inv_n * lam_d_2pi
        ax, az = a * inv_sx, a * inv_sz
        a2 = inv_n * lam_d_2pi_e2
        ax2, az2 = a2 * (inv_sx * inv_sx), a2 * (inv_sz * inv_sz)
        f32 = lambda v: float(np.float32(v))  # noqa: E731
        m = np.array([
            f32(S[b] * (w.xStep * w.zStep * 1.E+06) if (scan_x and scan_z) else 0.),
            f32(S[b + 1] * inv_n if scan_x else w.xStart),
            f32(S[b + 2] * ax if scan_x else 0.),
            f32(S[b + 3] * inv_n if scan_z else w.zStart),
            f32(S[b + 4] * az if scan_z else 0.),
            f32(S[b + 5] * inv_n if scan_x else w.xStart * w.xStart),
            f32(S[b + 6] * ax if scan_x else 0.),
            f32(S[b + 7] * ax2 if scan_x else 0.),
            f32(S[b + 8] * inv_n if scan_z else w.zStart * w.zStart),
            f32(S[b + 9] * az if scan_z else 0.),
            f32(S[b + 10] * az2 if scan_z else 0.)])
        out.append(m)
    return out[0], out[1]


def compute_rad_moments(w: Wfr):
    """srTGenOptElem::ComputeRadMoments (sroptelm.cpp:1608-2092), coordinate representation, ne = 1:
    the quadratic phase of the wavefront radius is removed first (TreatStronglyOscillatingTerm 'r'
    when WaveFrontTermCanBeTreated; re-added after, so only a local copy is changed here), the
    power limits found on the intensity, then the sums normalised into w.momX / w.momZ."""
    if w.nx <= 1 and w.nz <= 1:
        return
    if w.Pres != 0:
        raise NotImplementedError("moments of a wavefront in the angular representation are not restated")
    ex, ey = w.ex, w.ey
    if w.Pres == 0 and _wavefront_term_can_be_treated(w):
        save = (w.ex, w.ey)
        _treat_strongly_oscillating(w, 'r')
        ex, ey = w.ex, w.ey
        w.ex, w.ey = save
    lims = find_intensity_limits_inds(total_intensity(ex, ey), w)
    S, _, _ = moment_sums(ex, ey, w, lims)
    w.momX, w.momZ = moments_from_sums(S, w)


def _lagrange4(t):
    """Cubic Lagrange weights on nodes -1, 0, 1, 2 (the reference's SetupInterpolAux02 /
    InterpolF polynomial, sroptelm.h:560-640, is this interpolant in monomial form)."""
    return np.stack([-t * (t - 1.) * (t - 2.) / 6., (t + 1.) * (t - 1.) * (t - 2.) / 2.,
                     -(t + 1.) * t * (t - 2.) / 2., (t + 1.) * t * (t - 1.) / 6.])


def _resize_core(old: Wfr, new: Wfr, quad_treat):
    """RadResizeCore (sroptelm.cpp:3038-3337) for ne == 1, vectorised over new points.
    Includes the low-order fallback (CheckForLowOrderInterp, sroptelm.h:700-760) and the
    amplitude correction by the interpolated intensity (ImproveReAndIm, sroptelm.h:690)."""
    ixS, ixE, izS, izE = new.AuxLong1, new.AuxLong2, new.AuxLong3, new.AuxLong4
    outx = np.zeros((new.nz, new.nx), np.complex128)
    outy = np.zeros((new.nz, new.nx), np.complex128)
    if ixE < ixS or izE < izS:
        return outx, outy
    ix = np.arange(ixS, ixE + 1)
    iz = np.arange(izS, izE + 1)
    xStepInv, zStepInv = 1. / old.xStep, 1. / old.zStep

    def axis(iv, start_new, step_new, start_old, step_old, inv, n_old):
        a = start_new + iv * step_new
        ic = ((a - start_old) * inv + 1.E-06).astype(np.int64)
        rel = a - (start_old + ic * step_old)
        st = ic - 1
        st = np.where(ic == n_old - 1, ic - 3, st)
        rel = np.where(ic == n_old - 1, rel + 2. * step_old, rel)
        st = np.where(ic == n_old - 2, ic - 2, st)
        rel = np.where(ic == n_old - 2, rel + step_old, rel)
        st = np.where(ic == 0, ic, st)
        rel = np.where(ic == 0, rel - step_old, rel)
        return ic, st, rel * inv
    ixc, ixst, xr = axis(ix, new.xStart, new.xStep, old.xStart, old.xStep, xStepInv, old.nx)
    izc_all, izst_all, zr_all = axis(iz, new.zStart, new.zStep, old.zStart, old.zStep, zStepInv, old.nz)
    CH = max(1, 2 ** 22 // max(1, ix.size))          # rows per chunk (bounded memory)
    for z0 in range(0, iz.size, CH):
        sl = slice(z0, min(iz.size, z0 + CH))
        _resize_rows(old, outx, outy, ix, iz[sl], ixc, ixst, xr, izc_all[sl], izst_all[sl], zr_all[sl], ixS, izS + z0)
    return outx, outy


def _resize_rows(old, outx, outy, ix, iz, ixc, ixst, xr, izc, izst, zr, ixS, izS):
    wx = _lagrange4(xr)          # [4, nX]
    wz = _lagrange4(zr)          # [4, nZ]
    irx = np.clip(ixc - ixst, 0, 2)
    irz = np.clip(izc - izst, 0, 2)
    for src, dst in ((old.ex, outx), (old.ey, outy)):
        blk = np.empty((4, 4, iz.size, ix.size), np.complex128)   # [dz, dx, Z, X]
        for dz in range(4):
            rows = src[izst + dz]
            for dx in range(4):
                blk[dz, dx] = rows[:, ixst + dx]
        re_, im_ = blk.real, blk.imag
        inten = re_ * re_ + im_ * im_
        low = np.any((re_ == 0.) | (im_ == 0.), axis=(0, 1))
        W = wz[:, None, :, None] * wx[None, :, None, :]
        F = np.sum(W * blk, axis=(0, 1))
        FI = np.maximum(np.sum(W * inten, axis=(0, 1)), 0.)
        # low-order (bilinear on the 2x2 sub-cell picked by the clipped relative indices,
        # evaluated with the same xRel/zRel: reproduces the reference also at grid edges)
        X = xr[None, :]
        Z = zr[:, None]
        r0 = irz[:, None] * np.ones_like(irx)[None, :]
        c0 = np.ones_like(irz)[:, None] * irx[None, :]
        Zi = np.arange(iz.size)[:, None] * np.ones(ix.size, np.int64)[None, :]
        Xi = np.ones(iz.size, np.int64)[:, None] * np.arange(ix.size)[None, :]

        def pick(arr, dr, dc):
            return arr[r0 + dr, c0 + dc, Zi, Xi]
        f00, f10, f01, f11 = pick(blk, 0, 0), pick(blk, 0, 1), pick(blk, 1, 0), pick(blk, 1, 1)
        FL = f00 + (f10 - f00) * X + (f01 - f00) * Z + (f00 - f01 - f10 + f11) * X * Z
        i00, i10, i01, i11 = pick(inten, 0, 0), pick(inten, 0, 1), pick(inten, 1, 0), pick(inten, 1, 1)
        FIL = np.maximum(i00 + (i10 - i00) * X + (i01 - i00) * Z + (i00 - i01 - i10 + i11) * X * Z, 0.)
        F = np.where(low, FL, F)
        FI = np.where(low, FIL, FI)
        app = np.abs(F) ** 2
        fac = np.where(app != 0., np.sqrt(np.where(app != 0., FI / np.where(app != 0., app, 1.), 1.)), 1.)
        dst[izS:izS + iz.size, ixS:ixS + ix.size] = F * fac


def _resize_core_only_larger_range(old: Wfr, new: Wfr):
    """RadResizeCore_OnlyLargerRange (sroptelm.cpp:4231-4306)."""
    outx = np.zeros((new.nz, new.nx), np.complex128)
    outy = np.zeros((new.nz, new.nx), np.complex128)
    ixS, ixE, izS, izE = new.AuxLong1, new.AuxLong2, new.AuxLong3, new.AuxLong4
    ix = np.arange(ixS, ixE + 1)
    iz = np.arange(izS, izE + 1)
    xo = ((new.xStart + ix * new.xStep - old.xStart) * (1. / old.xStep) + 1.E-08).astype(np.int64)
    zo = ((new.zStart + iz * new.zStep - old.zStart) * (1. / old.zStep) + 1.E-08).astype(np.int64)
    outx[izS:izE + 1, ixS:ixE + 1] = old.ex[zo][:, xo]
    outy[izS:izE + 1, ixS:ixE + 1] = old.ey[zo][:, xo]
    return outx, outy


def _tune_step_keep_interp_limits(old: Wfr, new: Wfr, pm, axis, ic):
    """TuneStepToKeepInterpLimitsTheSameAtResize (cpp/src/core/sroptel3.cpp:537-623): where the new
    mesh reaches past the old one's first / last node, its step (and start) are tuned so that the
    new nodes land on the old mesh's limits, keeping node ic of the old mesh at the new centre."""
    if axis == 'x':
        nStart, nStep, oStart, oStep, nNp = new.xStart, new.xStep, old.xStart, old.xStep, new.nx
        OldEndInterp = old.xStart + (old.nx - 1) * old.xStep
    else:
        nStart, nStep, oStart, oStep, nNp = new.zStart, new.zStep, old.zStart, old.zStep, new.nz
        OldEndInterp = old.zStart + (old.nz - 1) * old.zStep
    NewEndInterp = nStart + (nNp - 1) * nStep
    left = nStart <= oStart
    right = NewEndInterp >= OldEndInterp
    if not (left or right):
        return
    cArg = oStart + ic * oStep
    half = nNp >> 1
    if left and not right:
        dist = cArg - nStart
        nStep = dist / float(int(dist / nStep + 1.E-10))
        nStart = cArg - half * nStep
    elif right and not left:
        dist = OldEndInterp - cArg
        nStep = dist / float(int(dist / nStep + 1.E-10))
        nStart = cArg - half * nStep
    else:
        OldRange = OldEndInterp - oStart
        if pm != 1.:
            nIn = int(OldRange / nStep + 1.E-10)
            nLeft = int((oStart - nStart) / nStep + 1.E-10)
            nStep = OldRange / float(nIn)
            nStart = oStart - nLeft * nStep
        else:
            nStep = OldRange / float(nNp - 1)
            nStart = oStart
    if axis == 'x':
        new.xStart, new.xStep = nStart, nStep
    else:
        new.zStart, new.zStep = nStart, nStep


def rad_resize_gen(w: Wfr, pxm, pxd, pzm, pzd, shift_type=0, xCenShift=0., zCenShift=0., other_side=False):
    """RadResizeGen (sroptelm.cpp:2242-3036), ne == 1, no per-polarisation memory fallback."""
    if pxm == 1. and pxd == 1. and pzm == 1. and pzd == 1. and shift_type <= 0:
        return
    RelCenPosX = RelCenPosZ = 0.5
    RelCenPosTol = 1.e-06
    if shift_type & 1:
        rxTot = w.xStep * (w.nx - 1)
        rxLeft = xCenShift - w.xStart
        if rxLeft > 0. and xCenShift < (w.xStart + rxTot):
            RelCenPosX = rxLeft / rxTot
    if shift_type & 2:
        rzTot = w.zStep * (w.nz - 1)
        rzLeft = zCenShift - w.zStart
        if rzLeft > 0. and zCenShift < (w.zStart + rzTot):
            RelCenPosZ = rzLeft / rzTot
    nxOld, nzOld = w.nx, w.nz
    xStartOld, zStartOld = w.xStart, w.zStart
    xStepOld, zStepOld = w.xStep, w.zStep
    xRangeOld, zRangeOld = xStepOld * nxOld, zStepOld * nzOld
    useStartTrOther = (abs(xStartOld + 0.5 * xRangeOld) > 0.5 * w.xStep) or (abs(zStartOld + 0.5 * zRangeOld) > 0.5 * w.zStep)
    pxmIn, pxdIn, pzmIn, pzdIn = pxm, pxd, pzm, pzd
    if other_side:
        to = 1 if w.Pres == 0 else 0
        if useStartTrOther:
            w.xStart = -(w.nx >> 1) * w.xStep
            w.zStart = -(w.nz >> 1) * w.zStep
            xs, zs = w.xStart - xStartOld, w.zStart - zStartOld
            w.xWfrMin += xs; w.xWfrMax += xs
            w.zWfrMin += zs; w.zWfrMax += zs
        set_rad_repres(w, to)
        pxm, pxd, pzm, pzd = pxd, pxm, pzd, pzm
    old = w
    new = Wfr(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in w.__dict__.items()})
    pxTot, pzTot = pxm * pxd, pzm * pzd
    NewNx, NewNz = w.nx, w.nz
    changed = (pxTot != 1.) or (pzTot != 1.)
    if changed:
        v = pxTot * NewNx
        iv = int(v)
        NewNx = iv + 1 if (v - iv) >= 0.5 else iv
        v = pzTot * NewNz
        iv = int(v)
        NewNz = iv + 1 if (v - iv) >= 0.5 else iv
        NewNx = next_correct_number_for_fft(NewNx)
        NewNz = next_correct_number_for_fft(NewNz)
        new.nx, new.nz = NewNx, NewNz
    iXc = w.nx >> 1
    centerOffset = False
    if abs(RelCenPosX - 0.5) > RelCenPosTol:
        xcAppr = w.xStart + w.nx * w.xStep * RelCenPosX
        iXc = _int_offset_coord(w.xStart, w.xStep, xcAppr)
        centerOffset = True
    Xc = w.xStart + w.xStep * iXc
    iZc = w.nz >> 1
    if abs(RelCenPosZ - 0.5) > RelCenPosTol:
        zcAppr = w.zStart + w.nz * w.zStep * RelCenPosZ
        iZc = _int_offset_coord(w.zStart, w.zStep, zcAppr)
        centerOffset = True
    Zc = w.zStart + w.zStep * iZc

    def preserve(axis):
        """PreserveLogicsOfWfrLimitsAtRangeResizing (srradstr.cpp:1598)."""
        if axis == 'x':
            tol = 0.01 * new.xStep
            if abs(old.xWfrMin - old.xStart) < tol and abs(old.xStart + old.nx * old.xStep - old.xWfrMax) < tol:
                new.xWfrMin, new.xWfrMax = new.xStart, new.xStart + new.nx * new.xStep
            else:
                new.xWfrMin, new.xWfrMax = old.xWfrMin, old.xWfrMax
        else:
            tol = 0.01 * new.zStep
            if abs(old.zWfrMin - old.zStart) < tol and abs(old.zStart + old.nz * old.zStep - old.zWfrMax) < tol:
                new.zWfrMin, new.zWfrMax = new.zStart, new.zStart + new.nz * new.zStep
            else:
                new.zWfrMin, new.zWfrMax = old.zWfrMin, old.zWfrMax
    if centerOffset:
        # centre of the new mesh at node iXc / iZc of the old one (sroptelm.cpp:2383-2433)
        NewNxLeftHalf = NewNx >> 1
        new.xStep = w.xStep / pxd
        new.xStart = Xc - NewNxLeftHalf * new.xStep
        NewNxEndInterp = new.xStart + (NewNx - 1) * new.xStep
        OldNxEndInterp = w.xStart + (w.nx - 1) * w.xStep
        _tune_step_keep_interp_limits(w, new, pxm, 'x', iXc)
        new.AuxLong1 = _int_offset_coord(new.xStart, new.xStep, w.xStart) if new.xStart < w.xStart else 0
        new.AuxLong2 = _int_offset_coord(new.xStart, new.xStep, OldNxEndInterp) if NewNxEndInterp > OldNxEndInterp \
            else NewNx - 1
        if pxm > 1.:
            preserve('x')
        else:
            if new.xStart > new.xWfrMin:
                new.xWfrMin = new.xStart
            xEndNew = new.xStart + new.nx * new.xStep
            if xEndNew < new.xWfrMax:
                new.xWfrMax = xEndNew
        NewNzLeftHalf = NewNz >> 1
        new.zStep = w.zStep / pzd
        new.zStart = Zc - NewNzLeftHalf * new.zStep
        _tune_step_keep_interp_limits(w, new, pzm, 'z', iZc)
        # (the reference's z branch starts one node later and takes the end limits after the tuning)
        new.AuxLong3 = 1 + _int_offset_coord(new.zStart, new.zStep, w.zStart) if new.zStart < w.zStart else 0
        NewNzEndInterp = new.zStart + (NewNz - 1) * new.zStep
        OldNzEndInterp = w.zStart + (w.nz - 1) * w.zStep
        new.AuxLong4 = _int_offset_coord(new.zStart, new.zStep, OldNzEndInterp) if NewNzEndInterp > OldNzEndInterp \
            else NewNz - 1
        if pzm > 1.:
            preserve('z')
        else:
            if new.zStart > new.zWfrMin:
                new.zWfrMin = new.zStart
            zEndNew = new.zStart + new.nz * new.zStep
            if zEndNew < new.zWfrMax:
                new.zWfrMax = zEndNew
    else:
        xMagOld = (w.nx - 1) * w.xStep
        if pxm > 1.:
            NxInner = int(NewNx / pxm) if pxd != 1. else w.nx
            d = NewNx - NxInner
            left = d >> 1
            if (left << 1) != d:
                left += 1
            new.xStep = xMagOld / (NxInner - 1)
            new.xStart = w.xStart - left * new.xStep
            new.AuxLong1 = left
            new.AuxLong2 = left + NxInner - 1
            preserve('x')
        else:
            xEndOld = w.xStart + (w.nx - 1) * w.xStep
            xMid = 0.5 * (w.xStart + xEndOld)
            xMagNew = xMagOld * pxm
            new.xStep = xMagNew / (NewNx - 1)
            if pxd == 1:
                new.xStep = w.xStep
                xMagNew = (NewNx - 1) * new.xStep
            new.xStart = xMid - 0.5 * xMagNew
            new.AuxLong1 = 0
            new.AuxLong2 = NewNx - 1
            if new.xStart > new.xWfrMin:
                new.xWfrMin = new.xStart
            if (new.xStart + xMagNew) < new.xWfrMax:
                new.xWfrMax = new.xStart + xMagNew
        zMagOld = (w.nz - 1) * w.zStep
        if pzm > 1.:
            NzInner = int(NewNz / pzm) if pzd != 1. else w.nz
            d = NewNz - NzInner
            left = d >> 1
            if (left << 1) != d:
                left += 1
            new.zStep = zMagOld / (NzInner - 1)
            new.zStart = w.zStart - left * new.zStep
            new.AuxLong3 = left
            new.AuxLong4 = left + NzInner - 1
            preserve('z')
        else:
            zEndOld = w.zStart + (w.nz - 1) * w.zStep
            zMid = 0.5 * (w.zStart + zEndOld)
            zMagNew = zMagOld * pzm
            new.zStep = zMagNew / (NewNz - 1)
            if pzd == 1:
                new.zStep = w.zStep
                zMagNew = (NewNz - 1) * new.zStep
            new.zStart = zMid - 0.5 * zMagNew
            new.AuxLong3 = 0
            new.AuxLong4 = NewNz - 1
            if new.zStart > new.zWfrMin:
                new.zWfrMin = new.zStart
            if (new.zStart + zMagNew) < new.zWfrMax:
                new.zWfrMax = new.zStart + zMagNew


    grow = (pxmIn * pxdIn * pzmIn * pzdIn) >= 1.
    if grow and changed:
        new.srwl_roundtrip()                         # ModifyWfrNeNxNz before the core
    # RadResizeCore (sroptelm.cpp:3038)
    RelStepTol = 1.e-05
    only_larger = (pxd == 1. and pzd == 1. and pxm >= 1. and pzm >= 1.) and \
        (abs(old.xStep - new.xStep) < RelStepTol and abs(old.zStep - new.zStep) < RelStepTol)
    if only_larger:
        ex, ey = _resize_core_only_larger_range(old, new)
    else:
        treated = False
        origQX, origQZ = old.QuadX, old.QuadZ
        if _wavefront_term_can_be_treated(old) and old.Pres < 1:
            new.QuadX, new.QuadZ = old.QuadX, old.QuadZ
            _treat_strongly_oscillating(old, 'r')
            treated = True
        ex, ey = _resize_core(old, new, treated)
        new.ex, new.ey = ex, ey
        if treated:
            _treat_strongly_oscillating(new, 'a')
            ex, ey = new.ex, new.ey
        new.QuadX, new.QuadZ = origQX, origQZ
    new.ex, new.ey = ex, ey
    if (not grow) and changed:
        new.srwl_roundtrip()                         # ModifyWfrNeNxNz after the core
    for k, v in new.__dict__.items():
        setattr(w, k, v)
    if other_side:
        to = 1 if w.Pres == 0 else 0
        set_rad_repres(w, to)
        if useStartTrOther:
            xcOld = xStartOld + (nxOld >> 1) * xStepOld
            w.xStart = xcOld - (w.nx >> 1) * w.xStep
            zcOld = zStartOld + (nzOld >> 1) * zStepOld
            w.zStart = zcOld - (w.nz >> 1) * w.zStep
            w.set_full_range()


# ----------------------------------------------------------------------------------------
# Container (srTCompositeOptElem, cpp/src/core/sroptcnt.cpp:87-425)
# ----------------------------------------------------------------------------------------


def _pp(pp, i, default):
    return pp[i] if (pp is not None and len(pp) > i) else default


def _element(w: Wfr, el, anal):
    """One element of a chain; a nested container ('container', elements, props) propagates every
    element inside it (nested containers included) with the outer entry's treatment, its own
    parameter lists unused (srTCompositeOptElem::PropagateRadiation, sroptcnt.h:52-76)."""
    kind = el[0]
    if kind == 'drift':
        drift(w, el[1], el[2], anal)
    elif kind == 'lens':
        lens(w, el[1], el[2], el[3], el[4])
    elif kind == 'aperture':
        aperture(w, el[1], el[2], el[3], el[4], el[5], el[6])
    elif kind == 'transmission':
        transmission(w, *el[1:])
    elif kind == 'container':
        for sub in el[1]:
            _element(w, tuple(sub), anal)
    else:
        raise ValueError("UNKNOWN_OPTICAL_ELEMENT")


def propagate(w: Wfr, elements, props, after=None):
    """srTCompositeOptElem ctor (sroptcnt.cpp:87-221) + PropagateRadiationGuided (:254-425).

    ``elements``: list of tuples ('drift', L, treat) | ('aperture', shape, ap_or_ob, Dx, Dy, x, y)
    | ('lens', Fx, Fy, x, y) | ('transmission', arTr, nx, ny, rx, ry, x, y, extTr, Fx, Fy)
    | ('container', elements, props).
    ``props``: list of per-element propagation parameter lists
    (len(props) may be len(elements)+1 for a post-resize).  ``after(k, w)``, when given, sees the
    wavefront after element k and, with k = len(elements), after the post-resize: the points where
    PropagateRadiationGuided extracts intensities (sroptcnt.cpp:398, :421)."""
    if (w.nx <= 1) or (w.nz <= 1):
        raise ValueError("CAN_NOT_PROPAGATE_1D_RAD")
    tolRes = 1.e-04
    for i, el in enumerate(elements):
        pp = props[i] if i < len(props) else None
        anal = 0
        if pp is not None:
            if int(_pp(pp, 0, 0)) or int(_pp(pp, 1, 0)):
                raise NotImplementedError("auto-resize (pp[0]/pp[1]) is not restated")
            anal = int(_pp(pp, 3, 0))
            pxm, pxd, pzm, pzd = _pp(pp, 5, 1.), _pp(pp, 6, 1.), _pp(pp, 7, 1.), _pp(pp, 8, 1.)
            shift = int(_pp(pp, 9, 0))
            if abs(pxd - 1.) > tolRes or abs(pxm - 1.) > tolRes or abs(pzd - 1.) > tolRes or \
                    abs(pzm - 1.) > tolRes or shift > 0:
                rad_resize_gen(w, pxm, pxd, pzm, pzd, shift, _pp(pp, 10, 0.), _pp(pp, 11, 0.),
                               other_side=bool(int(_pp(pp, 4, 0))))
        _element(w, el, anal)
        if after is not None:
            after(i, w)
    n = len(elements)
    if n < len(props):
        pp = props[n]
        pxm, pxd, pzm, pzd = _pp(pp, 5, 1.), _pp(pp, 6, 1.), _pp(pp, 7, 1.), _pp(pp, 8, 1.)
        if abs(pxd - 1.) > tolRes or abs(pxm - 1.) > tolRes or abs(pzd - 1.) > tolRes or abs(pzm - 1.) > tolRes:
            rad_resize_gen(w, pxm, pxd, pzm, pzd, other_side=bool(int(_pp(pp, 4, 0))))
        if after is not None:
            after(n, w)
    return w


# ----------------------------------------------------------------------------------------
# Multi-electron loop pieces (srwl_wfr_emit_prop_multi_e, env/python/srwpy/srwlib.py:8506)
# ----------------------------------------------------------------------------------------


def electron_offset(ex, ey, mesh, sc, dx0, dxp, dy0, dyp, de=0.):
    """SRWLWfr.sim_src_offset with _move_mesh=True (env/python/srwpy/srwlib.py:2803-2849): the kick
    of srTOptAngle::RadPointModifier (cpp/src/core/sroptang.h:64-79; phase 5.06773065e6 e (x' x + y' z)
    in FP64 on the unshifted mesh, field stored back as FP32), then the mesh moved by
    (x + x' R, y + y' R), R = (Rx + Ry)/2, and xc += x, yc += y.  Returns (ex, ey, mesh, sc)."""
    ny, nx = ex.shape
    if de != 0.:        # photon energy of the electron's wavefront: E (1 + 2 de) (undulator harmonic shift)
        mesh = dict(mesh)
        mesh['eStart'] = mesh['eStart'] * (1. + 2. * de)
        mesh['eFin'] = mesh['eStart']
    xStep = (mesh['xFin'] - mesh['xStart']) / (nx - 1)
    zStep = (mesh['yFin'] - mesh['yStart']) / (ny - 1)
    x = mesh['xStart'] + np.arange(nx) * xStep
    z = mesh['yStart'] + np.arange(ny) * zStep
    ph = 5.06773065e+06 * mesh['eStart'] * (dxp * x[None, :] + dyp * z[:, None])
    f = np.exp(1j * ph)
    ex2 = (np.asarray(ex, np.complex128) * f).astype(np.complex64).astype(np.complex128)
    ey2 = (np.asarray(ey, np.complex128) * f).astype(np.complex64).astype(np.complex128)
    R = 0.5 * (sc['Rx'] + sc['Ry'])
    dx, dy = dx0 + dxp * R, dy0 + dyp * R
    m2 = dict(mesh)
    m2['xStart'] += dx
    m2['xFin'] += dx
    m2['yStart'] += dy
    m2['yFin'] += dy
    sc2 = dict(sc)
    sc2['xc'] = sc.get('xc', 0.) + dx0
    sc2['yc'] = sc.get('yc', 0.) + dy0
    return ex2, ey2, m2, sc2


def total_intensity(ex, ey):
    """srwlCalcIntFromElecField, single-electron intensity, polarisation 6 (total), vs x and y
    (cpp/src/core/srradmnp.cpp:681): |Ex|^2 + |Ey|^2 stored as FP32."""
    ex = np.asarray(ex, np.complex64)
    ey = np.asarray(ey, np.complex64)
    return (ex.real * ex.real + ex.imag * ex.imag + ey.real * ey.real + ey.imag * ey.imag).astype(np.float32)


def _hermite(n, x):
    """srTGsnBeam::HermitePolynomial (srgsnbm.cpp:97): physicists' Hermite polynomial by recursion."""
    if n == 0:
        return np.ones_like(x)
    if n == 1:
        return 2. * x
    return 2. * (x * _hermite(n - 1, x) - (n - 1) * _hermite(n - 2, x))


def calc_elec_field_gaussian(mesh, gb, unit_el_fld=1, part_z=0.):
    """srwlCalcElecFieldGaussian (cpp/src/lib/srwlib.cpp:544) for a single photon energy without
    automatic sampling (precPar[0] = 0): srTGsnBeam (srgsnbm.cpp:15-78), its frequency-domain field
    (CreateWavefrontElFieldFreqDomain, :230-310, SetupSourceConstantsFreqDomain :104-126,
    SetupProperPolariz srgsnbm.h:74), the wavefront scalars of AuxSetupActionsArbSrc
    (srradstr.cpp:324-349) and the moments (ComputeRadMoments of the FP32 field).  ``gb``: dict with
    the SRWLGsnBm fields.  Returns the Wfr (FP32-rounded field) and the 20 entries of the 4x4
    propagation matrix block InitialSetupOf4x4PropMatr writes (srradstr.h:399)."""
    Pi = 3.1415926535898
    sqrt_2 = math.sqrt(2.)
    SigmaX, SigmaZ = gb['sigX'] * sqrt_2, gb['sigY'] * sqrt_2
    mx, mz = int(gb['mx']), int(gb['my'])
    SigmaPhotEn = (0.5 * 6.58211889E-16 / gb['sigT']) * sqrt_2 if gb['sigT'] > 0 else 1.e+23
    PhotPerBW = -1.
    if gb['pulseEn'] > 0 and gb['sigT'] > 0:
        PhotPerBW = 6.2415096E+15 * gb['pulseEn'] / (math.sqrt(Pi) * SigmaPhotEn)
        if gb['repRate'] > 0:
            PhotPerBW *= gb['repRate']
    AuxConst = float(1 << (mx + mz)) * math.factorial(mx) * math.factorial(mz)
    NormConst = math.sqrt(PhotPerBW / (AuxConst * ((1.E+06) * Pi)))
    if unit_el_fld == 2:
        NormConst *= math.sqrt(1.602176462e-16)
    x0, dxds0, z0, dzds0, s0 = gb['x'], gb['xp'], gb['y'], gb['yp'], gb['z']
    PhEnConv = 1.239842E-06
    en = mesh['eStart']
    Robs = mesh['zStart'] - s0
    LongDist = Robs
    if LongDist == 0.:
        LongDist = 0.01 * (PhEnConv / en)
    InvTwoSigXe2, InvTwoSigZe2 = 0.5 / (SigmaX * SigmaX), 0.5 / (SigmaZ * SigmaZ)
    InvTwoSigPhotEnE2 = 0.5 / (SigmaPhotEn * SigmaPhotEn)
    Buf = (Pi * 1.) / (PhEnConv * LongDist)
    PropagMultX, PropagMultZ = Buf / InvTwoSigXe2, Buf / InvTwoSigZe2
    x0Prop, z0Prop = x0 + dxds0 * LongDist, z0 + dzds0 * LongDist
    nx, ny = int(mesh['nx']), int(mesh['ny'])
    xStep = (mesh['xFin'] - mesh['xStart']) / (nx - 1)
    zStep = (mesh['yFin'] - mesh['yStart']) / (ny - 1)
    ix = np.arange(nx)[None, :]
    iz = np.arange(ny)[:, None]
    x = (mesh['xStart'] - x0Prop) + ix * xStep
    z = (mesh['yStart'] - z0Prop) + iz * zStep
    x_mi_x0 = (mesh['xStart'] - x0) + ix * xStep
    z_mi_z0 = (mesh['yStart'] - z0) + iz * zStep
    xx, zz = x_mi_x0 + x0, z_mi_z0 + z0
    enMult = 2.53384080189E+06
    InvLongDist = 1. / LongDist
    PropRatX, PropRatZ = en * PropagMultX, en * PropagMultZ
    InvPropRatX, InvPropRatZ = 1. / PropRatX, 1. / PropRatZ
    SigMultX, SigMultZ = 1. + InvPropRatX * InvPropRatX, 1. + InvPropRatZ * InvPropRatZ
    DisMultX, DisMultZ = 1. + PropRatX * PropRatX, 1. + PropRatZ * PropRatZ
    PropInvTwoSigXe2, PropInvTwoSigZe2 = InvTwoSigXe2 / SigMultX, InvTwoSigZe2 / SigMultZ
    PropInvSigX, PropInvSigZ = math.sqrt(2. * PropInvTwoSigXe2), math.sqrt(2. * PropInvTwoSigZe2)
    PropInvRx, PropInvRz = InvLongDist / DisMultX, InvLongDist / DisMultZ
    xpMult = (1. / PropInvRx - LongDist) * dxds0
    zpMult = (1. / PropInvRz - LongDist) * dzds0
    NuX, NuZ = math.atan(InvPropRatX), math.atan(InvPropRatZ)
    Phase = en * enMult * ((x_mi_x0 * x_mi_x0 + 2 * LongDist * x0 * dxds0 + xpMult * (2 * xx - LongDist * dxds0)) * PropInvRx
                           + (z_mi_z0 * z_mi_z0 + 2 * LongDist * z0 * dzds0 + zpMult * (2 * zz - LongDist * dzds0)) * PropInvRz) \
        + (mx + 0.5) * NuX + (mz + 0.5) * NuZ
    TwoPI = 6.28318530717959
    Phase = Phase - TwoPI * np.trunc(Phase * (1. / TwoPI))
    arg = -(x * x) * PropInvTwoSigXe2 - (z * z) * PropInvTwoSigZe2
    if gb['avgPhotEn'] > 0:
        d = en - gb['avgPhotEn']
        arg = arg - d * d * InvTwoSigPhotEnE2
    BufA = NormConst * math.sqrt(PropInvSigX * PropInvSigZ) * np.exp(arg) * _hermite(mx, x * PropInvSigX) * \
        _hermite(mz, z * PropInvSigZ)
    ReA, ImA = BufA * np.cos(Phase), BufA * np.sin(Phase)
    c = 0.70710678118655
    zero = np.zeros_like(ReA)
    pol = int(gb['polar'])
    comps = {1: (ReA, ImA, zero, zero), 2: (zero, zero, ReA, ImA), 3: (c * ReA, c * ImA, c * ReA, c * ImA),
             4: (c * ReA, c * ImA, -c * ReA, -c * ImA), 5: (c * ReA, c * ImA, -c * ImA, c * ReA),
             6: (c * ReA, c * ImA, c * ImA, -c * ReA)}[pol]
    f32 = [np.asarray(v, np.float32) for v in comps]
    ex = (f32[0] + 1j * f32[1]).astype(np.complex64)
    ey = (f32[2] + 1j * f32[3]).astype(np.complex64)
    w = Wfr.from_srwl(ex, ey, mesh, Robs, Robs, 0.01 * abs(Robs), 0.01 * abs(Robs), x0, z0)
    compute_rad_moments(w)
    d = mesh['zStart'] - part_z
    prop = np.zeros(16)
    prop[[0, 5, 10, 15]] = 1.
    prop[1] = prop[11] = d
    return w, prop


def _formal_phase(re, im):
    """FormalPhase (srradmnp.h:434): the argument of re + i im from atan of the FP32 ratio, in the
    quadrant of (re, im) (-pi - ... pi, the reference's branch conventions and pi constants)."""
    re = np.asarray(re, np.float32)
    im = np.asarray(im, np.float32)
    with np.errstate(divide='ignore', invalid='ignore'):
        a = np.arctan((im / re).astype(np.float64))
    HalhPi, Pi = 1.5707963267949, 3.1415926535898
    out = np.where(re != 0, np.where(re < 0, np.where(im <= 0, a - Pi, a + Pi), a),
                   np.where(im == 0, 0., np.where(im > 0, HalhPi, -HalhPi)))
    return out


def intensity_component(ex, ey, pol, what):
    """srTRadGenManip::IntensityComponent (srradmnp.h:367-425) over whole arrays with its FP32 / FP64
    operation order.  what: 0 intensity, 2 phase (FP64 result), 3 Re E, 6 Im E (the reference's
    internal numbering); pol 0 linear horizontal, 1 vertical, 2 +45 deg, 3 135 deg, 4 circular right,
    5 circular left, 6 total; -1..-4 the Stokes components."""
    f32 = np.float32
    exr, exi = np.real(ex).astype(f32), np.imag(ex).astype(f32)
    eyr, eyi = np.real(ey).astype(f32), np.imag(ey).astype(f32)
    if pol == -1:
        return (exr * exr + exi * exi + eyr * eyr + eyi * eyi).astype(f32)
    if pol == -2:
        return (exr * exr + exi * exi - (eyr * eyr + eyi * eyi)).astype(f32)
    if pol == -3:
        return (2. * (exr * eyr + exi * eyi).astype(np.float64)).astype(f32)
    if pol == -4:
        return (2. * (exr * eyi - exi * eyr).astype(np.float64)).astype(f32)
    half = False
    if pol == 0:
        a, b = exr, exi
    elif pol == 1:
        a, b = eyr, eyi
    elif pol == 2:
        a, b, half = exr + eyr, exi + eyi, True
    elif pol == 3:
        a, b, half = exr - eyr, exi - eyi, True
    elif pol == 5:
        a, b, half = exr - eyi, exi + eyr, True
    elif pol == 4:
        a, b, half = exr + eyi, exi - eyr, True
    else:
        if what in (0, 1):
            return (exr * exr + exi * exi + eyr * eyr + eyi * eyi).astype(f32)
        if what == 2:
            return _formal_phase(exr, exi).astype(np.float32).astype(np.float64)
        return exr if what == 3 else exi
    if what in (0, 1):
        v = (a * a + b * b).astype(f32)
        return (0.5 * v.astype(np.float64)).astype(f32) if half else v
    if what == 2:       # IntensityComponent returns FP32: the phase too is rounded to FP32
        return _formal_phase(a, b).astype(np.float32).astype(np.float64)
    v = a if what == 3 else b
    return (0.70710678 * v.astype(np.float64)).astype(f32) if half else v


def calc_int_from_elec_field(ex, ey, pol, int_type, meth=None, prev=None):
    """srwlCalcIntFromElecField (cpp/src/lib/srwlib.cpp:757) for a single photon energy, vs x and y
    (ExtractSingleElecIntensity2DvsXZ, srradmnp.cpp:681): int_type 0 single-electron intensity, 4 phase
    (FP64), 5 Re E, 6 Im E; pol -5 gives the four Stokes components one after the other.  meth[0] = 1
    averages into prev over meth[1] earlier iterations, 2 adds to prev."""
    what = {0: 0, 4: 2, 5: 3, 6: 6}[int_type]
    pols = [-1, -2, -3, -4] if pol == -5 else [pol]
    res = [np.asarray(intensity_component(ex, ey, p, what)).ravel() for p in pols]
    res = np.concatenate(res)
    mode = 0 if meth is None else int(meth[0])
    if mode == 0 or prev is None:
        return res
    if what == 2:
        prev = np.asarray(prev, np.float64)
        if mode == 1:
            it = float(meth[1])
            return (prev * it + res) * (1. / (it + 1.))
        return prev + res
    prev = np.asarray(prev, np.float32)
    if mode == 1:
        it = float(meth[1])
        return ((prev.astype(np.float64) * it + res.astype(np.float64)) * (1. / (it + 1.))).astype(np.float32)
    return (prev + res).astype(np.float32)


def _setup_int_coord(start, step, n, arg):
    """SetupIntCoord (srradmnp.cpp:35): node below arg (truncation toward zero), the next node, and
    the relative distance from the first, clamped to the mesh ends."""
    if n <= 1:
        return 0, 0, 0.
    inv = 1. / step
    i0 = int((arg - start) * inv)
    if i0 < 0:
        i0 = i1 = 0
    elif i0 >= n - 1:
        i0 = i1 = n - 1
    else:
        i1 = i0 + 1
    return i0, i1, inv * (arg - i0 * step - start)


def calc_int_cut(ex, ey, mesh, pol, int_type, dep, x, y):
    """srwlCalcIntFromElecField for ne == 1 vs x at y (dep 1), vs y at x (dep 2) or at the point (x, y)
    (dep 0): ExtractSingleElecIntensity1DvsX / 1DvsZ / 1DvsE (srradmnp.cpp:224-680), each value
    IntensityComponentSimpleInterpol2D (srradmnp.h:353) of the four corners around it, FP32
    differences and FP64 weights; the phase takes the first corner."""
    f32, f64 = np.float32, np.float64
    what = {0: 0, 4: 2, 5: 3, 6: 6}[int_type]
    nz, nx = ex.shape
    xStep = (mesh['xFin'] - mesh['xStart']) / (nx - 1) if nx > 1 else 0.
    zStep = (mesh['yFin'] - mesh['yStart']) / (nz - 1) if nz > 1 else 0.
    x0, x1, ax = _setup_int_coord(mesh['xStart'], xStep, nx, x)
    z0, z1, az = _setup_int_coord(mesh['yStart'], zStep, nz, y)
    out = []
    for p in ([-1, -2, -3, -4] if pol == -5 else [pol]):
        I = np.asarray(intensity_component(ex, ey, p, what))
        if dep == 0:
            c = (I[z0, x0], I[z0, x1], I[z1, x0], I[z1, x1])
            a1, a2 = ax, az
        elif dep == 1:
            c = (I[z0, :], I[z0, :], I[z1, :], I[z1, :])
            a1, a2 = 0., az
        else:
            c = (I[:, x0], I[:, x0], I[:, x1], I[:, x1])
            a1, a2 = 0., ax
        I00, I10, I01, I11 = [np.atleast_1d(v) for v in c]
        if what == 2:
            out.append(I00.astype(f64))
            continue
        I00, I10, I01, I11 = [v.astype(f32) for v in (I00, I10, I01, I11)]
        t = ((I00 - I01) - I10) + I11
        r = t.astype(f64) * (a1 * a2) + (I10 - I00).astype(f64) * a1 + (I01 - I00).astype(f64) * a2 + I00.astype(f64)
        out.append(r.astype(f32))
    return np.concatenate(out)


def add_interp_bilinear(acc, acc_mesh, I, mesh):
    """acc += I interpolated on acc_mesh: SRWLStokes.avg_update_interp with _ord=1 and _sum=True
    (env/python/srwpy/srwlib.py:1116-1203; points outside the mesh add nothing)."""
    anx, any_ = acc_mesh['nx'], acc_mesh['ny']
    axs = (acc_mesh['xFin'] - acc_mesh['xStart']) / (anx - 1)
    ays = (acc_mesh['yFin'] - acc_mesh['yStart']) / (any_ - 1)
    ny, nx = I.shape
    xs = (mesh['xFin'] - mesh['xStart']) / (nx - 1)
    ys = (mesh['yFin'] - mesh['yStart']) / (ny - 1)
    xa = acc_mesh['xStart'] + np.arange(anx) * axs
    ya = acc_mesh['yStart'] + np.arange(any_) * ays
    ix0 = np.trunc((xa - mesh['xStart']) / xs + 1.e-09).astype(np.int64)
    iy0 = np.trunc((ya - mesh['yStart']) / ys + 1.e-09).astype(np.int64)
    okx = (ix0 >= 0) & (ix0 < nx - 1)
    oky = (iy0 >= 0) & (iy0 < ny - 1)
    ix0c = np.clip(ix0, 0, nx - 2)
    iy0c = np.clip(iy0, 0, ny - 2)
    tx = (xa - (mesh['xStart'] + xs * ix0c)) / xs
    ty = (ya - (mesh['yStart'] + ys * iy0c)) / ys
    I = np.asarray(I, np.float64)
    a00 = I[iy0c[:, None], ix0c[None, :]]
    f10 = I[iy0c[:, None], ix0c[None, :] + 1]
    f01 = I[iy0c[:, None] + 1, ix0c[None, :]]
    f11 = I[iy0c[:, None] + 1, ix0c[None, :] + 1]
    a10, a01, a11 = f10 - a00, f01 - a00, a00 - f01 - f10 + f11
    TX, TY = tx[None, :], ty[:, None]
    f = a00 + TX * (a10 + TY * a11) + TY * a01
    acc += np.where(oky[:, None] & okx[None, :], f, 0.)
    return acc
