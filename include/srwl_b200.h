/*
 * srwl_b200: B200-native (sm_100a) implementation of SRW's Fourier-optics wavefront
 * propagation -- srwlPropagElecField over SRWLOptC chains of drifts, thin lenses and
 * apertures/obstacles -- behind the reference's own C API.
 *
 * The structures below are declared with the same members, order and types as the reference's
 * public header (cpp/src/lib/srwlib.h:75-94, 239-276, 302-327, 523-531), so a C client compiled
 * against the reference header can link this library instead (the binary layouts agree).
 * Only the members this path reads or writes are documented.
 *
 * Error convention (srwlib.h): 0 = success, > 0 error number, < 0 warning number.  Error
 * numbers of the reference are kept; numbers >= 23900 are specific to this library.
 */
#ifndef SRWL_B200_H
#define SRWL_B200_H

#if defined(__GNUC__)
#define SRWG_API __attribute__((visibility("default")))
#else
#define SRWG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

struct SRWLStructParticle {
    double x, y, z;
    double xp, yp;
    double gamma;
    double relE0;
    int nq;
};
typedef struct SRWLStructParticle SRWLParticle;

struct SRWLStructParticleBeam {
    double Iavg;
    double nPart;
    SRWLParticle partStatMom1;
    double arStatMom2[21];
};
typedef struct SRWLStructParticleBeam SRWLPartBeam;

/* SRWLGsnBm (srwlib.h:211-222): a (Hermite-)Gaussian beam at its waist */
struct SRWLStructGaussianBeam {
    double x, y, z;
    double xp, yp;
    double avgPhotEn;
    double pulseEn;
    double repRate;
    char polar;
    double sigX, sigY;
    double sigT;
    char mx, my;
};
typedef struct SRWLStructGaussianBeam SRWLGsnBm;

struct SRWLStructRadMesh {
    double eStart, eFin, xStart, xFin, yStart, yFin, zStart;
    long ne, nx, ny;
    double nvx, nvy, nvz, hvx, hvy, hvz;
    double* arSurf;
    char type;
    long long itStart, itFin;
};
typedef struct SRWLStructRadMesh SRWLRadMesh;

struct SRWLStructWaveFront {
    char *arEx, *arEy;           /* float32 [ny][nx][ne][re,im] each, host memory */
    char *arExAux, *arEyAux;
    SRWLRadMesh mesh;
    double Rx, Ry;               /* instant wavefront radii */
    double dRx, dRy;             /* their errors */
    double xc, yc;               /* instant source centre */
    double avgPhotEn;
    char presCA;                 /* 0 coordinate, 1 angular representation */
    char presFT;
    char numTypeElFld;           /* 'f' */
    char unitElFld;
    char unitElFldAng;
    SRWLPartBeam partBeam;
    double* arElecPropMatr;
    double *arMomX, *arMomY;     /* 11*ne statistical moments per component */
    double* arWfrAuxData;
};
typedef struct SRWLStructWaveFront SRWLWfr;

struct SRWLStructOpticsDrift {
    double L;
    char treat;
};
typedef struct SRWLStructOpticsDrift SRWLOptD;

struct SRWLStructOpticsAperture {
    char shape;                  /* 'r' rectangular, 'c' circular */
    char ap_or_ob;               /* 'a' aperture, 'o' obstacle */
    double Dx, Dy;
    double x, y;
};
typedef struct SRWLStructOpticsAperture SRWLOptA;

struct SRWLStructOpticsLens {
    double Fx, Fy;
    double x, y;
};
typedef struct SRWLStructOpticsLens SRWLOptL;

/* SRWLOptT (srwlib.h:378-389): generic transmission; arTr holds (amplitude transmission, optical path
 * difference [m]) pairs of doubles, [ny][nx] for ne == 1 */
struct SRWLStructOpticsTransmission {
    double* arTr;
    SRWLRadMesh mesh;
    char extTr;
    double Fx, Fy;
};
typedef struct SRWLStructOpticsTransmission SRWLOptT;

struct SRWLStructOpticsContainer {
    void** arOpt;                /* element pointers */
    char** arOptTypes;           /* "drift", "aperture", "obstacle", "lens", "transmission", "container" */
    int nElem;
    double** arProp;             /* per-element propagation parameter lists */
    char* arPropN;               /* their lengths (9..17) */
    int nProp;                   /* nElem or nElem+1 (post-resize) */
};
typedef struct SRWLStructOpticsContainer SRWLOptC;

/* ---------------------------------------------------------------------------------------------
 * Reference C API entry points (same signatures and semantics)
 * ------------------------------------------------------------------------------------------- */

/* Replaces srwlPropagElecField (cpp/src/lib/srwlib.h:821, srwlib.cpp:1023).  Propagates the
 * wavefront in place through the optical container on the GPU (arParGPU = {nPar, device index
 * (1-based)} or NULL for device 0).  Field arrays are host memory owned by the caller; when the
 * mesh size changes the registered modification callback is called (action 2) to re-allocate
 * them before the result is written back.  nInt > 0 with arID / arI: intensities extracted after
 * the elements arID[0][i] (1-based; nElem + 1: after the post-resize) as the reference does
 * (srTCompositeOptElem::ExtractPropagatedIntensity, sroptcnt.cpp:429): polarisation arID[1][i],
 * intensity type arID[2][i] (0 single-electron intensity, 4 phase, 5 Re E, 6 Im E), dependence
 * arID[3][i] = 3 (vs x and y), representation arID[4][i] = 0; written to arI[i] (allocated with the
 * function registered by srwlUtiSetAllocArrayFunc when NULL), their meshes to arIM[i].  Other
 * extraction kinds return error 23900.  Not thread-safe, like the reference. */
SRWG_API int srwlPropagElecField(SRWLWfr* pWfr, SRWLOptC* pOpt, int nInt, char** arID, SRWLRadMesh* arIM, char** arI,
                        double* arParGPU);

/* Replaces srwlCalcElecFieldGaussian (cpp/src/lib/srwlib.h, srwlib.cpp:544) for a single photon energy
 * without automatic sampling (precPar NULL or precPar[0] = 0): fills arEx / arEy (host memory, the
 * wavefront's mesh) with the field computed on the GPU, and sets Rx, Ry, dRx, dRy, xc, yc, the
 * moments (recomputed from the field) and the 4x4 matrix block of arElecPropMatr as the reference
 * does.  Automatic sampling and time-domain wavefronts return error 23900. */
SRWG_API int srwlCalcElecFieldGaussian(SRWLWfr* pWfr, SRWLGsnBm* pGsnBm, double* precPar);

/* Replaces srwlCalcIntFromElecField (cpp/src/lib/srwlib.h:748, srwlib.cpp:757) for wavefronts at a
 * single photon energy (ne == 1) vs x and y (depType 3), vs x at y (1), vs y at x (2) or at the point
 * (x, y) (0; the cuts and the point interpolated between the neighbouring nodes as the reference's
 * 1D extractions do): intType 0 (single-electron intensity), 4 (phase; pInt holds doubles), 5 (Re E),
 * 6 (Im E); pol 0..6 and the Stokes components -1..-4 (-5: all four, one array after the other,
 * intensity only).  Vs x and y, arMeth[0] = 1 averages into pInt with arMeth[1] earlier iterations, 2
 * adds to it; NULL writes it.  Computed on the GPU (arParGPU as for srwlPropagElecField); other
 * intensity types, dependences and pFldTrj return error 23900. */
SRWG_API int srwlCalcIntFromElecField(char* pInt, SRWLWfr* pWfr, char pol, char intType, char depType, double e,
                                      double x, double y, double* arMeth, void* pFldTrj, double* arParGPU);

/* Replaces srwlUtiSetWfrModifFunc (srwlib.h:542): registers the client callback that
 * re-allocates wavefront arrays (action 2: allocate for the current mesh; 12: with backup). */
SRWG_API void srwlUtiSetWfrModifFunc(int (*pExtFunc)(int action, SRWLWfr* pWfrIn, char pol));

/* Replaces srwlUtiSetAllocArrayFunc (srwlib.h:549): registers the client function that allocates the
 * arrays of intensities extracted during srwlPropagElecField ('f' or 'd', len points) when the caller
 * passes arI[i] == NULL. */
SRWG_API void srwlUtiSetAllocArrayFunc(char* (*pExtFunc)(char type, long long len));

/* Replaces srwlUtiGetErrText (srwlib.h:574): copies the text of error/warning number erNo to t
 * (at least 2048 bytes). */
SRWG_API int srwlUtiGetErrText(char* t, int erNo);

/* ---------------------------------------------------------------------------------------------
 * Extensions (no counterpart in the reference): plan once, execute on device-resident fields.
 * ------------------------------------------------------------------------------------------- */

typedef struct srwgPlan srwgPlan;

/* Plans the propagation of a wavefront with pWfr's mesh and scalars (arrays are not read)
 * through pOpt on device `device` (0-based): runs the reference's mesh/radius bookkeeping on
 * the host and lowers the element chain into fused GPU passes. */
SRWG_API int srwgPlanCreate(const SRWLWfr* pWfr, const SRWLOptC* pOpt, int device, srwgPlan** ppPlan);

/* Writes the output mesh and scalars (Rx, Ry, dRx, dRy, xc, yc, presCA, moments when arMomX/Y
 * are non-NULL) of the planned propagation into pWfrOut; field arrays are not touched.  Where
 * the propagation recomputes the statistical moments from the field (an aperture that clips the
 * beam, an obstacle: srTAperture::PropagateRadMoments, sroptapt.cpp:248), the moments are those
 * of wavefront 0 of the last execution (the call waits for it); before any execution they are
 * the analytically propagated ones. */
SRWG_API int srwgPlanGetOutput(const srwgPlan* plan, SRWLWfr* pWfrOut);

/* The 11 + 11 output moments (arMomX / arMomY layout) of wavefront `index` of the last execution
 * (waits for it); for plans without a moment recomputation the analytically propagated ones. */
SRWG_API int srwgPlanGetMoments(const srwgPlan* plan, int index, double* momX, double* momY);

/* Input and output grid sizes, number of GPU kernels per execution, and the bytes of device
 * work space the plan holds (two buffers of the largest grid, both components). */
SRWG_API int srwgPlanInfo(const srwgPlan* plan, long* nxIn, long* nyIn, long* nxOut, long* nyOut, int* nKernels,
                 long long* workBytes);

/* Executes the plan on device arrays (interleaved complex FP32, [ny][nx]) on CUDA stream
 * `stream` (NULL = default stream).  dExIn/dEyIn are read only; the result (output mesh) is
 * written to dExOut/dEyOut, which must hold nxOut*nyOut complex values each. */
SRWG_API int srwgPlanExecute(srwgPlan* plan, const float* dExIn, const float* dEyIn, float* dExOut, float* dEyOut,
                    void* stream);

/* Executes the plan on a batch of n wavefronts of the same mesh: wavefront b reads
 * dExIn + b*strideIn (floats) and writes dExOut + b*strideOut. */
SRWG_API int srwgPlanExecuteBatch(srwgPlan* plan, int n, const float* dExIn, const float* dEyIn, long long strideIn,
                         float* dExOut, float* dEyOut, long long strideOut, void* stream);

/* As srwgPlanExecute, and records a CUDA event pair around every pass on `stream`; waits for
 * the stream and writes each pass's duration in milliseconds to kernelMs[0 .. nKernels-1]
 * (at most maxKernels values).  Returns the number of passes in *nTimed. */
SRWG_API int srwgPlanExecuteTimed(srwgPlan* plan, const float* dExIn, const float* dEyIn, float* dExOut,
                                  float* dEyOut, void* stream, float* kernelMs, int maxKernels, int* nTimed);

SRWG_API int srwgPlanDestroy(srwgPlan* plan);

/* Partially coherent (multi-electron) propagation on the device (no counterpart C API in the
 * reference: it is the per-electron loop of srwl_wfr_emit_prop_multi_e, env/python/srwpy/srwlib.py:8506).
 * Macro-electron wavefronts are the base wavefront with the source offset of SRWLWfr.sim_src_offset
 * (srwlib.py:2803, _move_mesh=True): an angular kick (x', y') and a mesh shift (x + x' R, y + y' R);
 * each is propagated through pOpt (planned like srwlPropagElecField) in batches of up to maxBatch
 * (one launch per pass per batch; useGraph: replayed as a CUDA graph), and its total intensity
 * (srwlCalcIntFromElecField, polarisation 6, vs x and y) is added, bilinearly interpolated onto
 * pAccMesh (avg_update_interp order 1, srwlib.py:1116), to an FP64 accumulator on the device.
 * srwgMultiEAdd takes 4 doubles per electron (x [m], x' [rad], y [m], y' [rad]); a null stream
 * means the library's stream, synchronised before the call returns.  srwgMultiEGetMean copies the
 * mean (sum / number of electrons) to host memory.  pOpt must stay valid while the object lives. */
typedef struct srwgMultiE srwgMultiE;
SRWG_API int srwgMultiECreate(const SRWLWfr* pBase, const SRWLOptC* pOpt, const SRWLRadMesh* pAccMesh, int maxBatch,
                              int useGraph, int device, srwgMultiE** out);
SRWG_API int srwgMultiEAdd(srwgMultiE* m, int n, const double* arOffsets, void* stream);
/* as srwgMultiEAdd with 5 doubles per electron: the fifth is the relative energy deviation d of the
 * electron, which rescales the photon energy of its wavefront to E (1 + 2 d) */
SRWG_API int srwgMultiEAddE(srwgMultiE* m, int n, const double* arOffsets, void* stream);
/* number of passes of a batch, whether the last one writes the total intensity (float) instead of
 * the two fields (then the accumulation reads one float per sample), and (desc, optional) the text
 * description of the passes as srwgPlanDescribe gives it */
SRWG_API int srwgMultiEInfo(srwgMultiE* m, int* nPasses, int* intensityPass, char* desc, int descLen);
/* adds 1 <= n <= maxBatch electrons (stride 4 or 5 doubles each) as ONE batch, without the CUDA graph,
 * with CUDA events around every pass: passMs[i] = device time of pass i [ms] (at most maxPasses
 * values), the last one the accumulation's; *nPasses = passes + 1.  Measurement aid (no reference
 * counterpart). */
SRWG_API int srwgMultiEAddTimed(srwgMultiE* m, int n, const double* arOffsets, int stride, void* stream,
                                float* passMs, int maxPasses, int* nPasses);
SRWG_API int srwgMultiEGetMean(srwgMultiE* m, double* arMean, long long* nElec, void* stream);
/* device address of the FP64 intensity sum (pAccMesh ny x nx) and the electron count, e.g. for a
 * sum over ranks; srwgMultiESetAccumulator makes the object add into caller-owned device memory */
SRWG_API int srwgMultiEAccumulator(srwgMultiE* m, double** dAcc, long long* nElec);
SRWG_API int srwgMultiESetAccumulator(srwgMultiE* m, double* dAcc);
SRWG_API int srwgMultiEReset(srwgMultiE* m, void* stream);
SRWG_API int srwgMultiEDestroy(srwgMultiE* m);

/* Learned resize-factor predictor (no counterpart in the reference, whose users set the resize
 * factors pp[5..8] by hand): kernels of a small FP32 MLP and of the wavefront features it reads.
 * All pointers are device memory of the current device; row-major matrices.
 *   srwgMlpGemm:        C = alpha op(A) op(B) + beta C, op(A) M x K, op(B) K x N (trans flags transpose)
 *   srwgMlpBiasAct:     Z += bias (per column); Y = act(Z), act 0 identity, 1 GELU (tanh form)
 *   srwgMlpActBackward: dY *= act'(Z)
 *   srwgMlpColSum:      db[j] = sum_i dZ[i][j]
 *   srwgMlpMse:         *loss += mean (out - target)^2 (FP64), dout = 2 (out - target) / n
 *   srwgMlpAdam:        Adam step t (>= 1) with bias correction
 *   srwgWfrFeatures:    total intensity averaged on 64 x 64 cells (dFeat[4096]) and the sums of the
 *                       weighted fit of the phase curvature left after removing k (x^2/R0x + z^2/R0z)/2
 *                       (dSums[4]: sum w x dphi, sum w x^2, the same in z; k = 2 pi / lambda) */
SRWG_API int srwgMlpGemm(int M, int N, int K, const float* A, int lda, int transA, const float* B, int ldb, int transB,
                         float* C, int ldc, float alpha, float beta, void* stream);
SRWG_API int srwgMlpBiasAct(float* Z, const float* bias, float* Y, int M, int N, int act, void* stream);
SRWG_API int srwgMlpActBackward(const float* Z, float* dY, long long n, int act, void* stream);
SRWG_API int srwgMlpColSum(const float* dZ, float* db, int M, int N, void* stream);
SRWG_API int srwgMlpMse(const float* out, const float* target, float* dout, double* loss, int n, void* stream);
SRWG_API int srwgMlpAdam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                         float eps, int t, void* stream);
SRWG_API int srwgWfrFeatures(const float* dEx, const float* dEy, int nx, int ny, double xStart, double xStep,
                             double zStart, double zStep, double k, double invRx0, double invRz0, float* dFeat,
                             double* dSums, void* stream);

/* Allocation-free propagation (no counterpart in the reference).  For callers that cannot call
 * cudaMalloc at run time -- programs that reserve all device memory at start-up and hand out
 * slices themselves, or whose device memory must go through their own caching allocator --
 * this runs the propagation of srwgPlanCreate + srwgPlanExecute without allocating any device
 * memory: the caller passes the input fields (dExIn/dEyIn, read only) and the output fields
 * (dExOut/dEyOut, outCapacity complex points each, device memory), and all intermediate data
 * lives in one fixed device array inside the library (11 MiB, held by every GPU that loads the
 * library until the process exits).  Limits: intermediate grids of at most 512 x 512 points,
 * 1 MiB of plan tables and 2 MiB of moment-pass results and scratch; larger propagations return
 * error 23904 (text: srwlUtiGetErrText).  Runs on the current device and `stream`; pWfrOut
 * (optional) receives the output mesh and scalars.  Where the propagation recomputes the moments
 * from the field and pWfrOut has moment arrays, the call waits for `stream` to read them back.
 * Every call copies its tables from host memory, so a call on a stream that is being captured
 * returns error 23903 without queuing anything.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) with that device current; make it before any stream capture.  Calls
 * share the array: calls that overlap on the GPU race. */
SRWG_API int srwgPropagElecFieldStatic(const SRWLWfr* pWfr, const SRWLOptC* pOpt, const float* dExIn,
                                       const float* dEyIn, float* dExOut, float* dEyOut, long long outCapacity,
                                       void* stream, SRWLWfr* pWfrOut);

/* Autotuned launch shapes (no counterpart in the reference, whose FFTs are FFTW's): kernel family
 * (1: the power-of-two pass, 3: the specialised pass of linen_lengths.h, which also serves the powers
 * of two listed there) and lines per CTA of the line passes with compile-time lengths, per axis
 * (0 rows, 1 columns) and line length N.  The library reads the table measured by srw_b200.tune from
 * models/line_tuning.txt beside its directory (or the file named by the environment variable
 * SRWG_TUNING; "" for the built-in defaults) at its first plan.
 *   srwgTuneSetFamily: sets the family of one entry (0: the length's default); error 23903 when the
 *                      family has no kernel for N
 *   srwgTuneSetLines:  sets the lines per CTA of one entry in its family (0 removes the entry);
 *                      error 23903 for an invalid shape
 *   srwgTuneGetFamily / srwgTuneGetLines: what plans use now (0: not a compile-time length)
 *   srwgTuneLoad:      replaces the table by a file's entries (NULL or "": defaults only) */
SRWG_API int srwgTuneSetFamily(int axis, int N, int family);
SRWG_API int srwgTuneSetLines(int axis, int N, int lines);
SRWG_API int srwgTuneGetFamily(int axis, int N, int* family);
SRWG_API int srwgTuneGetLines(int axis, int N, int* lines);
SRWG_API int srwgTuneLoad(const char* path, int* nEntries);

/* Bounded waits of the kernels (the specialised line passes wait for the bulk copies of their input
 * tiles): srwgSetWaitLimit sets the iteration limit of those waits (0: the built-in limit, far above
 * any copy's time); a wait that reaches it counts the event in a per-device counter, lets the copies
 * in flight land, and the CTA skips its work (the pass's output is then incomplete).
 * srwgGetWaitStatus reads that counter of `device` (and clears it when reset != 0). */
SRWG_API int srwgSetWaitLimit(long long iterations);
SRWG_API int srwgGetWaitStatus(int device, int* count, int reset);

/* The number of points a resize gives for a requested n: the next good FFT number at or above n
 * (NextCorrectNumberForFFT, cpp/src/ext/genmath/gmfft.cpp:156), as the planner uses it. */
SRWG_API long srwgNextFftNumber(long n);

/* Human-readable list of the planned passes (one line per kernel) into buf. */
SRWG_API int srwgPlanDescribe(const srwgPlan* plan, char* buf, int bufLen);

#ifdef __cplusplus
}
#endif

#endif /* SRWL_B200_H */
