// Host planner: the reference's per-element bookkeeping (meshes, radii, centres, moments) in FP64
// with the reference's operation order, lowered into fused GPU passes (kdesc.h).
#pragma once
#include <vector_types.h>

#include <string>
#include <vector>
#include "kdesc.h"
#include "../../include/srwl_b200.h"

namespace srwg {

// next good FFT number >= n (NextCorrectNumberForFFT, gmfft.cpp:156-228)
long next_correct_number_for_fft(long n);

// Subset of srTSRWRadStructAccessData (cpp/src/core/srradstr.h:67) used by this path, ne == 1.
struct WfrState {
    int nx = 0, nz = 0;
    double eStart = 0, xStart = 0, xStep = 0, zStart = 0, zStep = 0;
    double yStart = 0, avgPhotEn = 0;
    double RobsX = 0, RobsZ = 0, RobsXAbsErr = 0, RobsZAbsErr = 0, xc = 0, zc = 0;
    double xWfrMin = 0, xWfrMax = 0, zWfrMin = 0, zWfrMax = 0;
    int Pres = 0;
    double xStartTr = 0, zStartTr = 0;
    bool UseStartTrToShiftAtChangingRepresToCoord = false;
    long AuxLong1 = 0, AuxLong2 = 0, AuxLong3 = 0, AuxLong4 = 0;
    bool xLinOnly = false, zLinOnly = false;
    double dxcSub = 0, dzcSub = 0;
    bool QuadX = false, QuadZ = false;
    double momX[11] = {0}, momZ[11] = {0};
    double propM[20] = {0};      // 4x4 propagation matrix and 4-vector (SRWLWfr::arElecPropMatr)
    bool havePropM = false;
    bool haveMom = false;
};

// One step of the statistical-moment bookkeeping.  The steps are replayed on the host after the
// passes ran, with the moments the reference recomputes from the field (ComputeRadMoments) taken
// from the result slots of the MOM passes.
struct MomOp {
    int kind = 0;                      // MOP_MATRIX or MOP_APERTURE
    double ax[2][2] = {{0}}, az[2][2] = {{0}};   // transfer matrices (lens, drift)
    int clamp = 0;                     // drift: floor of the rms sizes at the diffraction limit
    double sx = 0, sz = 0;
    int obstacle = 0;                  // aperture: opening (centre, half sizes) for the 1.7 sigma check
    double cx = 0, cz = 0, hx = 0, hz = 0;
    int slot = -1;                     // result slot of the MOM pass (-1: no recomputation possible)
    int qx = 0, qz = 0;                // quadratic-term treatment flags a recomputation leaves behind
    int nx = 0, nz = 0;                // mesh and photon energy of the recomputation
    double eStart = 0, xStart = 0, xStep = 0, zStart = 0, zStep = 0;
};
enum { MOP_MATRIX = 1, MOP_APERTURE = 2, MOP_ESTIMATE = 3 };

// Planner::plan / resume: the plan stops at a stage boundary (its passes so far are complete and
// must run before planning can go on, because the next element depends on moments measured from
// the field)
#define SRWG_NEED_STAGE (-77)

enum ElemKind { E_DRIFT = 1, E_APERTURE = 2, E_LENS = 3, E_TRANSM = 4 };

struct ElemDesc {
    int kind = 0;
    double L = 0; int treat = 0;                            // drift
    char shape = 'r', apob = 'a'; double Dx = 0, Dy = 0;    // aperture / obstacle
    double Fx = 0, Fy = 0;                                  // lens, transmission
    double x = 0, y = 0;                                    // centre
    int outer = 0;                                          // index in the top-level container
    int tr = -1;                                            // transmission: index of its table copy
    int trNx = 0, trNz = 0, extTr = 0;
    double trXs = 0, trXf = 0, trZs = 0, trZf = 0;
};

struct PropDesc {
    int n = 0;
    double pp[17] = {0};
    double get(int i, double def) const { return i < n ? pp[i] : def; }
};

class Builder;

// one stand-alone MOM pass (ComputeRadMoments) on a wavefront in the state w, result slot 0: its
// descriptor, its point-wise tables, and the op that turns its sums into moments (moments_from_sums)
void fill_moment_desc(const WfrState& w, MomDesc& d, MomOp& op);
void single_moment_pass(const WfrState& w, KernelDesc& k, MomOp& op, std::vector<float2>& tables);
void moments_from_sums(const double* S, const MomOp& op, double* momX, double* momZ);

// fills the separable point-wise tables of every pass (tables.cpp)
void build_tables(std::vector<KernelDesc>& ks, std::vector<float2>& tables);

// an intensity extraction after an element (srwlPropagElecField's arID / arIM / arI lists): after
// element `elem` (0-based; the number of elements: after the post-resize), request `index`
struct IntReq {
    int elem = 0, index = 0;
    int pol = 6, type = 0, dep = 3, pres = 0;
};

// a planned extraction of the current stage: its pass writes bytes at off of the extraction buffer
struct IntOut {
    int index = 0, nx = 0, nz = 0;
    double xStart = 0, xStep = 0, zStart = 0, zStep = 0;
    long long off = 0, bytes = 0;
    char arType = 'f';
};

class Planner {
public:
    WfrState w;                          // evolves from the input to the output state
    WfrState in;
    std::vector<KernelDesc> kernels;
    int outBuf = 0;                      // buffer holding the result (0: the input itself)
    long long maxElems = 0;              // largest grid over all work buffers
    std::vector<float2> tables;          // separable point-wise tables of all passes (tables.cpp)
    std::string err;
    bool numMoments = true;              // emit MOM passes where the reference recomputes the moments
    int nMomSlots = 0;                   // MOM passes of the plan (result slots per wavefront)
    std::vector<MomOp> momOps;
    std::vector<IntReq> intReqs;         // intensity extractions asked for (set before plan())
    std::vector<IntOut> intOuts;         // those planned in the current stage
    long long intBytes = 0;              // extraction buffer of the current stage

    // the output moments from the input ones and the MOM passes' result slots (nMomSlots x
    // SRWG_MOM_SLOT doubles; unused when nMomSlots == 0)
    void replay_moments(const double* slots, double* momX, double* momZ, bool* quadX = nullptr,
                        bool* quadZ = nullptr) const;

    // flattens SRWLOptC (nested containers included) and plans; returns 0, an SRW error number, or
    // (with allowStages) SRWG_NEED_STAGE: `kernels` then hold a complete stage, which must run on
    // the field before resume() plans on with the stage's moment results
    int plan(const SRWLWfr* wfr, const SRWLOptC* opt);
    // slots: the result slots of every MOM pass so far (nMomSlots x SRWG_MOM_SLOT doubles)
    int resume(const double* slots);
    std::string describe() const;
    bool allowStages = false;            // staged planning (the one-shot entry point only)
    // a linear phase kx x + kz z + c (physical coordinates of the input mesh) applied to the input
    // field before the first element, fused into the first pass (the angular kick of a macro-electron)
    bool inPhase = false;
    double inKx = 0, inKz = 0, inC = 0;
    int nStages = 0;                     // stage boundaries passed
    WfrState stageIn;                    // mesh of the current stage's input

private:
    Builder* b = nullptr;
    std::vector<ElemDesc> els_;          // the flattened chain and the element reached
    std::vector<PropDesc> props_;
    size_t elemIdx_ = 0;
    bool resizeDone_ = false;            // the current element's pre-resize is planned
    std::vector<double> slotVals_;       // host copy of the result slots of completed stages
    int pendingEstSlot_ = -1;            // MOM pass of a pp[3]=1 radius estimate waiting for its stage
    MomOp pendingEstOp_;
    int run();
    int finalize();
    void emit_moment_pass(MomOp& op, bool certain);
    void extract_after(int elem);
    void estimate_rad(double L, double& effRx, double& effRz);
    int flatten(const SRWLOptC* opt, std::vector<ElemDesc>& els, std::vector<PropDesc>& props, bool nested);
    void set_full_range();
    void srwl_roundtrip();
    void set_rad_repres(int coord_or_ang);
    void fft2_emit(int dir, bool use_given, double& xStepTr, double& zStepTr, double& xStartTr, double& zStartTr);
    void drift(const ElemDesc& e, int anal);
    void drift_ang(const ElemDesc& e);
    void drift_to_waist(const ElemDesc& e);
    void drift_from_waist(const ElemDesc& e);
    void drift_beyond_parax(const ElemDesc& e);
    bool quadFlagsUncertain_ = false;    // QuadX/QuadZ depend on a moment recomputation decided on the device
    int drift_quad(const ElemDesc& e, int subtype);
    void drift_moments(double L);
    void record_matrix(const double ax[2][2], const double az[2][2], int clamp, double sx, double sz);
    void prop_4x4(const double E[16], const double e[4]);
    bool momProvisional = false;         // plan-time moments wait for a MOM pass's result
    void lens(const ElemDesc& e);
    void transmission(const ElemDesc& e);
    std::vector<std::vector<double>> trTables_;   // copies of the transmission tables (T, OPD pairs)
    void aperture(const ElemDesc& e);
    void phase_lin_subtract(double newXc, double newZc);
    void phase_lin_reset();
    void fix_abs_err();
    void mirror(int sx, int sz);
    int resize(double pxm, double pxd, double pzm, double pzd, int shift, double xcs, double zcs, bool other_side);
    void treat_quad(char add_or_rem);
    double diff_lim_spot(char xz, double L) const;
};

}  // namespace srwg
