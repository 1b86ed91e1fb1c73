// Kernel descriptors shared by the host planner and the sm_100a kernels.
//
// A propagation through an SRWLOptC chain is lowered by the planner (planner.cpp) into a short
// list of bandwidth-bound passes over the two field components (Ex, Ey; complex FP32,
// row-major [nz][nx], the reference's layout for ne == 1, srradstr.cpp:501):
//   * LINE passes: each CTA loads whole rows (axis 0) or tiles of whole columns (axis 1) into
//     shared memory, runs up to two 1D FFTs along the line with point-wise work folded in
//     between / before / after them, and stores the lines back;
//   * RESIZE passes: the 16-point bicubic gather of RadResizeCore (sroptelm.cpp:3038);
//   * PW passes: a standalone element-wise pass (only when nothing else can host the ops);
//   * MOM passes: read-only reductions for the statistical moments (no output field).
// All point-wise work of the reference (drift transfer functions, quadratic phases, lens,
// aperture masks, FFT centring sign/rotation, normalisation, shift tables, mirror) is expressed
// by the structs below and applied inside those passes.
#pragma once
#include <stdint.h>

#define SRWG_MAX_MASKS 4
#define SRWG_MAX_STAGES 12
#define SRWG_MAX_KERNELS 64

// Aperture / obstacle mask in physical coordinates (sroptapt.h:118-395).  The physical coordinate
// of kernel index i is x0 + i*dx (dx may be negative when the kernel's index order is mirrored).
struct PwMask {
    int type;        // 1: rectangle, 2: circle
    int obstacle;    // 0: aperture (zero outside), 1: obstacle (zero inside)
    double x0, dx, z0, dz;
    double cx, cz;   // centre
    double hx, hz;   // rectangle half sizes incl. the reference's 1e-10 m tolerance
    double r2;       // circle radius squared
};

// Point-wise operator: v <- mask(i,j) * scale * exp(i*phase(i,j)) * v, with i the x index and j the
// z index of the element in the kernel's index space.
struct PwOps {
    int has_quad;
    double Ai, Bi, Aj, Bj, C;            // phase += Ai i^2 + Bi i + Aj j^2 + Bj j + C   (FP64)
    int has_ang;                         // angular-representation drift (sroptdrf.h:615)
    double qx0, dqx, qz0, dqz;           // q coordinates of index (i, j)
    double c0, c1;                       // phase += c0 q^2 (1 + c1 q^2 + 2 (c1 q^2)^2)
    int has_scale;
    float sre, sim;                      // complex scale
    int nmask;
    PwMask mask[SRWG_MAX_MASKS];
    int ang_resid;                       // 1: only the non-separable part c0 q^2 c1 q^2 (1 + 2 c1 q^2)
    int has_bpx;                         // exact propagator beyond the paraxial approximation
    double bqx0, bdqx, bqz0, bdqz;       //   (sroptdrf.h:712): phase += kL * (sqrt(1 - lam^2 q^2) - 1
    double blam, bkL;                    //   + btreat), q the angular frequencies of index (i, j)
    int btreat;
    int has_tr;                          // transmission table (sroptgtr.h:163-310), bilinear, FP64:
    int tr_id, tr_nx, tr_nz, tr_outer;   //   table id (offset after planning), size, 1: zero outside
    long long tr_off;                    //   offset of the (T, OPD) doubles in the plan's tables (float2)
    double tr_x0, tr_dx, tr_z0, tr_dz;   //   physical coordinate of index (i, j)
    double tr_xs, tr_xstep, tr_zs, tr_zstep;   // the table's mesh
    double tr_k;                         //   2 pi / lambda: phase = k * OPD
};

// Separable factor tables (complex FP32, computed in FP64 on the host) of one point-wise chain:
// factor(k, line) = tab[k] * ltab[line] * (non-separable extras).  Offsets are in float2 units into
// the plan's table buffer; -1 when absent.
struct ChainTab {
    long long tab;
    long long ltab;
};

// Index-only side operations of one centred 1D DFT (Make2DFFT helpers, gmfft.h:232-480),
// per axis.  For a forward transform they are applied after the DFT (RepairSign then Rotate,
// x Mult, shift-after table); for an inverse transform rotation+sign and the shift-before table
// are applied before it and Mult and the shift-after table after it.
struct FftSide {
    int rs;              // sign (-1)^k + half rotation (even N)
    int has_shift;       // multiply by exp(i * shift_a * (k - N/2))
    double shift_a;
    float scale;         // real factor (1 if none)
};

struct LineDesc {
    int axis;            // 0: rows (transform along x), 1: columns (transform along z)
    int nx, nz;
    int f1;              // 0 none, +1 forward, -1 inverse: first transform along the line
    FftSide f1_pre, f1_post;
    int has_pw;
    PwOps pw;
    int mirror_along;    // reverse order along the line after the point-wise ops
    int mirror_lines;    // store line l at (nlines - 1 - l)
    int f2;              // second transform along the line
    FftSide f2_pre, f2_post;
    ChainTab t_pre, t_mid, t_fin;   // tables of the pre / middle / final chains
    int has_extra;                  // non-separable point-wise work of the middle chain
    PwOps extra;
    int zwin;                       // the input is zero outside lines [zl0, zl1] x along [za0, za1]
    int zl0, zl1, za0, za1;         //   (the output window of the resize that produced it)
    int zskip;                      // with zwin: the (zero) lines outside [zl0, zl1] are not written,
                                    //   the next pass loads only those lines' window
    int blk_out;                    // row pass: output in blocks of blk_out columns (0: row-major);
                                    //   column intensity pass (out_int): the intensity of column c at
                                    //   point i at ((c / blk_out) N + i) blk_out + c % blk_out
    int blk_in;                     // column pass: input in blocks of blk_in columns (0: row-major)
    int out_int;                    // last pass of a multi-electron batch on a specialised kernel: one
                                    //   CTA transforms both components of its lines and writes the
                                    //   total intensity |Ex|^2 + |Ey|^2 (float, dst[0]) instead of them
    int int_flat;                   // intensity pass whose output factors (the output chain's table,
    float int_scale;                //   the line factors) have one magnitude everywhere: they are not
                                    //   applied, the intensity is scaled by int_scale = that magnitude^2
};

struct ResizeDesc {
    int nxo, nzo, nxn, nzn;
    double xStartO, xStepO, zStartO, zStepO;   // old mesh
    double xStartN, xStepN, zStartN, zStepN;   // new mesh
    long ixStart, ixEnd, izStart, izEnd;       // AuxLong1..4
    int only_larger;                           // RadResizeCore_OnlyLargerRange
    int has_pw;
    PwOps pw;                                  // applied to the new points
    ChainTab t;                                // separable part of pw: tab over x, ltab over z
    int has_extra;
    PwOps extra;
    long long axx, axz;                        // per-axis gather tables (ResizeAxis), float2 offsets
    int has_pre;                               // point-wise work on the OLD mesh before resampling (a
    PwOps pre;                                 //   preceding element-wise pass folded into this one)
    ChainTab tp;                               // separable part of pre: tab over old x, ltab over old z
    int has_pre_extra;
    PwOps pre_extra;
    int tile_or, tile_oc;                      // tiled kernel: largest old-row / old-column extent of a
                                               //   tile of new points (0: not tiled)
    int skip_zero;                             // points outside the window are not written: the next
                                               //   pass treats them as zero (LineDesc::zwin)
};

// per new-mesh index along one axis: first old node of the 4-point stencil, clipped relative cell
// index for the low-order fallback, relative coordinate (old steps) w.r.t. node st+1; for the
// range-only resize `st` is the copied node.  Stored as two float2 (ints bit-cast).
struct ResizeAxis {
    int st, ir;
    float rel, pad;
};

struct PwDesc {
    int nx, nz;
    PwOps pw;
    int mirror_x, mirror_z;                    // output index flips
    ChainTab t;
    int has_extra;
    PwOps extra;
};

// Statistical moments of the field (ComputeRadMoments, sroptelm.cpp:1608-2092), coordinate
// representation: a read-only reduction of the field in buffer `src` after the point-wise work `pw`
// (the operators still pending on it, and the removal of the wavefront's quadratic phase) into the
// 22 weighted sums of one result slot.  The host turns the sums into moments after the run.
struct MomDesc {
    int nx, nz;
    double xStart, xStep, zStart, zStep;       // physical mesh of the field
    double ax, az;                             // 2 pi / (lambda R) * step, per axis
    PwOps pw;
    ChainTab t;                                // separable part of pw: tab over x, ltab over z
    int has_extra;
    PwOps extra;
    int slot;
    // intensity extraction passes (K_INT) only: polarisation, component (0 intensity, 2 phase,
    // 3 Re E, 6 Im E) and the byte offset of the output in the extraction buffer
    int ipol, iwhat;
    long long ioff;
};

#define SRWG_MOM_SLOT 32   // doubles per result slot: 22 sums, 4 power-limit indices, status

enum KernelKind { K_LINE = 1, K_RESIZE = 2, K_PW = 3, K_MOM = 4, K_INT = 5 };

// passes that only read the field (moments, intensity extraction)
inline bool reads_only(int kind) { return kind == K_MOM || kind == K_INT; }

struct KernelDesc {
    int kind;
    int src, dst;        // buffer ids: 0 = input, 1 = work A, 2 = work B
    LineDesc line;
    ResizeDesc rs;
    PwDesc pwk;
    MomDesc mom;
};
