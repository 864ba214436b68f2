// Device-side views of the GAMERA Model/Grid/State/Solver data, shared by
// every build variant of the step kernels and by the C ABI.
#pragma once
#include "gam_layout.cuh"

// Solar-wind boundary data (apps/wind.F90:206-391) for a constant wind: the
// blend weights and wind face fluxes depend only on the grid and the wind
// direction, so they are computed once on the host (libm acos/exp, the same
// expressions as wgtWind/RampDown) and stored for the 4 ghost layers:
// entry (n-1) + 4*(j + (Nj+1)*k) for ghost layer n = 1..4.
struct WindData {
    double state[8];    // rho, P, Vx, Vy, Vz, Bx, By, Bz
    const double* wC;   // weight at the ghost cell centre
    const double* wF;   // 3 x: weight at the I face ie+n+1, J face and K face of the ghost cell
    const double* sF;   // 3 x: wind flux through those faces
    long nw;            // entries per array
    // time series (gam_set_wind_series, apps/wind.F90 WindBC_T): n rows of
    // t, D, Vx, Vy, Vz, P, Bx, By, Bz, xBS, yBS, zBS; n = 0: the constant wind
    int n;
    double tMin, tMax, dtW, Bx0, ByC, BzC;
    const double* ts;
};

// The ionospheric inner boundary (bc[0] = 7) and its model hooks: tables
// computed on the host from the coupling fields (gam_set_ionosphere)
struct IonData {
    int on;            // the magnetosphere's hooks (HackE) run on this grid or tile
    int push, nIonP;   // PushIon on the first nIonP active shells
    double dtCpl;      // coupling time scale (code time)
    const double* Vg;  // ghost-cell velocity, 3 per (n-1) + 4 (jj + Nj kk), n = 1..4
    const double* Vp;  // PushIon's target velocity, 3 per (ii - G) + nIonP ((jj - G) + Njp (kk - G))
    const double* Ee;  // the first shell's J and K EMFs (IonEFix), 2 per jj + Nj kk
    // the wind's part (bc[1] = 4, constant wind): WindEFix and NudgeSW
    int wind;          // 1: apply them
    double vSW;        // DiffuseOuter's speed min(|vFr|, Ca)
    double dtSW0;      // NudgeSW's time scale
    const double* We;  // 7 per s + 4 (jj - G + (Njp+1) (kk - G)), s = 0..3 for i = ie-2+s: the blend
                       // weight of the I, J, K edges (negative: unchanged), their wind EMF, and
                       // DiffuseOuter's weight
    const double* Wn;  // NudgeSW's weight of the last active cell, per (jj - G) + Njp (kk - G)
};

// Ring averaging about the LFM axis (ringav.F90, gid "lfm"): rings are the k
// circles of the first NumR j rows next to each pole (GAM_BC_LFM sides),
// sliced by i (gam_set_rings)
struct RingData {
    int on, doS, doE;     // doS / doE: the pole at js / je+1 belongs to this grid
    int NumR, Np;         // rings per pole, cells per ring (Nkp)
    int recon;            // ring reconstruction: 0 PPM, 1 PLM, 2 PCM
    int nft;              // Fourier modes 0..nft removed from the fluxes (-1: none)
    int clean;            // CleanLoops
    double tScl;          // CleanLoops' scale (1 with doFastClean)
    double aScl;          // CleanRing's 2/Np (in default real)
    int Nch[32];          // chunks of ring 1..NumR
    int chunkStride;      // 5 (max chunks + 4): shared-memory chunk values of one ring
    const double* ftab;   // cos / sin (m phi_n): [(2 m + c) Np + n - 1], m = 0..2
    void* smoothE;        // smoothing EMFs, 3 components of the box (compute precision)
};

template <class R> struct DevParams {
    R gamma, gm1, CFL, pdmb, Vd0, cHogH, cHogM, dFloor, pFloor;
    int doMHD, doLFMLim, do25D, doBackground, up7;
    int doBoris;  // Boris correction with the speed of light Ca (init.F90:417-423)
    double Ca;
    int doAB3;    // third-order (AB3) predictor with ooState (init.F90:377)
    int bc[6];
    // CalcDT covers the ghost layer below / above the active range per
    // direction (1, the reference's isDT..ieDT); a tile drops it where a
    // neighbour's cells lie, the magnetosphere everywhere
    int dtKlo, dtKhi;
    int dtIlo, dtIhi, dtJlo, dtJhi;
    WindData wind;
    double inflow[8];  // uniform inner-I inflow (bc[0] = 6): rho, P, Vx, Vy, Vz, Bx, By, Bz
    IonData ion;       // ionospheric inner boundary and its hooks (bc[0] = 7)
    RingData ring;     // ring averaging about the LFM axis (bc[2] / bc[3] = 8)
};

template <class R> struct Geo {  // Grid_T arrays on the device (gamtypes.F90:168-250)
    const R* vol;    // cell
    const R* xyzcc;  // cell, 3
    const R* dl;     // cell, min(di,dj,dk)
    const R* face;   // face, 3
    const R* xfc;    // face, 9: x + 3*d
    const R* Tf;     // face, 27: n + 9*d
    const R* edge;   // edge, 3
    const R* Te;     // edge, 27: n + 9*d
    const R* Teb;    // edge, 12: q + 4*d
    // FP32 form only: face centroid minus cell centroid for the six faces of
    // a cell, x + 3*f with f = I-, I+, J-, J+, K-, K+ (computed in FP64, rounded
    // once). Replaces xfc and xyzcc in bFlux2Fld, whose absolute coordinates
    // lose the cell-size differences when rounded to FP32.
    const R* dxf;    // cell, 18
    const double* fcB0;    // face, 9  (background; FP64 in both forms)
    const double* bFlux0;  // face, 3
    const double* edgB0;   // edge, 6: c + 2*d
    const double* B0;      // cell, 3
    const double* dpB0;    // cell, 3
};

template <class R> struct StateBuf {
    R* Gas;  // cell, 5
    R* mf;   // face, 3
    R* B;    // cell, 3
};

template <class R> struct Work {
    R* QW;   // cell, 5: volume * primitives of the half state (BlockCon2Prim), the recon operand
    R* QB;   // cell, 3: volume * Bxyz of the half state
    R* Dh;   // cell, 1: half-state density (GetCornerD)
    R* Wn;   // cell, 5: limiter primitives (state n with lfmlim, else the half state)
    R* Bl;   // cell, 3: limiter Bxyz without lfmlim (= half-state Bxyz); lfmlim uses State%Bxyz
    R* VdV;  // cell, 3: volume * momentum / max(density, dFloor) of the half state
    R* abh;  // face, 3: area * (half-state flux / max(area, TINY)), the EdgeLRs recon operand
    R* bn;   // face, 3: limiter flux / max(area, TINY)
    R* Bnf;  // face, 3: half-state flux / area
    R* AVf;  // cell, 9: area(dT1) * Vf(x) for edge direction eD at x + 3*eD
    R* E;    // edge, 3
    R* gF;   // face, 15: gas flux v + 5*d (already times face area)
    R* mF;   // face, 9: magnetic flux x + 3*d
    // differentiation form only (null in the step): the flux kernels' face
    // states, 22 per face and direction, q + 22*d: WL, WR (5 each), MagL,
    // MagR (3 each), VaD and the diffusion sums dW (5)
    R* fsv;
    // differentiation form only: the edge kernels' corner values, 10 per
    // edge and direction, q + 10*eD: Dc, bT1L, bT1R, fA1, bT2L, bT2R, fA2, VC (3)
    R* esv;
};
constexpr int GAM_FSV_NC = 22;
constexpr int GAM_ESV_NC = 10;

struct Range {  // inclusive box-index range
    int i0, i1, j0, j1, k0, k1;
};


// Everything one step launch needs.
template <class R> struct Ctx {
    GamBox b;
    DevParams<R> P;
    Geo<R> g;
    StateBuf<R> st[2];   // double buffer: st[cur] = State (n), st[1-cur] = oState (n-1) -> State (n+1)
    R* oomf;             // doAB3: ooState face fluxes (n-2), refreshed from oState by k_update_faces
    Work<R> w;
    GamScalars* sc;
    double gamma, gm1;
    int kvar;  // launch-configuration variant for tuning runs (GAM_KVAR); 0 = the tuned default
    // side streams and fork/join events of the step graph (independent
    // kernels of a step run as parallel branches); null: one stream
    cudaStream_t aux[5];
    cudaEvent_t ev[8];
};
