// ORACLE -- test infrastructure only. CPU restatement of the GAMERA MHD step of
// the Kaiju/MAGE reference (Fortran 2008 + OpenMP), used as the checker for the
// CUDA implementation and as the timed CPU baseline. Nothing in the product
// imports, links or calls this file.
//
// Each routine follows one Fortran routine of the reference, cited as
// file:line (paths relative to the reference project root), and keeps its
// data layout (column-major, i fastest, nG = 4 ghosts, lower bound isg = 1-nG),
// its 16-wide i-bricks (BRICKSIZE, CMakeLists.txt:44-47), its loop order and the
// evaluation order of every arithmetic expression (Fortran evaluates a+b+c as
// (a+b)+c, and x**2.0 is folded to x*x by the compiler). Intent: bitwise the
// same arithmetic as an IEEE-strict build of the reference.
//
// Build variants (oracle/Makefile):
//   strict : -O2 -fno-fast-math -ffp-contract=off, libm erfc/exp  (parity oracle)
//   gm     : as strict but erfc/exp from mage_b200/csrc/gam_math.cuh, so the
//            only remaining difference to the GPU is FMA contraction / order
//   fast   : -O3 -march=native -ffast-math, mirroring the reference Release
//            flags (cmake/compilers.cmake:49,138); timed CPU baseline.
//
// Choices where the reference source cannot pin the arithmetic (no Fortran
// compiler is available to run it):
//   * NORM2 is evaluated with gfortran's scaled algorithm (norm2s below);
//   * default-real literals follow standard Fortran kinds: only sqrt(2.0) in
//     initBW (prob.F90:246-252) is inexact and is taken in single precision;
//   * dot_product is the sequential sum starting from 0.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef GAM_ORACLE_OWN_MATH
#include "../mage_b200/csrc/gam_math.cuh"
#define O_ERFC(x) gam::gam_erfc(x)
#define O_EXP(x) gam::gam_exp(x)
#else
#define O_ERFC(x) std::erfc(x)
#define O_EXP(x) std::exp(x)
#endif

namespace orc {

// ---------------------------------------------------------------- constants
// src/base/kdefs.F90:14-21, src/base/defs/gdefs.F90:8-30
static const double TINY = 1.0e-12, HUGE_ = 1.0e12;
static const double PI = 3.141592653589793;  // 4*atan(1) in double
enum { NVAR = 5, NDIM = 3, recLen = 8, limLen = 4, vecLen = 16, Nr2 = 4, Nl2 = 2 };
// stress.F90:20-25: the nuclear option's threshold cLim, and sqrt(2.0) of its
// interface speed: a default-real (single precision) constant in the
// reference, which gfortran folds to the float 1.41421354
static const double cLim = 1.5;
static const double SQRT2_R4 = (double)1.41421354f;
enum { DEN = 0, MOMX = 1, MOMY = 2, MOMZ = 3, ENERGY = 4 };
enum { VELX = 1, VELY = 2, VELZ = 3, PRESSURE = 4 };
enum { IDIR = 0, JDIR = 1, KDIR = 2 };
enum { XDIR = 0, YDIR = 1, ZDIR = 2 };
enum { NORMX = 0, NORMY, NORMZ, TAN1X, TAN1Y, TAN1Z, TAN2X, TAN2Y, TAN2Z };
enum { XNQI = 0, YNQI, XNQJ, YNQJ };
enum { LEFT = 0, RIGHT = 1 };
static const int SgnLR[2] = {-1, 1};  // stress.F90:19

// boundary kinds (a subset of bcs.F90 / apps/wind.F90; BC_INFLOW is a uniform
// inflow of this library, with no counterpart in the reference)
enum { BC_PERIODIC = 0, BC_NONE = 1, BC_ZEROGRAD = 2, BC_SPHIN = 3, BC_WIND = 4, BC_INFLOW = 6, BC_ION = 7, BC_LFM = 8 };

// interpolation weights, recon.F90:22-23,28-29
static double interpWgt[8], interpWgt6[8], Up7C[7];
static void init_weights() {
    const int w8[8] = {-3, 29, -139, 533, 533, -139, 29, -3};
    const int w6[8] = {0, 1, -8, 37, 37, -8, 1, 0};
    const int u7[7] = {-3, 25, -101, 319, 214, -38, 4};
    for (int n = 0; n < 8; n++) interpWgt[n] = (double)w8[n] / 840.0;
    for (int n = 0; n < 8; n++) interpWgt6[n] = (double)w6[n] / 60.0;
    for (int n = 0; n < 7; n++) Up7C[n] = (double)u7[n] / 420.0;
}

// Gauss-Legendre 12 point, quadrature.F90:10-27
static const double gA[12] = {
    0.1252334085114689154724, 0.3678314989981801937527, 0.5873179542866174472967,
    0.7699026741943046870369, 0.9041172563704748566785, 0.9815606342467192506906,
    -0.1252334085114689154724, -0.3678314989981801937527, -0.5873179542866174472967,
    -0.7699026741943046870369, -0.9041172563704748566785, -0.9815606342467192506906};
static const double gWgt[12] = {
    0.2491470458134027850006, 0.233492536538354808761, 0.203167426723065921749,
    0.160078328543346226335, 0.1069393259953184309603, 0.0471753363865118271946,
    0.2491470458134027850006, 0.233492536538354808761, 0.203167426723065921749,
    0.160078328543346226335, 0.1069393259953184309603, 0.0471753363865118271946};

// ---------------------------------------------------------------- arrays
// Fortran array A(l0:u0, l1:u1, l2:u2, 0:nc-1), column-major.
struct F4 {
    std::vector<double> v;
    int l0 = 0, l1 = 0, l2 = 0, n0 = 0, n1 = 0, n2 = 0, nc = 0;
    void alloc(int a0, int b0, int a1, int b1, int a2, int b2, int ncomp, double fill = 0.0) {
        l0 = a0; l1 = a1; l2 = a2;
        n0 = b0 - a0 + 1; n1 = b1 - a1 + 1; n2 = b2 - a2 + 1; nc = ncomp;
        v.assign((size_t)n0 * n1 * n2 * nc, fill);
    }
    inline size_t idx(int i, int j, int k, int c) const {
        return (size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * ((size_t)(k - l2) + (size_t)n2 * c));
    }
    inline double& operator()(int i, int j, int k, int c = 0) { return v[idx(i, j, k, c)]; }
    inline double operator()(int i, int j, int k, int c = 0) const { return v[idx(i, j, k, c)]; }
    inline double* comp(int c) { return v.data() + (size_t)n0 * n1 * n2 * c; }
    inline const double* comp(int c) const { return v.data() + (size_t)n0 * n1 * n2 * c; }
    void fill(double x) { std::fill(v.begin(), v.end(), x); }
};

struct Params {  // mirrored by oracle/oracle.py (ctypes)
    int Nip, Njp, Nkp;
    int doMHD, doLFMLim, do25D, doBackground, up7, fixedTimestep;
    double gamma, CFL, pdmb, Vd0, cHogH, cHogM, dFloor, pFloor;
    double tFin, dt0, limDT0, fixedDT;
    int bc[6];
    int noMetric;  // 1: allocate the metric with its fill values only (arrays set by the caller)
    double M0;           // dipole moment (code units) of the background field, m = (0,0,M0)
    double wind[8];      // constant solar wind: rho, P, Vx, Vy, Vz, Bx, By, Bz (code units)
    double inflow[8];    // uniform inner-I inflow state, same order as wind
    int doBoris;         // physics/doBoris (init.F90:417-423)
    double Ca;           // physics/Ca: the Boris speed of light (code units)
    int doAB3;           // sim/doAB3 (init.F90:377): third-order predictor with ooState
    // ring averaging about the LFM axis (ring/doRing with ring/gid = "lfm"):
    // ringNumR rings (0: off), chunks per ring, ring/rngrec (0 PPM, 1 PLM,
    // 2 PCM), ringknobs/NMag, ringknobs/doClean, ringknobs/doFastClean
    int ringNumR;
    int ringNch[32];
    int ringRecon, ringNFT, ringClean, ringFast;
};

struct Model {
    double gamma, CFL, Vd0, cHogH, cHogM;
    double t = 0, tFin, dt = 0, dt0 = 0, limDT0;
    int ts = 0;
    bool fixedTimestep, doMHD, doLFMLim, do25D, doBackground, up7;
    double M0 = 0.0;
    double wind[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double inflow[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool doBoris = false;
    double Ca = 0.0;
    bool doAB3 = false;
    // solar-wind time series of WindBC_T (apps/wind.F90:28-53, readWind
    // :619-763), code units, 0-based rows; n = 0: the constant wind above
    struct WindSeries {
        int n = 0;
        std::vector<double> tW, Q, B, xyzBS;  // Q: n x (D, Vx, Vy, Vz, P); B, xyzBS: n x 3
        double tMin = 0, tMax = 0, dtW = 0, Bx0 = 0, ByC = 0, BzC = 0;
    } ws;
    // ionospheric inner boundary (IonInnerBC_T, voltron/ICs/earthcmi.F90:33-48)
    // and the magnetosphere hooks that come with it (EFix, PerStep)
    struct Ion {
        std::vector<double> inExyz;  // (1:PsiSh, jsg:jeg, ksg:keg, 1:3), PsiSh = 5 (cmidefs.F90:13)
        std::vector<double> inEijk;  // (1:PsiSh+1, jsg:jeg+1, ksg:keg+1, 1:3)
        double M0 = 0.0, dtCpl = 0.0;
        bool doIonPush = true;
        int nIonP = 1;
        double dtSW0 = 0.0;  // NudgeSW's time scale: one minute of the wind series (apps/wind.F90:414)
    } ion;
};

struct Grid {
    int Nip, Njp, Nkp, Ni, Nj, Nk;
    int is, ie, js, je, ks, ke, isg, ieg, jsg, jeg, ksg, keg;
    int isDT, ieDT, jsDT, jeDT, ksDT, keDT;
    F4 xyz, xyzcc, xfc, di, dj, dk, volume, Tf, Te, Teb, face, edge;
    F4 fcB0, edgB0, B0, bFlux0, dpB0;  // background (cell-sized, background.F90:43-47)
    int bc[6];
    // ring averaging about the LFM axis (Model%Ring, ringutils.F90:37-236 for
    // gid "lfm": the pole along k, Np = Nkp, slices over i); doS / doE: the
    // grid holds the pole at js / je+1 (J boundary GAM_BC_LFM)
    struct Ring {
        bool on = false, doS = false, doE = false, doClean = true, doFast = true;
        int NumR = 0, Np = 0, recon = 0, NFTMAG = 1;
        int Nch[32] = {0};
    } ring;
    // allocation helpers
    void cellArr(F4& a, int nc, double f = 0.0) const { a.alloc(isg, ieg, jsg, jeg, ksg, keg, nc, f); }
    void faceArr(F4& a, int nc, double f = 0.0) const { a.alloc(isg, ieg + 1, jsg, jeg + 1, ksg, keg + 1, nc, f); }
};

struct State {
    double time = -HUGE_;
    F4 Gas, magFlux, Efld, Bxyz;
};

// ringutils.F90:650-659 WrapK
static inline int WrapK(int k, int Np) {
    int kp = k + Np / 2;
    if (kp > Np) kp = kp - Np;
    return kp;
}
// ringutils.F90:521-586 lfmIJKfc: face-centred conjugate of face d
static void lfmIJKcc(const Grid& G, int i, int j, int k, int& ip, int& jp, int& kp);
static void lfmIJKfc(const Grid& G, int d, int i, int j, int k, int& ip, int& jp, int& kp) {
    const int Np = G.Nkp;
    ip = i;
    if (d == 0) {
        lfmIJKcc(G, i, j, k, ip, jp, kp);
        return;
    }
    kp = k;
    if (k < G.ks) kp = k + Np;
    if (d == 1 && k > G.ke) kp = k - Np;
    if (d == 2 && k > G.ke + 1) kp = k - Np;
    jp = j;
    if (d == 1) {  // J faces: the pole face itself is seen once
        if (G.ring.doS && j < G.js) {
            jp = G.js + (G.js - j);
            kp = WrapK(k, Np);
        }
        if (G.ring.doE && j > G.je + 1) {
            jp = G.je + 1 - (j - G.je) + 1;
            kp = WrapK(k, Np);
        }
    } else {
        if (G.ring.doS && j < G.js) {
            jp = G.js + (G.js - j) - 1;
            kp = WrapK(k, Np);
        }
        if (G.ring.doE && j > G.je) {
            jp = G.je - (j - G.je) + 1;
            kp = WrapK(k, Np);
        }
    }
}

// global limiter parameters (recon.F90:27 pdmb, gdefs.F90:12 floors)
static double pdmb = 0.75, dFloor = TINY, pFloor = TINY;

static inline double sgn(double b) { return std::copysign(1.0, b); }  // sign(1.0,b)

// gfortran NORM2: scaled sum of squares
static inline double norm2s(const double* a, int n) {
    double scale = 1.0, res = 0.0;
    for (int q = 0; q < n; q++) {
        if (a[q] != 0.0) {
            double ax = std::fabs(a[q]);
            if (scale < ax) {
                double val = scale / ax;
                res = 1.0 + res * val * val;
                scale = ax;
            } else {
                double val = ax / scale;
                res += val * val;
            }
        }
    }
    return scale * std::sqrt(res);
}
static inline void cross(const double* a, const double* b, double* c) {  // math.F90:265-274
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double* a, const double* b) {
    double s = 0.0;
    for (int q = 0; q < 3; q++) s += a[q] * b[q];
    return s;
}
// math.F90:332-343 normVec
static inline void normVec(const double* a, double* out) {
    double nA = std::sqrt(dot3(a, a));
    for (int x = 0; x < 3; x++) out[x] = nA <= TINY ? 0.0 : a[x] / nA;
}

// ---------------------------------------------------------------- EOS
// gamutils.F90:301-321 CellC2P
static void CellC2P(const Model& M, const double* Con, double* Prim) {
    double rho = Con[DEN];
    double Vx = Con[MOMX] / rho, Vy = Con[MOMY] / rho, Vz = Con[MOMZ] / rho;
    double E = Con[ENERGY];
    double KinE = 0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
    Prim[DEN] = std::max(rho, dFloor);
    Prim[VELX] = Vx;
    Prim[VELY] = Vy;
    Prim[VELZ] = Vz;
    Prim[PRESSURE] = std::max((M.gamma - 1) * (E - KinE), pFloor);
}
// gamutils.F90:362-383 CellP2C
static void CellP2C(const Model& M, const double* Prim, double* Con) {
    double rho = std::max(Prim[DEN], dFloor);
    double Vx = Prim[VELX], Vy = Prim[VELY], Vz = Prim[VELZ];
    double IntE = std::max(Prim[PRESSURE], pFloor) / (M.gamma - 1);
    double KinE = 0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
    Con[DEN] = rho;
    Con[MOMX] = rho * Vx;
    Con[MOMY] = rho * Vy;
    Con[MOMZ] = rho * Vz;
    Con[ENERGY] = IntE + KinE;
}

// ---------------------------------------------------------------- loaders
// gamutils.F90:64-130 gamLoadBlock / gamLoadBlockI. Qb[n][i], n = 0..2*Nx2-1
// stands for offset n-Nx2 along direction d from (iS,j,k).
static inline void loadBlock(const Grid& G, const double* Q, bool iface, int iS, int j, int k, int iMax,
                             int d, int Nx2, double (*Qb)[vecLen]) {
    long ni = iface ? G.Ni + 1 : G.Ni, nj = iface ? G.Nj + 1 : G.Nj;
    long l0 = (iS - G.isg) + (long)(j - G.jsg) * ni + (long)(k - G.ksg) * ni * nj;
    long nSt = (d == IDIR) ? 1 : (d == JDIR ? ni : ni * nj);
    for (int n = 0; n < 2 * Nx2; n++)
        for (int i = 0; i < vecLen; i++) Qb[n][i] = 0.0;
    for (int n = -Nx2; n < Nx2; n++) {
        long l = l0 + nSt * n;
        for (int i = 0; i < iMax; i++) Qb[n + Nx2][i] = Q[l + i];
    }
}

// ---------------------------------------------------------------- recon
// recon.F90:202-214 Central8
static inline void Central8(const double (*Qb)[vecLen], double* Qi) {
    for (int i = 0; i < vecLen; i++) {
        double s = 0.0;
        for (int n = 0; n < recLen; n++) s += interpWgt[n] * Qb[n][i];
        Qi[i] = s;
    }
}
// recon.F90:231-272 pdmLR
static inline void pdmLR(const double (*Qb)[vecLen], const double* Qi, double* Ql, double* Qr) {
    for (int i = 0; i < vecLen; i++) {
        double v0 = Qb[0][i], v1 = Qb[1][i], v2 = Qb[2][i], v3 = Qb[3][i];
        double maxV = std::max(v1, v2), minV = std::min(v1, v2);
        double vN = std::max(minV, std::min(Qi[i], maxV));
        double dv0 = pdmb * (v1 - v0), dv1 = pdmb * (v2 - v1), dv2 = pdmb * (v3 - v2);
        double s0 = sgn(dv0), s1 = sgn(dv1), s2 = sgn(dv2);
        double q0 = std::fabs(s0 + s1), q1 = std::fabs(s1 + s2);
        double dvL = vN - v1, dvR = v2 - vN;
        Ql[i] = vN - s1 * std::max(0.0, std::fabs(dvL) - q0 * std::fabs(dv0));
        Qr[i] = vN + s1 * std::max(0.0, std::fabs(dvR) - q1 * std::fabs(dv2));
    }
}
// recon.F90:275-301 PDM
static inline double PDM(double q0, double q1, double q2, double qI) {
    double maxQ = std::max(q1, q2), minQ = std::min(q1, q2);
    double qN = std::max(minQ, std::min(qI, maxQ));
    double dq0 = pdmb * (q1 - q0), dq1 = pdmb * (q2 - q1);
    double s0 = sgn(dq0), s1 = sgn(dq1);
    double s01 = std::fabs(s0 + s1);
    double dqL = qN - q1;
    return qN - s1 * std::max(0.0, std::fabs(dqL) - s01 * std::fabs(dq0));
}
// recon.F90:304-310 Up7
static inline double Up7(double q0, double q1, double q2, double q3, double q4, double q5, double q6) {
    return q0 * Up7C[0] + q1 * Up7C[1] + q2 * Up7C[2] + q3 * Up7C[3] + q4 * Up7C[4] + q5 * Up7C[5] +
           q6 * Up7C[6];
}
// recon.F90:125-158 Cen8LRs and :162-198 Up7LRs (the GetLRs choice, init.F90:441-454)
static bool g_up7 = false;
static void GetLRs(const double (*dV)[vecLen], const double (*nQ)[vecLen], const double (*Q)[vecLen],
                   const double* Vi, double* Ql, double* Qr) {
    double QdV[recLen][vecLen];
    for (int n = 0; n < recLen; n++)
        for (int i = 0; i < vecLen; i++) QdV[n][i] = dV[n][i] * Q[n][i];
    if (!g_up7) {
        double Qi[vecLen];
        Central8(QdV, Qi);
        for (int i = 0; i < vecLen; i++) Qi[i] = Qi[i] / Vi[i];
        pdmLR(nQ, Qi, Ql, Qr);
    } else {
        for (int i = 0; i < vecLen; i++) {
            Ql[i] = Up7(QdV[0][i], QdV[1][i], QdV[2][i], QdV[3][i], QdV[4][i], QdV[5][i], QdV[6][i]) / Vi[i];
            Qr[i] = Up7(QdV[7][i], QdV[6][i], QdV[5][i], QdV[4][i], QdV[3][i], QdV[2][i], QdV[1][i]) / Vi[i];
            Ql[i] = PDM(nQ[0][i], nQ[1][i], nQ[2][i], Ql[i]);
            Qr[i] = PDM(nQ[3][i], nQ[2][i], nQ[1][i], Qr[i]);
        }
    }
}
// recon.F90:96-122 BlockLRs
static void BlockLRs(const double (*VolB)[vecLen], const double (*nQb)[limLen][vecLen],
                     const double (*Qb)[recLen][vecLen], double (*Ql)[vecLen], double (*Qr)[vecLen], int NumV) {
    double Vi[vecLen];
    Central8(VolB, Vi);
    for (int nv = 0; nv < NumV; nv++) GetLRs(VolB, nQb[nv], Qb[nv], Vi, Ql[nv], Qr[nv]);
}
// recon.F90:39-93 BlockStateLRs with its BlockCon2Prim
static void BlockCon2Prim(const Model& M, const double (*inCon)[recLen][vecLen], double (*oPrim)[recLen][vecLen],
                          int xLen) {
    for (int n = 0; n < xLen; n++)
        for (int i = 0; i < vecLen; i++) {
            double D = std::max(inCon[DEN][n][i], dFloor);
            double Mx = inCon[MOMX][n][i], My = inCon[MOMY][n][i], Mz = inCon[MOMZ][n][i];
            double E = inCon[ENERGY][n][i];
            double KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
            double P = std::max((M.gamma - 1) * (E - KinE), pFloor);
            oPrim[DEN][n][i] = D;
            oPrim[VELX][n][i] = Mx / D;
            oPrim[VELY][n][i] = My / D;
            oPrim[VELZ][n][i] = Mz / D;
            oPrim[PRESSURE][n][i] = P;
        }
}

// ---------------------------------------------------------------- fluxes
// stress.F90:432-511 GasKinFlux
static void GasKinFlux(const Model& M, int q, const double (*PrimLRB)[vecLen], const double (*TfB)[vecLen],
                       double (*gFlxB)[vecLen], double (*dW)[vecLen]) {
    const double s = (double)SgnLR[q];
    for (int i = 0; i < vecLen; i++) {
        double D = PrimLRB[DEN][i], P = PrimLRB[PRESSURE][i];
        double Vx = PrimLRB[VELX][i], Vy = PrimLRB[VELY][i], Vz = PrimLRB[VELZ][i];
        double E = 0.5 * D * (Vx * Vx + Vy * Vy + Vz * Vz) + P / (M.gamma - 1);
        double lambda = D / (2 * P);
        double Vn = TfB[NORMX][i] * Vx + TfB[NORMY][i] * Vy + TfB[NORMZ][i] * Vz;
        double Vt1 = TfB[TAN1X][i] * Vx + TfB[TAN1Y][i] * Vy + TfB[TAN1Z][i] * Vz;
        double Vt2 = TfB[TAN2X][i] * Vx + TfB[TAN2Y][i] * Vy + TfB[TAN2Z][i] * Vz;
        double Vn0 = 0.5 * O_ERFC(s * std::sqrt(lambda) * Vn);
        double Vn1 = Vn * Vn0 - 0.5 * s * O_EXP(-(lambda * Vn * Vn)) / std::sqrt(PI * lambda);
        gFlxB[DEN][i] = gFlxB[DEN][i] + D * Vn1;
        gFlxB[ENERGY][i] = gFlxB[ENERGY][i] + (E + 0.5 * P) * Vn1 + 0.5 * P * Vn0 * Vn;
        double fMn = D * Vn * Vn1 + P * Vn0;
        double fMt1 = D * Vt1 * Vn1;
        double fMt2 = D * Vt2 * Vn1;
        double fMx = TfB[NORMX][i] * fMn + TfB[TAN1X][i] * fMt1 + TfB[TAN2X][i] * fMt2;
        double fMy = TfB[NORMY][i] * fMn + TfB[TAN1Y][i] * fMt1 + TfB[TAN2Y][i] * fMt2;
        double fMz = TfB[NORMZ][i] * fMn + TfB[TAN1Z][i] * fMt1 + TfB[TAN2Z][i] * fMt2;
        gFlxB[MOMX][i] = gFlxB[MOMX][i] + fMx;
        gFlxB[MOMY][i] = gFlxB[MOMY][i] + fMy;
        gFlxB[MOMZ][i] = gFlxB[MOMZ][i] + fMz;
        dW[DEN][i] = dW[DEN][i] + s * D;
        dW[MOMX][i] = dW[MOMX][i] + s * D * Vx;
        dW[MOMY][i] = dW[MOMY][i] + s * D * Vy;
        dW[MOMZ][i] = dW[MOMZ][i] + s * D * Vz;
        dW[ENERGY][i] = dW[ENERGY][i] + s * E;
    }
}
// stress.F90:513-599 MagKinFlux
static void MagKinFlux(const Model& M, int q, const double (*PrimLRB)[vecLen], const double (*MagLRB)[vecLen],
                       const double* Bn, const double (*TfB)[vecLen], double (*mFlxB)[vecLen],
                       const double (*B0)[vecLen], const double* B0n, double* bbD, double* VaD) {
    const double s = (double)SgnLR[q];
    for (int i = 0; i < vecLen; i++) {
        double D = PrimLRB[DEN][i], P = PrimLRB[PRESSURE][i];
        double Bx = MagLRB[XDIR][i], By = MagLRB[YDIR][i], Bz = MagLRB[ZDIR][i];
        double B0x = B0[XDIR][i], B0y = B0[YDIR][i], B0z = B0[ZDIR][i];
        double dPb = 0.5 * (Bx * Bx + By * By + Bz * Bz);
        double Va2;
        if (M.doBackground) {
            double sx = Bx + B0x, sy = By + B0y, sz = Bz + B0z;
            Va2 = (sx * sx + sy * sy + sz * sz) / D;
            bbD[i] = bbD[i] + 0.5 * (sx * sx + sy * sy + sz * sz);
        } else {
            Va2 = 2 * dPb / D;
            bbD[i] = bbD[i] + 0.5 * (Bx * Bx + By * By + Bz * Bz);
        }
        double Vac2 = M.doBoris ? Va2 / (1 + (Va2 / (M.Ca * M.Ca))) : Va2;  // Boris-corrected Va^2
        double Vx = PrimLRB[VELX][i], Vy = PrimLRB[VELY][i], Vz = PrimLRB[VELZ][i];
        double Nx = TfB[NORMX][i], Ny = TfB[NORMY][i], Nz = TfB[NORMZ][i];
        double Vn = Nx * Vx + Ny * Vy + Nz * Vz;
        double lambda = 1 / (2 * P / D + Vac2);
        double Vn0 = 0.5 * O_ERFC(s * std::sqrt(lambda) * Vn);
        VaD[i] = VaD[i] + 0.5 * std::sqrt(Vac2);
        mFlxB[XDIR][i] = mFlxB[XDIR][i] + Vn0 * (dPb * Nx - Bx * Bn[i]);
        mFlxB[YDIR][i] = mFlxB[YDIR][i] + Vn0 * (dPb * Ny - By * Bn[i]);
        mFlxB[ZDIR][i] = mFlxB[ZDIR][i] + Vn0 * (dPb * Nz - Bz * Bn[i]);
        if (M.doBackground) {
            double BdB0 = B0x * Bx + B0y * By + B0z * Bz;
            mFlxB[XDIR][i] = mFlxB[XDIR][i] + Vn0 * (-(B0x * Bn[i]) - Bx * B0n[i] + BdB0 * Nx);
            mFlxB[YDIR][i] = mFlxB[YDIR][i] + Vn0 * (-(B0y * Bn[i]) - By * B0n[i] + BdB0 * Ny);
            mFlxB[ZDIR][i] = mFlxB[ZDIR][i] + Vn0 * (-(B0z * Bn[i]) - Bz * B0n[i] + BdB0 * Nz);
        }
    }
}

// gFlx(i,j,k,nv,d) stored as F4 with component nv + 5*d; mFlx with x + 3*d
// stress.F90:204-429 Fluxes
static void Fluxes(const Model& M, const Grid& G, const State& nS, const State& hS, int iB, int j, int k, int dN,
                   F4& gFlx, F4& mFlx) {
    int ie = G.ie + (dN == IDIR ? 1 : 0);
    int iMax = std::min((int)vecLen, ie - iB + 1);
    int isB = iB;

    double VolB[recLen][vecLen];
    double ConB[NVAR][recLen][vecLen], MagB[NDIM][recLen][vecLen];
    double nConB[NVAR][limLen][vecLen], nMagB[NDIM][limLen][vecLen];
    double TfB[9][vecLen], faB[vecLen];
    double PrimL[NVAR][vecLen], PrimR[NVAR][vecLen], MagL[NDIM][vecLen], MagR[NDIM][vecLen];
    double gFlxB[NVAR][vecLen], mFlxB[NDIM][vecLen], dW[NVAR][vecLen], VaD[vecLen], bbD[vecLen];
    double B0[NDIM][vecLen], B0n[vecLen], Bn[vecLen];
    std::memset(gFlxB, 0, sizeof(gFlxB));
    std::memset(mFlxB, 0, sizeof(mFlxB));
    std::memset(dW, 0, sizeof(dW));
    std::memset(VaD, 0, sizeof(VaD));
    std::memset(bbD, 0, sizeof(bbD));
    std::memset(TfB, 0, sizeof(TfB));
    std::memset(faB, 0, sizeof(faB));
    std::memset(B0, 0, sizeof(B0));
    std::memset(Bn, 0, sizeof(Bn));
    std::memset(B0n, 0, sizeof(B0n));
    std::memset(MagL, 0, sizeof(MagL));
    std::memset(MagR, 0, sizeof(MagR));

    loadBlock(G, G.volume.comp(0), false, iB, j, k, iMax, dN, Nr2, VolB);
    for (int i = 0; i < iMax; i++) {
        for (int n = 0; n < 9; n++) TfB[n][i] = G.Tf(isB + i, j, k, n + 9 * dN);
        faB[i] = G.face(isB + i, j, k, dN);
    }
    if (M.doMHD) {
        for (int nv = 0; nv < NDIM; nv++) {
            loadBlock(G, hS.Bxyz.comp(nv), false, iB, j, k, iMax, dN, Nr2, MagB[nv]);
            const State& lS = M.doLFMLim ? nS : hS;
            loadBlock(G, lS.Bxyz.comp(nv), false, iB, j, k, iMax, dN, Nl2, nMagB[nv]);
        }
        BlockLRs(VolB, nMagB, MagB, MagL, MagR, NDIM);
        for (int i = 0; i < iMax; i++) Bn[i] = hS.magFlux(isB + i, j, k, dN) / faB[i];
        if (M.doBackground) {
            for (int i = 0; i < iMax; i++) {
                for (int d = 0; d < NDIM; d++) B0[d][i] = G.fcB0(isB + i, j, k, d + 3 * dN);
                B0n[i] = G.bFlux0(isB + i, j, k, dN) / faB[i];
            }
        }
    }
    for (int nv = 0; nv < NVAR; nv++) {
        loadBlock(G, hS.Gas.comp(nv), false, iB, j, k, iMax, dN, Nr2, ConB[nv]);
        const State& lS = M.doLFMLim ? nS : hS;
        loadBlock(G, lS.Gas.comp(nv), false, iB, j, k, iMax, dN, Nl2, nConB[nv]);
    }
    {  // BlockStateLRs
        double PrimB[NVAR][recLen][vecLen], nPrimB[NVAR][recLen][vecLen];
        double nConB8[NVAR][recLen][vecLen];
        for (int nv = 0; nv < NVAR; nv++)
            for (int n = 0; n < limLen; n++)
                for (int i = 0; i < vecLen; i++) nConB8[nv][n][i] = nConB[nv][n][i];
        BlockCon2Prim(M, nConB8, nPrimB, limLen);
        BlockCon2Prim(M, ConB, PrimB, recLen);
        double nPrim4[NVAR][limLen][vecLen];
        for (int nv = 0; nv < NVAR; nv++)
            for (int n = 0; n < limLen; n++)
                for (int i = 0; i < vecLen; i++) nPrim4[nv][n][i] = nPrimB[nv][n][i];
        BlockLRs(VolB, nPrim4, PrimB, PrimL, PrimR, NVAR);
    }
    if (M.doMHD) {
        MagKinFlux(M, LEFT, PrimL, MagL, Bn, TfB, mFlxB, B0, B0n, bbD, VaD);
        MagKinFlux(M, RIGHT, PrimR, MagR, Bn, TfB, mFlxB, B0, B0n, bbD, VaD);
        if (M.doBoris) {  // stress.F90:335-349 Boris hogs on the magnetic fluxes
            for (int i = 0; i < iMax; i++)
                for (int x = 0; x < NDIM; x++) {
                    double deeV = PrimR[VELX + x][i] - PrimL[VELX + x][i];
                    double deeP = bbD[i] * deeV / (M.Ca * M.Ca);
                    mFlxB[x][i] = mFlxB[x][i] - M.cHogM * VaD[i] * deeP;
                }
        }
        for (int nv = 0; nv < NDIM; nv++)
            for (int i = 0; i < iMax; i++) mFlx(isB + i, j, k, nv + 3 * dN) = faB[i] * mFlxB[nv][i];
    }
    std::memset(gFlxB, 0, sizeof(gFlxB));
    std::memset(dW, 0, sizeof(dW));
    GasKinFlux(M, LEFT, PrimL, TfB, gFlxB, dW);
    GasKinFlux(M, RIGHT, PrimR, TfB, gFlxB, dW);
    const double alphaS = 1.0;
    for (int nv = 0; nv < NVAR; nv++)
        for (int i = 0; i < iMax; i++) gFlxB[nv][i] = gFlxB[nv][i] - alphaS * M.cHogH * VaD[i] * dW[nv][i];
    if (M.doBoris) {  // stress.F90:399-417 the "nuclear option" (doNuke = T, cLim = 1.5)
        for (int i = 0; i < iMax; i++) {
            double vl[3] = {PrimL[VELX][i], PrimL[VELY][i], PrimL[VELZ][i]};
            double vr[3] = {PrimR[VELX][i], PrimR[VELY][i], PrimR[VELZ][i]};
            double vL = norm2s(vl, 3), vR = norm2s(vr, 3);
            double Vn = std::sqrt(vL * vL + vR * vR) / SQRT2_R4;
            if (Vn >= cLim * M.Ca)
                for (int nv = 0; nv < NVAR; nv++) {
                    double dCon = ConB[nv][Nr2][i] - ConB[nv][Nr2 - 1][i];
                    gFlxB[nv][i] = gFlxB[nv][i] - M.Ca * dCon;
                }
        }
    }
    for (int nv = 0; nv < NVAR; nv++)
        for (int i = 0; i < iMax; i++) gFlx(isB + i, j, k, nv + 5 * dN) = faB[i] * gFlxB[nv][i];
}

// stress.F90:41-198 CalcStress
// ringutils.F90:662-678 RingFlux: no flux through the pole faces, then
// FixGasFluxLFM (gamdebug.F90:91-124): the K fluxes of the two periodic k
// ends set to their mean
static void RingFlux(const Model& M, const Grid& G, F4& gFlx, F4& mFlx) {
    const int jz[2] = {G.js, G.je + 1};
    const bool on[2] = {G.ring.doS, G.ring.doE};
    for (int p = 0; p < 2; p++) {
        if (!on[p]) continue;
        for (int k = G.ksg; k <= G.keg; k++)
            for (int i = G.isg; i <= G.ieg; i++) {
                for (int nv = 0; nv < NVAR; nv++) gFlx(i, jz[p], k, nv + 5 * JDIR) = 0.0;
                if (M.doMHD)
                    for (int x = 0; x < NDIM; x++) mFlx(i, jz[p], k, x + 3 * JDIR) = 0.0;
            }
    }
    if (!M.doMHD) return;
    for (int j = G.js; j <= G.je; j++)
        for (int i = G.is; i <= G.ie; i++) {
            for (int nv = 0; nv < NVAR; nv++) {
                const double gF = 0.5 * (gFlx(i, j, G.ks, nv + 5 * KDIR) + gFlx(i, j, G.ke + 1, nv + 5 * KDIR));
                gFlx(i, j, G.ks, nv + 5 * KDIR) = gF;
                gFlx(i, j, G.ke + 1, nv + 5 * KDIR) = gF;
            }
            for (int x = 0; x < NDIM; x++) {
                const double mF = 0.5 * (mFlx(i, j, G.ks, x + 3 * KDIR) + mFlx(i, j, G.ke + 1, x + 3 * KDIR));
                mFlx(i, j, G.ks, x + 3 * KDIR) = mF;
                mFlx(i, j, G.ke + 1, x + 3 * KDIR) = mF;
            }
        }
}
static void CalcStress(const Model& M, const Grid& G, const State& nS, const State& hS, F4& gFlx, F4& mFlx,
                       F4& dGasH, F4& dGasM) {
    int nFlx = M.do25D ? 2 : 3;
    int ks = G.ks, ke = M.do25D ? G.ks : G.ke;
#pragma omp parallel
    {
        for (int d = 0; d < nFlx; d++) {
            if (d == IDIR) {
#pragma omp for collapse(2) nowait
                for (int k = ks; k <= ke; k++)
                    for (int j = G.js; j <= G.je; j++)
                        for (int iB = G.is; iB <= G.ie + 1; iB += vecLen) Fluxes(M, G, nS, hS, iB, j, k, d, gFlx, mFlx);
            } else if (d == JDIR) {
#pragma omp for collapse(2) nowait
                for (int k = ks; k <= ke; k++)
                    for (int iB = G.is; iB <= G.ie; iB += vecLen)
                        for (int j = G.js; j <= G.je + 1; j++) Fluxes(M, G, nS, hS, iB, j, k, d, gFlx, mFlx);
            } else {
#pragma omp for collapse(2) nowait
                for (int j = G.js; j <= G.je; j++)
                    for (int iB = G.is; iB <= G.ie; iB += vecLen)
                        for (int k = ks; k <= ke + 1; k++) Fluxes(M, G, nS, hS, iB, j, k, d, gFlx, mFlx);
            }
        }
    }
    if (G.ring.on) RingFlux(M, G, gFlx, mFlx);  // stress.F90:137-139
    // HackFlux = IonFlux (earthcmi.F90:357-404) on the inner tile with rings:
    // the I fluxes of the first face ring at each pole set to their ring mean
    if (G.ring.on && G.bc[0] == BC_ION) {
        const int jr[2] = {G.je, G.js};
        const bool on[2] = {G.ring.doE, G.ring.doS};
        for (int p = 0; p < 2; p++) {
            if (!on[p]) continue;
            if (M.doMHD)
                for (int x = 0; x < NDIM; x++) {
                    double s = 0.0;
                    for (int k = G.ks; k <= G.ke; k++) s = s + mFlx(G.is, jr[p], k, x + 3 * IDIR);
                    const double avg = s / G.ring.Np;
                    for (int k = G.ks; k <= G.ke; k++) mFlx(G.is, jr[p], k, x + 3 * IDIR) = avg;
                }
            for (int nv = 0; nv < NVAR; nv++) {
                double s = 0.0;
                for (int k = G.ks; k <= G.ke; k++) s = s + gFlx(G.is, jr[p], k, nv + 5 * IDIR);
                const double avg = s / G.ring.Np;
                for (int k = G.ks; k <= G.ke; k++) gFlx(G.is, jr[p], k, nv + 5 * IDIR) = avg;
            }
        }
    }
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++) {
                double dV = G.volume(i, j, k);
                for (int nv = 0; nv < NVAR; nv++)
                    dGasH(i, j, k, nv) = (gFlx(i, j, k, nv + 5 * IDIR) - gFlx(i + 1, j, k, nv + 5 * IDIR) +
                                          gFlx(i, j, k, nv + 5 * JDIR) - gFlx(i, j + 1, k, nv + 5 * JDIR) +
                                          gFlx(i, j, k, nv + 5 * KDIR) - gFlx(i, j, k + 1, nv + 5 * KDIR)) /
                                         dV;
                if (M.doMHD) {
                    for (int x = 0; x < NDIM; x++) {
                        dGasM(i, j, k, x) = (mFlx(i, j, k, x + 3 * IDIR) - mFlx(i + 1, j, k, x + 3 * IDIR) +
                                             mFlx(i, j, k, x + 3 * JDIR) - mFlx(i, j + 1, k, x + 3 * JDIR) +
                                             mFlx(i, j, k, x + 3 * KDIR) - mFlx(i, j, k + 1, x + 3 * KDIR)) /
                                            dV;
                        if (M.doBackground) dGasM(i, j, k, x) = dGasM(i, j, k, x) + G.dpB0(i, j, k, x);
                    }
                }
            }
}

// ---------------------------------------------------------------- E field
static void getNormalPlane(int dN, int* e1, int* e2) {  // metric.F90:174-190
    e1[0] = e1[1] = e1[2] = 0;
    e2[0] = e2[1] = e2[2] = 0;
    if (dN == IDIR) { e1[1] = 1; e2[2] = 1; }
    else if (dN == JDIR) { e1[0] = 1; e2[2] = 1; }
    else { e1[0] = 1; e2[1] = 1; }
}
// fields.F90:235-285 Mom2Face
static void Mom2Face(const Grid& G, const F4& W, double (*VfB)[vecLen], int iB, int j, int k, int iMax, int dT) {
    double VolB[recLen][vecLen], DenB[recLen][vecLen], MomB[3][recLen][vecLen], VelB[3][recLen][vecLen];
    double dV[vecLen];
    loadBlock(G, G.volume.comp(0), false, iB, j, k, iMax, dT, Nr2, VolB);
    loadBlock(G, W.comp(DEN), false, iB, j, k, iMax, dT, Nr2, DenB);
    for (int d = 0; d < 3; d++) loadBlock(G, W.comp(MOMX + d), false, iB, j, k, iMax, dT, Nr2, MomB[d]);
    for (int d = 0; d < 3; d++)
        for (int i = 0; i < vecLen; i++) VfB[d][i] = 0.0;
    for (int n = 0; n < recLen; n++)
        for (int i = 0; i < iMax; i++)
            for (int d = 0; d < 3; d++) VelB[d][n][i] = VolB[n][i] * MomB[d][n][i] / std::max(DenB[n][i], dFloor);
    for (int i = 0; i < iMax; i++) {
        double s = 0.0;
        for (int n = 0; n < recLen; n++) s += interpWgt[n] * VolB[n][i];
        dV[i] = std::max(s, TINY);
    }
    for (int d = 0; d < 3; d++)
        for (int i = 0; i < iMax; i++) {
            double s = 0.0;
            for (int n = 0; n < recLen; n++) s += interpWgt[n] * VelB[d][n][i];
            VfB[d][i] = s / dV[i];
        }
}
// fields.F90:457-517 GetCornerV
static void GetCornerV(const Grid& G, const F4& Vf, double* v1, double* v2, double* vDiff, int iB, int j, int k,
                       int iMax, int dN, int dT1, int dT2) {
    double AreaB[recLen][vecLen], VelB[recLen][vecLen], VxyzC[3][vecLen], dA[vecLen];
    std::memset(VxyzC, 0, sizeof(VxyzC));
    std::memset(dA, 0, sizeof(dA));
    loadBlock(G, G.face.comp(dT1), true, iB, j, k, iMax, dT2, Nr2, AreaB);
    for (int i = 0; i < iMax; i++) {
        double s = 0.0;
        for (int n = 0; n < recLen; n++) s += interpWgt[n] * AreaB[n][i];
        dA[i] = std::max(s, TINY);
    }
    for (int d = 0; d < 3; d++) {
        loadBlock(G, Vf.comp(d), false, iB, j, k, iMax, dT2, Nr2, VelB);
        for (int i = 0; i < iMax; i++) {
            double s = 0.0;
            for (int n = 0; n < recLen; n++) s += interpWgt[n] * (AreaB[n][i] * VelB[n][i]);
            VxyzC[d][i] = s / dA[i];
        }
    }
    for (int i = 0; i < iMax; i++) {
        int iG = iB + i;
        v1[i] = VxyzC[XDIR][i] * G.Te(iG, j, k, TAN1X + 9 * dN) + VxyzC[YDIR][i] * G.Te(iG, j, k, TAN1Y + 9 * dN) +
                VxyzC[ZDIR][i] * G.Te(iG, j, k, TAN1Z + 9 * dN);
        v2[i] = VxyzC[XDIR][i] * G.Te(iG, j, k, TAN2X + 9 * dN) + VxyzC[YDIR][i] * G.Te(iG, j, k, TAN2Y + 9 * dN) +
                VxyzC[ZDIR][i] * G.Te(iG, j, k, TAN2Z + 9 * dN);
        vDiff[i] = std::sqrt(v1[i] * v1[i] + v2[i] * v2[i]);
    }
}
// fields.F90:427-454 GetCornerD
static void GetCornerD(const Grid& G, const F4& Gas, double* Dc, int iB, int j, int k, int iMax, int dN) {
    int e1[3], e2[3];
    getNormalPlane(dN, e1, e2);
    for (int i = 0; i < iMax; i++) {
        int iG = iB + i;
        Dc[i] = 0.25 * (Gas(iG, j, k, DEN) + Gas(iG - e1[0], j - e1[1], k - e1[2], DEN) +
                        Gas(iG - e2[0], j - e2[1], k - e2[2], DEN) +
                        Gas(iG - e1[0] - e2[0], j - e1[1] - e2[1], k - e1[2] - e2[2], DEN));
    }
}
// fields.F90:288-362 EdgeLRs
static void EdgeLRs(const Model& M, const Grid& G, const F4& bFluxn, const F4& bFluxHf, double* bL, double* bR,
                    double* fA, int iB, int j, int k, int iMax, int dN, int dT1, int dT2) {
    double AreaB[recLen][vecLen], VolB[recLen][vecLen], nAreaB[limLen][vecLen];
    double MagB[1][recLen][vecLen], nMagB[1][limLen][vecLen], MagLB[1][vecLen], MagRB[1][vecLen];
    for (int i = 0; i < vecLen; i++) fA[i] = bL[i] = bR[i] = 0.0;
    std::memset(VolB, 0, sizeof(VolB));
    loadBlock(G, G.face.comp(dT1), true, iB, j, k, iMax, dT2, Nr2, AreaB);
    loadBlock(G, bFluxHf.comp(dT1), true, iB, j, k, iMax, dT2, Nr2, MagB[0]);
    loadBlock(G, G.face.comp(dT1), true, iB, j, k, iMax, dT2, Nl2, nAreaB);
    loadBlock(G, (M.doLFMLim ? bFluxn : bFluxHf).comp(dT1), true, iB, j, k, iMax, dT2, Nl2, nMagB[0]);
    for (int i = 0; i < iMax; i++) {
        for (int n = 0; n < recLen; n++) VolB[n][i] = AreaB[n][i];
        for (int n = 0; n < recLen; n++) MagB[0][n][i] = MagB[0][n][i] / std::max(AreaB[n][i], TINY);
        for (int n = 0; n < limLen; n++) nMagB[0][n][i] = nMagB[0][n][i] / std::max(nAreaB[n][i], TINY);
    }
    BlockLRs(VolB, nMagB, MagB, MagLB, MagRB, 1);
    for (int i = 0; i < vecLen; i++) {
        bL[i] = MagLB[0][i];
        bR[i] = MagRB[0][i];
    }
    for (int i = 0; i < iMax; i++) {
        double s = 0.0;
        for (int n = 0; n < recLen; n++) s += interpWgt[n] * AreaB[n][i];
        fA[i] = s;
        bL[i] = bL[i] * fA[i];
        bR[i] = bR[i] * fA[i];
    }
}
// fields.F90:365-424 GetCornerB
static void GetCornerB(const Model& M, const Grid& G, const F4& bFluxn, const F4& bFluxHf, double* b1, double* b2,
                       double* Jd, int iB, int j, int k, int iMax, int dN, int dT1, int dT2) {
    double bT1L[vecLen], bT1R[vecLen], fA1[vecLen], bT2L[vecLen], bT2R[vecLen], fA2[vecLen];
    EdgeLRs(M, G, bFluxn, bFluxHf, bT1L, bT1R, fA1, iB, j, k, iMax, dN, dT1, dT2);
    EdgeLRs(M, G, bFluxn, bFluxHf, bT2L, bT2R, fA2, iB, j, k, iMax, dN, dT2, dT1);
    for (int i = 0; i < iMax; i++) {
        int iG = iB + i;
        double xni = G.Teb(iG, j, k, XNQI + 4 * dN), yni = G.Teb(iG, j, k, YNQI + 4 * dN);
        double xnj = G.Teb(iG, j, k, XNQJ + 4 * dN), ynj = G.Teb(iG, j, k, YNQJ + 4 * dN);
        double detT = 1.0 / (xni * ynj - xnj * yni);
        double bT1 = 0.5 * (bT1L[i] + bT1R[i]) / fA1[i];
        double bT2 = 0.5 * (bT2L[i] + bT2R[i]) / fA2[i];
        double db1 = (bT1R[i] - bT1L[i]) / fA1[i];
        double db2 = (bT2R[i] - bT2L[i]) / fA2[i];
        Jd[i] = db2 - db1;
        b1[i] = detT * (ynj * bT1 - yni * bT2);
        b2[i] = detT * (-(xnj * bT1) + xni * bT2);
        if (M.doBackground) {
            b1[i] = b1[i] + G.edgB0(iG, j, k, 0 + 2 * dN);
            b2[i] = b2[i] + G.edgB0(iG, j, k, 1 + 2 * dN);
        }
    }
}
// fields.F90:70-232 CalcElecField
static void CalcElecField(const Model& M, const Grid& G, const State& nS, const State& hS, F4& Vf, F4& E) {
    E.fill(0.0);
    for (int eD = 0; eD < 3; eD++) {
        int dT1, dT2, ie, je, ke;
        if (eD == IDIR) {
            dT1 = JDIR; dT2 = KDIR;
            ie = G.ie; je = G.je + 1; ke = G.ke + 1;
#pragma omp parallel for collapse(2)
            for (int k = G.ksg; k <= G.keg; k++)
                for (int iB = G.isg; iB <= G.ieg; iB += vecLen)
                    for (int j = G.js; j <= G.je + 1; j++) {
                        int iMax = std::min((int)vecLen, G.ieg - iB + 1);
                        double VelB[3][vecLen];
                        Mom2Face(G, hS.Gas, VelB, iB, j, k, iMax, dT1);
                        for (int i = 0; i < iMax; i++)
                            for (int d = 0; d < 3; d++) Vf(iB + i, j, k, d) = VelB[d][i];
                    }
        } else if (eD == JDIR) {
            dT1 = KDIR; dT2 = IDIR;
            ie = G.ie + 1; je = G.je; ke = G.ke + 1;
#pragma omp parallel for collapse(2)
            for (int j = G.jsg; j <= G.jeg; j++)
                for (int iB = G.isg; iB <= G.ieg; iB += vecLen)
                    for (int k = G.ks; k <= G.ke + 1; k++) {
                        int iMax = std::min((int)vecLen, G.ieg - iB + 1);
                        double VelB[3][vecLen];
                        Mom2Face(G, hS.Gas, VelB, iB, j, k, iMax, dT1);
                        for (int i = 0; i < iMax; i++)
                            for (int d = 0; d < 3; d++) Vf(iB + i, j, k, d) = VelB[d][i];
                    }
        } else {
            dT1 = IDIR; dT2 = JDIR;
            ie = G.ie + 1; je = G.je + 1; ke = G.ke;
#pragma omp parallel for collapse(2)
            for (int k = G.ksg; k <= G.keg; k++)
                for (int j = G.jsg; j <= G.jeg; j++)
                    for (int iB = G.is; iB <= G.ie + 1; iB += vecLen) {
                        int iMax = std::min((int)vecLen, G.ie + 1 - iB + 1);
                        double VelB[3][vecLen];
                        Mom2Face(G, hS.Gas, VelB, iB, j, k, iMax, dT1);
                        for (int i = 0; i < iMax; i++)
                            for (int d = 0; d < 3; d++) Vf(iB + i, j, k, d) = VelB[d][i];
                    }
        }
#pragma omp parallel for collapse(2)
        for (int k = G.ks; k <= ke; k++)
            for (int j = G.js; j <= je; j++)
                for (int iB = G.is; iB <= ie; iB += vecLen) {
                    int iMax = std::min((int)vecLen, ie - iB + 1);
                    double v1[vecLen], v2[vecLen], vDiff[vecLen], Dc[vecLen], b1[vecLen], b2[vecLen], Jd[vecLen];
                    for (int i = 0; i < vecLen; i++) vDiff[i] = 0.0;
                    GetCornerV(G, Vf, v1, v2, vDiff, iB, j, k, iMax, eD, dT1, dT2);
                    GetCornerD(G, hS.Gas, Dc, iB, j, k, iMax, eD);
                    GetCornerB(M, G, nS.magFlux, hS.magFlux, b1, b2, Jd, iB, j, k, iMax, eD, dT1, dT2);
                    for (int i = 0; i < iMax; i++) {
                        int iG = iB + i;
                        double vA = std::sqrt(b1[i] * b1[i] + b2[i] * b2[i]) / std::sqrt(Dc[i]);
                        if (M.doBoris) vA = M.Ca * vA / std::sqrt(M.Ca * M.Ca + vA * vA);  // fields.F90:211-213
                        vDiff[i] = vDiff[i] + vA;
                        vDiff[i] = std::min(vDiff[i], M.CFL * G.edge(iG, j, k, eD) / M.dt);
                        double e = -(v1[i] * b2[i] - v2[i] * b1[i]) + M.Vd0 * vDiff[i] * Jd[i];
                        E(iG, j, k, eD) = e * G.edge(iG, j, k, eD);
                    }
                }
    }
}
// fields.F90:18-51 E2Flux
static void E2Flux(const Grid& G, F4& magFlux, const F4& E, double dt) {
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke + 1; k++)
        for (int j = G.js; j <= G.je + 1; j++)
            for (int i = G.is; i <= G.ie + 1; i++) {
                double dfi = E(i, j + 1, k, KDIR) - E(i, j, k, KDIR) - E(i, j, k + 1, JDIR) + E(i, j, k, JDIR);
                double dfj = E(i, j, k + 1, IDIR) - E(i, j, k, IDIR) - E(i + 1, j, k, KDIR) + E(i, j, k, KDIR);
                double dfk = E(i + 1, j, k, JDIR) - E(i, j, k, JDIR) - E(i, j + 1, k, IDIR) + E(i, j, k, IDIR);
                magFlux(i, j, k, IDIR) = magFlux(i, j, k, IDIR) - dt * dfi;
                magFlux(i, j, k, JDIR) = magFlux(i, j, k, JDIR) - dt * dfj;
                magFlux(i, j, k, KDIR) = magFlux(i, j, k, KDIR) - dt * dfk;
            }
}

// ---------------------------------------------------------------- field from flux
// gridutils.F90:648-680 gamCellBxyz
static inline void gamCellBxyz(const Grid& G, const F4& mf, int i, int j, int k, double* B) {
    double dV = G.volume(i, j, k);
    double fI = mf(i, j, k, IDIR), fJ = mf(i, j, k, JDIR), fK = mf(i, j, k, KDIR);
    double fIp = mf(i + 1, j, k, IDIR), fJp = mf(i, j + 1, k, JDIR), fKp = mf(i, j, k + 1, KDIR);
    double Div = fIp - fI + fJp - fJ + fKp - fK;
    for (int x = 0; x < 3; x++) {
        double xfI = G.xfc(i, j, k, x + 3 * IDIR), xfJ = G.xfc(i, j, k, x + 3 * JDIR), xfK = G.xfc(i, j, k, x + 3 * KDIR);
        double xfIp = G.xfc(i + 1, j, k, x + 3 * IDIR), xfJp = G.xfc(i, j + 1, k, x + 3 * JDIR),
               xfKp = G.xfc(i, j, k + 1, x + 3 * KDIR);
        double b = (fIp * xfIp + fJp * xfJp + fKp * xfKp - fI * xfI - fJ * xfJ - fK * xfK) / dV;
        B[x] = b - Div * G.xyzcc(i, j, k, x) / dV;
    }
}
// ringutils.F90:393-444 RingFlux2FieldFix: the cells across the pole take
// the Bxyz of their conjugate
static void RingFlux2FieldFix(const Grid& G, F4& Bxyz) {
    if (!G.ring.on || !(G.ring.doS || G.ring.doE)) return;
    for (int k = G.ksg; k <= G.keg; k++)
        for (int i = G.isg; i <= G.ieg; i++)
            for (int n = 1; n <= 4; n++) {
                int ip, jp, kp;
                if (G.ring.doS) {
                    lfmIJKcc(G, i, G.js - n, k, ip, jp, kp);
                    for (int x = 0; x < 3; x++) Bxyz(i, G.js - n, k, x) = Bxyz(ip, jp, kp, x);
                }
                if (G.ring.doE) {
                    lfmIJKcc(G, i, G.je + n, k, ip, jp, kp);
                    for (int x = 0; x < 3; x++) Bxyz(i, G.je + n, k, x) = Bxyz(ip, jp, kp, x);
                }
            }
}
// gridutils.F90:281-301 bFlux2Fld
static void bFlux2Fld(const Grid& G, const F4& magFlux, F4& Bxyz) {
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int i = G.isg; i <= G.ieg; i++) {
                double B[3];
                gamCellBxyz(G, magFlux, i, j, k, B);
                for (int x = 0; x < 3; x++) Bxyz(i, j, k, x) = B[x];
            }
    RingFlux2FieldFix(G, Bxyz);
}

// ---------------------------------------------------------------- update
// mhdgroup.F90:299-329 CellMaxwell
static void CellMaxwell(const Model& M, double* U, const double* dGasM, double dt) {
    double D = std::max(U[DEN], dFloor);
    double Mx = U[MOMX], My = U[MOMY], Mz = U[MOMZ], TotE = U[ENERGY];
    double KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
    double P = std::max((M.gamma - 1) * (TotE - KinE), pFloor);
    Mx = Mx + dt * dGasM[XDIR];
    My = My + dt * dGasM[YDIR];
    Mz = Mz + dt * dGasM[ZDIR];
    KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
    U[DEN] = D;
    U[MOMX] = Mx;
    U[MOMY] = My;
    U[MOMZ] = Mz;
    U[ENERGY] = KinE + P / (M.gamma - 1);
}
// mhdgroup.F90:334-382 CellBoris, single fluid; B2 and B0 are total fields
// (background included) at n+1 and n, U2 the hydro-updated state, U0 State n
static void CellBoris(const Model& M, double* U2, const double* U0, const double* B2, const double* B0,
                      const double* dGasH, const double* dGasM, double Ca, double dt) {
    double W2[NVAR];
    CellC2P(M, U2, W2);
    double D2 = std::max(W2[DEN], dFloor);
    double P2 = std::max(W2[PRESSURE], pFloor);
    double D0 = std::max(U0[DEN], dFloor);
    double V0[3] = {U0[MOMX] / D0, U0[MOMY] / D0, U0[MOMZ] / D0};
    double B1[3], dPGas[3], dPMag[3], bhat1[3], dMom[3];
    for (int x = 0; x < 3; x++) B1[x] = 0.5 * (B2[x] + B0[x]);
    double alpha = dot3(B1, B1) / (D2 * Ca * Ca);
    double dRho = dt * dGasH[DEN];
    for (int x = 0; x < 3; x++) {
        dPGas[x] = dt * dGasH[MOMX + x];
        dPMag[x] = dt * dGasM[x];
    }
    double pCon = 1.0 / (1.0 + alpha);
    normVec(B1, bhat1);
    if (alpha > TINY) {
        double sum[3];
        for (int x = 0; x < 3; x++) sum[x] = dPGas[x] + dPMag[x];
        double pg = dot3(dPGas, bhat1), ps = dot3(sum, bhat1), pv = dot3(V0, bhat1);
        for (int x = 0; x < 3; x++)
            dMom[x] = pg * bhat1[x] + pCon * (sum[x] - ps * bhat1[x]) + alpha * pCon * dRho * (V0[x] - pv * bhat1[x]);
    } else {
        for (int x = 0; x < 3; x++) dMom[x] = dPGas[x] + dPMag[x];
    }
    W2[DEN] = D2;
    for (int x = 0; x < 3; x++) W2[VELX + x] = (D0 * V0[x] + dMom[x]) / D2;
    W2[PRESSURE] = P2;
    CellP2C(M, W2, U2);
}
static void CopyState(const Grid& G, const State& a, State& b) {  // mhdgroup.F90:202-256
    b.Gas.v = a.Gas.v;
    b.Bxyz.v = a.Bxyz.v;
    b.magFlux.v = a.magFlux.v;
    b.time = a.time;
}
static void PoleE(const Grid& G, F4& E);
// mhdgroup.F90:79-200 applyUpdate (single fluid)
static void applyUpdate(const Model& M, const Grid& G, State& S, State& oS, State& ooS, double dt, const F4& dGasH,
                        const F4& dGasM, F4& E) {
    if (M.doAB3) CopyState(G, oS, ooS);
    CopyState(G, S, oS);
    S.time = S.time + dt;
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++)
                for (int nv = 0; nv < NVAR; nv++)  // CellReynolds with Model%dt (mhdgroup.F90:121)
                    S.Gas(i, j, k, nv) = S.Gas(i, j, k, nv) + M.dt * dGasH(i, j, k, nv);
    if (!M.doMHD) return;
    if (G.ring.on && (G.ring.doS || G.ring.doE)) PoleE(G, E);  // mhdgroup.F90:140-142
    E2Flux(G, S.magFlux, E, dt);
    bFlux2Fld(G, S.magFlux, S.Bxyz);
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++) {
                double U[NVAR], dPm[NDIM];
                for (int nv = 0; nv < NVAR; nv++) U[nv] = S.Gas(i, j, k, nv);
                for (int x = 0; x < NDIM; x++) dPm[x] = dGasM(i, j, k, x);
                if (M.doBoris) {
                    double oU[NVAR], B[3], oB[3], dPg[NVAR];
                    for (int nv = 0; nv < NVAR; nv++) {
                        oU[nv] = oS.Gas(i, j, k, nv);
                        dPg[nv] = dGasH(i, j, k, nv);
                    }
                    for (int x = 0; x < 3; x++) {
                        B[x] = S.Bxyz(i, j, k, x);
                        oB[x] = oS.Bxyz(i, j, k, x);
                        if (M.doBackground) {
                            B[x] = B[x] + G.B0(i, j, k, x);
                            oB[x] = oB[x] + G.B0(i, j, k, x);
                        }
                    }
                    CellBoris(M, U, oU, B, oB, dPg, dPm, M.Ca, dt);
                } else {
                    CellMaxwell(M, U, dPm, dt);
                }
                for (int nv = 0; nv < NVAR; nv++) S.Gas(i, j, k, nv) = U[nv];
            }
}
// mhdgroup.F90:709-717 ExtrapAB2
static inline double ExtrapAB2(double dt, double Q, double oQ, double odt) {
    double dQ = (Q - oQ) / odt;
    return Q + dt * dQ;
}
// mhdgroup.F90:721-731 ExtrapAB3
static inline double ExtrapAB3(double dt, double Q, double oQ, double ooQ, double odt, double oodt) {
    double dQ = (Q - oQ) / odt;
    double odQ = (oQ - ooQ) / oodt;
    double tScl = (dt + odt) / (odt + oodt);
    return Q + dt * dQ + dt * tScl * (dQ - odQ);
}
// mhdgroup.F90:444-615 Predictor + PredictCell (single fluid). With doAB3 the
// face fluxes use ooState (:466-470) but the gas takes its third level from
// oState (ooQ = oState%Gas, :500-502), as the reference does.
static void Predictor(const Model& M, const Grid& G, const State& S, const State& oS, const State& ooS, State& pS,
                      double pdt) {
    double odt = S.time - oS.time;
    double oodt = M.doAB3 ? oS.time - ooS.time : 0.0;
    if (M.doMHD) {
#pragma omp parallel for collapse(2)
        for (int k = G.ksg; k <= G.keg + 1; k++)
            for (int j = G.jsg; j <= G.jeg + 1; j++)
                for (int i = G.isg; i <= G.ieg + 1; i++)
                    for (int d = 0; d < 3; d++)
                        pS.magFlux(i, j, k, d) =
                            M.doAB3 ? ExtrapAB3(pdt, S.magFlux(i, j, k, d), oS.magFlux(i, j, k, d),
                                                ooS.magFlux(i, j, k, d), odt, oodt)
                                    : ExtrapAB2(pdt, S.magFlux(i, j, k, d), oS.magFlux(i, j, k, d), odt);
    }
    bFlux2Fld(G, pS.magFlux, pS.Bxyz);
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int i = G.isg; i <= G.ieg; i++) {
                double Q[NVAR], oQ[NVAR], W[NVAR], oW[NVAR], pW[NVAR], pQ[NVAR];
                for (int nv = 0; nv < NVAR; nv++) {
                    Q[nv] = S.Gas(i, j, k, nv);
                    oQ[nv] = oS.Gas(i, j, k, nv);
                }
                CellC2P(M, oQ, oW);
                CellC2P(M, Q, W);
                if (M.doAB3) {
                    double ooW[NVAR];
                    CellC2P(M, oQ, ooW);  // ooQ = oState%Gas
                    for (int nv = 0; nv < NVAR; nv++) pW[nv] = ExtrapAB3(pdt, W[nv], oW[nv], ooW[nv], odt, oodt);
                } else {
                    for (int nv = 0; nv < NVAR; nv++) pW[nv] = ExtrapAB2(pdt, W[nv], oW[nv], odt);
                }
                pW[DEN] = std::max(pW[DEN], dFloor);
                pW[PRESSURE] = std::max(pW[PRESSURE], pFloor);
                CellP2C(M, pW, pQ);
                for (int nv = 0; nv < NVAR; nv++) pS.Gas(i, j, k, nv) = pQ[nv];
            }
}

// ---------------------------------------------------------------- BCs
// bcs.F90:279-450 periodic_{i,o}bc{I,J,K}
static inline bool isCellCenterG(const Grid& G, int i, int j, int k) {
    return k <= G.keg && j <= G.jeg && i <= G.ieg && k >= G.ksg && j >= G.jsg && i >= G.isg;
}
static void periodic_ibcI(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int j = G.jsg; j <= G.jeg + 1; j++)
            for (int n = 1; n <= 4; n++) {
                int ig = G.is - n, is2 = G.ie - n + 1;
                if (isCellCenterG(G, ig, j, k)) {
                    for (int v = 0; v < NVAR; v++) S.Gas(ig, j, k, v) = S.Gas(is2, j, k, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(ig, j, k, x) = S.Bxyz(is2, j, k, x);
                }
                for (int x = 0; x < 3; x++) S.magFlux(ig, j, k, x) = S.magFlux(is2, j, k, x);
            }
}
static void periodic_obcI(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int j = G.jsg; j <= G.jeg + 1; j++)
            for (int n = 1; n <= 4; n++) {
                int ig = G.ie + n, is2 = G.is + n - 1;
                if (isCellCenterG(G, ig, j, k)) {
                    for (int v = 0; v < NVAR; v++) S.Gas(ig, j, k, v) = S.Gas(is2, j, k, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(ig, j, k, x) = S.Bxyz(is2, j, k, x);
                }
                S.magFlux(ig, j, k, JDIR) = S.magFlux(is2, j, k, JDIR);
                S.magFlux(ig, j, k, KDIR) = S.magFlux(is2, j, k, KDIR);
                S.magFlux(ig + 1, j, k, IDIR) = S.magFlux(G.is + n, j, k, IDIR);
            }
}
static void periodic_ibcJ(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int i = G.isg; i <= G.ieg + 1; i++)
            for (int n = 1; n <= 4; n++) {
                int jg = G.js - n, js2 = G.je - n + 1;
                if (isCellCenterG(G, i, jg, k)) {
                    for (int v = 0; v < NVAR; v++) S.Gas(i, jg, k, v) = S.Gas(i, js2, k, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, jg, k, x) = S.Bxyz(i, js2, k, x);
                }
                for (int x = 0; x < 3; x++) S.magFlux(i, jg, k, x) = S.magFlux(i, js2, k, x);
            }
}
static void periodic_obcJ(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int i = G.isg; i <= G.ieg + 1; i++)
            for (int n = 1; n <= 4; n++) {
                int jg = G.je + n, js2 = G.js + n - 1;
                if (isCellCenterG(G, i, jg, k)) {
                    for (int v = 0; v < NVAR; v++) S.Gas(i, jg, k, v) = S.Gas(i, js2, k, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, jg, k, x) = S.Bxyz(i, js2, k, x);
                }
                S.magFlux(i, jg, k, IDIR) = S.magFlux(i, js2, k, IDIR);
                S.magFlux(i, jg, k, KDIR) = S.magFlux(i, js2, k, KDIR);
                S.magFlux(i, jg + 1, k, JDIR) = S.magFlux(i, G.js + n, k, JDIR);
            }
}
static void periodic_ibcK(const Model& M, const Grid& G, State& S) {
    if (M.do25D) {
        for (int n = 1; n <= 4; n++) {
            int kg = G.ks - n;
            for (int j = G.jsg; j <= G.jeg; j++)
                for (int i = G.isg; i <= G.ieg; i++) {
                    for (int v = 0; v < NVAR; v++) S.Gas(i, j, kg, v) = S.Gas(i, j, G.ks, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, j, kg, x) = S.Bxyz(i, j, G.ks, x);
                }
            for (int j = G.jsg; j <= G.jeg + 1; j++)
                for (int i = G.isg; i <= G.ieg + 1; i++)
                    for (int x = 0; x < 3; x++) S.magFlux(i, j, kg, x) = S.magFlux(i, j, G.ks, x);
        }
        return;
    }
    for (int j = G.jsg; j <= G.jeg + 1; j++)
        for (int i = G.isg; i <= G.ieg + 1; i++)
            for (int n = 1; n <= 4; n++) {
                int kg = G.ks - n, ks2 = G.ke - n + 1;
                if (isCellCenterG(G, i, j, kg)) {
                    for (int v = 0; v < NVAR; v++) S.Gas(i, j, kg, v) = S.Gas(i, j, ks2, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, j, kg, x) = S.Bxyz(i, j, ks2, x);
                }
                for (int x = 0; x < 3; x++) S.magFlux(i, j, kg, x) = S.magFlux(i, j, ks2, x);
            }
}
static void periodic_obcK(const Model& M, const Grid& G, State& S) {
    if (M.do25D) {
        for (int n = 1; n <= 4; n++) {
            int kg = G.ks + n;
            for (int j = G.jsg; j <= G.jeg; j++)
                for (int i = G.isg; i <= G.ieg; i++) {
                    for (int v = 0; v < NVAR; v++) S.Gas(i, j, kg, v) = S.Gas(i, j, G.ks, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, j, kg, x) = S.Bxyz(i, j, G.ks, x);
                }
            for (int j = G.jsg; j <= G.jeg + 1; j++)
                for (int i = G.isg; i <= G.ieg + 1; i++)
                    for (int x = 0; x < 3; x++) S.magFlux(i, j, kg, x) = S.magFlux(i, j, G.ks, x);
        }
        return;
    }
    for (int j = G.jsg; j <= G.jeg + 1; j++)
        for (int i = G.isg; i <= G.ieg + 1; i++)
            for (int n = 1; n <= 4; n++) {
                int kg = G.ke + n, ks2 = G.ks + n - 1;
                if (isCellCenterG(G, i, j, kg)) {
                    for (int v = 0; v < NVAR; v++) S.Gas(i, j, kg, v) = S.Gas(i, j, ks2, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, j, kg, x) = S.Bxyz(i, j, ks2, x);
                }
                S.magFlux(i, j, kg, IDIR) = S.magFlux(i, j, ks2, IDIR);
                S.magFlux(i, j, kg, JDIR) = S.magFlux(i, j, ks2, JDIR);
                S.magFlux(i, j, kg + 1, KDIR) = S.magFlux(i, j, G.ks + n, KDIR);
            }
}
// step.F90:17-55 EnforceBCs (single domain: every boundary is owned)
static void SphIn(const Grid& G, State& S);
static void zeroGrad_ibcJ(const Grid& G, State& S);
static void zeroGrad_obcJ(const Grid& G, State& S);
static void WindBC(const Model& M, const Grid& G, State& S);
static void InflowBC(const Model& M, const Grid& G, State& S);
static void zeroGrad_obcI(const Grid& G, State& S);
static void IonInner(const Model& M, const Grid& G, State& S);
static void lfmPole(const Grid& G, State& S, int p);
static void EnforceBCs(const Model& M, const Grid& G, State& S) {
    if (G.bc[0] == BC_PERIODIC) periodic_ibcI(G, S);
    else if (G.bc[0] == BC_SPHIN) SphIn(G, S);
    else if (G.bc[0] == BC_INFLOW) InflowBC(M, G, S);
    else if (G.bc[0] == BC_ION) IonInner(M, G, S);
    if (G.bc[1] == BC_PERIODIC) periodic_obcI(G, S);
    else if (G.bc[1] == BC_WIND) WindBC(M, G, S);
    else if (G.bc[1] == BC_ZEROGRAD) zeroGrad_obcI(G, S);
    if (G.bc[2] == BC_PERIODIC) periodic_ibcJ(G, S);
    else if (G.bc[2] == BC_ZEROGRAD) zeroGrad_ibcJ(G, S);
    else if (G.bc[2] == BC_LFM) lfmPole(G, S, 0);
    if (G.bc[3] == BC_PERIODIC) periodic_obcJ(G, S);
    else if (G.bc[3] == BC_ZEROGRAD) zeroGrad_obcJ(G, S);
    else if (G.bc[3] == BC_LFM) lfmPole(G, S, 1);
    if (G.bc[4] == BC_PERIODIC) periodic_ibcK(M, G, S);
    if (G.bc[5] == BC_PERIODIC) periodic_obcK(M, G, S);
}


// ---------------------------------------------------------------- ionosphere
// The ionospheric inner boundary of the magnetosphere and its model hooks,
// as voltron/ICs/earthcmi.F90 sets them up (the reference's default Voltron
// IC file), for a grid without rings (Model%Ring%doS = doE = F): PsiSh = 5,
// PsiSt = -3 (cmidefs.F90:13-14); single fluid, no ingestion.
static const int PsiSh = 5, PsiSt = -3;
static double inExyz(const Model& M, const Grid& G, int s, int j, int k, int x) {  // s = 1..PsiSh
    const long nj = G.jeg - G.jsg + 1, nk = G.keg - G.ksg + 1;
    return M.ion.inExyz[(s - 1) + PsiSh * ((j - G.jsg) + nj * ((k - G.ksg) + nk * x))];
}
static double inEijk(const Model& M, const Grid& G, int s, int j, int k, int x) {  // s = 1..PsiSh+1
    const long nj = G.jeg - G.jsg + 2, nk = G.keg - G.ksg + 2;
    return M.ion.inEijk[(s - 1) + (PsiSh + 1) * ((j - G.jsg) + nj * ((k - G.ksg) + nk * x))];
}
// ringutils.F90:482-518 lfmIJKcc: k into the active range; with rings, a
// ghost j across the pole maps to its conjugate (mirrored j, k + Np/2)
static void lfmIJKcc(const Grid& G, int i, int j, int k, int& ip, int& jp, int& kp) {
    const int Np = G.Nkp;
    ip = i;
    if (k < G.ks) kp = k + Np;
    else if (k > G.ke) kp = k - Np;
    else kp = k;
    jp = j;
    if (G.ring.doS && j < G.js) {
        jp = G.js + (G.js - j) - 1;
        kp = WrapK(k, Np);
    }
    if (G.ring.doE && j > G.je) {
        jp = G.je - (j - G.je) + 1;
        kp = WrapK(k, Np);
    }
}
// math.F90:265-274 cross, :332-343 normVec, :365-376 Vec2Perp
static void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static void normVec3(const double* a, double* n) {
    const double nA = std::sqrt(dot3(a, a));
    for (int x = 0; x < 3; x++) n[x] = nA <= TINY ? 0.0 : a[x] / nA;
}
static void Vec2Perp(const double* A, const double* n, double* P) {
    const double d = dot3(A, n);
    for (int x = 0; x < 3; x++) P[x] = A[x] - d * n[x];
}
static void Dipole(double M0, const double* r, double* A);
// E x B / |B|^2 in the dipole at xyz (earthcmi.F90:484-490, 624-629)
static void ExB(const Model& M, const double* xyz, const double* E, double* Veb) {
    double Bd[3], c[3];
    Dipole(M.ion.M0, xyz, Bd);
    cross3(E, Bd, c);
    const double bb = dot3(Bd, Bd);
    for (int x = 0; x < 3; x++) Veb[x] = c[x] / bb;
}
// msphingest.F90:268-372 CellPlasmaBC, single fluid without ingestion data:
// the active cell's density and pressure, the E x B velocity perpendicular
// to the radius plus the inward part of its radial component
static void CellPlasmaBC(const Model& M, double* gU, const double* pU, const double* Veb, const double* rHat) {
    double pW[5], gW[5] = {0, 0, 0, 0, 0}, Vp[3];
    const double Vr = dot3(Veb, rHat);
    CellC2P(M, pU, pW);
    gW[DEN] = pW[DEN];
    gW[PRESSURE] = pW[PRESSURE];
    Vec2Perp(Veb, rHat, Vp);
    const double vin = std::min(Vr, 0.0);
    for (int x = 0; x < 3; x++) gW[VELX + x] = Vp[x] + vin * rHat[x];
    CellP2C(M, gW, gU);
}
// earthcmi.F90:441-583 IonInner (rings off)
static void IonInner(const Model& M, const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int j = G.jsg; j <= G.jeg + 1; j++)
            for (int n = 1; n <= 4; n++) {
                const int ig = G.is - n, ip = G.is + n - 1, np = 4 - n + 1;
                if (k <= G.keg && j <= G.jeg) {  // isCellCenterG
                    int idip, jp, kp;
                    lfmIJKcc(G, ig, j, k, idip, jp, kp);
                    const double xc[3] = {G.xyzcc(idip, jp, kp, XDIR), G.xyzcc(idip, jp, kp, YDIR),
                                          G.xyzcc(idip, jp, kp, ZDIR)};
                    const double E[3] = {inExyz(M, G, np, jp, kp, 0), inExyz(M, G, np, jp, kp, 1),
                                         inExyz(M, G, np, jp, kp, 2)};
                    double Veb[3], rHat[3], gU[5], pU[5];
                    ExB(M, xc, E, Veb);
                    normVec3(xc, rHat);
                    for (int v = 0; v < NVAR; v++) pU[v] = S.Gas(ip, jp, kp, v);
                    CellPlasmaBC(M, gU, pU, Veb, rHat);
                    for (int v = 0; v < NVAR; v++) S.Gas(ig, j, k, v) = gU[v];
                }
                // isGoodFaceIJK (gridutils.F90:985-1015): the faces of the box
                if (j <= G.jeg && k <= G.keg) S.magFlux(ig, j, k, IDIR) = 0.0;
                if (k <= G.keg) S.magFlux(ig, j, k, JDIR) = 0.0;
                if (j <= G.jeg) S.magFlux(ig, j, k, KDIR) = 0.0;
            }
    // Bxyz of each ghost from the fluxes of its conjugate cell (:530-543)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int n = 1; n <= 4; n++) {
                const int ig = G.is - n;
                int ip, jp, kp;
                lfmIJKcc(G, ig, j, k, ip, jp, kp);
                double B[3];
                gamCellBxyz(G, S.magFlux, ip, jp, kp, B);
                for (int x = 0; x < 3; x++) S.Bxyz(ig, j, k, x) = B[x];
            }
    // the ghosts across the pole take their conjugate's Bxyz (:545-572)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int i = G.isg; i <= G.is - 1; i++)
            for (int n = 1; n <= 4; n++) {
                int ip, jp, kp;
                if (G.ring.doS) {
                    lfmIJKcc(G, i, G.js - n, k, ip, jp, kp);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, G.js - n, k, x) = S.Bxyz(ip, jp, kp, x);
                }
                if (G.ring.doE) {
                    lfmIJKcc(G, i, G.je + n, k, ip, jp, kp);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, G.je + n, k, x) = S.Bxyz(ip, jp, kp, x);
                }
            }
}
// HackE = EFix (earthcmi.F90:321-354): IonEFix (msphutils.F90:214-240),
// WindEFix with the wind outside (below), then FixEFieldLFM
// (gamdebug.F90:149-175)
static void IonEFix(const Model& M, const Grid& G, State& S) {
    if (PsiSh + PsiSt >= 1) {  // the inner tile holds shell is = 1
        const int is0 = 1 - PsiSt + 1;
        for (int k = G.ksg; k <= G.keg; k++)
            for (int j = G.jsg; j <= G.jeg; j++) {
                S.Efld(G.is, j, k, JDIR) = G.edge(G.is, j, k, JDIR) * inEijk(M, G, is0, j, k, 1);
                S.Efld(G.is, j, k, KDIR) = G.edge(G.is, j, k, KDIR) * inEijk(M, G, is0, j, k, 2);
            }
    }
}
static void FixEFieldLFM(const Grid& G, F4& E) {
    for (int j = G.js; j <= G.je + 1; j++)
        for (int i = G.is; i <= G.ie + 1; i++) {
            const double Ei = 0.5 * (E(i, j, G.ks, IDIR) + E(i, j, G.ke + 1, IDIR));
            const double Ej = 0.5 * (E(i, j, G.ks, JDIR) + E(i, j, G.ke + 1, JDIR));
            E(i, j, G.ks, IDIR) = Ei;
            E(i, j, G.ke + 1, IDIR) = Ei;
            E(i, j, G.ks, JDIR) = Ej;
            E(i, j, G.ke + 1, JDIR) = Ej;
        }
}

// ---------------------------------------------------------------- ring averaging
// Ring averaging about the LFM axis (ringav.F90, ringrecon.F90, ringutils.F90
// for Model%Ring%GridID = "lfm"): rings are the k circles of the first NumR
// j rows next to each pole, sliced by i; with the reference's defaults
// (doShift, doVClean, doMassRA and multifluid off; NFTVEL unused).
enum { SPOLE = 1, EPOLE = 2 };
static const int NFTMAX = 2;
// ringav.F90:394-430 PoleE: K EMFs on the pole zero, I EMFs on the pole
// their ring mean, then FixEFieldLFM
static void PoleE(const Grid& G, F4& E) {
    const int Np = G.ring.Np;
    const int jp[2] = {G.js, G.je + 1};
    const bool on[2] = {G.ring.doS, G.ring.doE};
    for (int nS = G.is; nS <= G.ie + 1; nS++)
        for (int p = 0; p < 2; p++) {
            if (!on[p]) continue;
            for (int k = G.ksg; k <= G.keg; k++) E(nS, jp[p], k, KDIR) = 0.0;
            double s = 0.0;
            for (int k = G.ks; k <= G.ke; k++) s = s + E(nS, jp[p], k, IDIR);
            const double avg = s / Np;
            for (int k = G.ksg; k <= G.keg; k++) E(nS, jp[p], k, IDIR) = avg;
        }
    FixEFieldLFM(G, E);
}
// math.F90:192-197 minmod (sign() as copysign, min() as a < b)
static inline double fmin2(double a, double b) { return b < a ? b : a; }
static inline double minmod(double x, double y) {
    return 0.5 * (std::copysign(1.0, x) + std::copysign(1.0, y)) * fmin2(std::fabs(x), std::fabs(y));
}
// ringrecon.F90:251-285 PPM_IntLR, :235-249 PLM_IntLR, :224-232 PCM_IntLR
static void RingLR(int recon, double fm2, double fm1, double f, double fp1, double fp2, double& vm, double& vp) {
    if (recon == 2) {
        vm = f;
        vp = f;
        return;
    }
    if (recon == 1) {
        const double dwL = f - fm1, dwR = fp1 - f, dwC = (fp1 - fm1) / 2.0;
        const double min1 = fmin2(2 * std::fabs(dwL), 2 * std::fabs(dwR));
        const double min2 = fmin2(min1, std::fabs(dwC));
        const double dwM = std::copysign(min2, dwC);
        vp = f + 0.5 * dwM;
        vm = f - 0.5 * dwM;
        return;
    }
    const double dvm2 = fm1 - fm2, dvm1 = f - fm1, dvp1 = fp1 - f, dvp2 = fp2 - fp1;
    double dvc = 0.5 * (dvm2 + dvm1), SM = 2.0 * minmod(dvm2, dvm1);
    const double Sm1 = minmod(dvc, SM);
    dvc = 0.5 * (dvm1 + dvp1);
    SM = 2.0 * minmod(dvm1, dvp1);
    const double Sp1 = minmod(dvc, SM);
    dvc = 0.5 * (dvp2 + dvp1);
    SM = 2.0 * minmod(dvp2, dvp1);
    const double Sp2 = minmod(dvc, SM);
    vp = 0.5 * (f + fp1) - (Sp2 - Sp1) / 6.0;
    vm = 0.5 * (f + fm1) - (Sp1 - Sm1) / 6.0;
    double ap = vp - f, am = vm - f;
    if (ap * am >= 0.0) {
        ap = 0.0;
        am = 0.0;
    } else {
        if (std::fabs(ap) >= 2.0 * std::fabs(am)) ap = -2.0 * am;
        if (std::fabs(am) >= 2.0 * std::fabs(ap)) am = -2.0 * ap;
    }
    vp = f + ap;
    vm = f + am;
}
// ringrecon.F90:34-91 ReconstructRing: the chunk values (each chunk's first
// element, all equal after chunk averaging) with 2 periodic ghosts, an
// interval L/R per chunk, and the parabola's cell averages within it
static void ReconstructRing(const Grid& G, double* rW, int Nc) {
    const int Np = G.ring.Np, dJ = Np / Nc, Ng = 2;
    std::vector<double> chW(Nc + 2 * Ng);
    auto ch = [&](int n) -> double& { return chW[n - 1 + Ng]; };  // n = 1-Ng .. Nc+Ng
    for (int n = 1; n <= Nc; n++) ch(n) = rW[(n - 1) * dJ];
    for (int n = 1; n <= Ng; n++) {
        ch(1 - n) = ch(Nc - n + 1);
        ch(Nc + n) = ch(n);
    }
    for (int n = 1; n <= Nc; n++) {
        const int mS = 1 + (n - 1) * dJ;
        double fL, fR;
        RingLR(G.ring.recon, ch(n - 2), ch(n - 1), ch(n), ch(n + 1), ch(n + 2), fL, fR);
        const double f = ch(n);
        const double a = 3 * (fL + fR - 2 * f), b = 2 * (3 * f - fR - 2 * fL), c = fL;
        for (int m = 1; m <= dJ; m++) {
            const double fI = (a / 3.0) * (3 * m * m - 3 * m + 1) / (dJ * dJ) + 0.5 * b * (2 * m - 1) / dJ + c;
            rW[mS + m - 2] = fI;
        }
    }
}
// ringav.F90:433-493 CleanRing / DirtyRing: Fourier modes 0..numFT of a ring
// at the cell centres phi_n = (n - 1/2) 2 pi / Np removed and put back
static void CleanRing(const Grid& G, double* Q, double cFT[NFTMAX + 1][2], int numFT) {
    const int Np = G.ring.Np;
    for (int m = 0; m <= NFTMAX; m++) cFT[m][0] = cFT[m][1] = 0.0;
    const double aScl = (double)(2.0f / (float)Np), dp = 2.0 * PI / Np;  // 2.0/Np in default real
    for (int n = 1; n <= Np; n++) {
        const double phi = dp * n - 0.5 * dp;
        for (int m = 0; m <= numFT; m++) {
            cFT[m][0] = cFT[m][0] + Q[n - 1] * std::cos(1.0 * m * phi);
            cFT[m][1] = cFT[m][1] + Q[n - 1] * std::sin(1.0 * m * phi);
        }
    }
    for (int c = 0; c < 2; c++) cFT[0][c] = 0.5 * aScl * cFT[0][c];
    for (int m = 1; m <= numFT; m++)
        for (int c = 0; c < 2; c++) cFT[m][c] = 1.0 * aScl * cFT[m][c];
    for (int n = 1; n <= Np; n++) {
        const double phi = dp * n - 0.5 * dp;
        for (int m = 0; m <= numFT; m++)
            Q[n - 1] = Q[n - 1] - cFT[m][0] * std::cos(1.0 * m * phi) - cFT[m][1] * std::sin(1.0 * m * phi);
    }
}
static void DirtyRing(const Grid& G, double* Q, const double cFT[NFTMAX + 1][2], int numFT) {
    const int Np = G.ring.Np;
    const double dp = 2.0 * PI / Np;
    for (int n = 1; n <= Np; n++) {
        const double phi = dp * n - 0.5 * dp;
        for (int m = 0; m <= numFT; m++)
            Q[n - 1] = Q[n - 1] + cFT[m][0] * std::cos(1.0 * m * phi) + cFT[m][1] * std::sin(1.0 * m * phi);
    }
}
// ringav.F90:212-344 CalcSmoothE: per slice and ring, the face fluxes through
// the ring (J faces -> I EMFs, I faces -> J EMFs) cleaned of their low Fourier
// modes, chunk-averaged, reconstructed and dirtied again; the change of each
// face's flux accumulated along the chunk into the EMF that makes it
static void CalcSmoothE(const Grid& G, const State& S, F4& SmoothE, int pole) {
    const int Np = G.ring.Np;
    const int fDIRS[2] = {JDIR, IDIR}, eDIRS[2] = {IDIR, JDIR};
    const double eScls[2] = {1.0, -1.0};
    std::vector<double> bFlx(3 * Np), dEr(3 * Np), rFlx(Np), raFlx(Np), dFlx(Np);
    for (int nS = G.is; nS <= G.ie + 1; nS++)
        for (int nR = 1; nR <= G.ring.NumR; nR++) {
            const int NumCh = G.ring.Nch[nR - 1], dC = Np / NumCh;
            // PullRingI (ringutils.F90:760-800)
            for (int n = 0; n < Np; n++) {
                const int k = G.ks + n;
                if (pole == SPOLE) {
                    bFlx[n] = S.magFlux(nS, G.js + nR - 1, k, IDIR);
                    bFlx[Np + n] = S.magFlux(nS, G.js + nR, k, JDIR);
                    bFlx[2 * Np + n] = S.magFlux(nS, G.js + nR - 1, k, KDIR);
                } else {
                    for (int d = 0; d < 3; d++) bFlx[d * Np + n] = S.magFlux(nS, G.je - nR + 1, k, d);
                }
            }
            std::fill(dEr.begin(), dEr.end(), 0.0);
            for (int dd = 0; dd < 2; dd++) {
                const int fD = fDIRS[dd], eD = eDIRS[dd];
                const double eScl = eScls[dd];
                for (int n = 0; n < Np; n++) rFlx[n] = bFlx[fD * Np + n];
                double cFT[NFTMAX + 1][2];
                CleanRing(G, rFlx.data(), cFT, G.ring.NFTMAG);
                for (int c = 1; c <= NumCh; c++) {
                    const int lRs = 1 + (c - 1) * dC, lRe = lRs + dC - 1;
                    double s = 0.0;
                    for (int l = lRs; l <= lRe; l++) s = s + rFlx[l - 1];
                    for (int l = lRs; l <= lRe; l++) raFlx[l - 1] = s / dC;
                }
                ReconstructRing(G, raFlx.data(), NumCh);
                DirtyRing(G, raFlx.data(), cFT, G.ring.NFTMAG);
                for (int n = 0; n < Np; n++) dFlx[n] = raFlx[n] - bFlx[fD * Np + n];
                for (int c = 1; c <= NumCh; c++) {
                    const int lRs = 1 + (c - 1) * dC;
                    double cumFlx = -dFlx[lRs - 1];
                    for (int m = 2; m <= dC; m++) {
                        dEr[eD * Np + lRs + m - 2] = eScl * cumFlx;
                        cumFlx = cumFlx - dFlx[lRs + m - 2];
                    }
                }
            }
            for (int n = 0; n < Np; n++) {
                const int k = G.ks + n;
                if (pole == SPOLE) {
                    SmoothE(nS, G.js + nR, k, IDIR) = dEr[n];
                    SmoothE(nS, G.js + nR - 1, k, JDIR) = dEr[Np + n];
                    SmoothE(nS, G.js + nR - 1, k, KDIR) = dEr[2 * Np + n];
                } else {
                    for (int d = 0; d < 3; d++) SmoothE(nS, G.je - nR + 1, k, d) = dEr[d * Np + n];
                }
            }
            if (pole == SPOLE) {
                SmoothE(nS, G.js + nR, G.ke + 1, IDIR) = SmoothE(nS, G.js + nR, G.ks, IDIR);
                SmoothE(nS, G.js + nR - 1, G.ke + 1, JDIR) = SmoothE(nS, G.js + nR - 1, G.ks, JDIR);
            } else {
                SmoothE(nS, G.je - nR + 1, G.ke + 1, IDIR) = SmoothE(nS, G.je - nR + 1, G.ks, IDIR);
                SmoothE(nS, G.je - nR + 1, G.ke + 1, JDIR) = SmoothE(nS, G.je - nR + 1, G.ks, JDIR);
            }
        }
}
// ringav.F90:347-391 CleanLoops: the K flux through the first ring's cells
// (the faces around the pole) loses its ring mean
static void CleanLoops(const Grid& G, State& S) {
    const int Np = G.ring.Np;
    const double tScl = G.ring.doFast ? 1.0 : (double)(1.0f / (float)Np);  // 1.0/Np in default real
    const int jr[2] = {G.js, G.je};
    const bool on[2] = {G.ring.doS, G.ring.doE};
    for (int nS = G.is; nS <= G.ie + 1; nS++)
        for (int p = 0; p < 2; p++) {
            if (!on[p]) continue;
            double s = 0.0;
            for (int k = G.ks; k <= G.ke; k++) s = s + S.magFlux(nS, jr[p], k, KDIR);
            const double avgFlx = s / Np;
            for (int k = G.ks; k <= G.ke + 1; k++)
                S.magFlux(nS, jr[p], k, KDIR) = S.magFlux(nS, jr[p], k, KDIR) - tScl * avgFlx;
        }
}
// ringutils.F90:804-856 Gas2Ring / Ring2Gas (doMassRA = F: rho, momentum,
// internal energy)
static void Gas2Ring(const Model& M, double* W) {
    const double D = std::max(W[DEN], dFloor);
    const double KinE = 0.5 * (W[MOMX] * W[MOMX] + W[MOMY] * W[MOMY] + W[MOMZ] * W[MOMZ]) / D;
    const double P = std::max((M.gamma - 1) * (W[ENERGY] - KinE), pFloor);
    W[DEN] = D;
    W[ENERGY] = P / (M.gamma - 1);
}
static void Ring2Gas(const Model& M, double* W) {
    const double D = std::max(W[DEN], dFloor);
    double P = (M.gamma - 1) * W[ENERGY];
    P = std::max(P, pFloor);
    const double KinE = 0.5 * (W[MOMX] * W[MOMX] + W[MOMY] * W[MOMY] + W[MOMZ] * W[MOMZ]) / D;
    W[DEN] = D;
    W[ENERGY] = KinE + P / (M.gamma - 1);
}
// ringav.F90:78-210 SmoothGas: per slice and ring the ring variables are
// chunk-averaged and reconstructed, then written back as gas
static void SmoothGas(const Model& M, const Grid& G, State& S, int pole) {
    const int Np = G.ring.Np;
    std::vector<double> rW(NVAR * Np), raW(NVAR * Np);
    for (int nS = G.is; nS <= G.ie; nS++)
        for (int nR = 1; nR <= G.ring.NumR; nR++) {
            const int NumCh = G.ring.Nch[nR - 1], dC = Np / NumCh;
            const int jr = pole == SPOLE ? G.js + nR - 1 : G.je - nR + 1;
            for (int n = 0; n < Np; n++) {
                double W[NVAR];
                for (int v = 0; v < NVAR; v++) W[v] = S.Gas(nS, jr, G.ks + n, v);
                Gas2Ring(M, W);
                for (int v = 0; v < NVAR; v++) rW[v * Np + n] = W[v];
            }
            for (int v = 0; v < NVAR; v++)
                for (int c = 1; c <= NumCh; c++) {
                    const int lRs = 1 + (c - 1) * dC, lRe = lRs + dC - 1;
                    double s = 0.0;
                    for (int l = lRs; l <= lRe; l++) s = s + rW[v * Np + l - 1];
                    for (int l = lRs; l <= lRe; l++) raW[v * Np + l - 1] = s / dC;
                }
            for (int v = 0; v < NVAR; v++) ReconstructRing(G, raW.data() + v * Np, NumCh);
            for (int n = 0; n < Np; n++) {
                double W[NVAR];
                for (int v = 0; v < NVAR; v++) W[v] = raW[v * Np + n];
                Ring2Gas(M, W);
                for (int v = 0; v < NVAR; v++) S.Gas(nS, jr, G.ks + n, v) = W[v];
            }
        }
}
// ringav.F90:26-75 RingAverage (after the update, mhdgroup.F90:69-74)
static void RingAverage(const Model& M, const Grid& G, State& S, F4& SmoothE) {
    SmoothE.fill(0.0);
    if (G.ring.doS) CalcSmoothE(G, S, SmoothE, SPOLE);
    if (G.ring.doE) CalcSmoothE(G, S, SmoothE, EPOLE);
    PoleE(G, SmoothE);
    E2Flux(G, S.magFlux, SmoothE, 1.0);
    if (G.ring.doClean) CleanLoops(G, S);
    bFlux2Fld(G, S.magFlux, S.Bxyz);
    if (G.ring.doS) SmoothGas(M, G, S, SPOLE);
    if (G.ring.doE) SmoothGas(M, G, S, EPOLE);
}
// ringutils.F90:242-391 RingGridFix: the CFL length along k of ring cells
// scaled by their chunk size, the ghost metric across the pole taken from the
// conjugate cells and faces (J and K face normals reversed)
static void RingGridFix(Grid& G) {
    const Grid::Ring& R = G.ring;
    for (int iR = 1; iR <= R.NumR; iR++) {
        const int dJ = R.Np / R.Nch[iR - 1];
        for (int k = G.ksg; k <= G.keg; k++)
            for (int i = G.isg; i <= G.ieg; i++) {
                if (R.doS) G.dk(i, G.js + iR - 1, k) = dJ * G.dk(i, G.js + iR - 1, k);
                if (R.doE) G.dk(i, G.je - iR + 1, k) = dJ * G.dk(i, G.je - iR + 1, k);
            }
    }
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int i = G.isg; i <= G.ieg + 1; i++)
            for (int n = 1; n <= 4; n++)
                for (int p = 0; p < 2; p++) {
                    if (!(p == 0 ? R.doS : R.doE)) continue;
                    const int jg = p == 0 ? G.js - n : G.je + n;
                    int ip, jp, kp;
                    if (k <= G.keg && i <= G.ieg) {
                        lfmIJKcc(G, i, jg, k, ip, jp, kp);
                        G.volume(i, jg, k) = G.volume(ip, jp, kp);
                        G.di(i, jg, k) = G.di(ip, jp, kp);
                        G.dj(i, jg, k) = G.dj(ip, jp, kp);
                        G.dk(i, jg, k) = G.dk(ip, jp, kp);
                    }
                    for (int d = 0; d < 3; d++) {
                        const int jf = (d == JDIR && p == 1) ? jg + 1 : jg;  // the E side's first ghost J face
                        const double sg = d == IDIR ? 1.0 : -1.0;
                        lfmIJKfc(G, d, i, jf, k, ip, jp, kp);
                        for (int x = 0; x < 3; x++)
                            G.Tf(i, jf, k, NORMX + x + 9 * d) = sg * G.Tf(ip, jp, kp, NORMX + x + 9 * d);
                        G.face(i, jf, k, d) = G.face(ip, jp, kp, d);
                    }
                }
}
// bcs.F90:1019-1106 lfmIn / lfmOut: ghost cells across the pole take their
// conjugate's gas and Bxyz, ghost faces its flux (J and K fluxes reversed)
static void lfmPole(const Grid& G, State& S, int p) {
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int i = G.isg; i <= G.ieg + 1; i++)
            for (int n = 1; n <= 4; n++) {
                const int jg = p == 0 ? G.js - n : G.je + n;
                int ip, jp, kp;
                if (isCellCenterG(G, i, jg, k)) {
                    lfmIJKcc(G, i, jg, k, ip, jp, kp);
                    for (int v = 0; v < NVAR; v++) S.Gas(i, jg, k, v) = S.Gas(ip, jp, kp, v);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, jg, k, x) = S.Bxyz(ip, jp, kp, x);
                }
                lfmIJKfc(G, IDIR, i, jg, k, ip, jp, kp);
                S.magFlux(i, jg, k, IDIR) = S.magFlux(ip, jp, kp, IDIR);
                const int jf = p == 0 ? jg : jg + 1;
                lfmIJKfc(G, JDIR, i, jf, k, ip, jp, kp);
                S.magFlux(i, jf, k, JDIR) = -S.magFlux(ip, jp, kp, JDIR);
                lfmIJKfc(G, KDIR, i, jg, k, ip, jp, kp);
                S.magFlux(i, jg, k, KDIR) = -S.magFlux(ip, jp, kp, KDIR);
            }
}
// HackStep = PerStep (earthcmi.F90:224-263): PushIon (:586-663), then
// NudgeSW with the wind outside (below)
static void PushIon(const Model& M, const Grid& G, State& S) {
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.is + M.ion.nIonP - 1; i++) {
                const double xcc[3] = {G.xyzcc(i, j, k, XDIR), G.xyzcc(i, j, k, YDIR), G.xyzcc(i, j, k, ZDIR)};
                const double E[3] = {inExyz(M, G, PsiSh, j, k, 0), inExyz(M, G, PsiSh, j, k, 1),
                                     inExyz(M, G, PsiSh, j, k, 2)};
                double Veb[3], rHat[3], Vp[3], pCon[5], pW[5];
                ExB(M, xcc, E, Veb);
                normVec3(xcc, rHat);
                Vec2Perp(Veb, rHat, Vp);
                for (int v = 0; v < NVAR; v++) pCon[v] = S.Gas(i, j, k, v);
                CellC2P(M, pCon, pW);
                if (pCon[DEN] < 0.0) continue;  // RhoMin(BLK) = 0
                const int dN = i - G.is + 1;
                double dt = M.dt / (dN * M.ion.dtCpl);
                dt = std::min(dt, 1.0);
                for (int x = 0; x < 3; x++) {
                    const double dV = Vp[x] - pW[VELX + x];
                    pW[VELX + x] = pW[VELX + x] + dt * dV;
                }
                CellP2C(M, pW, pCon);
                for (int v = 0; v < NVAR; v++) S.Gas(i, j, k, v) = pCon[v];
            }
}

// The wind's part of the same hooks, for the constant wind (a series of
// constant rows with ByC = BzC = 0, so RefreshWind's front velocity is
// (-|V|, 0, 0)): WindEFix (apps/wind.F90:489-566) with DiffuseOuter
// (:570-616, doSWDiffuse = T) in HackE, NudgeSW (:394-486) in HackStep.
static double wgtWind(const double* V, const double* xyz);
static double Con2Fast(const Model& M, const double* gCon, const double* B);
static void DiffuseOuter(const Model& M, const Grid& G, const State& S, int i, int j, int k, double vSW, double* Ed) {
    double Jd[3] = {0.0, 0.0, 0.0};
    double bP = S.magFlux(i, j, k, JDIR) / std::max(G.face(i, j, k, JDIR), TINY);
    double bM = S.magFlux(i - 1, j, k, JDIR) / std::max(G.face(i - 1, j, k, JDIR), TINY);
    double db2 = bP - bM;
    bP = S.magFlux(i, j, k, IDIR) / G.face(i, j, k, IDIR);
    bM = S.magFlux(i, j - 1, k, IDIR) / G.face(i, j - 1, k, IDIR);
    double db1 = bP - bM;
    Jd[KDIR] = db2 - db1;
    bP = S.magFlux(i, j, k, IDIR) / G.face(i, j, k, IDIR);
    bM = S.magFlux(i, j, k - 1, IDIR) / G.face(i, j, k - 1, IDIR);
    db2 = bP - bM;
    bP = S.magFlux(i, j, k, KDIR) / G.face(i, j, k, KDIR);
    bM = S.magFlux(i - 1, j, k, KDIR) / G.face(i - 1, j, k, KDIR);
    db1 = bP - bM;
    Jd[JDIR] = db2 - db1;
    const double dl = std::sqrt(G.edge(i, j, k, JDIR) * G.edge(i, j, k, KDIR));
    const double Vd = std::min(vSW, M.CFL * dl / M.dt);
    Ed[IDIR] = 0.0;
    Ed[JDIR] = Vd * Jd[JDIR] * dl;
    Ed[KDIR] = Vd * Jd[KDIR] * dl;
}
static void WindEFix(const Model& M, const Grid& G, State& S) {
    const double V[3] = {M.wind[2], M.wind[3], M.wind[4]}, B[3] = {M.wind[5], M.wind[6], M.wind[7]};
    const double vFr[3] = {-norm2s(V, 3), 0.0, 0.0};
    const double vSW = std::min(norm2s(vFr, 3), M.doBoris ? M.Ca : HUGE_);
    double c[3], swE[3];
    cross3(V, B, c);
    for (int x = 0; x < 3; x++) swE[x] = -c[x];
    for (int k = G.ks; k <= G.ke + 1; k++)
        for (int j = G.js; j <= G.je + 1; j++)
            for (int i = G.ie - 2; i <= G.ie + 1; i++) {
                double wSW = 0.0;
                for (int n = 0; n < 3; n++) {
                    const int i2 = n == IDIR ? i + 1 : i, j2 = n == JDIR ? j + 1 : j, k2 = n == KDIR ? k + 1 : k;
                    double e1[3], e2[3], ecc[3], de[3];
                    for (int x = 0; x < 3; x++) {
                        e1[x] = G.xyz(i, j, k, x);
                        e2[x] = G.xyz(i2, j2, k2, x);
                        ecc[x] = 0.5 * (e1[x] + e2[x]);
                        de[x] = e2[x] - e1[x];
                    }
                    wSW = wgtWind(V, ecc);
                    if (wSW > TINY) {
                        if (i <= G.ie) wSW = wSW / (1.0 + G.ie + 1 - i);
                        const double mhdE = S.Efld(i, j, k, n);
                        S.Efld(i, j, k, n) = (1.0 - wSW) * mhdE + wSW * dot3(swE, de);
                    }
                }
                if (i == G.ie + 1) {
                    double Ed[3];
                    DiffuseOuter(M, G, S, i, j, k, vSW, Ed);
                    for (int x = 0; x < 3; x++) S.Efld(i, j, k, x) = S.Efld(i, j, k, x) + wSW * Ed[x];
                }
            }
    if (G.ring.on) {  // the pole's EMFs of these shells (:549-564)
        const int jp[2] = {G.je + 1, G.js};
        const bool on[2] = {G.ring.doE, G.ring.doS};
        for (int n = G.ie - 2; n <= G.ie + 1; n++)
            for (int p = 0; p < 2; p++) {
                if (!on[p]) continue;
                double s = 0.0;
                for (int k = G.ks; k <= G.ke; k++) s = s + S.Efld(n, jp[p], k, IDIR);
                const double avgEi = s / G.ring.Np;
                for (int k = G.ksg; k <= G.keg; k++) {
                    S.Efld(n, jp[p], k, IDIR) = avgEi;
                    S.Efld(n, jp[p], k, KDIR) = 0.0;
                }
            }
    }
}
static void NudgeSW(const Model& M, const Grid& G, State& S) {
    const double V[3] = {M.wind[2], M.wind[3], M.wind[4]};
    const int ip = G.ie;
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++) {
            const double xcc[3] = {G.xyzcc(ip, j, k, XDIR), G.xyzcc(ip, j, k, YDIR), G.xyzcc(ip, j, k, ZDIR)};
            const double wSW = wgtWind(V, xcc);
            if (wSW > TINY) {
                const double dtSW = std::max(M.ion.dtSW0 / wSW, M.dt);
                const double gW_sw[5] = {M.wind[0], M.wind[2], M.wind[3], M.wind[4], M.wind[1]};
                double gCon[5], gW_mhd[5], gW[5];
                for (int v = 0; v < NVAR; v++) gCon[v] = S.Gas(ip, j, k, v);
                CellC2P(M, gCon, gW_mhd);
                for (int v = 0; v < NVAR; v++) gW[v] = gW_mhd[v] + (M.dt / dtSW) * (gW_sw[v] - gW_mhd[v]);
                CellP2C(M, gW, gCon);
                for (int v = 0; v < NVAR; v++) S.Gas(ip, j, k, v) = gCon[v];
            }
        }
    if (G.ring.on && G.ring.doE) {  // the small ring about the axis flows out (:458-484)
        for (int k = G.ks; k <= G.ke; k++)
            for (int n = 0; n <= 1; n++) {
                const int i = G.ie, j = G.je + n;
                if (S.Gas(i, j, k, MOMX) > 0) {
                    double gCon[5], gW[5], B[3];
                    for (int v = 0; v < NVAR; v++) gCon[v] = S.Gas(i, j, k, v);
                    for (int x = 0; x < 3; x++) B[x] = S.Bxyz(i, j, k, x);
                    const double Cx = Con2Fast(M, gCon, B);
                    CellC2P(M, gCon, gW);
                    gW[VELX] = -Cx;
                    CellP2C(M, gW, gCon);
                    for (int v = 0; v < NVAR; v++) S.Gas(i, j, k, v) = gCon[v];
                }
            }
    }
}

// ---------------------------------------------------------------- dt
// gridutils.F90:49-106 CellDT (single fluid, no resistivity, no Boris)
static inline double CellDT(const Model& M, const Grid& G, const State& S, int i, int j, int k) {
    double rho = S.Gas(i, j, k, DEN);
    double Vx = S.Gas(i, j, k, MOMX) / rho, Vy = S.Gas(i, j, k, MOMY) / rho, Vz = S.Gas(i, j, k, MOMZ) / rho;
    double MagV = std::sqrt(Vx * Vx + Vy * Vy + Vz * Vz);
    double ke = 0.5 * rho * (MagV * MagV);
    double e = S.Gas(i, j, k, ENERGY) - ke;
    double P = (M.gamma - 1) * e;
    double Cs = std::sqrt(M.gamma * P / rho);
    double Vfl = MagV, Valf = 0.0, Vdiff = 0.0;
    if (M.doMHD) {
        double Bx = S.Bxyz(i, j, k, XDIR), By = S.Bxyz(i, j, k, YDIR), Bz = S.Bxyz(i, j, k, ZDIR);
        if (M.doBackground) {
            Bx = Bx + G.B0(i, j, k, XDIR);
            By = By + G.B0(i, j, k, YDIR);
            Bz = Bz + G.B0(i, j, k, ZDIR);
        }
        double MagB = std::sqrt(Bx * Bx + By * By + Bz * Bz);
        Valf = MagB / std::sqrt(rho);
        if (M.doBoris) Valf = M.Ca * Valf / std::sqrt(M.Ca * M.Ca + Valf * Valf);  // gridutils.F90:91-93
    }
    double vCFL = Vfl + std::sqrt(Cs * Cs + Valf * Valf) + Vdiff;
    double dl = std::min(std::min(G.di(i, j, k), G.dj(i, j, k)), G.dk(i, j, k));
    return M.CFL * dl / vCFL;
}
enum { ST_OK = 0, ST_DT_BAD = 1, ST_DT_DISASTER = 2 };
// step.F90:58-168 CalcDT; failure cases return a status instead of stopping
static double CalcDT(Model& M, const Grid& G, const State& S, int* status) {
    *status = ST_OK;
    if (M.fixedTimestep) return M.dt;
    double dtOld = M.dt, dtMin = HUGE_;
#pragma omp parallel for collapse(2) reduction(min : dtMin)
    for (int k = G.ksDT; k <= G.keDT; k++)
        for (int j = G.jsDT; j <= G.jeDT; j++)
            for (int i = G.isDT; i <= G.ieDT; i++) dtMin = std::min(CellDT(M, G, S, i, j, k), dtMin);
    bool isDisaster = (dtMin == HUGE_), isBad = false;
    double dt = dtMin;
    if (M.ts > 0) {
        if (dtOld / dtMin >= 10) isBad = true;
        if (M.dt0 > TINY && dtMin / M.dt0 <= M.limDT0) isBad = true;
        if (dtMin <= TINY) isDisaster = true;
    }
    if (isDisaster) *status = ST_DT_DISASTER;
    else if (isBad) *status = ST_DT_BAD;
    if (M.t + dt > M.tFin) dt = std::max(M.tFin - M.t, TINY);
    if (M.dt0 > TINY && dt > 10.0 * M.dt0) dt = 10.0 * M.dt0;
    return dt;
}

// ---------------------------------------------------------------- geometry
// quadrature.F90:331-343 faceDeltas
static void faceDeltas(const double* f0, const double* f1, const double* f2, const double* f3, double* dx,
                       double* dy, double* dz) {
    dx[0] = f1[0] - f0[0]; dx[1] = f2[0] - f0[0]; dx[2] = f3[0] + f0[0] - f2[0] - f1[0];
    dy[0] = f1[1] - f0[1]; dy[1] = f2[1] - f0[1]; dy[2] = f3[1] + f0[1] - f2[1] - f1[1];
    dz[0] = f1[2] - f0[2]; dz[1] = f2[2] - f0[2]; dz[2] = f3[2] + f0[2] - f2[2] - f1[2];
}
// quadrature.F90:159-221 GaussianFaceIntegral for the two lazy integrands the
// metric needs (IdVec -> area, rVec -> first moment); metric.F90:302-327
static void GaussianFaceIntegral(const double* f0, const double* f1, const double* f2, const double* f3, bool rvec,
                                 double* fInt) {
    double dx[3], dy[3], dz[3];
    faceDeltas(f0, f1, f2, f3, dx, dy, dz);
    fInt[0] = fInt[1] = fInt[2] = 0.0;
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) {
            double eta = 0.5 * (1 + gA[i]), psi = 0.5 * (1 + gA[j]);
            double w = gWgt[i] * gWgt[j];
            double xp = f0[0] + dx[0] * eta + dx[1] * psi + dx[2] * eta * psi;
            double yp = f0[1] + dy[0] * eta + dy[1] * psi + dy[2] * eta * psi;
            double zp = f0[2] + dz[0] * eta + dz[1] * psi + dz[2] * eta * psi;
            double Ax = rvec ? xp : 1.0, Ay = rvec ? yp : 1.0, Az = rvec ? zp : 1.0;
            double etaV[3] = {dx[0] + dx[2] * psi, dy[0] + dy[2] * psi, dz[0] + dz[2] * psi};
            double psiV[3] = {dx[1] + dx[2] * eta, dy[1] + dy[2] * eta, dz[1] + dz[2] * eta};
            double c[3];
            cross(etaV, psiV, c);
            double area = 0.25 * norm2s(c, 3) * w;
            fInt[0] = fInt[0] + area * Ax;
            fInt[1] = fInt[1] + area * Ay;
            fInt[2] = fInt[2] + area * Az;
        }
}
static inline double DetJ(const double J[3][3]) {  // math.F90:470-478 (J[row][col])
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}
// quadrature.F90:42-100 GaussianVolumeIntegral; W(x,y,z) -> 5 values
template <class Fn>
static void GaussianVolumeIntegral(const double xyzC[8][3], Fn W, double* wInt) {
    static const int iS[8] = {-1, +1, +1, -1, -1, +1, +1, -1};
    static const int jS[8] = {-1, -1, +1, +1, -1, -1, +1, +1};
    static const int kS[8] = {-1, -1, -1, -1, +1, +1, +1, +1};
    for (int v = 0; v < 5; v++) wInt[v] = 0.0;
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++)
            for (int k = 0; k < 12; k++) {
                double wijk = gWgt[i] * gWgt[j] * gWgt[k];
                double iScl[8], jScl[8], kScl[8];
                for (int n = 0; n < 8; n++) {
                    iScl[n] = iS[n] < 0 ? 1 - gA[i] : 1 + gA[i];
                    jScl[n] = jS[n] < 0 ? 1 - gA[j] : 1 + gA[j];
                    kScl[n] = kS[n] < 0 ? 1 - gA[k] : 1 + gA[k];
                }
                double xp[3], Jac[3][3];
                for (int x = 0; x < 3; x++) {
                    double s = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                    for (int n = 0; n < 8; n++) s += xyzC[n][x] * (iScl[n] * jScl[n] * kScl[n]);
                    for (int n = 0; n < 8; n++) s1 += xyzC[n][x] * ((double)iS[n] * jScl[n] * kScl[n]);
                    for (int n = 0; n < 8; n++) s2 += xyzC[n][x] * (iScl[n] * (double)jS[n] * kScl[n]);
                    for (int n = 0; n < 8; n++) s3 += xyzC[n][x] * (iScl[n] * jScl[n] * (double)kS[n]);
                    xp[x] = 0.125 * s;
                    Jac[x][0] = 0.125 * s1;
                    Jac[x][1] = 0.125 * s2;
                    Jac[x][2] = 0.125 * s3;
                }
                double dJ = std::fabs(DetJ(Jac));
                double Wp[5];
                W(xp[0], xp[1], xp[2], Wp);
                for (int v = 0; v < 5; v++) wInt[v] = wInt[v] + dJ * wijk * Wp[v];
            }
}
static void cellCoords(const Grid& G, int i, int j, int k, double xyzC[8][3]) {  // metric.F90:153-171
    const int o[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int n = 0; n < 8; n++)
        for (int x = 0; x < 3; x++) xyzC[n][x] = G.xyz(i + o[n][0], j + o[n][1], k + o[n][2], x);
}
static void faceCoords(const Grid& G, int i, int j, int k, int d, double* f0, double* f1, double* f2,
                       double* f3) {  // metric.F90:98-128
    int a1[3], a2[3];
    if (d == IDIR) { int t1[3] = {0, 1, 0}, t2[3] = {0, 0, 1}; std::memcpy(a1, t1, 12); std::memcpy(a2, t2, 12); }
    else if (d == JDIR) { int t1[3] = {0, 0, 1}, t2[3] = {1, 0, 0}; std::memcpy(a1, t1, 12); std::memcpy(a2, t2, 12); }
    else { int t1[3] = {1, 0, 0}, t2[3] = {0, 1, 0}; std::memcpy(a1, t1, 12); std::memcpy(a2, t2, 12); }
    for (int x = 0; x < 3; x++) {
        f0[x] = G.xyz(i, j, k, x);
        f1[x] = G.xyz(i + a1[0], j + a1[1], k + a1[2], x);
        f2[x] = G.xyz(i + a2[0], j + a2[1], k + a2[2], x);
        f3[x] = G.xyz(i + a1[0] + a2[0], j + a1[1] + a2[1], k + a1[2] + a2[2], x);
    }
}
// init.F90:1075-1137 ebGeom
static void ebGeom(const Grid& G, F4& Teb, int c0, int dNorm, int dT1, int dT2) {
    int ie = G.ie + 1;
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke + 1; k++)
        for (int j = G.js; j <= G.je + 1; j++)
            for (int iB = G.is; iB <= ie; iB += vecLen) {
                int iMax = std::min((int)vecLen, ie - iB + 1);
                double fArB[recLen][vecLen], N[3][recLen][vecLen];
                loadBlock(G, G.face.comp(dT1), true, iB, j, k, iMax, dT2, Nr2, fArB);
                for (int x = 0; x < 3; x++) loadBlock(G, G.Tf.comp(NORMX + x + 9 * dT1), true, iB, j, k, iMax, dT2, Nr2, N[x]);
                for (int i = 0; i < iMax; i++) {
                    int iG = iB + i;
                    double fAi = 0.0;
                    for (int n = 0; n < recLen; n++) fAi += interpWgt6[n] * fArB[n][i];
                    double Nec[3];
                    for (int x = 0; x < 3; x++) {
                        double s = 0.0;
                        for (int n = 0; n < recLen; n++) s += (N[x][n][i] * fArB[n][i]) * interpWgt6[n];
                        Nec[x] = s / fAi;
                    }
                    double t1[3] = {G.Te(iG, j, k, TAN1X + 9 * dNorm), G.Te(iG, j, k, TAN1Y + 9 * dNorm),
                                    G.Te(iG, j, k, TAN1Z + 9 * dNorm)};
                    double t2[3] = {G.Te(iG, j, k, TAN2X + 9 * dNorm), G.Te(iG, j, k, TAN2Y + 9 * dNorm),
                                    G.Te(iG, j, k, TAN2Z + 9 * dNorm)};
                    double dxT = dot3(Nec, t1), dyT = dot3(Nec, t2);
                    double dScl = std::sqrt(dxT * dxT + dyT * dyT);
                    if (dScl <= TINY) dScl = 1.0;
                    Teb(iG, j, k, c0 + 0 + 4 * dNorm) = dxT / dScl;
                    Teb(iG, j, k, c0 + 1 + 4 * dNorm) = dyT / dScl;
                }
            }
}
static void RingGridFix(Grid& G);
// init.F90:793-1072 Corners2Grid
static void Corners2Grid(const Model& M, Grid& G) {
    G.cellArr(G.xyzcc, 3);
    G.faceArr(G.xfc, 9);
    G.faceArr(G.face, 3, 1.0);
    G.faceArr(G.Tf, 27);
    for (int d = 0; d < 3; d++) {
        int DelI = d == IDIR, DelJ = d == JDIR, DelK = d == KDIR;
#pragma omp parallel for collapse(2)
        for (int k = G.ksg; k <= G.keg + DelK; k++)
            for (int j = G.jsg; j <= G.jeg + DelJ; j++)
                for (int i = G.isg; i <= G.ieg + DelI; i++) {
                    double f0[3], f1[3], f2[3], f3[3], fInt[3];
                    faceCoords(G, i, j, k, d, f0, f1, f2, f3);
                    GaussianFaceIntegral(f0, f1, f2, f3, false, fInt);
                    double fA = fInt[0];
                    GaussianFaceIntegral(f0, f1, f2, f3, true, fInt);
                    for (int x = 0; x < 3; x++) G.xfc(i, j, k, x + 3 * d) = fInt[x] / fA;
                    G.face(i, j, k, d) = fA;
                    double dT1[3], dT2[3];
                    for (int x = 0; x < 3; x++) {
                        if (d == IDIR) {
                            dT1[x] = 0.5 * (G.xyz(i, j + 1, k + 1, x) - G.xyz(i, j, k + 1, x)) +
                                     0.5 * (G.xyz(i, j + 1, k, x) - G.xyz(i, j, k, x));
                            dT2[x] = 0.5 * (G.xyz(i, j + 1, k + 1, x) - G.xyz(i, j + 1, k, x)) +
                                     0.5 * (G.xyz(i, j, k + 1, x) - G.xyz(i, j, k, x));
                        } else if (d == JDIR) {
                            dT1[x] = 0.5 * (G.xyz(i + 1, j, k + 1, x) - G.xyz(i + 1, j, k, x)) +
                                     0.5 * (G.xyz(i, j, k + 1, x) - G.xyz(i, j, k, x));
                            dT2[x] = 0.5 * (G.xyz(i + 1, j, k + 1, x) - G.xyz(i, j, k + 1, x)) +
                                     0.5 * (G.xyz(i + 1, j, k, x) - G.xyz(i, j, k, x));
                        } else {
                            dT1[x] = 0.5 * (G.xyz(i + 1, j + 1, k, x) - G.xyz(i, j + 1, k, x)) +
                                     0.5 * (G.xyz(i + 1, j, k, x) - G.xyz(i, j, k, x));
                            dT2[x] = 0.5 * (G.xyz(i + 1, j + 1, k, x) - G.xyz(i + 1, j, k, x)) +
                                     0.5 * (G.xyz(i, j + 1, k, x) - G.xyz(i, j, k, x));
                        }
                    }
                    double c[3], eN[3], eT1[3], eT2[3], c2[3];
                    cross(dT1, dT2, c);
                    double nc = norm2s(c, 3);
                    for (int x = 0; x < 3; x++) eN[x] = c[x] / nc;
                    double n2 = norm2s(dT2, 3);
                    for (int x = 0; x < 3; x++) eT2[x] = dT2[x] / n2;
                    cross(eT2, eN, c2);
                    double nc2 = norm2s(c2, 3);
                    for (int x = 0; x < 3; x++) eT1[x] = c2[x] / nc2;
                    for (int x = 0; x < 3; x++) {
                        G.Tf(i, j, k, NORMX + x + 9 * d) = eN[x];
                        G.Tf(i, j, k, TAN1X + x + 9 * d) = eT1[x];
                        G.Tf(i, j, k, TAN2X + x + 9 * d) = eT2[x];
                    }
                }
    }
    G.cellArr(G.volume, 1);
    G.cellArr(G.di, 1);
    G.cellArr(G.dj, 1);
    G.cellArr(G.dk, 1);
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int i = G.isg; i <= G.ieg; i++) {
                double xyzC[8][3], ijkDV[5];
                cellCoords(G, i, j, k, xyzC);
                GaussianVolumeIntegral(xyzC, [](double x, double y, double z, double* W) {
                    W[0] = 1; W[1] = x; W[2] = y; W[3] = z; W[4] = 0;
                }, ijkDV);
                G.volume(i, j, k) = ijkDV[0];
                for (int x = 0; x < 3; x++) G.xyzcc(i, j, k, x) = ijkDV[1 + x] / ijkDV[0];
            }
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int i = G.isg; i <= G.ieg; i++) {
                double fA = std::max(G.face(i + 1, j, k, IDIR), G.face(i, j, k, IDIR));
                G.di(i, j, k) = G.volume(i, j, k) / fA;
                fA = std::max(G.face(i, j + 1, k, JDIR), G.face(i, j, k, JDIR));
                G.dj(i, j, k) = G.volume(i, j, k) / fA;
                fA = std::max(G.face(i, j, k + 1, KDIR), G.face(i, j, k, KDIR));
                G.dk(i, j, k) = G.volume(i, j, k) / fA;
            }
    if (G.ring.on) RingGridFix(G);  // init.F90:960
    G.faceArr(G.edge, 3, 1.0);
    G.faceArr(G.Te, 27);
    for (int d = 0; d < 3; d++) {
        int is = G.isg, ie = G.ieg + 1, js = G.jsg, je = G.jeg + 1, ks = G.ksg, ke = G.keg + 1;
        if (d == IDIR) { ie = G.ieg; ks = G.ksg + 1; ke = G.keg; }
        else if (d == JDIR) { je = G.jeg; is = G.isg + 1; ie = G.ieg; }
        else { ke = G.keg; js = G.jsg + 1; je = G.jeg; }
#pragma omp parallel for collapse(2)
        for (int k = ks; k <= ke; k++)
            for (int j = js; j <= je; j++)
                for (int i = is; i <= ie; i++) {
                    double dEdge[3], eAvg[3];
                    for (int x = 0; x < 3; x++) {
                        if (d == IDIR) {
                            dEdge[x] = G.xyz(i + 1, j, k, x) - G.xyz(i, j, k, x);
                            eAvg[x] = 0.5 * (G.xyz(i, j, k + 1, x) - G.xyz(i, j, k - 1, x) + G.xyz(i + 1, j, k + 1, x) -
                                             G.xyz(i + 1, j, k - 1, x));
                        } else if (d == JDIR) {
                            dEdge[x] = G.xyz(i, j + 1, k, x) - G.xyz(i, j, k, x);
                            eAvg[x] = 0.5 * (G.xyz(i + 1, j, k, x) - G.xyz(i - 1, j, k, x) + G.xyz(i + 1, j + 1, k, x) -
                                             G.xyz(i - 1, j + 1, k, x));
                        } else {
                            dEdge[x] = G.xyz(i, j, k + 1, x) - G.xyz(i, j, k, x);
                            eAvg[x] = 0.5 * (G.xyz(i, j + 1, k, x) - G.xyz(i, j - 1, k, x) + G.xyz(i, j + 1, k + 1, x) -
                                             G.xyz(i, j - 1, k + 1, x));
                        }
                    }
                    double eN[3], eT1[3], eT2[3], c[3];
                    double nE = norm2s(dEdge, 3);
                    for (int x = 0; x < 3; x++) eN[x] = dEdge[x] / nE;
                    cross(eAvg, eN, c);
                    double nc = norm2s(c, 3);
                    for (int x = 0; x < 3; x++) eT1[x] = c[x] / nc;
                    cross(eN, eT1, c);
                    nc = norm2s(c, 3);
                    for (int x = 0; x < 3; x++) eT2[x] = c[x] / nc;
                    G.edge(i, j, k, d) = norm2s(dEdge, 3);
                    for (int x = 0; x < 3; x++) {
                        G.Te(i, j, k, NORMX + x + 9 * d) = eN[x];
                        G.Te(i, j, k, TAN1X + x + 9 * d) = eT1[x];
                        G.Te(i, j, k, TAN2X + x + 9 * d) = eT2[x];
                    }
                }
    }
    G.faceArr(G.Teb, 12, 1.0);
    for (int dNorm = 0; dNorm < 3; dNorm++) {
        int T1 = (dNorm + 1) % 3, T2 = (dNorm + 2) % 3;
        ebGeom(G, G.Teb, XNQI, dNorm, T1, T2);
        ebGeom(G, G.Teb, XNQJ, dNorm, T2, T1);
    }
    (void)M;
}
// init.F90:511-530 SetDomain (single domain owns all boundaries)
static void SetDomain(Grid& G) {
    G.isDT = G.is - 1; G.ieDT = G.ie + 1;
    G.jsDT = G.js - 1; G.jeDT = G.je + 1;
    G.ksDT = G.ks - 1; G.keDT = G.ke + 1;
}

// ---------------------------------------------------------------- problems
// prob.F90:74-119 initOT2D
static void initOT2D(const Model& M, const Grid& G, State& S) {
    double Rho0 = 25.0 / (36.0 * PI), P0 = 5 / (12.0 * PI), B0 = 1 / std::sqrt(4.0 * PI);
    for (int k = G.ks; k <= G.ke + 1; k++)
        for (int j = G.js; j <= G.je + 1; j++)
            for (int i = G.is; i <= G.ie + 1; i++) {
                double xc = G.xyzcc(i, j, k, 0), yc = G.xyzcc(i, j, k, 1);
                S.Gas(i, j, k, DEN) = Rho0;
                double Vx = -std::sin(2 * PI * yc), Vy = std::sin(2 * PI * xc), Vz = 0.0;
                double KinE = 0.5 * Rho0 * (Vx * Vx + Vy * Vy + Vz * Vz);
                S.Gas(i, j, k, MOMX) = Vx * Rho0;
                S.Gas(i, j, k, MOMY) = Vy * Rho0;
                S.Gas(i, j, k, MOMZ) = Vz * Rho0;
                S.Gas(i, j, k, ENERGY) = KinE + P0 / (M.gamma - 1);
                S.magFlux(i, j, k, XDIR) = (-B0 * std::sin(2 * PI * yc)) * G.face(i, j, k, XDIR);
                S.magFlux(i, j, k, YDIR) = (B0 * std::sin(4 * PI * xc)) * G.face(i, j, k, YDIR);
                S.magFlux(i, j, k, ZDIR) = 0.0;
            }
}
struct BWParams { double x0, y0, z0, D0, P0, pRat, dRat, rC, B0; };
// gridutils.F90:193-237 VectorPot2Flux, with quadrature.F90:345-370 GaussianEdgeIntegral
template <class Fn> static void VectorPot2Flux(const Grid& G, State& S, Fn Axyz) {
    auto edgeInt = [&](const double* e1, const double* e2, double* eInt) {
        double dR2[3], xBar[3];
        for (int x = 0; x < 3; x++) { dR2[x] = 0.5 * (e2[x] - e1[x]); xBar[x] = 0.5 * (e2[x] + e1[x]); }
        eInt[0] = eInt[1] = eInt[2] = 0.0;
        for (int i = 0; i < 12; i++) {
            double xp[3], Ap[3];
            for (int x = 0; x < 3; x++) xp[x] = xBar[x] + gA[i] * dR2[x];
            Axyz(xp, Ap);
            for (int x = 0; x < 3; x++) eInt[x] = eInt[x] + 0.5 * gWgt[i] * Ap[x];
        }
    };
    F4 lA;
    G.cellArr(lA, 3);
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg - 1; k++)
        for (int j = G.jsg; j <= G.jeg - 1; j++)
            for (int i = G.isg; i <= G.ieg - 1; i++) {
                double e0[3], eI[3], eJ[3], eK[3], t[3], dd[3];
                for (int x = 0; x < 3; x++) {
                    e0[x] = G.xyz(i, j, k, x); eI[x] = G.xyz(i + 1, j, k, x);
                    eJ[x] = G.xyz(i, j + 1, k, x); eK[x] = G.xyz(i, j, k + 1, x);
                }
                edgeInt(eI, e0, t);
                for (int x = 0; x < 3; x++) dd[x] = eI[x] - e0[x];
                lA(i, j, k, IDIR) = dot3(t, dd);
                edgeInt(eJ, e0, t);
                for (int x = 0; x < 3; x++) dd[x] = eJ[x] - e0[x];
                lA(i, j, k, JDIR) = dot3(t, dd);
                edgeInt(eK, e0, t);
                for (int x = 0; x < 3; x++) dd[x] = eK[x] - e0[x];
                lA(i, j, k, KDIR) = dot3(t, dd);
            }
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg - 1; k++)
        for (int j = G.jsg; j <= G.jeg - 1; j++)
            for (int i = G.isg; i <= G.ieg - 1; i++) {
                S.magFlux(i, j, k, IDIR) = lA(i, j, k, JDIR) - lA(i, j, k + 1, JDIR) + lA(i, j + 1, k, KDIR) - lA(i, j, k, KDIR);
                S.magFlux(i, j, k, JDIR) =
                    -(lA(i, j, k, IDIR) - lA(i, j, k + 1, IDIR) + lA(i + 1, j, k, KDIR) - lA(i, j, k, KDIR));
                S.magFlux(i, j, k, KDIR) = lA(i, j, k, IDIR) - lA(i, j + 1, k, IDIR) + lA(i + 1, j, k, JDIR) - lA(i, j, k, JDIR);
            }
}

// Counter-based uniform deviate in [-1, 1) (SplitMix64 of seed and index).
static inline double rng_uniform(uint64_t seed, uint64_t idx) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ULL + idx + 0x632BE59BD9B4E019ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}
// Dipole-in-wind start: the constant wind state in every active cell with a
// relative density perturbation amp*u (u from rng_uniform keyed by the
// Fortran cell index), and the wind's uniform field as face fluxes of the
// potential A = (B x r)/2. The dipole itself is the background field (AddB0).
static void initDipoleWind(const Model& M, const Grid& G, State& S, uint64_t seed, double amp) {
    const double* w = M.wind;
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++) {
                uint64_t idx = (uint64_t)(i - G.isg) + (uint64_t)G.Ni * ((uint64_t)(j - G.jsg) + (uint64_t)G.Nj * (uint64_t)(k - G.ksg));
                double u = rng_uniform(seed, idx);
                double W[5] = {w[0] * (1.0 + amp * u), w[2], w[3], w[4], w[1]};
                double U[5];
                CellP2C(M, W, U);
                for (int v = 0; v < 5; v++) S.Gas(i, j, k, v) = U[v];
            }
    const double B[3] = {w[5], w[6], w[7]};
    VectorPot2Flux(G, S, [&](const double* p, double* A) {
        A[0] = 0.5 * (B[1] * p[2] - B[2] * p[1]);
        A[1] = 0.5 * (B[2] * p[0] - B[0] * p[2]);
        A[2] = 0.5 * (B[0] * p[1] - B[1] * p[0]);
    });
}

// prob.F90:190-298 initBW (doB0 = F, doBz = F), with gridutils.F90:144-189
// GasIC2State and :193-237 VectorPot2Flux
static void initBW(const Model& M, const Grid& G, State& S, const BWParams& bp) {
    const double bScl = bp.B0 / (double)std::sqrt(2.0f);  // default-real sqrt(2.0)
    const double bSclz = 0.0;
    auto W = [&](double x, double y, double z, double* Wp) {
        double R = std::sqrt((x - bp.x0) * (x - bp.x0) + (y - bp.y0) * (y - bp.y0) + (z - bp.z0) * (z - bp.z0));
        double D = bp.D0, P = bp.P0;
        if (R <= bp.rC) { D = bp.dRat * D; P = bp.pRat * P; }
        Wp[0] = D; Wp[1] = 0.0; Wp[2] = 0.0; Wp[3] = 0.0; Wp[4] = P;
    };
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++) {
                double xyzC[8][3], ijkW[5];
                cellCoords(G, i, j, k, xyzC);
                double dV = G.volume(i, j, k);
                GaussianVolumeIntegral(xyzC, W, ijkW);
                for (int v = 0; v < 5; v++) ijkW[v] = ijkW[v] / dV;
                double D = ijkW[DEN];
                double Mx = D * ijkW[VELX], My = D * ijkW[VELY], Mz = D * ijkW[VELZ];
                double P = ijkW[PRESSURE];
                double KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
                double IntE = P / (M.gamma - 1.0);
                S.Gas(i, j, k, DEN) = D;
                S.Gas(i, j, k, MOMX) = Mx;
                S.Gas(i, j, k, MOMY) = My;
                S.Gas(i, j, k, MOMZ) = Mz;
                S.Gas(i, j, k, ENERGY) = IntE + KinE;
            }
    if (!M.doMHD) return;
    VectorPot2Flux(G, S, [&](const double* p, double* A) {
        A[0] = 0.0;
        A[1] = bSclz * p[0];
        A[2] = bScl * (p[1] - p[0]);
    });
}

// ---------------------------------------------------------------- the reference's test problems
// Default-real literals of the reference (single precision under gfortran),
// as the double they become in mixed expressions
static inline double R4(double x) { return (double)(float)x; }

// gridutils.F90:144-189 GasIC2State: cell averages of the primitive function W
template <class Fn> static void GasIC2State(const Model& M, const Grid& G, State& S, Fn W) {
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++) {
                double xyzC[8][3], ijkW[5];
                cellCoords(G, i, j, k, xyzC);
                double dV = G.volume(i, j, k);
                GaussianVolumeIntegral(xyzC, W, ijkW);
                for (int v = 0; v < 5; v++) ijkW[v] = ijkW[v] / dV;
                double D = ijkW[DEN];
                double Mx = D * ijkW[VELX], My = D * ijkW[VELY], Mz = D * ijkW[VELZ];
                double P = ijkW[PRESSURE];
                double KinE = 0.5 * (Mx * Mx + My * My + Mz * Mz) / D;
                double IntE = P / (M.gamma - 1.0);
                S.Gas(i, j, k, DEN) = D;
                S.Gas(i, j, k, MOMX) = Mx;
                S.Gas(i, j, k, MOMY) = My;
                S.Gas(i, j, k, MOMZ) = Mz;
                S.Gas(i, j, k, ENERGY) = IntE + KinE;
            }
}
// pointwise gas at the cell centres of is..ie+1 (the loops of initADV1D,
// initADV2D, initLoop, prob.F90:690, 758, 461) with zero face fluxes there
template <class Fn> static void PointGas(const Model& M, const Grid& G, State& S, Fn W, bool zeroFlux) {
    for (int k = G.ks; k <= G.ke + 1; k++)
        for (int j = G.js; j <= G.je + 1; j++)
            for (int i = G.is; i <= G.ie + 1; i++) {
                double Wp[5];
                W(G.xyzcc(i, j, k, 0), G.xyzcc(i, j, k, 1), G.xyzcc(i, j, k, 2), Wp);
                double Rho = Wp[0], Vx = Wp[1], Vy = Wp[2], Vz = Wp[3], P = Wp[4];
                S.Gas(i, j, k, DEN) = Rho;
                S.Gas(i, j, k, MOMX) = Rho * Vx;
                S.Gas(i, j, k, MOMY) = Rho * Vy;
                S.Gas(i, j, k, MOMZ) = Rho * Vz;
                double KinE = 0.5 * Rho * (Vx * Vx + Vy * Vy + Vz * Vz);
                S.Gas(i, j, k, ENERGY) = KinE + P / (M.gamma - 1);
                if (zeroFlux)
                    for (int d = 0; d < 3; d++) S.magFlux(i, j, k, d) = 0.0;
            }
}
// prob.F90:671-736 initADV1D: four shapes advected at speed 1 on [-1, 1]
static void initADV1D(const Model& M, const Grid& G, State& S) {
    PointGas(M, G, S, [](double xc, double, double, double* W) {
        double Rho0 = R4(0.1);
        double a = (xc + R4(0.7)) / R4(0.05);
        double Rho1 = std::exp(-(a * a));
        double Rho2 = std::fabs(xc + R4(0.3)) <= R4(0.1) ? 1.0 : 0.0;
        double Rho3 = std::fabs(xc - R4(0.1)) <= R4(0.1) ? 1.0 - std::fabs(10.0 * (xc - R4(0.1))) : 0.0;
        double q = (double)(0.1f * 0.1f) - (xc - 0.5) * (xc - 0.5);  // 0.1**2: a default-real constant
        double Rho4 = q >= 0 ? 10.0 * std::sqrt(q) : 0.0;
        W[0] = Rho0 + Rho1 + Rho2 + Rho3 + Rho4;
        W[1] = 1.0; W[2] = 0.0; W[3] = 0.0; W[4] = 1.0;
    }, true);
}
// prob.F90:739-797 initADV2D: a disc of twice the density advected at V0
// along alpha (degrees from y), zero field
static void initADV2D(const Model& M, const Grid& G, State& S, double V0, double alpha) {
    const double Rho0 = 1.0, P0 = 1.0, R0 = 0.3, x0 = 0.0, y0 = 0.0;
    PointGas(M, G, S, [&](double xc, double yc, double, double* W) {
        double r = std::sqrt((xc - x0) * (xc - x0) + (yc - y0) * (yc - y0));
        W[0] = r < R0 ? Rho0 * 2.0 : Rho0;
        W[1] = V0 * std::sin(alpha * PI / 180.0);
        W[2] = V0 * std::cos(alpha * PI / 180.0);
        W[3] = 0.0;
        W[4] = P0;
    }, true);
}
// prob.F90:436-500 initLoop: a weak field loop (Az = max(0, A0 (R0 - r)))
// advected at V0 along alpha
static void initLoop2D(const Model& M, const Grid& G, State& S, double V0, double alpha) {
    const double Rho0 = 1.0, P0 = 1.0, Vz0 = 0.0, A0 = 1.0e-3, R0 = 0.3, x0 = 0.0, y0 = 0.0;
    PointGas(M, G, S, [&](double, double, double, double* W) {
        W[0] = Rho0;
        W[1] = V0 * std::sin(alpha * PI / 180.0);
        W[2] = V0 * std::cos(alpha * PI / 180.0);
        W[3] = Vz0;
        W[4] = P0;
    }, false);
    VectorPot2Flux(G, S, [&](const double* p, double* A) {
        double r = std::sqrt((p[0] - x0) * (p[0] - x0) + (p[1] - y0) * (p[1] - y0));
        A[0] = 0.0;
        A[1] = 0.0;
        A[2] = std::max(0.0, A0 * (R0 - r));
    });
}
// prob.F90:1027-1083 initALFVEN: circularly polarised Alfven wave along alp
static void initAlfven(const Model& M, const Grid& G, State& S, double alp) {
    const double Rho0 = 1.0, P0 = R4(0.1), B_para = 1.0, V_para = 0.0;
    GasIC2State(M, G, S, [&](double x, double y, double, double* W) {
        double ph = 2 * PI * (x * std::cos(alp) + y * std::sin(alp));
        W[0] = Rho0;
        W[1] = V_para * std::cos(alp) - R4(0.1) * std::sin(ph) * std::sin(alp);
        W[2] = V_para * std::sin(alp) + R4(0.1) * std::sin(ph) * std::cos(alp);
        W[3] = R4(0.1) * std::cos(ph);
        W[4] = P0;
    });
    VectorPot2Flux(G, S, [&](const double* p, double* A) {
        double x = p[0], y = p[1], z = p[2];
        double ph = 2 * PI * (x * std::cos(alp) + y * std::sin(alp));
        A[0] = B_para * std::sin(alp) * z;
        A[1] = -1.0 * B_para * std::cos(alp) * z + R4(0.1) * std::sin(ph) / (2 * PI * std::cos(alp));
        A[2] = R4(0.1) * std::cos(ph) / (2 * PI);
    });
}

// ---------------------------------------------------------------- background field
// msphutils.F90:534-551 Dipole, m = (0,0,M0)
static void Dipole(double M0, const double* r, double* A) {
    double rad = norm2s(r, 3);
    double m[3] = {0.0, 0.0, M0};
    double d = dot3(m, r);
    double p5 = std::pow(rad, 5.0), p3 = std::pow(rad, 3.0);
    for (int x = 0; x < 3; x++) A[x] = 3 * d * r[x] / p5 - m[x] / p3;
}
// quadrature.F90:105-151 GaussianFaceFlux
template <class Fn>
static double GaussianFaceFlux(const double* f0, const double* f1, const double* f2, const double* f3, Fn Axyz) {
    double dx[3], dy[3], dz[3];
    faceDeltas(f0, f1, f2, f3, dx, dy, dz);
    double flx = 0.0;
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) {
            double eta = 0.5 * (1 + gA[i]), psi = 0.5 * (1 + gA[j]);
            double w = gWgt[i] * gWgt[j];
            double p[3] = {f0[0] + dx[0] * eta + dx[1] * psi + dx[2] * eta * psi,
                           f0[1] + dy[0] * eta + dy[1] * psi + dy[2] * eta * psi,
                           f0[2] + dz[0] * eta + dz[1] * psi + dz[2] * eta * psi};
            double A[3];
            Axyz(p, A);
            double etaV[3] = {dx[0] + dx[2] * psi, dy[0] + dy[2] * psi, dz[0] + dz[2] * psi};
            double psiV[3] = {dx[1] + dx[2] * eta, dy[1] + dy[2] * eta, dz[1] + dz[2] * eta};
            double c[3], N[3];
            cross(etaV, psiV, c);
            for (int x = 0; x < 3; x++) N[x] = 0.25 * w * c[x];
            flx = flx + dot3(N, A);
        }
    return flx;
}
// quadrature.F90:159-221 GaussianFaceIntegral (first moment only) and
// :223-280 GaussianFaceStress, for a vector field
template <class Fn>
static void GaussianFaceIntStress(const double* f0, const double* f1, const double* f2, const double* f3, Fn Axyz,
                                  double* fInt, double* Mbb) {
    double dx[3], dy[3], dz[3];
    faceDeltas(f0, f1, f2, f3, dx, dy, dz);
    for (int x = 0; x < 3; x++) fInt[x] = Mbb[x] = 0.0;
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) {
            double eta = 0.5 * (1 + gA[i]), psi = 0.5 * (1 + gA[j]);
            double w = gWgt[i] * gWgt[j];
            double p[3] = {f0[0] + dx[0] * eta + dx[1] * psi + dx[2] * eta * psi,
                           f0[1] + dy[0] * eta + dy[1] * psi + dy[2] * eta * psi,
                           f0[2] + dz[0] * eta + dz[1] * psi + dz[2] * eta * psi};
            double B[3];
            Axyz(p, B);
            double etaV[3] = {dx[0] + dx[2] * psi, dy[0] + dy[2] * psi, dz[0] + dz[2] * psi};
            double psiV[3] = {dx[1] + dx[2] * eta, dy[1] + dy[2] * eta, dz[1] + dz[2] * eta};
            double c[3], dS[3];
            cross(etaV, psiV, c);
            double area = 0.25 * norm2s(c, 3) * w;
            for (int x = 0; x < 3; x++) fInt[x] = fInt[x] + area * B[x];
            for (int x = 0; x < 3; x++) dS[x] = 0.25 * w * c[x];
            double BB = dot3(B, B), BdS = dot3(B, dS);
            for (int x = 0; x < 3; x++) Mbb[x] = Mbb[x] + 0.5 * BB * dS[x] - B[x] * BdS;
        }
}
// quadrature.F90:345-370 GaussianEdgeIntegral
template <class Fn>
static void GaussianEdgeIntegral(const double* e1, const double* e2, Fn Axyz, double* eInt) {
    double dR2[3], xBar[3];
    for (int x = 0; x < 3; x++) { dR2[x] = 0.5 * (e2[x] - e1[x]); xBar[x] = 0.5 * (e2[x] + e1[x]); }
    eInt[0] = eInt[1] = eInt[2] = 0.0;
    for (int i = 0; i < 12; i++) {
        double xp[3], Ap[3];
        for (int x = 0; x < 3; x++) xp[x] = xBar[x] + gA[i] * dR2[x];
        Axyz(xp, Ap);
        for (int x = 0; x < 3; x++) eInt[x] = eInt[x] + 0.5 * gWgt[i] * Ap[x];
    }
}
// background.F90:20-167 AddB0 for the dipole
static void AddB0(const Model& M, Grid& G) {
    G.cellArr(G.fcB0, 9);
    G.cellArr(G.edgB0, 6);
    G.cellArr(G.B0, 3);
    G.cellArr(G.bFlux0, 3);
    G.cellArr(G.dpB0, 3);
    F4 fS;  // faceStress(i,j,k,d,x) at x + 3*d
    G.cellArr(fS, 9);
    const double M0 = M.M0;
    auto B0f = [M0](const double* p, double* A) { Dipole(M0, p, A); };
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int i = G.isg; i <= G.ieg; i++) {
                for (int d = 0; d < 3; d++) {
                    double f0[3], f1[3], f2[3], f3[3], fInt[3], Mbb[3];
                    faceCoords(G, i, j, k, d, f0, f1, f2, f3);
                    G.bFlux0(i, j, k, d) = GaussianFaceFlux(f0, f1, f2, f3, B0f);
                    GaussianFaceIntStress(f0, f1, f2, f3, B0f, fInt, Mbb);
                    for (int x = 0; x < 3; x++) G.fcB0(i, j, k, x + 3 * d) = fInt[x] / G.face(i, j, k, d);
                    for (int x = 0; x < 3; x++) fS(i, j, k, x + 3 * d) = Mbb[x];
                }
                for (int d = 0; d < 3; d++) {
                    double e1[3], e2[3], eInt[3];
                    int o[3] = {d == 0, d == 1, d == 2};
                    for (int x = 0; x < 3; x++) {
                        e1[x] = G.xyz(i, j, k, x);
                        e2[x] = G.xyz(i + o[0], j + o[1], k + o[2], x);
                    }
                    GaussianEdgeIntegral(e1, e2, B0f, eInt);
                    G.edgB0(i, j, k, 0 + 2 * d) = eInt[XDIR] * G.Te(i, j, k, TAN1X + 9 * d) +
                                                  eInt[YDIR] * G.Te(i, j, k, TAN1Y + 9 * d) +
                                                  eInt[ZDIR] * G.Te(i, j, k, TAN1Z + 9 * d);
                    G.edgB0(i, j, k, 1 + 2 * d) = eInt[XDIR] * G.Te(i, j, k, TAN2X + 9 * d) +
                                                  eInt[YDIR] * G.Te(i, j, k, TAN2Y + 9 * d) +
                                                  eInt[ZDIR] * G.Te(i, j, k, TAN2Z + 9 * d);
                }
                double xyzC[8][3], ijkB[5];
                cellCoords(G, i, j, k, xyzC);
                GaussianVolumeIntegral(xyzC, [M0](double x, double y, double z, double* W) {
                    double p[3] = {x, y, z}, A[3];
                    Dipole(M0, p, A);
                    W[0] = A[0]; W[1] = A[1]; W[2] = A[2]; W[3] = 0.0; W[4] = 0.0;
                }, ijkB);
                for (int x = 0; x < 3; x++) G.B0(i, j, k, x) = ijkB[x] / G.volume(i, j, k);
            }
#pragma omp parallel for collapse(2)
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++)
                for (int x = 0; x < 3; x++)
                    G.dpB0(i, j, k, x) = -(fS(i + 1, j, k, x + 0) - fS(i, j, k, x + 0) + fS(i, j + 1, k, x + 3) -
                                           fS(i, j, k, x + 3) + fS(i, j, k + 1, x + 6) - fS(i, j, k, x + 6)) /
                                         G.volume(i, j, k);
}

// ---------------------------------------------------------------- more BCs
// bcs.F90:934-957 SphIn
static void SphIn(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int n = 1; n <= 4; n++) {
                int ig = G.is - n;
                for (int v = 0; v < NVAR; v++) S.Gas(ig, j, k, v) = S.Gas(G.is, j, k, v);
                for (int x = 0; x < 3; x++) S.magFlux(ig, j, k, x) = S.magFlux(G.is, j, k, x);
                for (int x = 0; x < 3; x++) S.Bxyz(ig, j, k, x) = S.Bxyz(G.is, j, k, x);
            }
}
// bcs.F90:853-892 zeroGrad_ibcJ / zeroGrad_obcJ
static void zeroGrad_ibcJ(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg; k++)
        for (int n = 1; n <= 4; n++)
            for (int i = G.isg; i <= G.ieg; i++) {
                for (int v = 0; v < NVAR; v++) S.Gas(i, G.js - n, k, v) = S.Gas(i, G.js, k, v);
                for (int x = 0; x < 3; x++) S.magFlux(i, G.js - n, k, x) = S.magFlux(i, G.js, k, x);
            }
}
static void zeroGrad_obcJ(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg; k++)
        for (int n = 1; n <= 4; n++)
            for (int i = G.isg; i <= G.ieg; i++) {
                for (int v = 0; v < NVAR; v++) S.Gas(i, G.je + n, k, v) = S.Gas(i, G.je, k, v);
                S.magFlux(i, G.je + n, k, IDIR) = S.magFlux(i, G.je, k, IDIR);
                S.magFlux(i, G.je + n, k, KDIR) = S.magFlux(i, G.je, k, KDIR);
                S.magFlux(i, G.je + n + 1, k, JDIR) = S.magFlux(i, G.je + 1, k, JDIR);
            }
}
// bcs.F90:820-850 zeroGrad_obcI: gas copied from the last active cell, ghost
// face fluxes from that cell's field projected on each face (Bxyz untouched)
static void zeroGrad_obcI(const Grid& G, State& S) {
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++) {
            double B[3];
            gamCellBxyz(G, S.magFlux, G.ie, j, k, B);
            for (int n = 1; n <= 4; n++) {
                const int ig = G.ie + n;
                for (int v = 0; v < NVAR; v++) S.Gas(ig, j, k, v) = S.Gas(G.ie, j, k, v);
                for (int d = 0; d < 3; d++) {
                    const int fi = d == IDIR ? ig + 1 : ig;
                    double nH[3] = {G.Tf(fi, j, k, NORMX + 9 * d), G.Tf(fi, j, k, NORMY + 9 * d),
                                    G.Tf(fi, j, k, NORMZ + 9 * d)};
                    S.magFlux(fi, j, k, d) = G.face(fi, j, k, d) * dot3(B, nH);
                }
            }
        }
}
// Uniform inflow through the inner I side (a boundary of this library, shaped
// like zeroGrad_obcI): every ghost cell gets the state {rho, P, V, B}, its
// I face (is-n) and J, K faces the flux face * (n . B), and its Bxyz the
// gamCellBxyz of those fluxes (as WindBC does for its ghosts).
static void InflowBC(const Model& M, const Grid& G, State& S) {
    const double* w = M.inflow;  // rho, P, V(3), B(3)
    const double Bin[3] = {w[5], w[6], w[7]};
    double gW[5] = {w[0], w[2], w[3], w[4], w[1]}, gCon[5];
    CellP2C(M, gW, gCon);
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int n = 1; n <= 4; n++) {
                const int ig = G.is - n;
                for (int v = 0; v < NVAR; v++) S.Gas(ig, j, k, v) = gCon[v];
                for (int d = 0; d < 3; d++) {
                    double nH[3] = {G.Tf(ig, j, k, NORMX + 9 * d), G.Tf(ig, j, k, NORMY + 9 * d),
                                    G.Tf(ig, j, k, NORMZ + 9 * d)};
                    S.magFlux(ig, j, k, d) = G.face(ig, j, k, d) * dot3(Bin, nH);
                }
            }
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int n = 1; n <= 4; n++) {
                double B[3];
                gamCellBxyz(G, S.magFlux, G.is - n, j, k, B);
                for (int x = 0; x < 3; x++) S.Bxyz(G.is - n, j, k, x) = B[x];
            }
}
// math.F90:97-111 RampDown
static inline double RampDown(double r, double rC, double lC) {
    if (r <= rC) return 1.0;
    if (r >= rC + lC) return 0.0;
    double rScl = (r - rC) / lC;
    double eArg = -1.0 / (1.0 - rScl * rScl);
    return std::exp(eArg + 1.0);
}
// apps/wind.F90:180-203 wgtWind for a constant wind velocity V
static double wgtWind(const double* V, const double* xyz) {
    double nHat[3], vHat[3], mv[3];
    normVec(xyz, nHat);
    normVec(V, vHat);
    for (int x = 0; x < 3; x++) mv[x] = -vHat[x];
    double dTh = std::acos(dot3(mv, nHat)) * 180.0 / PI;
    return RampDown(dTh, 90.0, 90.0);
}
// gamutils.F90:238-253 CellPress2Cs and :255-269 Con2Fast (Boris off)
static double Con2Fast(const Model& M, const double* gCon, const double* B) {
    double rho = std::max(gCon[DEN], dFloor);
    double Vx = gCon[MOMX] / rho, Vy = gCon[MOMY] / rho, Vz = gCon[MOMZ] / rho;
    double KinE = 0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
    double P = std::max((M.gamma - 1) * (gCon[ENERGY] - KinE), pFloor);
    double Cs = std::sqrt(M.gamma * P / rho);
    double D = gCon[DEN];
    double MagB = norm2s(B, 3);
    double Va = MagB / std::sqrt(D);
    if (M.doBoris) Va = M.Ca * Va / std::sqrt(M.Ca * M.Ca + Va * Va);  // gamutils.F90:356-358
    return std::sqrt(Cs * Cs + Va * Va);
}
// apps/wind.F90:825-868 InterpWgts; the reference keeps doWindInterp = F, so
// the weights are always (1, 0): the wind holds the row at or below t
static void InterpWgts(const Model::WindSeries& W, double t, double& w0, double& w1, int& i0, int& i1) {
    if (t >= W.tMax) {
        i0 = W.n; i1 = i0; w0 = 1.0; w1 = 0.0;
    } else if (t <= W.tMin) {
        i0 = 1; i1 = i0; w0 = 1.0; w1 = 0.0;
    } else {
        i0 = (int)std::floor((t - W.tMin) / W.dtW) + 1;
        i1 = i0 + 1;
        if (i1 <= W.n) {
            double dT = W.tW[i1 - 1] - W.tW[i0 - 1];
            w0 = (W.tW[i1 - 1] - t) / dT;
            w1 = (t - W.tW[i0 - 1]) / dT;
        } else {
            i1 = W.n; i0 = i1 - 1; w0 = 0.0; w1 = 1.0;
        }
    }
    w0 = 1.0;  // doWindInterp = F (wind.F90:19, :862-866)
    w1 = 0.0;
}
// apps/wind.F90:766-809 InterpWind (no spin-up sequence: a null field before tMin)
static void InterpWind(const Model::WindSeries& W, double t, double& D, double& P, double* V, double* B) {
    double w0, w1;
    int i0, i1;
    InterpWgts(W, t, w0, w1, i0, i1);
    const int a = i0 - 1, b = i1 - 1;
    D = w0 * W.Q[5 * a + 0] + w1 * W.Q[5 * b + 0];
    P = w0 * W.Q[5 * a + 4] + w1 * W.Q[5 * b + 4];
    for (int x = 0; x < 3; x++) V[x] = w0 * W.Q[5 * a + 1 + x] + w1 * W.Q[5 * b + 1 + x];
    for (int x = 0; x < 3; x++) B[x] = w0 * W.B[3 * a + x] + w1 * W.B[3 * b + x];
    B[0] = W.Bx0 + W.ByC * B[1] + W.BzC * B[2];
    if (t <= W.tMin) B[0] = B[1] = B[2] = 0.0;
}
// apps/wind.F90:812-822 PlaceWind and :116-157 RefreshWind at time t
static void RefreshWind(const Model::WindSeries& W, double t, double* xyzW, double* vFr) {
    double w0, w1;
    int i0, i1;
    InterpWgts(W, t, w0, w1, i0, i1);
    for (int x = 0; x < 3; x++) xyzW[x] = w0 * W.xyzBS[3 * (i0 - 1) + x] + w1 * W.xyzBS[3 * (i1 - 1) + x];
    double D, P, V0[3], B[3];
    InterpWind(W, t, D, P, V0, B);
    double vSpd = -norm2s(V0, 3);
    double bcc = std::sqrt(W.ByC * W.ByC + W.BzC * W.BzC);
    double btt = std::sqrt(1 + bcc * bcc);
    if (bcc > TINY) {
        double CosBp = W.ByC / bcc, SinBp = W.BzC / bcc;
        double CosF = 1.0 / btt, SinF = bcc / btt;
        vFr[0] = vSpd * (CosF * CosF);
        vFr[1] = -(vSpd * CosF * SinF * CosBp);
        vFr[2] = -(vSpd * CosF * SinF * SinBp);
    } else {
        vFr[0] = vSpd; vFr[1] = 0.0; vFr[2] = 0.0;
    }
}
// apps/wind.F90:160-176 GetWindAt: the wind rewound by the lag time to xyz
static void GetWindAt(const Model::WindSeries& W, const double* xyzW, const double* vFr, const double* xyz,
                      double t, double& D, double& P, double* V, double* B) {
    double vMag = norm2s(vFr, 3);
    double d[3] = {xyz[0] - xyzW[0], xyz[1] - xyzW[1], xyz[2] - xyzW[2]};
    double DelT = dot3(d, vFr) / (vMag * vMag);
    InterpWind(W, t - DelT, D, P, V, B);
}
// apps/wind.F90:180-203 wgtWind with the wind at xyz and t
static double wgtWindTS(const Model::WindSeries& W, const double* xyzW, const double* vFr, const double* xyz,
                        double t) {
    double nHat[3], vHat[3], mv[3], D, P, V[3], B[3];
    normVec(xyz, nHat);
    GetWindAt(W, xyzW, vFr, xyz, t, D, P, V, B);
    normVec(V, vHat);
    for (int x = 0; x < 3; x++) mv[x] = -vHat[x];
    double dTh = std::acos(dot3(mv, nHat)) * 180.0 / PI;
    return RampDown(dTh, 90.0, 90.0);
}

// apps/wind.F90:206-374 WindBC with a constant wind (GetWindAt is then
// independent of position and time), single fluid, no ring
static void WindBC(const Model& M, const Grid& G, State& S) {
    const double MinMach = 1.0;
    const double* w = M.wind;  // rho, P, V(3), B(3)
    const double Vsw[3] = {w[2], w[3], w[4]}, Bsw[3] = {w[5], w[6], w[7]};
    const int ip = G.ie;
    // a time series: RefreshWind at Model%t, then the wind at each point's lag time
    const bool ts = M.ws.n > 0;
    double xyzW[3] = {0.0, 0.0, 0.0}, vFr[3] = {-1.0, 0.0, 0.0};
    if (ts) RefreshWind(M.ws, M.t, xyzW, vFr);
    auto weight = [&](const double* xyz) { return ts ? wgtWindTS(M.ws, xyzW, vFr, xyz, M.t) : wgtWind(Vsw, xyz); };
    auto windAt = [&](const double* xyz, double& D, double& P, double* V, double* B) {
        if (ts) {
            GetWindAt(M.ws, xyzW, vFr, xyz, M.t, D, P, V, B);
            return;
        }
        D = w[0];
        P = w[1];
        for (int x = 0; x < 3; x++) {
            V[x] = Vsw[x];
            B[x] = Bsw[x];
        }
    };
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg + 1; k++)
        for (int j = G.jsg; j <= G.jeg + 1; j++)
            for (int n = 1; n <= 4; n++) {
                const int ig = G.ie + n;
                if (isCellCenterG(G, ig, j, k)) {
                    double gW_sw[5] = {0, 0, 0, 0, 0}, gW_in[5] = {0, 0, 0, 0, 0};
                    double xcc[3] = {G.xyzcc(ig, j, k, 0), G.xyzcc(ig, j, k, 1), G.xyzcc(ig, j, k, 2)};
                    double wSW = weight(xcc);
                    double wMHD = 1.0 - wSW;
                    if (wSW > TINY) {
                        double D, P, V[3], B[3];
                        windAt(xcc, D, P, V, B);
                        gW_sw[DEN] = D;
                        gW_sw[PRESSURE] = P;
                        for (int x = 0; x < 3; x++) gW_sw[VELX + x] = V[x];
                    }
                    if (wMHD > TINY) {
                        double gCon[5], B_in[3];
                        for (int v = 0; v < 5; v++) gCon[v] = S.Gas(ip, j, k, v);
                        for (int x = 0; x < 3; x++) B_in[x] = S.Bxyz(ip, j, k, x);
                        CellC2P(M, gCon, gW_in);
                        double Cx = Con2Fast(M, gCon, B_in);
                        double V[3] = {gW_in[VELX], gW_in[VELY], gW_in[VELZ]};
                        double nHat[3] = {G.Tf(ip + 1, j, k, NORMX), G.Tf(ip + 1, j, k, NORMY), G.Tf(ip + 1, j, k, NORMZ)};
                        if (dot3(V, nHat) < MinMach * Cx) {
                            double dn = dot3(V, nHat);
                            for (int x = 0; x < 3; x++) V[x] = V[x] - dn * nHat[x] + MinMach * Cx * nHat[x];
                        }
                        for (int x = 0; x < 3; x++) gW_in[VELX + x] = V[x];
                    }
                    double gW[5], gCon[5];
                    for (int v = 0; v < 5; v++) gW[v] = wSW * gW_sw[v] + wMHD * gW_in[v];
                    CellP2C(M, gW, gCon);
                    for (int v = 0; v < 5; v++) S.Gas(ig, j, k, v) = gCon[v];
                }
                // face fluxes: I at ig+1, J and K at ig
                {
                    double xf[3] = {G.xfc(ig + 1, j, k, 0), G.xfc(ig + 1, j, k, 1), G.xfc(ig + 1, j, k, 2)};
                    double wSW = weight(xf);
                    double nH[3] = {G.Tf(ig + 1, j, k, NORMX), G.Tf(ig + 1, j, k, NORMY), G.Tf(ig + 1, j, k, NORMZ)};
                    double D, P, V[3], Bf[3];
                    windAt(xf, D, P, V, Bf);
                    double swFlx = G.face(ig + 1, j, k, IDIR) * dot3(nH, Bf);  // Project2Face, bcs.F90:250-263
                    double inFlx = S.magFlux(ip + 1, j, k, IDIR);
                    S.magFlux(ig + 1, j, k, IDIR) = wSW * swFlx + (1 - wSW) * inFlx;
                }
                for (int d = 1; d < 3; d++) {
                    double xf[3] = {G.xfc(ig, j, k, 0 + 3 * d), G.xfc(ig, j, k, 1 + 3 * d), G.xfc(ig, j, k, 2 + 3 * d)};
                    double wSW = weight(xf);
                    double nH[3] = {G.Tf(ig, j, k, NORMX + 9 * d), G.Tf(ig, j, k, NORMY + 9 * d), G.Tf(ig, j, k, NORMZ + 9 * d)};
                    double D, P, V[3], Bf[3];
                    windAt(xf, D, P, V, Bf);
                    double swFlx = G.face(ig, j, k, d) * dot3(nH, Bf);
                    double inFlx = S.magFlux(ip, j, k, d);
                    S.magFlux(ig, j, k, d) = wSW * swFlx + (1 - wSW) * inFlx;
                }
            }
    // Bxyz of each ghost from its conjugate cell's fluxes (:335-347), then
    // the ghosts across the pole from their conjugate (:349-373)
#pragma omp parallel for collapse(2)
    for (int k = G.ksg; k <= G.keg; k++)
        for (int j = G.jsg; j <= G.jeg; j++)
            for (int n = 1; n <= 4; n++) {
                int ip, jp, kp;
                lfmIJKcc(G, G.ie + n, j, k, ip, jp, kp);
                double B[3];
                gamCellBxyz(G, S.magFlux, ip, jp, kp, B);
                for (int x = 0; x < 3; x++) S.Bxyz(G.ie + n, j, k, x) = B[x];
            }
    for (int k = G.ksg; k <= G.keg; k++)
        for (int i = G.ie + 1; i <= G.ieg; i++)
            for (int n = 1; n <= 4; n++) {
                int ip, jp, kp;
                if (G.ring.doS) {
                    lfmIJKcc(G, i, G.js - n, k, ip, jp, kp);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, G.js - n, k, x) = S.Bxyz(ip, jp, kp, x);
                }
                if (G.ring.doE) {
                    lfmIJKcc(G, i, G.je + n, k, ip, jp, kp);
                    for (int x = 0; x < 3; x++) S.Bxyz(i, G.je + n, k, x) = S.Bxyz(ip, jp, kp, x);
                }
            }
}

// ---------------------------------------------------------------- app
struct App {
    Model M;
    Grid G;
    State S, oS, ooS, hS;
    F4 gFlx, mFlx, dGasH, dGasM, Vf;
    F4 SmoothE;  // ring averaging's smoothing EMFs
    int status = 0;
};

static void allocState(const Grid& G, State& S) {
    G.cellArr(S.Gas, NVAR);
    G.faceArr(S.magFlux, 3);
    G.cellArr(S.Efld, 3);
    G.cellArr(S.Bxyz, 3);
}

// mhdgroup.F90:16-76 AdvanceMHD
static void AdvanceMHD(App& A, double dt) {
    if (std::fabs(A.oS.time - A.S.time) < TINY) A.oS.time = A.S.time - A.M.dt;
    Predictor(A.M, A.G, A.S, A.oS, A.ooS, A.hS, 0.5 * dt);
    if (A.M.doMHD) {
        CalcElecField(A.M, A.G, A.S, A.hS, A.Vf, A.S.Efld);
        if (A.G.bc[0] == BC_ION) {  // HackE
            IonEFix(A.M, A.G, A.S);
            if (A.G.bc[1] == BC_WIND) WindEFix(A.M, A.G, A.S);
            FixEFieldLFM(A.G, A.S.Efld);
        }
    }
    CalcStress(A.M, A.G, A.S, A.hS, A.gFlx, A.mFlx, A.dGasH, A.dGasM);
    applyUpdate(A.M, A.G, A.S, A.oS, A.ooS, dt, A.dGasH, A.dGasM, A.S.Efld);
    if (A.G.ring.on && (A.G.ring.doS || A.G.ring.doE)) RingAverage(A.M, A.G, A.S, A.SmoothE);
}
// gamapp.F90:73-113 stepGamera + UpdateStateData
static int stepGamera(App& A) {
    AdvanceMHD(A, A.M.dt);
    if (A.G.bc[0] == BC_ION) {  // HackStep
        if (A.M.ion.doIonPush) PushIon(A.M, A.G, A.S);
        if (A.G.bc[1] == BC_WIND) NudgeSW(A.M, A.G, A.S);
    }
    A.M.ts = A.M.ts + 1;
    A.M.t = A.M.t + A.M.dt;
    int st;
    A.M.dt = CalcDT(A.M, A.G, A.S, &st);
    if (st != ST_OK) return st;  // the reference stops here (step.F90:143-153)
    EnforceBCs(A.M, A.G, A.S);
    bFlux2Fld(A.G, A.S.magFlux, A.S.Bxyz);
    return ST_OK;
}

}  // namespace orc

// ====================================================================== C API
using namespace orc;

extern "C" {

struct OrcScalars {
    double t, dt, dt0, time, otime;
    int ts, status;
    double ootime;
};

void* orc_create(const Params* p, const double* xyz) {
    init_weights();
    App* A = new App();
    Model& M = A->M;
    Grid& G = A->G;
    M.gamma = p->gamma; M.CFL = p->CFL; M.Vd0 = p->Vd0; M.cHogH = p->cHogH; M.cHogM = p->cHogM;
    M.tFin = p->tFin; M.dt0 = p->dt0; M.limDT0 = p->limDT0;
    M.fixedTimestep = p->fixedTimestep != 0;
    M.dt = M.fixedTimestep ? p->fixedDT : 0.0;
    M.doMHD = p->doMHD != 0; M.doLFMLim = p->doLFMLim != 0; M.do25D = p->do25D != 0;
    M.doBackground = p->doBackground != 0; M.up7 = p->up7 != 0;
    M.M0 = p->M0;
    for (int n = 0; n < 8; n++) M.wind[n] = p->wind[n];
    for (int n = 0; n < 8; n++) M.inflow[n] = p->inflow[n];
    M.doBoris = p->doBoris != 0;
    M.Ca = p->Ca;
    M.doAB3 = p->doAB3 != 0;
    g_up7 = M.up7;
    pdmb = p->pdmb; dFloor = p->dFloor; pFloor = p->pFloor;
    G.Nip = p->Nip; G.Njp = p->Njp; G.Nkp = p->Nkp;
    G.Ni = G.Nip + 8; G.Nj = G.Njp + 8; G.Nk = G.Nkp + 8;
    G.is = 1; G.ie = G.Nip; G.js = 1; G.je = G.Njp; G.ks = 1; G.ke = G.Nkp;
    G.isg = G.is - 4; G.ieg = G.ie + 4; G.jsg = G.js - 4; G.jeg = G.je + 4; G.ksg = G.ks - 4; G.keg = G.ke + 4;
    for (int n = 0; n < 6; n++) G.bc[n] = p->bc[n];
    if (p->ringNumR > 0) {  // InitRings (ringutils.F90:37-236), gid "lfm", single domain
        G.ring.on = true;
        G.ring.doS = p->bc[2] == BC_LFM;
        G.ring.doE = p->bc[3] == BC_LFM;
        G.ring.NumR = p->ringNumR;
        G.ring.Np = p->Nkp;
        for (int n = 0; n < p->ringNumR && n < 32; n++) G.ring.Nch[n] = p->ringNch[n];
        G.ring.recon = p->ringRecon;
        G.ring.NFTMAG = p->ringNFT;
        G.ring.doClean = p->ringClean != 0;
        G.ring.doFast = p->ringFast != 0;
    }
    G.faceArr(G.xyz, 3);
    std::memcpy(G.xyz.v.data(), xyz, G.xyz.v.size() * sizeof(double));
    SetDomain(G);
    if (p->noMetric) {
        G.cellArr(G.xyzcc, 3); G.faceArr(G.xfc, 9); G.faceArr(G.face, 3, 1.0); G.faceArr(G.Tf, 27);
        G.cellArr(G.volume, 1); G.cellArr(G.di, 1); G.cellArr(G.dj, 1); G.cellArr(G.dk, 1);
        G.faceArr(G.edge, 3, 1.0); G.faceArr(G.Te, 27); G.faceArr(G.Teb, 12, 1.0);
    } else {
        Corners2Grid(M, G);
        if (M.doBackground) AddB0(M, G);
    }
    allocState(G, A->S);
    A->S.time = M.t;  // allocState sets State%time = Model%t (gamutils.F90:199)
    allocState(G, A->oS);
    allocState(G, A->ooS);
    allocState(G, A->hS);
    G.cellArr(A->gFlx, 15);
    G.cellArr(A->mFlx, 9);
    G.cellArr(A->dGasH, 5);
    G.cellArr(A->dGasM, 3);
    G.cellArr(A->Vf, 3);
    if (G.ring.on) G.cellArr(A->SmoothE, 3);
    return A;
}

void orc_destroy(void* h) { delete (App*)h; }

// the coupling fields and settings of the ionospheric inner boundary
void orc_set_ionosphere(void* h, const double* inE, const double* inEe, double M0, double dtCpl, int doIonPush,
                        int nIonP, double dtSW0) {
    App* A = (App*)h;
    const Grid& G = A->G;
    const long nj = G.jeg - G.jsg + 1, nk = G.keg - G.ksg + 1;
    A->M.ion.inExyz.assign(inE, inE + PsiSh * nj * nk * 3);
    A->M.ion.inEijk.assign(inEe, inEe + (PsiSh + 1) * (nj + 1) * (nk + 1) * 3);
    A->M.ion.M0 = M0;
    A->M.ion.dtCpl = dtCpl;
    A->M.ion.doIonPush = doIonPush != 0;
    A->M.ion.nIonP = nIonP;
    A->M.ion.dtSW0 = dtSW0;
    // the magnetosphere's DT bounds: the active cells only (earthcmi.F90:136-142)
    Grid& Gw = A->G;
    Gw.isDT = Gw.is; Gw.ieDT = Gw.ie;
    Gw.jsDT = Gw.js; Gw.jeDT = Gw.je;
    Gw.ksDT = Gw.ks; Gw.keDT = Gw.ke;
}

// Pointers to internal Fortran-ordered arrays, for numpy views.
// which: 0 Gas,1 magFlux,2 Bxyz,3 oGas,4 omagFlux,5 oBxyz,6 xyzcc,7 xfc,8 volume,
// 9 di,10 dj,11 dk,12 Tf,13 Te,14 Teb,15 face,16 edge,17 Efld,18 hGas,19 hmagFlux,20 hBxyz,
// 21 dGasH, 22 dGasM, 23 xyz
double* orc_array(void* h, int which, long* n) {
    App* A = (App*)h;
    F4* a = nullptr;
    switch (which) {
        case 0: a = &A->S.Gas; break;
        case 1: a = &A->S.magFlux; break;
        case 2: a = &A->S.Bxyz; break;
        case 3: a = &A->oS.Gas; break;
        case 4: a = &A->oS.magFlux; break;
        case 5: a = &A->oS.Bxyz; break;
        case 6: a = &A->G.xyzcc; break;
        case 7: a = &A->G.xfc; break;
        case 8: a = &A->G.volume; break;
        case 9: a = &A->G.di; break;
        case 10: a = &A->G.dj; break;
        case 11: a = &A->G.dk; break;
        case 12: a = &A->G.Tf; break;
        case 13: a = &A->G.Te; break;
        case 14: a = &A->G.Teb; break;
        case 15: a = &A->G.face; break;
        case 16: a = &A->G.edge; break;
        case 17: a = &A->S.Efld; break;
        case 18: a = &A->hS.Gas; break;
        case 19: a = &A->hS.magFlux; break;
        case 20: a = &A->hS.Bxyz; break;
        case 21: a = &A->dGasH; break;
        case 22: a = &A->dGasM; break;
        case 23: a = &A->G.xyz; break;
        case 24: a = &A->G.fcB0; break;
        case 25: a = &A->G.bFlux0; break;
        case 26: a = &A->G.edgB0; break;
        case 27: a = &A->G.B0; break;
        case 28: a = &A->G.dpB0; break;
        case 29: a = &A->ooS.Gas; break;
        case 30: a = &A->ooS.magFlux; break;
        case 31: a = &A->ooS.Bxyz; break;
        default: *n = 0; return nullptr;
    }
    *n = (long)a->v.size();
    return a->v.data();
}

void orc_ic_ot(void* h) {
    App* A = (App*)h;
    initOT2D(A->M, A->G, A->S);
}
void orc_ic_dipole_wind(void* h, double amp, unsigned long long seed) {
    App* A = (App*)h;
    initDipoleWind(A->M, A->G, A->S, (uint64_t)seed, amp);
}
void orc_set_background_noalloc(void* h) {  // allocate the B0 arrays (caller fills them)
    App* A = (App*)h;
    A->G.cellArr(A->G.fcB0, 9); A->G.cellArr(A->G.edgB0, 6); A->G.cellArr(A->G.B0, 3);
    A->G.cellArr(A->G.bFlux0, 3); A->G.cellArr(A->G.dpB0, 3);
}
void orc_ic_bw(void* h, const double* bwp) {
    App* A = (App*)h;
    BWParams bp{bwp[0], bwp[1], bwp[2], bwp[3], bwp[4], bwp[5], bwp[6], bwp[7], bwp[8]};
    initBW(A->M, A->G, A->S, bp);
}

// init.F90:190-244 (CalcGridInfo after the IC): Bxyz, oState, first BCs, first dt.
int orc_init_finish(void* h) {
    App* A = (App*)h;
    A->oS.Gas.v = A->S.Gas.v;
    if (A->M.doMHD) {
        bFlux2Fld(A->G, A->S.magFlux, A->S.Bxyz);
        A->oS.magFlux.v = A->S.magFlux.v;
        A->oS.Bxyz.v = A->S.Bxyz.v;
    }
    EnforceBCs(A->M, A->G, A->S);
    CopyState(A->G, A->S, A->oS);
    A->oS.Efld.v = A->S.Efld.v;
    if (A->M.doAB3) CopyState(A->G, A->S, A->ooS);  // init.F90:232
    int st;
    A->M.dt = CalcDT(A->M, A->G, A->S, &st);
    A->oS.time = A->S.time - A->M.dt;
    if (A->M.doAB3) A->ooS.time = A->oS.time - A->M.dt;  // init.F90:238-241
    return st;
}

void orc_set_time(void* h, double t) {
    App* A = (App*)h;
    A->M.t = t;
    A->S.time = t;
}

int orc_step(void* h, int n) {
    App* A = (App*)h;
    for (int s = 0; s < n; s++) {
        int st = stepGamera(*A);
        if (st != ST_OK) { A->status = st; return st; }
    }
    return ST_OK;
}

void orc_scalars(void* h, OrcScalars* o) {
    App* A = (App*)h;
    o->t = A->M.t; o->dt = A->M.dt; o->dt0 = A->M.dt0; o->time = A->S.time; o->otime = A->oS.time;
    o->ts = A->M.ts; o->status = A->status;
    o->ootime = A->ooS.time;
}
void orc_set_scalars(void* h, const OrcScalars* o) {
    App* A = (App*)h;
    A->M.t = o->t; A->M.dt = o->dt; A->M.dt0 = o->dt0; A->S.time = o->time; A->oS.time = o->otime;
    A->M.ts = o->ts;
    A->ooS.time = o->ootime;
}

// gridutils.F90:717-770 DivB (sequential sum, no background)
// the solar-wind time series (code units; xyzBS may be null: the bow-shock
// marker at the origin, readWind's default, apps/wind.F90:731)
void orc_set_wind_series(void* h, int n, const double* t, const double* rho, const double* P, const double* V,
                         const double* B, const double* xyzBS, double Bx0, double ByC, double BzC) {
    App* A = (App*)h;
    Model::WindSeries& W = A->M.ws;
    W.n = n;
    W.tW.assign(t, t + n);
    W.Q.assign(5 * (size_t)n, 0.0);
    W.B.assign(3 * (size_t)n, 0.0);
    W.xyzBS.assign(3 * (size_t)n, 0.0);
    for (int r = 0; r < n; r++) {
        W.Q[5 * r + 0] = rho[r];
        for (int x = 0; x < 3; x++) W.Q[5 * r + 1 + x] = V[3 * r + x];
        W.Q[5 * r + 4] = P[r];
        for (int x = 0; x < 3; x++) W.B[3 * r + x] = B[3 * r + x];
        W.B[3 * r + 0] = Bx0 + ByC * W.B[3 * r + 1] + BzC * W.B[3 * r + 2];  // readWind :723-727
        if (xyzBS)
            for (int x = 0; x < 3; x++) W.xyzBS[3 * r + x] = xyzBS[3 * r + x];
    }
    W.tMin = *std::min_element(W.tW.begin(), W.tW.end());
    W.tMax = *std::max_element(W.tW.begin(), W.tW.end());
    W.dtW = n > 1 ? W.tW[1] - W.tW[0] : 1.0;
    for (int r = 1; r + 1 < n; r++) W.dtW = std::min(W.dtW, W.tW[r + 1] - W.tW[r]);
    W.Bx0 = Bx0; W.ByC = ByC; W.BzC = BzC;
}

// the reference's test problems (prob.F90), parameters as in its decks
void orc_ic_case(void* h, int which, double a, double b) {
    App* A = (App*)h;
    switch (which) {
        case 0: initADV1D(A->M, A->G, A->S); break;
        case 1: initADV2D(A->M, A->G, A->S, a, b); break;
        case 2: initLoop2D(A->M, A->G, A->S, a, b); break;
        default: initAlfven(A->M, A->G, A->S, a); break;
    }
}

double orc_divb(void* h) {
    App* A = (App*)h;
    const Grid& G = A->G;
    const F4& mf = A->S.magFlux;
    double tot = 0.0;
    for (int k = G.ks; k <= G.ke; k++)
        for (int j = G.js; j <= G.je; j++)
            for (int i = G.is; i <= G.ie; i++) {
                double dFi = mf(i, j, k, IDIR) - mf(i + 1, j, k, IDIR);
                double dFj = mf(i, j, k, JDIR) - mf(i, j + 1, k, JDIR);
                double dFk = mf(i, j, k, KDIR) - mf(i, j, k + 1, KDIR);
                double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
                if (A->M.doBackground) {  // gridutils.F90:749-753 (doTot)
                    dFi0 = G.bFlux0(i, j, k, IDIR) - G.bFlux0(i + 1, j, k, IDIR);
                    dFj0 = G.bFlux0(i, j, k, JDIR) - G.bFlux0(i, j + 1, k, JDIR);
                    dFk0 = G.bFlux0(i, j, k, KDIR) - G.bFlux0(i, j, k + 1, KDIR);
                }
                tot = tot + std::fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
            }
    return tot;
}

// RingAverage alone on the current state (ringav.F90:26-75), the call that
// tests/voltron/testring.pf (ringAvgConservationTest) makes; 1 if the grid
// has no rings
int orc_ring_average(void* h) {
    App* A = (App*)h;
    if (!A->G.ring.on) return 1;
    RingAverage(A->M, A->G, A->S, A->SmoothE);
    return 0;
}

// Known-answer hooks for tests/gamera/testgamutils.pf
void orc_c2p(double gamma, const double* con, double* prim) {
    Model M; M.gamma = gamma;
    dFloor = TINY; pFloor = TINY;
    CellC2P(M, con, prim);
}
void orc_p2c(double gamma, const double* prim, double* con) {
    Model M; M.gamma = gamma;
    dFloor = TINY; pFloor = TINY;
    CellP2C(M, prim, con);
}
double orc_erfc(double x) { return O_ERFC(x); }
double orc_exp(double x) { return O_EXP(x); }
int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
