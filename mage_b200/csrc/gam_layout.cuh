// Device data layout of the GAMERA grid and state.
//
// Every 3-D field (cell-, face- or edge-centred) lives in one padded box of
// (sx, Nj+1, Nk+1) elements, i fastest, sx = Ni+1 rounded up to a multiple of
// 8 so rows start on 64-byte boundaries. Box index ii = i - isg (Fortran index
// i, isg = 1-nG), so cell, face and edge (i,j,k) share one linear index and a
// stencil step along direction d is the constant stride s[d]. Cell arrays
// leave the last i/j/k layer unused. Multi-component arrays store component c
// at offset c*fs, fs rounded up to 32 elements.
#pragma once
#include <stdint.h>

#define GAM_NG 4

struct GamBox {
    int Nip, Njp, Nkp;  // active cells
    int Ni, Nj, Nk;     // cells incl. ghosts
    int sx;             // i pitch (elements) = j stride
    long sk;            // k stride = sx*(Nj+1)
    long nbox;          // elements of one field = sk*(Nk+1)
    long fs;            // component stride (>= nbox, multiple of 32)
};

static inline GamBox gam_make_box(int Nip, int Njp, int Nkp) {
    GamBox b;
    b.Nip = Nip; b.Njp = Njp; b.Nkp = Nkp;
    b.Ni = Nip + 2 * GAM_NG; b.Nj = Njp + 2 * GAM_NG; b.Nk = Nkp + 2 * GAM_NG;
    b.sx = ((b.Ni + 1) + 7) / 8 * 8;
    b.sk = (long)b.sx * (b.Nj + 1);
    b.nbox = b.sk * (b.Nk + 1);
    b.fs = (b.nbox + 31) / 32 * 32;
    return b;
}

// The ring configuration the metric needs (RingGridFix): rings per pole and
// their chunks, which poles this grid holds
struct GamRingGeo {
    int on, doS, doE, NumR, Np;
    int Nch[32];
};

// Scalars of Model_T / State_T that change every step; they live in device
// memory so a sequence of steps runs without host round trips.
struct GamScalars {
    double t, dt, dt0, time, otime, tFin, limDT0, CFL;
    double odt, pdt;                   // this step's AB2 spacing and half step
    unsigned long long dtmin_bits;     // running min of the cell dt (bits of a positive double)
    int ts;
    int status;                        // 0 ok, 4 dt bad, 5 dt disaster
    int halted;                        // set once a step failed; later kernels return at once
    int fixedTimestep;
    int nbad;                          // cells whose dt is not a finite positive number
    double ootime, oodt;               // ooState time and oState - ooState spacing (doAB3)
    // bounds-check build (GAM_BOUNDS_CHECK): first failed index check
    int oob;                           // 1 once a check failed
    int oobKernel;                     // for_each_kernel id (15: halo, 16: other)
    long long oobIndex;                // the offending linear box index
    long long oobLimit;                // indices must be < this (0: the box size)
};
