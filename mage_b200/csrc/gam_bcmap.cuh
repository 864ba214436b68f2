// Boundary-copy map of the whole-step kernels (gam_stepadj.cu): the box
// geometry, the ghost rules of the periodic and zero-gradient boundaries
// composed into one source index per box position, and the tables of the
// adjoint of that gather (host). Host- and device-callable, so
// that the host test suite checks the map against the PyTorch restatement's
// (mage_b200/diffstep.py, Grid._bc_maps) without a GPU.
#pragma once
#ifdef __CUDACC__
#define GAM_HD __host__ __device__
#else
#define GAM_HD
#endif
#include <vector>

#include "../../include/gamgpu.h"

namespace gam_stepadj {

constexpr int G = 4;  // ghost layers (nG, init.F90:327)

struct Box {
    int Nip, Njp, Nkp, Ni, Nj, Nk;  // active cells; cells with ghosts
    int nx, ny, nz;                 // box extents Ni+1, Nj+1, Nk+1
    long n;                         // elements of one component
    int bc[6];
};

inline Box make_box(const gam_params* p) {
    Box b;
    b.Nip = p->Nip; b.Njp = p->Njp; b.Nkp = p->Nkp;
    b.Ni = b.Nip + 2 * G; b.Nj = b.Njp + 2 * G; b.Nk = b.Nkp + 2 * G;
    b.nx = b.Ni + 1; b.ny = b.Nj + 1; b.nz = b.Nk + 1;
    b.n = (long)b.nx * b.ny * b.nz;
    for (int s = 0; s < 6; s++) b.bc[s] = p->bc[s];
    return b;
}

// lower / upper ghost rule of one axis with nn active cells; `normal`: the
// face flux of this axis' direction, whose upper face G+nn is active
GAM_HD inline int lo_rule(int kind, int x, int nn) {
    if (x < G) {
        if (kind == GAM_BC_PERIODIC) return x + nn;
        if (kind == GAM_BC_ZEROGRAD) return G;
    }
    return x;
}
GAM_HD inline int hi_rule(int kind, int x, int nn, bool normal) {
    const bool m = normal ? (x >= G + nn + 1 && x <= G + nn + 4) : (x >= G + nn && x <= G + nn + 3);
    if (m) {
        if (kind == GAM_BC_PERIODIC) return x - nn;
        if (kind == GAM_BC_ZEROGRAD) return normal ? G + nn : G + nn - 1;
    }
    return x;
}
// flat source index of box position (i, j, k); comp -1: cell values, 0/1/2:
// face fluxes of direction comp. K rule, then J (over the cell ranges of i and
// k only when J is not periodic), then I.
GAM_HD inline long bc_source(const Box& b, int comp, int i, int j, int k) {
    if (comp < 0 && (i >= b.Ni || j >= b.Nj || k >= b.Nk)) return ((long)k * b.ny + j) * b.nx + i;
    int sk = k;
    if (b.bc[4] == GAM_BC_PERIODIC) sk = hi_rule(GAM_BC_PERIODIC, lo_rule(GAM_BC_PERIODIC, k, b.Nkp), b.Nkp, comp == 2);
    const int sjm = hi_rule(b.bc[3], lo_rule(b.bc[2], j, b.Njp), b.Njp, comp == 1);
    const bool cond = b.bc[2] == GAM_BC_PERIODIC || (i < b.Ni && sk < b.Nk);
    const int sj = cond ? sjm : j;
    int si = i;
    if (b.bc[0] == GAM_BC_PERIODIC) si = hi_rule(GAM_BC_PERIODIC, lo_rule(GAM_BC_PERIODIC, i, b.Nip), b.Nip, comp == 0);
    return ((long)sk * b.ny + sj) * b.nx + si;
}

// box position of flat index t, in 32-bit arithmetic (a box holds fewer than
// 2^31 elements; 64-bit division is a long instruction sequence)
GAM_HD inline bool pos_of(const Box& b, long t, int& i, int& j, int& k) {
    if (t >= b.n) return false;
    const unsigned u = (unsigned)t, q = u / (unsigned)b.nx;
    i = (int)(u - q * (unsigned)b.nx);
    k = (int)(q / (unsigned)b.ny);
    j = (int)(q - (unsigned)k * (unsigned)b.ny);
    return true;
}

// The adjoint of the gather out[t] = in[src(t)] as tables, built on the host
// once per configuration and field (comp as for bc_source): code[s] = (1 if
// src(s) = s) + 2 (row + 1), row -1 where no other position copies s; the
// rows, one per position s that others copy (s ascending), list those
// positions t in ascending order (src from rowStart[row] to rowStart[row+1]).
// The adjoint at s is then (in[s] if code bit 0) + the sum over its row in
// that order: the same bits on every call.
inline void bc_adj_tables(const Box& b, int comp, std::vector<int>& code, std::vector<int>& rowStart,
                          std::vector<int>& src) {
    const long n = b.n;
    std::vector<int> from((size_t)n), cnt((size_t)n, 0), rowOf((size_t)n, -1);
    for (long t = 0; t < n; t++) {
        int i, j, k;
        pos_of(b, t, i, j, k);
        from[t] = (int)bc_source(b, comp, i, j, k);
        if (from[t] != t) cnt[from[t]]++;
    }
    code.assign((size_t)n, 0);
    rowStart.assign(1, 0);
    int rows = 0;
    for (long s = 0; s < n; s++) {
        if (cnt[s]) {
            rowOf[s] = rows++;
            rowStart.push_back(rowStart.back() + cnt[s]);
        }
        code[s] = (from[s] == s ? 1 : 0) + 2 * (rowOf[s] + 1);
    }
    src.assign((size_t)rowStart.back(), 0);
    std::vector<int> fill((size_t)rows, 0);
    for (long t = 0; t < n; t++)
        if (from[t] != t) {
            const int r = rowOf[from[t]];
            src[rowStart[r] + fill[r]++] = (int)t;
        }
}

}  // namespace gam_stepadj
