// oqg_dev.cuh -- device-side data layout of one QG basin.
//
// Fields are stored per basin as [layer][j][pitch] arrays of the handle's
// storage type T (double, or float in OQG_MIXED), x fastest like the
// reference's Fortran (nxp, nyp, nl) arrays, with rows padded to a pitch that
// is a multiple of 32 elements.  The two time levels of p and q live in four
// buffers whose roles swap every step (parity `par`):
//   p = F[par], pm = F[1-par], q = F[2+par], qm = F[3-par].
// A step writes q_new over qm and p_new over pm, so after it the parity flips.
#pragma once

#include <cstdint>

#define OQG_NLMAX 8
#define OQG_MAXRAD 16

namespace oqg {

// Scalars of the constraint equations and the step counter.  Two copies,
// by step parity: a step with parity `par` reads st[par] and its assembly
// kernel (CTA 0) writes the next values to st[1-par].
struct DevState {
    double dpi[OQG_NLMAX], dpip[OQG_NLMAX];              // mass constraint (constraint.F90:63-67)
    double cs[OQG_NLMAX], cn[OQG_NLMAX];                 // channel momentum constraints
    double csp[OQG_NLMAX], cnp[OQG_NLMAX];
    long long nt;                                        // steps done (nt-1 of the next)
    long long pad_;
};

// Forcing scalars that depend only on the forcing fields.
struct DevForcing {
    double ent_xn;                                       // area integral of ent layer 1
    double int_Be_s[OQG_NLMAX], int_Be_n[OQG_NLMAX];     // channel ent strip integrals
    double txis, txin;
};

// Device error bits
#define OQG_DERR_TIMEOUT 2   // a bounded wait for a tile load ran out

// Number of per-tile channel strip quantities per layer (vorticity kernel)
#define OQG_NQ 10

struct BasinDev {
    // geometry
    int nxp, nyp, nl, cyclic;
    int px;        // field row pitch (elements)
    int nxin;      // x-transform input length: box nxp-2, channel nxp-1
    int nk;        // wavenumbers per row: box nxp-2 (real), channel N/2+1 (complex)
    int ny;        // rows of the transform problem: nyp-2
    int M;         // complex FFT length: box 2(nxp-1), channel nxp-1
    int nrad, rad[OQG_MAXRAD];
    int pr;        // pitch of the modal right-hand side rows (elements of T)
    int pk;        // pitch of spectral rows (T for a box, complex T2 for a channel)
    int tiles_x, tiles_y;
    int vty;       // rows per tile of the vorticity kernel
    int kt;        // 0-based topography / drag layer
    int dz_sign, tau_sign, topo_active, suppress_period;
    double dx, dy, fnot, beta;
    double fx, fy, fx_bc, fy_bc;     // 1/dx^2, 1/dy^2 and the mixed-BC factors
    double jac_fac;                  // 1/(3 (2dx)(2dy) f0)
    double a_tri, ftnorm;
    double qb_fac;                   // ocqbdy factor bcco dxm2/(bcco/2+1)/f0
    double bc_half1;                 // bcco/2 + 1 (dPdx_2bc, dPdy_2bc)
    double c2[OQG_NLMAX], c4[OQG_NLMAX];   // ah2/f0, ah4/f0
    double c_ent1, c_wind, c_ent2, c_drag;
    double h[OQG_NLMAX], gp[OQG_NLMAX], ah2[OQG_NLMAX], ah4[OQG_NLMAX];
    double delek;
    double ctl2m[OQG_NLMAX * OQG_NLMAX];   // column-major (k, m)
    double ctm2l[OQG_NLMAX * OQG_NLMAX];   // column-major (m, k)
    double amat[OQG_NLMAX * OQG_NLMAX];    // column-major (k, l)
    double rdm2[OQG_NLMAX];
    // box constraint solve: cdhoc and its LU (column-major, n = nl-1)
    double cdhoc[OQG_NLMAX * OQG_NLMAX], lu[OQG_NLMAX * OQG_NLMAX];
    int piv[OQG_NLMAX];
    // channel homogeneous constants
    double hc1s[OQG_NLMAX], hc2s[OQG_NLMAX], hc1n[OQG_NLMAX], hc2n[OQG_NLMAX], hbsi;
    // device buffers
    void *F[4];                 // p/pm/q/qm roles by parity
    const void *wekp;           // [nyp][px] T
    const void *ent;            // [nl-1][nyp][px] T or null
    const double *ddyn;         // [nyp][px] or null
    const double *yprel;        // [nyp] y - yl/2 (box.F90:142-145)
    const void *tmaps;          // box: OQG_NTMAP tensor maps (128 bytes each) or null
    void *rhs;                  // [nl][ny][pr] T
    void *spec;                 // [nl][ny][pk] T or T2
    const void *tw;             // [M] T2 per-stage FFT twiddles (fft_stage_twiddles)
    const double *piv_tab;      // Thomas pivots 1/(b - a gam), compressed
    const int *piv_off;         // [nl*nk] offset into piv_tab
    const int *piv_len;         // [nl*nk] stored length (beyond: fixed point)
    const double *dst_w;        // [nk] sum_i of the inverse DST basis (box)
    const void *hsb;            // box: [nl-1][nyp][px] T hom_sol_bc
    const double *hbt;          // channel: [nyp] barotropic homogeneous solution
    const double *hbc1, *hbc2;  // channel: [nl][nyp]
    double *part_tile;          // [tiles][nl][OQG_NQ]
    double *part_col;           // [y-solve CTAs][2]: dst_w-weighted column sums and
                                // their compensations
    DevState *st;               // [2] by step parity
    DevForcing *frc;
    double *ent_rows;           // [nyp][2] row sums of the ent area integral and their
                                // compensations
    void *inh_g;                // modal rows in global memory, [nl][nyp][px] (8-byte
                                // slots): wide grids, and every box (k_xinv_rows)
    int *err;                   // device error bits
    // launch bookkeeping
    int k4_rows;                // interior rows per CTA of the assembly launch
    int xinv_sep;               // the inverse transforms run as k_xinv_rows and the
                                // assembly as k_xinv_asm (boxes; always when wide)
    int xinv_split;             // k_xinv keeps its modal rows in inh_g
    int asm_items;              // k_xinv_asm work items of this basin (256-point runs
                                // interleaved over them)
    void *scal_g;               // with xinv_sep: the step's scalar phase results,
                                // written once per step by k_xinv_rows
    double tdt_m;               // leapfrog step of this member when a launch
                                // passes tdt = 0 (ensembles: one per member)
    unsigned wait_limit;        // polls of a first wait for a tile load before
                                // it reports a timeout (drains use the full limit)
};

// Division of ints in [0, 2^31) by a divisor d >= 1 fixed for a loop, by a
// multiply-high and a shift (Granlund and Montgomery's method with a 33-bit
// multiplier 2^32 + m): q = (umulhi(m, n) + n) >> s, s = ceil(log2 d),
// m = floor(2^32 (2^s - d) / d) + 1.
struct FastDiv {
    unsigned m = 1;
    int s = 0;
    FastDiv() = default;
    __host__ __device__ __forceinline__ explicit FastDiv(int d) {
        s = 0;
        while ((1u << s) < (unsigned)d) ++s;
        m = (unsigned)(((1ull << 32) * ((1ull << s) - (unsigned long long)d)) / (unsigned long long)d + 1ull);
    }
    __device__ __forceinline__ int div(int n) const {
        return (int)((__umulhi(m, (unsigned)n) + (unsigned)n) >> s);
    }
};

// One entry of a launch's work list: which basin and which block of it.
struct Work {
    int member;
    int block;
};

template <class T> struct C2;
template <> struct C2<double> { typedef double2 t; };
template <> struct C2<float> { typedef float2 t; };

}  // namespace oqg
