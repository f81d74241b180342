// rb_internal.h -- device-side problem record shared by the host ABI code and the kernels.
//
// One DevProblem describes one SN solve resident in HBM: its tables (uploaded once), its
// work buffers (Krylov vectors, angular-flux scratch) and its result slots. The kernels
// read it through a device pointer; nothing here is visible across the C ABI.
#pragma once
#include <stdint.h>

#define RB_MAXNM 16   // largest cell system (Nm5) handled by the sweep kernels
#define RB_MAXFACE 16 // largest face-moment count
#define RB_MAXORD 8   // largest closure order per axis
#define RB_MAXMAT 64  // materials per problem held in shared memory
#define RB_OCT_MAXCTA 1024  // CTAs of a team the 3D octant sweep can pace with progress flags

// mixed form: in-group tolerance floor of a solve with the FP32 operator (its noise floor is near
// 1e-7), and the tolerance of the first Krylov solve before the FP64 defect correction
#define RB_MIXED_TOL 1e-7
#define RB_MIXED_TOL1 1e-5

// status bits written by the device into DevProblem::status
#define RB_DEV_OK 0
#define RB_DEV_NOT_CONVERGED 1   // informational: some group hit max_iter (reference prints only)
#define RB_DEV_BAD_TABLE 2       // a material id out of range or a singular cell system
#define RB_DEV_TIMEOUT 4         // a bounded wait gave up

struct DevProblem {
    // ---- sizes ------------------------------------------------------------------------
    int ndims, nx, ny, nz;
    long long ncell;
    int nd, np, nm5, nmf[3], nm4, nfmax, npsurf, ng, nmat, ls, oE, csd, solver_type;
    int accel, maxit, restart, depth, precision;
    double tol;
    int np_source;
    long long nphi, nstate, off_b[3], nb[3];
    long long fcells[3];  // boundary face cells per axis
    int noct;          // direction groups: 1 (1D), 4 quadrants (2D), 8 octants (3D)
    int oct_start[9];  // device directions of group o: [oct_start[o], oct_start[o+1]); 2D/3D
                       // problems hold their directions sorted by group (bit 0: μ < 0,
                       // bit 1: η < 0, bit 2: ξ < 0), the reference's order inside a group
    int nvec;          // Krylov vectors allocated in `vecs`
    long long vstride; // distance between Krylov vectors: nstate rounded up to even (the pad stays 0)
    // ---- tables (device pointers) --------------------------------------------------------
    const double *dx, *dy, *dz;
    const int *mat;    // [ncell] 0-based material
    const double *cosv;   // [3][nd] direction cosines
    const double *mn;     // [nd,np]  Mn (column-major: mn[n + nd*p])
    const double *dn;     // [np,nd]  Dn (dn[p + np*n])
    const int *pl;        // [np]
    const double *mnfp;   // [nd,np]  Mn·ℳ (Fokker-Planck solvers) or null
    const double *frow_m; // [3][nd][npsurf] half-range incoming row (zeros when none)
    const double *frow_d; // [3][nd][npsurf] half-range outgoing row
    // mixed form, 2D/3D: the operators of the tensor-core products packed in split TF32
    // (rb_tc.cuh): Mn (and Mn·ℳ) for M2D, Dn for D2M; null when not built
    const float *tc_m2d, *tc_d2m;
    // Closure tables, per direction n and spatial axis a (a < 3), factored so that the cell
    // system of flux_xD_BTE/BFP is  S = Σt·I + Σ_a h_a·G_a + Scsd[mat],
    //   q = Qn + Σ_a h_a·Gsrc_a·F_a − (EsA·S⁺ − EsB·S⁻)·F_E,   F_a' = ω₁·F_a + Gout_a·𝚽n.
    const double *G;      // [nd][3][nm*nm]   (i + nm*j)
    const double *Gsrc;   // [nd][3][nm*nfmax] (j + nm*f), f < nfa = face moments of axis a
    const double *Gout;   // [nd][3][nm*nfmax] (f + nfa*j)
    const int *tang;      // [nd] 1D tangential direction (|μ| ≤ 1e-10): no x-face update
    double w1[4];         // ω₁ of each axis (x,y,z,E)
    const double *Kcsd;   // [oE][nm*nm] stopping-power moment matrices
    const double *Bcsd;   // [nm*nm]      S⁺ matrix
    const double *EsA, *EsB; // [nm*nE]  energy-face source coefficients (j + nm*e)
    const double *Eout;   // [nE*nm]      energy-face closure (e + nE*j)
    // cross sections (reference layouts)
    const double *sigma_t;  // [ng,nmat]
    const double *sigma_s;  // [nmat,ng,ng,ls+1]
    const double *s_minus, *s_plus, *s_mom, *t_mom, *e_width;
    const double *vol;      // [ng][nphi] fixed volume sources (group-major) or null
    const double *pvol;     // [ng][nphi] particle source of a coupled transport (rb_transport) or null
    const double *surf[6];  // [ng, np_source, face cells] or null
    int bc[6];
    // ---- work ---------------------------------------------------------------------------
    double *flux;      // [ng][nphi] group-major flux moments
    double *vecs;      // [nvec][vstride] Krylov / fixed-point vectors
    double *qlout;     // [nphi] out-of-group + volume source of the current group
    double *qnout;     // [nd*nm5*ncell] Mn·Qlout
    double *psi;       // [nd*nm5*ncell] angular source / angular flux (in place)
    float *psi32;      // [nd*nm5*ncell] mixed form: FP32 angular source / flux
    double *kmat;      // [nmat][np] per-group in-group Σs of each moment's Legendre order
    double *scsd;      // [nmat][nm5*nm5] per-group CSD part of the cell matrix
    double *fexit;     // 1D: [nd][RB_MAXFACE] exit faces; 2D/3D: per-direction exits and z-face plane
    unsigned long long *oct_flags;  // [RB_OCT_MAXCTA] 3D octant sweep: steps each CTA has published
    double *phiE_a, *phiE_b; // [nd*nm4*ncell] energy-face fluxes (in / out, swapped per group)
    double *cutoff;    // [nphi]
    // ---- results ------------------------------------------------------------------------
    double *rho, *resid;
    int *iters, *conv;
    long long *passes;
    int *status;
};
