// rb_kernels.cuh -- one transport pass of a 1D problem, spread over a team (thread-block cluster).
//
// A pass (sn_inner_pass.jl:17-137) is three phases separated by team barriers:
//   M2D   ψ[n,is,c] = Mn·Qlout + K[mat(c)]·𝚽[:,is,c],  K = Mn·(diag Σs_l + T·ℳ) built per group:
//         the in-group scattering source (scattering_source.jl:25-30) and the Fokker-Planck
//         source (fokker_planck_source.jl:29-33) folded into the moment-to-discrete product.
//   sweep sn_sweep_1D.jl:51-123 with flux_1D_BTE / flux_1D_BFP. Along one direction the
//         incoming face flux obeys an affine recurrence F_{k+1} = A_k·F_k + b_k (the closure
//         solved for the outgoing face), so the cells are cut into chunks: every thread composes
//         its chunk's map, one thread per direction chains the chunk maps from the boundary
//         flux, and every thread re-sweeps its chunk from its now-known incoming flux. All
//         threads work instead of one per direction.
//   D2M   𝚽[p,is,c] = Σ_n Dn[p,n]·ψ[n,is,c] (direction order, as the reference accumulates)
//         and the outgoing boundary moments; for the Krylov matvec the output is z − A·z.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "rb_internal.h"
#include "rb_team.cuh"

#define RB_MAXRESTART 48
#define RB_MAXDEPTH 16
#define RB_THREADS 256
#define RB_SCAN_NF 2      // scan path for face-moment counts up to this (every fixed 1D shape)
#define RB_MAXCLUSTER 16
#define RB_TILE_DOUBLES 2688  // largest staging of team_product (16-deep panels, 32x128 tile, padded)

namespace rb {

// ------------------------------------------------------------------------------------------
// state algebra (krylov_state.jl:53-114) over [𝚽 | boundary in-moments]. Every loop issues the
// loads of RB_VU strided elements before using them, so each thread keeps that many memory
// requests in flight instead of one.
// ------------------------------------------------------------------------------------------
#define RB_VU 8  // elements per thread whose loads are in flight together in a vector loop
#define RB_VLOOP(t, N, LOAD, USE)                                                          \
    {                                                                                      \
        const long long T_ = (t).size();                                                   \
        for (long long q0_ = (t).rank(); q0_ < (N); q0_ += RB_VU * T_) {                   \
            _Pragma("unroll") for (int u_ = 0; u_ < RB_VU; u_++) {                         \
                const long long q = q0_ + u_ * T_;                                         \
                if (q < (N)) { LOAD }                                                      \
            }                                                                              \
            _Pragma("unroll") for (int u_ = 0; u_ < RB_VU; u_++) {                         \
                const long long q = q0_ + u_ * T_;                                         \
                if (q < (N)) { USE }                                                       \
            }                                                                              \
        }                                                                                  \
    }

// Krylov vectors: element pairs (16-byte loads) over [0, vstride), vstride even and every
// vector 16-byte aligned. CTA r of the team takes the contiguous pair range
// [np·r/C, np·(r+1)/C) and its threads stride through it, RB_VU2 pairs each in flight.
#define RB_VU2 8
#define RB_VPAIRS(t, NP, LOAD, USE)                                                         \
    {                                                                                      \
        const long long np_ = (NP);                                                        \
        const long long p1_ = np_ * ((t).crank + 1) / (t).ncta;                            \
        for (long long b_ = np_ * (t).crank / (t).ncta + threadIdx.x; b_ < p1_;           \
             b_ += RB_VU2 * blockDim.x) {                                                  \
            _Pragma("unroll") for (int u_ = 0; u_ < RB_VU2; u_++) {                        \
                const long long q = b_ + u_ * blockDim.x;                                  \
                if (q < p1_) { LOAD }                                                      \
            }                                                                              \
            _Pragma("unroll") for (int u_ = 0; u_ < RB_VU2; u_++) {                        \
                const long long q = b_ + u_ * blockDim.x;                                  \
                if (q < p1_) { USE }                                                       \
            }                                                                              \
        }                                                                                  \
    }
// the same with D pairs in flight per thread (loops over three or four vectors use fewer, so that
// their values and addresses stay in registers)
#define RB_VPAIRS_D(t, NP, D, LOAD, USE)                                                    \
    {                                                                                      \
        const long long np_ = (NP);                                                        \
        const long long p1_ = np_ * ((t).crank + 1) / (t).ncta;                            \
        for (long long b_ = np_ * (t).crank / (t).ncta + threadIdx.x; b_ < p1_;           \
             b_ += (D) * blockDim.x) {                                                     \
            _Pragma("unroll") for (int u_ = 0; u_ < (D); u_++) {                           \
                const long long q = b_ + u_ * blockDim.x;                                  \
                if (q < p1_) { LOAD }                                                      \
            }                                                                              \
            _Pragma("unroll") for (int u_ = 0; u_ < (D); u_++) {                           \
                const long long q = b_ + u_ * blockDim.x;                                  \
                if (q < p1_) { USE }                                                       \
            }                                                                              \
        }                                                                                  \
    }
#define RB_D2(p) reinterpret_cast<double2 *>(p)
#define RB_CD2(p) reinterpret_cast<const double2 *>(p)

// dot product of two Krylov vectors (np pairs)
template <class Team>
__device__ double vdot2(Team &t, const double *a, const double *b, long long np) {
    const double2 *a2 = RB_CD2(a), *b2 = RB_CD2(b);
    double s = 0.0;
    double2 xa[RB_VU2], xb[RB_VU2];
    RB_VPAIRS(t, np, { xa[u_] = a2[q]; xb[u_] = b2[q]; }, {
        s += xa[u_].x * xb[u_].x;
        s += xa[u_].y * xb[u_].y;
    })
    return t.sum(s);
}

template <class Team>
__device__ double vdot(Team &t, const double *a, const double *b, long long n) {
    double s = 0.0, xa[RB_VU], xb[RB_VU];
    RB_VLOOP(t, n, { xa[u_] = a[q]; xb[u_] = b[q]; }, { s += xa[u_] * xb[u_]; (void)q; })
    return t.sum(s);
}
template <class Team>
__device__ void vaxpy(Team &t, double al, const double *x, double *y, long long n) {
    double xx[RB_VU], yy[RB_VU];
    RB_VLOOP(t, n, { xx[u_] = x[q]; yy[u_] = y[q]; }, { y[q] = yy[u_] + al * xx[u_]; })
    t.sync();
}
template <class Team>
__device__ void vcopy(Team &t, double *d, const double *s, long long n) {
    double xx[RB_VU];
    RB_VLOOP(t, n, { xx[u_] = s[q]; }, { d[q] = xx[u_]; })
    t.sync();
}
template <class Team>
__device__ void vzero(Team &t, double *d, long long n) {
    for (long long i = t.rank(); i < n; i += t.size()) d[i] = 0.0;
    t.sync();
}
// y = a·x + b·y
template <class Team>
__device__ void vlin(Team &t, double a, const double *x, double b, double *y, long long n) {
    double xx[RB_VU], yy[RB_VU];
    RB_VLOOP(t, n, { xx[u_] = x[q]; yy[u_] = y[q]; }, { y[q] = a * xx[u_] + b * yy[u_]; })
    t.sync();
}

// ------------------------------------------------------------------------------------------
// cell solve: Gaussian elimination with partial pivoting (the arithmetic of Julia's `𝒮\Q`,
// sn_1D_bte.jl:55 / sn_1D_bfp.jl:101) on an NM×NM system in registers, NR right-hand sides
// ------------------------------------------------------------------------------------------
template <typename R, int NM, int NR>
__device__ __forceinline__ void lu_solve(R (&S)[NM * NM], R (&q)[NR][NM]) {
    if (NM == 1) {
        const R inv = R(1) / S[0];
#pragma unroll
        for (int r = 0; r < NR; r++) q[r][0] = q[r][0] * inv;
        return;
    }
#pragma unroll
    for (int k = 0; k < NM; k++) {
        int p = k;
        R mx = fabs(S[k + NM * k]);
#pragma unroll
        for (int i = k + 1; i < NM; i++)
            if (fabs(S[i + NM * k]) > mx) { mx = fabs(S[i + NM * k]); p = i; }
#pragma unroll
        for (int i = k + 1; i < NM; i++) {
            if (i == p) {
#pragma unroll
                for (int j = 0; j < NM; j++) { R tmp = S[k + NM * j]; S[k + NM * j] = S[i + NM * j]; S[i + NM * j] = tmp; }
#pragma unroll
                for (int r = 0; r < NR; r++) { R tq = q[r][k]; q[r][k] = q[r][i]; q[r][i] = tq; }
            }
        }
        const R inv = R(1) / S[k + NM * k];
#pragma unroll
        for (int i = k + 1; i < NM; i++) {
            const R f = S[i + NM * k] * inv;
#pragma unroll
            for (int j = k + 1; j < NM; j++) S[i + NM * j] -= f * S[k + NM * j];
#pragma unroll
            for (int r = 0; r < NR; r++) q[r][i] -= f * q[r][k];
        }
    }
#pragma unroll
    for (int i = NM - 1; i >= 0; i--) {
        const R inv = R(1) / S[i + NM * i];
#pragma unroll
        for (int r = 0; r < NR; r++) {
            R s = q[r][i];
#pragma unroll
            for (int j = i + 1; j < NM; j++) s -= S[i + NM * j] * q[r][j];
            q[r][i] = s * inv;
        }
    }
}

template <typename R>
__device__ void lu_solve_rt(R *S, R *q, int n) {  // S is n×n, leading dimension n
#pragma unroll 1
    for (int k = 0; k < n; k++) {
        int p = k;
        R mx = fabs(S[k + n * k]);
#pragma unroll 1
        for (int i = k + 1; i < n; i++)
            if (fabs(S[i + n * k]) > mx) { mx = fabs(S[i + n * k]); p = i; }
        if (p != k) {
#pragma unroll 1
            for (int j = 0; j < n; j++) { R tmp = S[k + n * j]; S[k + n * j] = S[p + n * j]; S[p + n * j] = tmp; }
            R tq = q[k]; q[k] = q[p]; q[p] = tq;
        }
        const R inv = R(1) / S[k + n * k];
#pragma unroll 1
        for (int i = k + 1; i < n; i++) {
            const R f = S[i + n * k] * inv;
#pragma unroll 1
            for (int j = k + 1; j < n; j++) S[i + n * j] -= f * S[k + n * j];
            q[i] -= f * q[k];
        }
    }
#pragma unroll 1
    for (int i = n - 1; i >= 0; i--) {
        R s = q[i];
#pragma unroll 1
        for (int j = i + 1; j < n; j++) s -= S[i + n * j] * q[j];
        q[i] = s / S[i + n * i];
    }
}

// ------------------------------------------------------------------------------------------
// per-CTA shared state
// ------------------------------------------------------------------------------------------
// The tensor-core state of a CTA (rb_tc.cuh): TMEM base address, the MMA-completion mbarriers
// of the two column stages and the parities of their next phases (bit s). ready = 0 in kernels
// that do not allocate TMEM.
struct TcState {
    uint64_t mbar[2];
    unsigned tmem;
    unsigned phase;
    int ready;
};

struct alignas(16) GroupShared {
    double sigt[RB_MAXMAT];
    double sp[RB_MAXMAT];   // S⁺/ΔE
    double sm[RB_MAXMAT];   // S⁻/ΔE
    double tg[RB_MAXMAT];
    // accelerator scalars (each CTA keeps an identical copy)
    double H[(RB_MAXRESTART + 1) * RB_MAXRESTART];
    double cs[RB_MAXRESTART], sn[RB_MAXRESTART], g[RB_MAXRESTART + 1], y[RB_MAXRESTART];
    double A[RB_MAXDEPTH * RB_MAXDEPTH], b[RB_MAXDEPTH];
    union alignas(16) {
        // sweep scan: per thread-chunk affine map (A: NF×NF, b: NF) and the chunk's incoming flux
        struct {
            double chA[RB_THREADS][RB_SCAN_NF * RB_SCAN_NF];
            double chb[RB_THREADS][RB_SCAN_NF];
            double chF[RB_THREADS][RB_SCAN_NF];
        };
        // M2D / D2M: a tile of columns of the moment or angular arrays
        double tile[RB_TILE_DOUBLES];
    };
    TeamShared team;
    TcState tc;
    unsigned oct_epoch;  // 3D octant sweeps run so far in this solve (identical in every CTA)
};

// Incoming x-face flux of a 1D direction: surface source into moment 1 plus the lagged
// reflective / periodic in-moments (sn_sweep_1D.jl:60-91).
__device__ __forceinline__ void boundary_in_1d(const DevProblem &P, int n, const double *zin_b, int np_source,
                                               int ig, double *f0) {
    const int nf = P.nmf[0];
    const bool fwd = P.cosv[n] >= 0.0;
    const int face = fwd ? 0 : 1, side = fwd ? 0 : 1;
    const double *mrow = P.frow_m + (long long)P.npsurf * n;
    for (int f = 0; f < nf; f++) f0[f] = 0.0;
    const double *src = P.surf[face];
    if (src)
        for (int p = 0; p < np_source; p++) f0[0] += mrow[p] * src[ig + (long long)P.ng * p];
    const int bcv = P.bc[face];
    if (bcv != 0) {
        const int rside = (bcv == 1) ? side : 1 - side;
        for (int p = 0; p < P.npsurf; p++)
            for (int is = 0; is < nf; is++)
                f0[is] += mrow[p] * zin_b[p + (long long)P.npsurf * (is + (long long)nf * rside)];
    }
}

// One cell of the closure in compile-time shapes. map() keeps the face dependence symbolic:
// F_out = A·F_in + b. step() updates F in place and writes ψ (𝚽n) and the energy-face outputs.
template <typename R, int NM, int NF, int NE, bool CSD, typename PS = double>
struct Cell1D {
    const DevProblem &P;
    const GroupShared &gs;
    int n, nd;
    bool tang;
    double amu;
    R Gr[NM * NM], Gs[NM * NF], Go[NF * NM];
    R w1x, w1E;
    const double *phiE_in;
    double *phiE_out;
    long long ld;   // ψ element (n, j, c) sits at psi[n + ld·(j + NM·(c − c0))]
    int c0;
    const int *matp;       // material of cell c at matp[c − c0] (the cell tables start at cell c0)
    const double *dxp;     // width of cell c at dxp[c − c0]
    const double *scsdp;   // CSD block of the cell matrix per material

    __device__ Cell1D(const DevProblem &P_, const GroupShared &gs_, int n_, const double *pEi, double *pEo,
                      long long ld_ = -1, int c0_ = 0, const int *matp_ = nullptr, const double *dxp_ = nullptr,
                      const double *scsdp_ = nullptr)
        : P(P_), gs(gs_), n(n_), nd(P_.nd), phiE_in(pEi), phiE_out(pEo), ld(ld_ < 0 ? P_.nd : ld_), c0(c0_),
          matp(matp_ ? matp_ : P_.mat + c0_), dxp(dxp_ ? dxp_ : P_.dx + c0_), scsdp(scsdp_ ? scsdp_ : P_.scsd) {
        tang = P.tang[n] != 0;
        amu = fabs(P.cosv[n]);
        const long long tb = (long long)n * 3;  // axis-0 block of direction n
#pragma unroll
        for (int k = 0; k < NM * NM; k++) Gr[k] = (R)P.G[tb * NM * NM + k];
#pragma unroll
        for (int k = 0; k < NM * NF; k++) { Gs[k] = (R)P.Gsrc[tb * NM * P.nfmax + k]; Go[k] = (R)P.Gout[tb * NM * P.nfmax + k]; }
        w1x = (R)P.w1[0];
        w1E = (R)P.w1[3];
    }

    // assemble S and the face-independent part q0 = Qn − E·F_E of cell c
    __device__ __forceinline__ void assemble(int c, const PS *psi, R (&S)[NM * NM], R (&q0)[NM], R &h,
                                             R (&FE)[NE]) const {
        const int m = matp[c - c0];
        h = tang ? R(0) : (R)(amu / dxp[c - c0]);
        const R sig = (R)gs.sigt[m];
#pragma unroll
        for (int i = 0; i < NM; i++)
#pragma unroll
            for (int j = 0; j < NM; j++) S[i + NM * j] = (i == j ? sig : R(0)) + h * Gr[i + NM * j];
        const PS *pc = psi + n + ld * NM * (c - c0);
#pragma unroll
        for (int j = 0; j < NM; j++) q0[j] = (R)pc[ld * j];
        if (CSD) {
            const double *Sc = scsdp + (long long)m * NM * NM;
#pragma unroll
            for (int k2 = 0; k2 < NM * NM; k2++) S[k2] += (R)Sc[k2];
#pragma unroll
            for (int e = 0; e < NE; e++) FE[e] = phiE_in ? (R)phiE_in[n + (long long)nd * (e + (long long)NE * c)] : R(0);
            const R spl = (R)gs.sp[m], smn = (R)gs.sm[m];
#pragma unroll
            for (int j = 0; j < NM; j++) {
                R a = R(0);
#pragma unroll
                for (int e = 0; e < NE; e++) a += ((R)P.EsA[j + NM * e] * spl - (R)P.EsB[j + NM * e] * smn) * FE[e];
                q0[j] -= a;
            }
        }
    }

    __device__ __forceinline__ void map(int c, const PS *psi, R (&A)[NF * NF], R (&b)[NF]) const {
        R S[NM * NM], q[NF + 1][NM], h, FE[NE];
        assemble(c, psi, S, q[0], h, FE);
#pragma unroll
        for (int f = 0; f < NF; f++)
#pragma unroll
            for (int j = 0; j < NM; j++) q[f + 1][j] = h * Gs[j + NM * f];
        lu_solve<R, NM, NF + 1>(S, q);
        if (tang) {  // the x face passes through unchanged (sn_1D_bte.jl:57)
#pragma unroll
            for (int f = 0; f < NF; f++) {
                b[f] = R(0);
#pragma unroll
                for (int g = 0; g < NF; g++) A[f + NF * g] = (f == g) ? R(1) : R(0);
            }
            return;
        }
#pragma unroll
        for (int f = 0; f < NF; f++) {
            R bb = R(0);
#pragma unroll
            for (int j = 0; j < NM; j++) bb += Go[f + NF * j] * q[0][j];
            b[f] = bb;
#pragma unroll
            for (int g = 0; g < NF; g++) {
                R a = (f == g) ? w1x : R(0);
#pragma unroll
                for (int j = 0; j < NM; j++) a += Go[f + NF * j] * q[g + 1][j];
                A[f + NF * g] = a;
            }
        }
    }

    __device__ __forceinline__ void step(int c, PS *psi, R (&F)[NF]) const {
        R S[NM * NM], q[1][NM], h, FE[NE];
        assemble(c, psi, S, q[0], h, FE);
#pragma unroll
        for (int j = 0; j < NM; j++) {
            R a = R(0);
#pragma unroll
            for (int f = 0; f < NF; f++) a += Gs[j + NM * f] * F[f];
            q[0][j] += h * a;
        }
        lu_solve<R, NM, 1>(S, q);
        if (!tang) {
            R Fo[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) {
                R a = w1x * F[f];
#pragma unroll
                for (int j = 0; j < NM; j++) a += Go[f + NF * j] * q[0][j];
                Fo[f] = a;
            }
#pragma unroll
            for (int f = 0; f < NF; f++) F[f] = Fo[f];
        }
        if (CSD) {
#pragma unroll
            for (int e = 0; e < NE; e++) {
                R a = w1E * FE[e];
#pragma unroll
                for (int j = 0; j < NM; j++) a += (R)P.Eout[e + NE * j] * q[0][j];
                phiE_out[n + (long long)nd * (e + (long long)NE * c)] = (double)a;
            }
        }
        PS *pc = psi + n + ld * NM * (c - c0);
#pragma unroll
        for (int j = 0; j < NM; j++) pc[ld * j] = (PS)q[0][j];
    }
};

// The sweep phase with the chunked scan. Directions are dealt to the CTAs of the team round
// robin; within a CTA the directions it owns share its threads, `chunks` threads each.
template <typename R, int NM, int NF, int NE, bool CSD, class Team, typename PS = double>
__device__ void sweep1d_scan(Team &t, const DevProblem &P, GroupShared &gs, const double *zin_b, int np_source,
                             const double *phiE_in, double *phiE_out, int ig, PS *psi) {
    const int nd = P.nd, nx = P.nx;
    const int ncta = (int)t.ncta, crank = (int)t.crank;
    const int my_dirs = (nd - crank + ncta - 1) / ncta;  // directions n = crank + k·ncta
    const int nthr = blockDim.x;
    int per_round = my_dirs < nthr ? my_dirs : nthr;
    if (per_round < 1) per_round = 1;
    int chunks = nthr / per_round;
    if (chunks > nx) chunks = nx;
    for (int k0 = 0; k0 < my_dirs; k0 += per_round) {
        const int dl = threadIdx.x / chunks, ch = threadIdx.x % chunks;
        const int kdir = k0 + dl;
        const bool active = (dl < per_round) && (kdir < my_dirs);
        const int n = crank + kdir * ncta;
        const int L = (nx + chunks - 1) / chunks;
        const int kb = min(nx, ch * L), ke = min(nx, kb + L);
        const bool fwd = active ? (P.cosv[n] >= 0.0) : true;
        if (active) {
            Cell1D<R, NM, NF, NE, CSD, PS> cell(P, gs, n, phiE_in, phiE_out);
            R Ac[NF * NF], bc[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) {
                bc[f] = R(0);
#pragma unroll
                for (int g = 0; g < NF; g++) Ac[f + NF * g] = (f == g) ? R(1) : R(0);
            }
            for (int k = kb; k < ke; k++) {
                R A[NF * NF], b[NF];
                cell.map(fwd ? k : nx - 1 - k, psi, A, b);
                R An[NF * NF], bn[NF];  // (A,b)∘(Ac,bc)
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    R s = b[f];
#pragma unroll
                    for (int g = 0; g < NF; g++) s += A[f + NF * g] * bc[g];
                    bn[f] = s;
#pragma unroll
                    for (int g = 0; g < NF; g++) {
                        R a = R(0);
#pragma unroll
                        for (int h2 = 0; h2 < NF; h2++) a += A[f + NF * h2] * Ac[h2 + NF * g];
                        An[f + NF * g] = a;
                    }
                }
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    bc[f] = bn[f];
#pragma unroll
                    for (int g = 0; g < NF; g++) Ac[f + NF * g] = An[f + NF * g];
                }
            }
#pragma unroll
            for (int f = 0; f < NF; f++) {
                gs.chb[threadIdx.x][f] = (double)bc[f];
#pragma unroll
                for (int g = 0; g < NF; g++) gs.chA[threadIdx.x][f + NF * g] = (double)Ac[f + NF * g];
            }
        }
        __syncthreads();
        // chain the chunk maps from the boundary flux (one thread per direction)
        if (active && ch == 0) {
            double F0[RB_MAXFACE];
            boundary_in_1d(P, n, zin_b, np_source, ig, F0);
            R F[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) F[f] = (R)F0[f];
            for (int c2 = 0; c2 < chunks; c2++) {
                const int tid = dl * chunks + c2;
#pragma unroll
                for (int f = 0; f < NF; f++) gs.chF[tid][f] = (double)F[f];
                R Fn[NF];
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    R s = (R)gs.chb[tid][f];
#pragma unroll
                    for (int g = 0; g < NF; g++) s += (R)gs.chA[tid][f + NF * g] * F[g];
                    Fn[f] = s;
                }
#pragma unroll
                for (int f = 0; f < NF; f++) F[f] = Fn[f];
            }
        }
        __syncthreads();
        // re-sweep every chunk from its incoming flux
        if (active) {
            Cell1D<R, NM, NF, NE, CSD, PS> cell(P, gs, n, phiE_in, phiE_out);
            R F[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) F[f] = (R)gs.chF[threadIdx.x][f];
            for (int k = kb; k < ke; k++) cell.step(fwd ? k : nx - 1 - k, psi, F);
            if (ch == chunks - 1)
#pragma unroll
                for (int f = 0; f < NF; f++) P.fexit[(long long)n * RB_MAXFACE + f] = (double)F[f];
        }
        __syncthreads();
    }
}

// Run-time shapes (nm up to RB_MAXNM): one thread per direction walks all cells.
static __device__ void sweep1d_dir_rt(const DevProblem &P, const GroupShared &gs, int n, const double *zin_b,
                               int np_source, const double *phiE_in, double *phiE_out, double *psi, int ig) {
    const int nx = P.nx, nd = P.nd, nm = P.nm5, nf = P.nmf[0], ne = P.nm4;
    const double mu = P.cosv[n];
    const bool fwd = mu >= 0.0;
    const bool tang = P.tang[n] != 0;
    double F[RB_MAXFACE], Fo[RB_MAXFACE], FE[RB_MAXFACE];
    boundary_in_1d(P, n, zin_b, np_source, ig, F);
    const long long tb = (long long)n * 3;
    const double *Gr = P.G + tb * nm * nm, *Gs = P.Gsrc + tb * nm * P.nfmax, *Go = P.Gout + tb * nm * P.nfmax;
    const double amu = fabs(mu);
    double S[RB_MAXNM * RB_MAXNM], q[RB_MAXNM];
#pragma unroll 1
    for (int k = 0; k < nx; k++) {
        const int c = fwd ? k : nx - 1 - k;
        const int m = P.mat[c];
        const double h = tang ? 0.0 : amu / P.dx[c];
        double *pc = psi + n + (long long)nd * nm * c;
#pragma unroll 1
        for (int e = 0; e < nm * nm; e++) S[e] = h * Gr[e] + (P.csd ? P.scsd[(long long)m * nm * nm + e] : 0.0);
#pragma unroll 1
        for (int i = 0; i < nm; i++) S[i + nm * i] += gs.sigt[m];
#pragma unroll 1
        for (int j = 0; j < nm; j++) {
            double a = 0.0;
#pragma unroll 1
            for (int f = 0; f < nf; f++) a += Gs[j + nm * f] * F[f];
            q[j] = pc[(long long)nd * j] + h * a;
        }
        if (P.csd) {
#pragma unroll 1
            for (int e = 0; e < ne; e++) FE[e] = phiE_in ? phiE_in[n + (long long)nd * (e + (long long)ne * c)] : 0.0;
#pragma unroll 1
            for (int j = 0; j < nm; j++) {
                double a = 0.0;
#pragma unroll 1
                for (int e = 0; e < ne; e++) a += (P.EsA[j + nm * e] * gs.sp[m] - P.EsB[j + nm * e] * gs.sm[m]) * FE[e];
                q[j] -= a;
            }
        }
        lu_solve_rt<double>(S, q, nm);
        if (!tang) {
#pragma unroll 1
            for (int f = 0; f < nf; f++) {
                double a = P.w1[0] * F[f];
#pragma unroll 1
                for (int j = 0; j < nm; j++) a += Go[f + nf * j] * q[j];
                Fo[f] = a;
            }
#pragma unroll 1
            for (int f = 0; f < nf; f++) F[f] = Fo[f];
        }
        if (P.csd) {
#pragma unroll 1
            for (int e = 0; e < ne; e++) {
                double a = P.w1[3] * FE[e];
#pragma unroll 1
                for (int j = 0; j < nm; j++) a += P.Eout[e + ne * j] * q[j];
                phiE_out[n + (long long)nd * (e + (long long)ne * c)] = a;
            }
        }
#pragma unroll 1
        for (int j = 0; j < nm; j++) pc[(long long)nd * j] = q[j];
    }
#pragma unroll 1
    for (int f = 0; f < nf; f++) P.fexit[(long long)n * RB_MAXFACE + f] = F[f];
}

template <typename R, typename PS, class Team>
__device__ bool sweep1d_fixed(Team &t, const DevProblem &P, GroupShared &gs, const double *zin_b, int np_source,
                              const double *pE, double *phiE_out, int ig, PS *psi) {
    const int nm = P.nm5, nf = P.nmf[0], ne = P.nm4;
    if (!P.csd) {
        if (nm == 1 && nf == 1) { sweep1d_scan<R, 1, 1, 1, false>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
        if (nm == 2 && nf == 1) { sweep1d_scan<R, 2, 1, 1, false>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
        if (nm == 3 && nf == 1) { sweep1d_scan<R, 3, 1, 1, false>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
    } else {
        if (nm == 1 && nf == 1 && ne == 1) { sweep1d_scan<R, 1, 1, 1, true>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
        if (nm == 2 && nf == 1 && ne == 2) { sweep1d_scan<R, 2, 1, 2, true>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
        if (nm == 2 && nf == 2 && ne == 1) { sweep1d_scan<R, 2, 2, 1, true>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
        if (nm == 4 && nf == 2 && ne == 2) { sweep1d_scan<R, 4, 2, 2, true>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, psi); return true; }
    }
    return false;
}

template <class Team>
__device__ void sweep1d(Team &t, const DevProblem &P, GroupShared &gs, const double *zin_b, int np_source,
                        const double *pE, double *phiE_out, int ig, int mixed) {
    if (mixed) {  // mixed form: FP32 sweep on the FP32 angular buffer
        if (sweep1d_fixed<float>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, P.psi32)) return;
        // other shapes: widen the buffer, sweep in FP64, narrow it back
        const long long nq = (long long)P.nd * P.nm5 * P.ncell;
        for (long long i = t.rank(); i < nq; i += t.size()) P.psi[i] = (double)P.psi32[i];
        t.sync();
        for (int n = t.rank(); n < P.nd; n += t.size()) sweep1d_dir_rt(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
        t.sync();
        for (long long i = t.rank(); i < nq; i += t.size()) P.psi32[i] = (float)P.psi[i];
        return;
    }
    if (sweep1d_fixed<double>(t, P, gs, zin_b, np_source, pE, phiE_out, ig, P.psi)) return;
    // other shapes: one thread per direction over the whole team
    for (int n = t.rank(); n < P.nd; n += t.size()) sweep1d_dir_rt(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
}

// ------------------------------------------------------------------------------------------
// moment <-> discrete products over column tiles. A column is one (is, c) pair; the moment array
// 𝚽[p,col] and the angular array ψ[n,col] store a column contiguously, so a tile of TC columns
// is one contiguous block, staged in shared memory with coalesced loads. The small operators
// (Mn, Mn·ℳ, Dn) are read through the read-only cache. Tiles are dealt to the team's CTAs.
// ------------------------------------------------------------------------------------------
// Team-wide product over column tiles: acc[i,col] = Σ_k Op[i,k]·w(k,col)·X[k mod nk, col] with
// Op = [A | B] (B optional, then k runs over 2·nk): a second operator applied to X under its own
// per-column scale is one longer contraction. In FP64 one accumulator serves both parts; in
// FP32 each part has its own and they are added in FP64, so a large Fokker-Planck term and
// the scattering term it nearly cancels are not summed in single precision. Output tiles of
// TR rows × TC columns are dealt to the team's CTAs; each thread owns a 4×4 block of a tile and
// the operand panels are staged in shared memory 16 values of k at a time, converted to the
// compute type T (double for the plain form, float for the mixed form).
template <class TX>
struct ProductArgs {
    const double *A, *B;   // [ni + lda·k] operators (B may be null)
    int lda, ni, nk;
    const TX *X;           // [k + ldx·col]
    int ldx;
    long long ncol;
};

template <typename T> struct Vec4;
template <> struct Vec4<double> {
    __device__ static void load(const double *p, double (&o)[4]) {
        const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
};
template <> struct Vec4<float> {
    __device__ static void load(const float *p, float (&o)[4]) {
        const float4 a = *reinterpret_cast<const float4 *>(p);
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    }
};

template <typename T, class TX, class Team, class Scale, class Pre, class Store>
__device__ void team_product(Team &t, GroupShared &gs, const ProductArgs<TX> &a, Scale scale, Pre pre, Store store) {
    constexpr int KC = 16;
    constexpr int EA = (KC * 128 + RB_THREADS - 1) / RB_THREADS;  // operator elements per thread
    constexpr int EX = (KC * 128 + RB_THREADS - 1) / RB_THREADS;  // column elements per thread
    // row tiles: the operator's rows split evenly into tiles of at most 128 (a multiple of 4), so
    // an 80-row operator is one tile of 80 rows, not 64 + 16
    const int ni4 = (a.ni + 3) & ~3;
    const int nrb0 = (ni4 + 127) / 128;
    const int TR = ((ni4 + nrb0 - 1) / nrb0 + 3) & ~3;
    int TC = (RB_THREADS / (TR / 4)) * 4;  // every thread owns a 4×4 block
    if (TC > 128) TC = 128;
    if ((TC + 4) * 16 + TR * 16 > (int)(RB_TILE_DOUBLES * sizeof(double) / sizeof(T))) TC = 64;
    const int nrb = (a.ni + TR - 1) / TR;
    const long long ncb = (a.ncol + TC - 1) / TC;
    const int nk = a.nk, nkt = a.B ? 2 * a.nk : a.nk;
    // padded row of the column panel (16 bytes more in FP64, 16 in FP32): the transposing
    // stores spread over the banks and every 4-column block stays 16-byte aligned
    const int TCP = TC + (sizeof(T) == 8 ? 2 : 4);
    T *As = reinterpret_cast<T *>(gs.tile), *Xs = As + KC * TR;
    const int ib = threadIdx.x % (TR / 4), cb = threadIdx.x / (TR / 4);
    const bool owner = cb < TC / 4;
    for (long long tl = t.crank; tl < (long long)nrb * ncb; tl += t.ncta) {
        const int i0 = (int)(tl % nrb) * TR;
        const long long c0 = (tl / nrb) * TC;
        constexpr bool SPLIT = sizeof(T) < 8;
        T acc[4][4], accb[SPLIT ? 4 : 1][SPLIT ? 4 : 1];
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) acc[x][y] = T(0);
        if (SPLIT)
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) accb[SPLIT ? x : 0][SPLIT ? y : 0] = T(0);
        // panels of the A part cover k < nk, those of the B part start at nk
        const int npa = (nk + KC - 1) / KC, npanel = a.B ? 2 * npa : npa;
        for (int ip = 0; ip < npanel; ip++) {
            const bool partb = ip >= npa;
            const int k0 = partb ? nk + (ip - npa) * KC : ip * KC;
            const int kend = partb ? nkt : nk;
            // every load of the panel is issued before the first shared-memory store
            double av[EA], xv[EX], sv[EX];
#pragma unroll
            for (int u = 0; u < EA; u++) {
                const int e = threadIdx.x + u * RB_THREADS;
                const int i = i0 + e % TR, k = k0 + e / TR;
                const bool in = e < KC * TR && i < a.ni && k < kend;
                const double *op = k < nk ? a.A : a.B;
                av[u] = in ? op[i + (long long)a.lda * (k < nk ? k : k - nk)] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < EX; u++) {
                const int e = threadIdx.x + u * RB_THREADS;
                const int k = k0 + e % KC;
                const long long col = c0 + e / KC;
                const bool in = e < KC * TC && k < kend && col < a.ncol;
                xv[u] = in ? (double)a.X[(k < nk ? k : k - nk) + (long long)a.ldx * col] : 0.0;
                sv[u] = in ? scale(k, col) : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < EA; u++) {
                const int e = threadIdx.x + u * RB_THREADS;
                if (e < KC * TR) As[e] = (T)av[u];
            }
#pragma unroll
            for (int u = 0; u < EX; u++) {
                const int e = threadIdx.x + u * RB_THREADS;
                if (e < KC * TC) Xs[(e % KC) * TCP + e / KC] = (T)(sv[u] * xv[u]);
            }
            __syncthreads();
            if (owner) {
#pragma unroll 4
                for (int kk = 0; kk < KC; kk++) {
                    T o[4], v[4];
                    Vec4<T>::load(As + kk * TR + ib * 4, o);
                    Vec4<T>::load(Xs + kk * TCP + cb * 4, v);
                    if (SPLIT && partb) {
#pragma unroll
                        for (int x = 0; x < 4; x++)
#pragma unroll
                            for (int y = 0; y < 4; y++) accb[SPLIT ? x : 0][SPLIT ? y : 0] += o[x] * v[y];
                    } else {
#pragma unroll
                        for (int x = 0; x < 4; x++)
#pragma unroll
                            for (int y = 0; y < 4; y++) acc[x][y] += o[x] * v[y];
                    }
                }
            }
        }
        if (owner) {  // epilogue: the loads `pre` makes for the 16 outputs first, then the stores
            double pv[4][4];
#pragma unroll
            for (int y = 0; y < 4; y++)
#pragma unroll
                for (int x = 0; x < 4; x++) {
                    const long long col = c0 + cb * 4 + y;
                    const int i = i0 + ib * 4 + x;
                    pv[x][y] = (col < a.ncol && i < a.ni) ? pre(i, col) : 0.0;
                }
#pragma unroll
            for (int y = 0; y < 4; y++) {
                const long long col = c0 + cb * 4 + y;
                if (col >= a.ncol) continue;
#pragma unroll
                for (int x = 0; x < 4; x++) {
                    const int i = i0 + ib * 4 + x;
                    if (i < a.ni)
                        store(i, col, SPLIT ? (double)acc[x][y] + (double)accb[SPLIT ? x : 0][SPLIT ? y : 0] : (double)acc[x][y],
                              pv[x][y]);
                }
            }
        }
    }
    __syncthreads();
}

// ψ[n,col] = add[n,col] + Σ_p Mn[n,p]·ys[mat,p]·𝚽[p,col] + Σ_p (Mn·ℳ)[n,p]·T[mat]·𝚽[p,col]
// (scaled == 0: ψ = Mn·src, the Mn·Qlout product of the group set-up). The mixed form computes
// it in FP32 into the FP32 angular buffer (the FP64 Mn·Qlout term is added before rounding).
template <class Team>
__device__ void m2d_tiles(Team &t, const DevProblem &P, GroupShared &gs, const double *src, const double *add,
                          int scaled, int mixed = 0) {
    const int nd = P.nd, np = P.np, nm = P.nm5;
    ProductArgs<double> a{P.mn, (scaled && P.mnfp) ? P.mnfp : nullptr, nd, nd, np, src, np, (long long)nm * P.ncell};
    const int *mat = P.mat;
    const double *ys = P.kmat;
    auto sc = [=, &gs] __device__(int k, long long col) {
        if (!scaled) return 1.0;
        const int m = mat[col / nm];
        return k < np ? ys[(long long)m * np + k] : gs.tg[m];
    };
    auto pre = [=] __device__(int i, long long col) { return add ? add[col * nd + i] : 0.0; };
    if (mixed && scaled) {
        float *psi = P.psi32;
        team_product<float>(t, gs, a, sc, pre, [=] __device__(int i, long long col, double v, double ad) {
            psi[col * nd + i] = (float)(ad + v);
        });
        return;
    }
    double *psi = P.psi;
    team_product<double>(t, gs, a, sc, pre, [=] __device__(int i, long long col, double v, double ad) {
        psi[col * nd + i] = ad + v;
    });
}

// zout[p,col] = Σ_n Dn[p,n]·ψ[n,col]   (matvec: zout = zin − that); FP32 product in the mixed
// form, written to the FP64 state.
template <class Team>
__device__ void d2m_tiles(Team &t, const DevProblem &P, GroupShared &gs, const double *zin, double *zout, int matvec,
                          int mixed = 0) {
    const int nd = P.nd, np = P.np, nm = P.nm5;
    auto one = [] __device__(int, long long) { return 1.0; };
    auto pre = [=] __device__(int i, long long col) { return matvec ? zin[col * np + i] : 0.0; };
    auto st = [=] __device__(int i, long long col, double v, double z) { zout[col * np + i] = matvec ? z - v : v; };
    if (mixed) {
        ProductArgs<float> a{P.dn, nullptr, np, np, nd, P.psi32, nd, (long long)nm * P.ncell};
        team_product<float>(t, gs, a, one, pre, st);
    } else {
        ProductArgs<double> a{P.dn, nullptr, np, np, nd, P.psi, nd, (long long)nm * P.ncell};
        team_product<double>(t, gs, a, one, pre, st);
    }
}

// ------------------------------------------------------------------------------------------
// the pass T(z) = A·z + c (homogeneous: A·z), sn_inner_pass.jl:17-137, for 1D problems.
// matvec != 0 writes zout = zin − A·zin instead (the Krylov operator of sn_one_speed.jl:147).
// ------------------------------------------------------------------------------------------
template <class Team>
__device__ void pass1d(Team &t, const DevProblem &P, GroupShared &gs, const double *zin, double *zout, int homog,
                       int matvec, int ig, const double *phiE_in, double *phiE_out, int mixed = 0) {
    const int nd = P.nd;
    // M2D over column tiles staged in shared memory
    m2d_tiles(t, P, gs, zin, homog ? nullptr : P.qnout, 1, mixed);
    t.sync();
    // sweep; homogeneous passes see no surface source and a zero incoming energy flux
    // (sn_inner_pass.jl:37-38)
    const int np_source = homog ? 0 : P.np_source;
    const double *zin_b = zin + P.off_b[0];
    const double *pE = (P.csd && !homog) ? phiE_in : nullptr;
    sweep1d(t, P, gs, zin_b, np_source, pE, phiE_out, ig, mixed);
    t.sync();
    // D2M over column tiles staged in shared memory; direction order kept per output
    d2m_tiles(t, P, gs, zin, zout, matvec, mixed);
    // outgoing boundary moments: side 1 (X+) collects μ ≥ 0, side 0 (X-) μ < 0
    const int nf = P.nmf[0], nps = P.npsurf;
    const long long nb = P.nb[0];
    for (long long o = t.rank(); o < nb; o += t.size()) {
        const int p = (int)(o % nps);
        const int is = (int)((o / nps) % nf);
        const int side = (int)(o / ((long long)nps * nf));
        double s = 0.0;
        for (int n = 0; n < nd; n++) {
            const bool fwd = P.cosv[n] >= 0.0;
            if ((side == 1) == fwd)
                s += P.frow_d[(long long)nps * n + p] * P.fexit[(long long)n * RB_MAXFACE + is];
        }
        const long long k = P.off_b[0] + o;
        zout[k] = matvec ? zin[k] - s : s;
    }
    t.sync();
}

}  // namespace rb
