// rb_kernels.cuh -- the device side of the SN solve.
//
// Design: one persistent launch solves a batch of problems. Each problem is owned by a
// "team" (one CTA for 1D problems); the team runs the whole group loop of
// sn_flux.jl:162-224 on the device: out-of-group source, the in-group accelerator
// (livolant / anderson / gmres / bicgstab, sn_one_speed.jl:122-187) and every transport pass
// (sn_inner_pass.jl:17-137), with no host round trip. Scalars the accelerators need (dots,
// norms, Hessenberg/Givens) are reduced inside the team in a fixed order, so results are
// deterministic and independent of which problems share the launch.
//
// A pass is three phases over the team's threads:
//   M2D   Qn[n,is,c] = Mn·Qlout + Σ_p K[mat(c)][n,p]·𝚽[p,is,c],  K = Mn·(diag Σs_l + T·ℳ)
//   sweep one thread per direction walks the cells upwind, solving the Nm5×Nm5 cell system of
//         the diamond-difference / DG closures in registers (sn_1D_bte.jl, sn_1D_bfp.jl)
//   D2M   𝚽[p,is,c] = Σ_n Dn[p,n]·ψ[n,is,c] and the outgoing boundary moments.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "rb_internal.h"

#define RB_MAXRESTART 48
#define RB_MAXDEPTH 16
#define RB_THREADS 256

namespace rb {

// ------------------------------------------------------------------------------------------
// team of one CTA: barrier and deterministic reductions
// ------------------------------------------------------------------------------------------
struct CtaTeam {
    double *red;  // shared scratch, >= nwarps doubles
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ int size() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    // Sum over the team; every thread receives the same bits (xor butterfly, then a fixed
    // warp order).
    __device__ double sum(double v) const {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if ((threadIdx.x & 31) == 0) red[w] = v;
        __syncthreads();
        double s = 0.0;
        for (int k = 0; k < nw; k++) s += red[k];
        __syncthreads();
        return s;
    }
    __device__ int any(int flag) const { return __syncthreads_or(flag); }
};

// ------------------------------------------------------------------------------------------
// state algebra (krylov_state.jl:53-114) over [𝚽 | boundary in-moments]
// ------------------------------------------------------------------------------------------
template <class Team>
__device__ double vdot(const Team &t, const double *a, const double *b, long long n) {
    double s = 0.0;
    for (long long i = t.rank(); i < n; i += t.size()) s += a[i] * b[i];
    return t.sum(s);
}
template <class Team>
__device__ void vaxpy(const Team &t, double al, const double *x, double *y, long long n) {
    for (long long i = t.rank(); i < n; i += t.size()) y[i] += al * x[i];
    t.sync();
}
template <class Team>
__device__ void vscale(const Team &t, double al, double *x, long long n) {
    for (long long i = t.rank(); i < n; i += t.size()) x[i] *= al;
    t.sync();
}
template <class Team>
__device__ void vcopy(const Team &t, double *d, const double *s, long long n) {
    for (long long i = t.rank(); i < n; i += t.size()) d[i] = s[i];
    t.sync();
}
template <class Team>
__device__ void vzero(const Team &t, double *d, long long n) {
    for (long long i = t.rank(); i < n; i += t.size()) d[i] = 0.0;
    t.sync();
}
// y = a·x + b·y
template <class Team>
__device__ void vlin(const Team &t, double a, const double *x, double b, double *y, long long n) {
    for (long long i = t.rank(); i < n; i += t.size()) y[i] = a * x[i] + b * y[i];
    t.sync();
}

// ------------------------------------------------------------------------------------------
// cell solve: Gaussian elimination with partial pivoting (the arithmetic of Julia's `𝒮\Q`,
// sn_1D_bte.jl:55 / sn_1D_bfp.jl:101). The compile-time version keeps the NM×NM system in
// registers; the run-time one serves the rarer large systems from local memory.
// ------------------------------------------------------------------------------------------
template <typename R, int NM>
__device__ __forceinline__ void lu_solve(R (&S)[NM * NM], R (&q)[NM]) {
    if (NM == 1) { q[0] = q[0] / S[0]; return; }
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
                R tq = q[k]; q[k] = q[i]; q[i] = tq;
            }
        }
        const R inv = R(1) / S[k + NM * k];
#pragma unroll
        for (int i = k + 1; i < NM; i++) {
            const R f = S[i + NM * k] * inv;
#pragma unroll
            for (int j = k + 1; j < NM; j++) S[i + NM * j] -= f * S[k + NM * j];
            q[i] -= f * q[k];
        }
    }
#pragma unroll
    for (int i = NM - 1; i >= 0; i--) {
        R s = q[i];
#pragma unroll
        for (int j = i + 1; j < NM; j++) s -= S[i + NM * j] * q[j];
        q[i] = s / S[i + NM * i];
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
// per-group constants of a problem, cached in shared memory
// ------------------------------------------------------------------------------------------
struct GroupShared {
    double sigt[RB_MAXMAT];
    double sp[RB_MAXMAT];   // S⁺/ΔE
    double sm[RB_MAXMAT];   // S⁻/ΔE
    double tg[RB_MAXMAT];
    // Krylov scalars
    double H[(RB_MAXRESTART + 1) * RB_MAXRESTART];
    double cs[RB_MAXRESTART], sn[RB_MAXRESTART], g[RB_MAXRESTART + 1], y[RB_MAXRESTART];
    double A[RB_MAXDEPTH * RB_MAXDEPTH], b[RB_MAXDEPTH];
    double red[32];
    int flag;
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

// ------------------------------------------------------------------------------------------
// the 1D sweep of one direction (sn_sweep_1D.jl:51-123 with flux_1D_BTE / flux_1D_BFP),
// compile-time shapes: NM cell moments, NF x-face moments, NE energy-face moments
// ------------------------------------------------------------------------------------------
template <typename R, int NM, int NF, int NE, bool CSD>
__device__ void sweep1d_dir(const DevProblem &P, const GroupShared &gs, int n, const double *zin_b,
                            int np_source, const double *phiE_in, double *phiE_out, double *psi, int ig) {
    const int nx = P.nx, nd = P.nd;
    const double mu = P.cosv[n];
    const bool fwd = mu >= 0.0;
    const bool tang = P.tang[n] != 0;
    R F[NF];
    {
        double f0[NF];
        boundary_in_1d(P, n, zin_b, np_source, ig, f0);
#pragma unroll
        for (int f = 0; f < NF; f++) F[f] = (R)f0[f];
    }
    const long long tb = (long long)n * 3;  // axis-0 block of direction n
    R Gr[NM * NM], Gs[NM * NF], Go[NF * NM];
#pragma unroll
    for (int k = 0; k < NM * NM; k++) Gr[k] = (R)P.G[tb * NM * NM + k];
#pragma unroll
    for (int k = 0; k < NM * NF; k++) { Gs[k] = (R)P.Gsrc[tb * NM * P.nfmax + k]; Go[k] = (R)P.Gout[tb * NM * P.nfmax + k]; }
    R EA[NM * NE], EB[NM * NE], EO[NE * NM];
    if (CSD) {
#pragma unroll
        for (int k = 0; k < NM * NE; k++) { EA[k] = (R)P.EsA[k]; EB[k] = (R)P.EsB[k]; EO[k] = (R)P.Eout[k]; }
    }
    const R w1x = (R)P.w1[0], w1E = (R)P.w1[3];
    const double amu = fabs(mu);
#pragma unroll 1
    for (int k = 0; k < nx; k++) {
        const int c = fwd ? k : nx - 1 - k;
        const int m = P.mat[c];
        const R h = tang ? R(0) : (R)(amu / P.dx[c]);
        R S[NM * NM], q[NM];
        const R sig = (R)gs.sigt[m];
        double *pc = psi + n + (long long)nd * NM * c;
#pragma unroll
        for (int i = 0; i < NM; i++)
#pragma unroll
            for (int j = 0; j < NM; j++) S[i + NM * j] = (i == j ? sig : R(0)) + h * Gr[i + NM * j];
#pragma unroll
        for (int j = 0; j < NM; j++) {
            R a = R(0);
#pragma unroll
            for (int f = 0; f < NF; f++) a += Gs[j + NM * f] * F[f];
            q[j] = (R)pc[(long long)nd * j] + h * a;
        }
        R FE[NE];
        if (CSD) {
            const double *Sc = P.scsd + (long long)m * NM * NM;
#pragma unroll
            for (int k2 = 0; k2 < NM * NM; k2++) S[k2] += (R)Sc[k2];
#pragma unroll
            for (int e = 0; e < NE; e++) FE[e] = phiE_in ? (R)phiE_in[n + (long long)nd * (e + (long long)NE * c)] : R(0);
            const R spl = (R)gs.sp[m], smn = (R)gs.sm[m];
#pragma unroll
            for (int j = 0; j < NM; j++) {
                R a = R(0);
#pragma unroll
                for (int e = 0; e < NE; e++) a += (EA[j + NM * e] * spl - EB[j + NM * e] * smn) * FE[e];
                q[j] -= a;
            }
        }
        lu_solve<R, NM>(S, q);
        if (!tang) {
            R Fo[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) {
                R a = w1x * F[f];
#pragma unroll
                for (int j = 0; j < NM; j++) a += Go[f + NF * j] * q[j];
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
                for (int j = 0; j < NM; j++) a += EO[e + NE * j] * q[j];
                phiE_out[n + (long long)nd * (e + (long long)NE * c)] = (double)a;
            }
        }
#pragma unroll
        for (int j = 0; j < NM; j++) pc[(long long)nd * j] = (double)q[j];
    }
#pragma unroll
    for (int f = 0; f < NF; f++) P.fexit[(long long)n * RB_MAXFACE + f] = (double)F[f];
}

// Run-time shapes (nm up to RB_MAXNM): the same arithmetic from local memory.
__device__ void sweep1d_dir_rt(const DevProblem &P, const GroupShared &gs, int n, const double *zin_b,
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

__device__ __forceinline__ void sweep1d_dispatch(const DevProblem &P, const GroupShared &gs, int n,
                                                 const double *zin_b, int np_source, const double *pE,
                                                 double *phiE_out, int ig) {
    const int nm = P.nm5, nf = P.nmf[0], ne = P.nm4;
    if (!P.csd) {
        if (nm == 1 && nf == 1) return sweep1d_dir<double, 1, 1, 1, false>(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
        if (nm == 2 && nf == 1) return sweep1d_dir<double, 2, 1, 1, false>(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
    } else {
        if (nm == 1 && nf == 1 && ne == 1) return sweep1d_dir<double, 1, 1, 1, true>(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
        if (nm == 4 && nf == 2 && ne == 2) return sweep1d_dir<double, 4, 2, 2, true>(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
    }
    sweep1d_dir_rt(P, gs, n, zin_b, np_source, pE, phiE_out, P.psi, ig);
}

// ------------------------------------------------------------------------------------------
// the pass T(z) = A·z + c (homogeneous: A·z), sn_inner_pass.jl:17-137, for 1D problems
// ------------------------------------------------------------------------------------------
template <class Team>
__device__ void pass1d(const Team &t, const DevProblem &P, const GroupShared &gs, const double *zin,
                       double *zout, int homog, int ig, const double *phiE_in, double *phiE_out) {
    const int nd = P.nd, np = P.np, nm = P.nm5;
    const long long ncell = P.ncell;
    const long long nq = (long long)nd * nm * ncell;
    // M2D with the in-group scattering and Fokker-Planck sources folded into K
    for (long long o = t.rank(); o < nq; o += t.size()) {
        const int n = (int)(o % nd);
        const long long r = o / nd;  // is + nm*c
        const long long c = r / nm;
        const int m = P.mat[c];
        const double *K = P.kmat + ((long long)m * nd + n) * np;
        const double *ph = zin + r * np;
        double s = homog ? 0.0 : P.qnout[o];
        for (int p = 0; p < np; p++) s += K[p] * ph[p];
        P.psi[o] = s;
    }
    t.sync();
    // sweep: one thread per direction; homogeneous passes see no surface source and a zero
    // incoming energy flux (sn_inner_pass.jl:37-38)
    const int np_source = homog ? 0 : P.np_source;
    const double *zin_b = zin + P.off_b[0];
    const double *pE = (P.csd && !homog) ? phiE_in : nullptr;
    for (int n = t.rank(); n < nd; n += t.size()) sweep1d_dispatch(P, gs, n, zin_b, np_source, pE, phiE_out, ig);
    t.sync();
    // D2M, accumulated in direction order as the reference does
    const long long nphi = P.nphi;
    for (long long o = t.rank(); o < nphi; o += t.size()) {
        const int p = (int)(o % np);
        const long long r = o / np;
        const double *ps = P.psi + r * nd;
        double s = 0.0;
        for (int n = 0; n < nd; n++) s += P.dn[p + (long long)np * n] * ps[n];
        zout[o] = s;
    }
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
        zout[P.off_b[0] + o] = s;
    }
    t.sync();
}

}  // namespace rb
