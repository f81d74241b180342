// rb_local1d.cuh -- the 1D transport pass with the cells split over the CTAs of the cluster.
//
// CTA r of a C-CTA cluster owns the contiguous cells [r·Lc, min(Nx, (r+1)·Lc)), Lc = ⌈Nx/C⌉,
// and keeps the angular array ψ of its cells in shared memory for the whole pass:
//   M2D    ψ[n, is, c] of its cells from the moments in HBM (a CTA-local tiled product),
//   sweep  every direction over its own cells: each thread composes the affine face map
//          F_out = A·F_in + b of a chunk of cells (sn_sweep_1D.jl:93-112 with the closure of
//          flux_1D_BTE / flux_1D_BFP), the chunk maps of a direction are composed into the
//          CTA's map, the CTA maps are exchanged through distributed shared memory (the one
//          cluster barrier inside the pass), every CTA chains the maps of the CTAs upstream of
//          it from the boundary flux (sn_sweep_1D.jl:60-91) and re-sweeps its chunks,
//   D2M    𝚽 = Dn·ψ of its cells straight into the output state.
// CTA 0 chains every CTA's map, which gives the exit flux of each direction, and writes the
// outgoing boundary moments (sn_sweep_1D.jl:115-121, lagged as sn_inner_pass.jl:127-134).
// So ψ never leaves the SM and a pass costs two cluster barriers (the map exchange and the
// end of the pass). The per-cell tables (material, width, the group's CSD blocks and in-group
// Σs) are copied into shared memory once per group.
#pragma once
#include <type_traits>

#include "rb_kernels.cuh"

namespace rb {

#define RB_LMAP (RB_SCAN_NF * RB_SCAN_NF + RB_SCAN_NF)  // doubles of one face map
#define RB_LKEYS 2  // distinct (material, width) cell kinds per CTA with factored cell operators

// a CTA-local team: team_product over this CTA's columns only
struct CtaTeam {
    unsigned crank = 0, ncta = 1;
};

// shape of the fixed-size cell systems (the instantiated closures)
__host__ __device__ __forceinline__ bool local1d_shape(const DevProblem &P) {
    const int nm = P.nm5, nf = P.nmf[0], ne = P.nm4;
    if (!P.csd) return nf == 1 && (nm == 1 || nm == 2 || nm == 3);
    return (nm == 1 && nf == 1 && ne == 1) || (nm == 2 && nf == 1 && ne == 2) || (nm == 2 && nf == 2 && ne == 1) ||
           (nm == 4 && nf == 2 && ne == 2);
}

// Krylov-vector slice of a CTA: the moments of its cells, and in the last CTA the boundary
// in-moments too; its largest length over the cluster
__host__ __device__ __forceinline__ long long local1d_slice(const DevProblem &P, int ncta) {
    const long long lc = (P.nx + ncta - 1) / ncta;
    return (long long)P.np * P.nm5 * lc + (P.nstate - P.nphi);
}

// bytes of the local region a problem needs on a cluster of `ncta` CTAs: face maps, exit
// fluxes, the group's in-group Σs per material and moment, the CSD cell blocks per material,
// the width and material of each owned cell, then ψ of the owned cells (which the
// Gram-Schmidt loop reuses for the basis vector in use) and the slice of w
__host__ __device__ __forceinline__ int local1d_kent(const DevProblem &P) {  // doubles per cell operator
    const int nm = P.nm5, nf = P.nmf[0];
    return nm * nm + nm * nf + nf * nf;
}
// (with_w: also the slice of w, for the Gram-Schmidt loop in shared memory)
__host__ __device__ __forceinline__ long long local1d_bytes(const DevProblem &P, int ncta, bool with_w = true) {
    const long long lc = (P.nx + ncta - 1) / ncta, nd = P.nd, nm = P.nm5;
    const long long psi = (nd + 1) * nm * lc, sl = local1d_slice(P, ncta);
    return 16 + nd * (RB_LMAP + RB_SCAN_NF) * 8 + (long long)P.nmat * P.np * 8 + (long long)P.nmat * nm * nm * 8 +
           (long long)RB_LKEYS * nd * local1d_kent(P) * 8 + lc * 8 + 2 * ((lc * 4 + 15) & ~15LL) +
           (with_w ? ((psi > sl ? psi : sl) + sl) * 8 : psi * 8);
}

// whether a problem takes the local pass on a cluster of `ncta` CTAs with `local_bytes` of
// shared memory beyond the per-CTA state
__host__ __device__ __forceinline__ bool local1d_ok(const DevProblem &P, int ncta, long long local_bytes) {
    return P.ndims == 1 && local1d_shape(P) && P.nd <= RB_THREADS && local1d_bytes(P, ncta, false) <= local_bytes;
}
// whether its Gram-Schmidt loop also keeps the slice of w in shared memory
__host__ __device__ __forceinline__ bool local1d_w(const DevProblem &P, int ncta, long long local_bytes) {
    return local1d_ok(P, ncta, local_bytes) && local1d_bytes(P, ncta, true) <= local_bytes;
}

struct Local1D {
    double *cmap;   // [nd][RB_LMAP] this CTA's face map per direction (A column-major, then b)
    double *fx;     // [nd][RB_SCAN_NF] exit flux per direction (CTA 0)
    double *kmat;   // [nmat][np] in-group Σs of each moment's Legendre order (this group)
    double *scsd;   // [nmat][nm·nm] CSD block of the cell matrix (this group)
    double *dx;     // [lc] widths of the owned cells
    int *mat;       // [lc] materials of the owned cells
    int *key;       // [lc] cell kind (index of its (material, width) pair) of the owned cells
    int *nkey;      // kinds among the owned cells; 0 when more than RB_LKEYS (per-cell solves)
    double *ktab;   // [RB_LKEYS][nd][kent] factored cell operators: S⁻¹, S⁻¹·h·Gsrc, the face map
    int kent;
    void *psi;      // [ncl][ldp] ψ of the local columns (double or float); in the Gram-Schmidt
                    // loop, the slice of the basis vector in use
    double *ws;     // the slice of w in the Gram-Schmidt loop
    long long ldp;  // leading dimension of ψ (nd + 1: odd, so column accesses spread over banks)
    int cb, ce;     // owned cells [cb, ce)
    long long e0, eb;  // slice element j < l1 is state element e0 + j, the rest eb + (j − l1)
    int l1, ls;        // length of the cell part and of the whole slice

    __device__ Local1D(const DevProblem &P, unsigned crank, unsigned ncta, void *base) {
        const int lc = (P.nx + (int)ncta - 1) / (int)ncta;
        cb = min(P.nx, (int)crank * lc);
        ce = min(P.nx, cb + lc);
        nkey = reinterpret_cast<int *>(base);
        cmap = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(base) + 16);
        fx = cmap + (long long)P.nd * RB_LMAP;
        kmat = fx + (long long)P.nd * RB_SCAN_NF;
        scsd = kmat + (long long)P.nmat * P.np;
        kent = local1d_kent(P);
        ktab = scsd + (long long)P.nmat * P.nm5 * P.nm5;
        dx = ktab + (long long)RB_LKEYS * P.nd * kent;
        mat = reinterpret_cast<int *>(dx + lc);
        key = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(mat) + ((lc * 4 + 15) & ~15));
        psi = reinterpret_cast<unsigned char *>(key) + ((lc * 4 + 15) & ~15);
        ldp = P.nd + 1;
        const long long np_ = (long long)(P.nd + 1) * P.nm5 * lc, sl = local1d_slice(P, (int)ncta);
        ws = reinterpret_cast<double *>(psi) + (np_ > sl ? np_ : sl);
        e0 = (long long)P.np * P.nm5 * cb;
        eb = P.nphi;
        l1 = (int)((long long)P.np * P.nm5 * (ce - cb));
        ls = l1 + (crank + 1 == ncta ? (int)(P.nstate - P.nphi) : 0);
    }
};

// Loop over the CTA's slice of a Krylov vector: element j of the slice is state element g,
// RB_SVU elements per thread in flight (a 4-CTA team's whole slice of a C2-sized state).
#define RB_SVU 40
#define RB_SLICE_LOOP(L, LOAD, USE)                                                         \
    {                                                                                      \
        const int l1_ = (L).l1, ls_ = (L).ls;                                              \
        const long long e0_ = (L).e0, eb_ = (L).eb;                                        \
        for (int j0_ = threadIdx.x; j0_ < ls_; j0_ += RB_SVU * blockDim.x) {               \
            _Pragma("unroll") for (int u_ = 0; u_ < RB_SVU; u_++) {                         \
                const int j = j0_ + u_ * blockDim.x;                                       \
                const long long g = j < l1_ ? e0_ + j : eb_ + (j - l1_);                   \
                if (j < ls_) { LOAD }                                                      \
                (void)g;                                                                   \
            }                                                                              \
            _Pragma("unroll") for (int u_ = 0; u_ < RB_SVU; u_++) {                         \
                const int j = j0_ + u_ * blockDim.x;                                       \
                const long long g = j < l1_ ? e0_ + j : eb_ + (j - l1_);                   \
                if (j < ls_) { USE }                                                       \
                (void)g;                                                                   \
            }                                                                              \
        }                                                                                  \
    }

// per-group copy of the tables the local pass reads per cell (after the group's constants are set)
__device__ __forceinline__ void local1d_group_setup(const DevProblem &P, Local1D &L) {
    const int nl = L.ce - L.cb;
    const int nk = P.nmat * P.np, ns = P.csd ? P.nmat * P.nm5 * P.nm5 : 0;
    for (int o = threadIdx.x; o < nk; o += blockDim.x) L.kmat[o] = P.kmat[o];
    for (int o = threadIdx.x; o < ns; o += blockDim.x) L.scsd[o] = P.scsd[o];
    for (int c = threadIdx.x; c < nl; c += blockDim.x) {
        L.dx[c] = P.dx[L.cb + c];
        L.mat[c] = P.mat[L.cb + c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the (material, width) kinds of the owned cells, in first-seen order
        int nk2 = 0, km[RB_LKEYS];
        double kd[RB_LKEYS];
        for (int c = 0; c < nl && nk2 >= 0; c++) {
            int k = 0;
            while (k < nk2 && !(km[k] == L.mat[c] && kd[k] == L.dx[c])) k++;
            if (k == nk2) {
                if (nk2 == RB_LKEYS) { nk2 = -1; break; }
                km[k] = L.mat[c];
                kd[k] = L.dx[c];
                nk2++;
            }
            L.key[c] = k;
        }
        *L.nkey = nk2 < 0 ? 0 : nk2;
    }
    __syncthreads();
}

// Factored cell operators of each (kind, direction): S = Σt·I + h·G + Scsd of flux_1D_BTE /
// flux_1D_BFP (sn_1D_bte.jl:42-46, sn_1D_bfp.jl:77-82) is the same for every cell of a kind,
// so it is solved once per group for the identity and h·Gsrc, giving S⁻¹, Y = S⁻¹·h·Gsrc and
// the face map A = ω₁·I + Gout·Y (the identity for a tangential direction).
template <int NM, int NF>
__device__ void local1d_factor(const DevProblem &P, const GroupShared &gs, Local1D &L) {
    const int nk = *L.nkey, nd = P.nd;
    for (int o = threadIdx.x; o < nk * nd; o += blockDim.x) {
        const int k = o / nd, n = o % nd;
        int c = 0;
        while (L.key[c] != k) c++;
        const int m = L.mat[c];
        const bool tang = P.tang[n] != 0;
        const double h = tang ? 0.0 : fabs(P.cosv[n]) / L.dx[c];
        const long long tb = (long long)n * 3;
        double S[NM * NM], q[NM + NF][NM];
#pragma unroll
        for (int i = 0; i < NM; i++)
#pragma unroll
            for (int j = 0; j < NM; j++)
                S[i + NM * j] = (i == j ? gs.sigt[m] : 0.0) + h * P.G[tb * NM * NM + i + NM * j] +
                                (P.csd ? L.scsd[(long long)m * NM * NM + i + NM * j] : 0.0);
#pragma unroll
        for (int r = 0; r < NM + NF; r++)
#pragma unroll
            for (int i = 0; i < NM; i++)
                q[r][i] = r < NM ? (r == i ? 1.0 : 0.0) : h * P.Gsrc[tb * NM * P.nfmax + i + NM * (r - NM)];
        lu_solve<double, NM, NM + NF>(S, q);
        double *T = L.ktab + (long long)o * L.kent;
#pragma unroll
        for (int j = 0; j < NM; j++)
#pragma unroll
            for (int i = 0; i < NM; i++) T[i + NM * j] = q[j][i];
#pragma unroll
        for (int f = 0; f < NF; f++)
#pragma unroll
            for (int i = 0; i < NM; i++) T[NM * NM + i + NM * f] = q[NM + f][i];
#pragma unroll
        for (int f = 0; f < NF; f++)
#pragma unroll
            for (int g = 0; g < NF; g++) {
                double a = (f == g) ? (tang ? 1.0 : P.w1[0]) : 0.0;
                if (!tang)
#pragma unroll
                    for (int j = 0; j < NM; j++) a += P.Gout[tb * NM * P.nfmax + f + NF * j] * q[NM + g][j];
                T[NM * NM + NM * NF + f + NF * g] = a;
            }
    }
    __syncthreads();
}

__device__ __forceinline__ void local1d_factor_fixed(const DevProblem &P, const GroupShared &gs, Local1D &L) {
    const int nm = P.nm5, nf = P.nmf[0];
    if (nm == 1 && nf == 1) local1d_factor<1, 1>(P, gs, L);
    else if (nm == 2 && nf == 1) local1d_factor<2, 1>(P, gs, L);
    else if (nm == 3 && nf == 1) local1d_factor<3, 1>(P, gs, L);
    else if (nm == 2 && nf == 2) local1d_factor<2, 2>(P, gs, L);
    else if (nm == 4 && nf == 2) local1d_factor<4, 2>(P, gs, L);
}

// One cell with the factored operator of its kind: the right-hand side q0 = Qn − E·F_E, then
// y = S⁻¹·q0; the face map is F_out = A·F_in + Gout·y and the cell moments are y + Y·F_in.
template <typename R, int NM, int NF, int NE, bool CSD, typename PS>
struct CellKey1D {
    const DevProblem &P;
    const GroupShared &gs;
    const Local1D &L;
    int n, nd;
    bool tang;
    R Go[NF * NM];
    R w1x, w1E;
    const double *phiE_in;
    double *phiE_out;

    __device__ CellKey1D(const DevProblem &P_, const GroupShared &gs_, const Local1D &L_, int n_, const double *pEi,
                         double *pEo)
        : P(P_), gs(gs_), L(L_), n(n_), nd(P_.nd), phiE_in(pEi), phiE_out(pEo) {
        tang = P.tang[n] != 0;
#pragma unroll
        for (int k = 0; k < NF * NM; k++) Go[k] = (R)P.Gout[(long long)n * 3 * NM * P.nfmax + k];
        w1x = (R)P.w1[0];
        w1E = (R)P.w1[3];
    }
    __device__ __forceinline__ const double *op(int lc) const {
        return L.ktab + ((long long)L.key[lc] * nd + n) * L.kent;
    }
    // y = S⁻¹·q0 of local cell lc; FE returns the incoming energy-face flux
    __device__ __forceinline__ void solve0(int lc, const PS *psi, R (&y)[NM], R (&FE)[NE]) const {
        R q0[NM];
        const PS *pc = psi + n + L.ldp * NM * lc;
#pragma unroll
        for (int j = 0; j < NM; j++) q0[j] = (R)pc[L.ldp * j];
        if (CSD) {
            const int m = L.mat[lc];
            const long long c = L.cb + lc;
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
        const double *T = op(lc);
#pragma unroll
        for (int i = 0; i < NM; i++) {
            R a = R(0);
#pragma unroll
            for (int j = 0; j < NM; j++) a += (R)T[i + NM * j] * q0[j];
            y[i] = a;
        }
    }
    __device__ __forceinline__ void map(int lc, const PS *psi, R (&A)[NF * NF], R (&b)[NF]) const {
        R y[NM], FE[NE];
        solve0(lc, psi, y, FE);
        const double *T = op(lc) + NM * NM + NM * NF;
#pragma unroll
        for (int f = 0; f < NF; f++) {
            R bb = R(0);
            if (!tang)
#pragma unroll
                for (int j = 0; j < NM; j++) bb += Go[f + NF * j] * y[j];
            b[f] = bb;
#pragma unroll
            for (int g = 0; g < NF; g++) A[f + NF * g] = (R)T[f + NF * g];
        }
    }
    __device__ __forceinline__ void step(int lc, PS *psi, R (&F)[NF]) const {
        R y[NM], FE[NE];
        solve0(lc, psi, y, FE);
        const double *Y = op(lc) + NM * NM;
#pragma unroll
        for (int i = 0; i < NM; i++) {
            R a = y[i];
#pragma unroll
            for (int f = 0; f < NF; f++) a += (R)Y[i + NM * f] * F[f];
            y[i] = a;
        }
        if (!tang) {
            R Fo[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) {
                R a = w1x * F[f];
#pragma unroll
                for (int j = 0; j < NM; j++) a += Go[f + NF * j] * y[j];
                Fo[f] = a;
            }
#pragma unroll
            for (int f = 0; f < NF; f++) F[f] = Fo[f];
        }
        if (CSD) {
            const long long c = L.cb + lc;
#pragma unroll
            for (int e = 0; e < NE; e++) {
                R a = w1E * FE[e];
#pragma unroll
                for (int j = 0; j < NM; j++) a += (R)P.Eout[e + NE * j] * y[j];
                phiE_out[n + (long long)nd * (e + (long long)NE * c)] = (double)a;
            }
        }
        PS *pc = psi + n + L.ldp * NM * lc;
#pragma unroll
        for (int j = 0; j < NM; j++) pc[L.ldp * j] = (PS)y[j];
    }
};

// compose (A,b) ← (A2,b2)∘(A,b): F ↦ A2·(A·F + b) + b2
template <typename R, int NF>
__device__ __forceinline__ void compose_map(const R (&A2)[NF * NF], const R (&b2)[NF], R (&A)[NF * NF], R (&b)[NF]) {
    R An[NF * NF], bn[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) {
        R s = b2[f];
#pragma unroll
        for (int g = 0; g < NF; g++) s += A2[f + NF * g] * b[g];
        bn[f] = s;
#pragma unroll
        for (int g = 0; g < NF; g++) {
            R a = R(0);
#pragma unroll
            for (int h = 0; h < NF; h++) a += A2[f + NF * h] * A[h + NF * g];
            An[f + NF * g] = a;
        }
    }
#pragma unroll
    for (int f = 0; f < NF; f++) {
        b[f] = bn[f];
#pragma unroll
        for (int g = 0; g < NF; g++) A[f + NF * g] = An[f + NF * g];
    }
}

// F ← A·F + b for a map stored as [A column-major | b]
template <typename R, int NF>
__device__ __forceinline__ void apply_map(const double *M, R (&F)[NF]) {
    R Fn[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) {
        R s = (R)M[NF * NF + f];
#pragma unroll
        for (int g = 0; g < NF; g++) s += (R)M[f + NF * g] * F[g];
        Fn[f] = s;
    }
#pragma unroll
    for (int f = 0; f < NF; f++) F[f] = Fn[f];
}

// The sweep over the local cells. Threads: direction n = tid / chunks, chunk = tid % chunks
// (nd ≤ blockDim.x is required). Ends with ψ of the local cells holding the angular flux and,
// in CTA 0, the outgoing boundary moments written to zout.
template <typename R, int NM, int NF, int NE, bool CSD, typename PS>
__device__ __noinline__ void sweep1d_local(ClusterTeam &t, const DevProblem &P, GroupShared &gs, Local1D &L,
                              const double *zin, double *zout, int matvec, int np_source, const double *phiE_in,
                              double *phiE_out, int ig) {
    const int nd = P.nd;
    const int nl = L.ce - L.cb;
    PS *psi = reinterpret_cast<PS *>(L.psi);
    int chunks = (int)blockDim.x / nd;
    if (chunks > nl) chunks = nl;
    if (chunks < 1) chunks = 1;
    const int dl = threadIdx.x / chunks, ch = threadIdx.x % chunks;
    const bool active = dl < nd && nl > 0;
    const int n = dl;
    const int lk = (nl + chunks - 1) / chunks;
    const int kb = min(nl, ch * lk), ke = min(nl, kb + lk);
    const bool fwd = active ? (P.cosv[n] >= 0.0) : true;
    const int cb = L.cb, ce = L.ce;
    const bool keyed = *L.nkey > 0;  // factored operators of the cell kinds (else per-cell solves)
    // 1. chunk maps
    if (active) {
        R Ac[NF * NF], bc[NF];
#pragma unroll
        for (int f = 0; f < NF; f++) {
            bc[f] = R(0);
#pragma unroll
            for (int g = 0; g < NF; g++) Ac[f + NF * g] = (f == g) ? R(1) : R(0);
        }
        if (keyed) {
            CellKey1D<R, NM, NF, NE, CSD, PS> cell(P, gs, L, n, phiE_in, phiE_out);
            for (int k = kb; k < ke; k++) {
                R A[NF * NF], b[NF];
                cell.map(fwd ? k : nl - 1 - k, psi, A, b);
                compose_map<R, NF>(A, b, Ac, bc);
            }
        } else {
            Cell1D<R, NM, NF, NE, CSD, PS> cell(P, gs, n, phiE_in, phiE_out, L.ldp, cb, L.mat, L.dx, L.scsd);
            for (int k = kb; k < ke; k++) {
                R A[NF * NF], b[NF];
                cell.map(fwd ? cb + k : ce - 1 - k, psi, A, b);
                compose_map<R, NF>(A, b, Ac, bc);
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
    // 2. the CTA's map of each direction (identity for a CTA without cells)
    if (dl < nd && ch == 0) {
        R A[NF * NF], b[NF];
#pragma unroll
        for (int f = 0; f < NF; f++) {
            b[f] = R(0);
#pragma unroll
            for (int g = 0; g < NF; g++) A[f + NF * g] = (f == g) ? R(1) : R(0);
        }
        if (nl > 0)
            for (int c2 = 0; c2 < chunks; c2++) {
                R A2[NF * NF], b2[NF];
                const int tid = dl * chunks + c2;
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    b2[f] = (R)gs.chb[tid][f];
#pragma unroll
                    for (int g = 0; g < NF; g++) A2[f + NF * g] = (R)gs.chA[tid][f + NF * g];
                }
                compose_map<R, NF>(A2, b2, A, b);
            }
        double *M = L.cmap + (long long)n * RB_LMAP;
#pragma unroll
        for (int f = 0; f < NF; f++) {
            M[NF * NF + f] = (double)b[f];
#pragma unroll
            for (int g = 0; g < NF; g++) M[f + NF * g] = (double)A[f + NF * g];
        }
    }
    t.sync();  // every CTA's maps visible to the cluster
    // 3. incoming flux of this CTA: the boundary flux through the maps of the CTAs upstream;
    //    CTA 0 goes on through every map for the exit flux
    const int C = (int)t.ncta, r = (int)t.crank;
    if (dl < nd && ch == 0 && (nl > 0 || r == 0)) {
        cg::cluster_group cl = cg::this_cluster();
        const bool fw = P.cosv[n] >= 0.0;
        double F0[RB_MAXFACE];
        boundary_in_1d(P, n, zin + P.off_b[0], np_source, ig, F0);
        R F[NF], Fin[NF];
#pragma unroll
        for (int f = 0; f < NF; f++) { F[f] = (R)F0[f]; Fin[f] = F[f]; }
        for (int s = 0; s < C; s++) {
            const int q = fw ? s : C - 1 - s;
            if (q == r) {
#pragma unroll
                for (int f = 0; f < NF; f++) Fin[f] = F[f];
                if (r != 0) break;
            }
            const double *M = cl.map_shared_rank(L.cmap, q) + (long long)n * RB_LMAP;
            apply_map<R, NF>(M, F);
        }
        if (r == 0)
#pragma unroll
            for (int f = 0; f < NF; f++) L.fx[(long long)n * RB_SCAN_NF + f] = (double)F[f];
        if (nl > 0)  // incoming flux of each chunk
            for (int c2 = 0; c2 < chunks; c2++) {
                const int tid = dl * chunks + c2;
                R Fn[NF];
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    gs.chF[tid][f] = (double)Fin[f];
                    R s = (R)gs.chb[tid][f];
#pragma unroll
                    for (int g = 0; g < NF; g++) s += (R)gs.chA[tid][f + NF * g] * Fin[g];
                    Fn[f] = s;
                }
#pragma unroll
                for (int f = 0; f < NF; f++) Fin[f] = Fn[f];
            }
    }
    __syncthreads();
    // 4. re-sweep each chunk from its incoming flux; ψ becomes the angular flux
    if (active) {
        R F[NF];
#pragma unroll
        for (int f = 0; f < NF; f++) F[f] = (R)gs.chF[threadIdx.x][f];
        if (keyed) {
            CellKey1D<R, NM, NF, NE, CSD, PS> cell(P, gs, L, n, phiE_in, phiE_out);
            for (int k = kb; k < ke; k++) cell.step(fwd ? k : nl - 1 - k, psi, F);
        } else {
            Cell1D<R, NM, NF, NE, CSD, PS> cell(P, gs, n, phiE_in, phiE_out, L.ldp, cb, L.mat, L.dx, L.scsd);
            for (int k = kb; k < ke; k++) cell.step(fwd ? cb + k : ce - 1 - k, psi, F);
        }
    }
    // 5. CTA 0: outgoing boundary moments, side 1 (X+) collects μ ≥ 0, side 0 (X-) μ < 0
    if (r == 0) {
        __syncthreads();
        const int nps = P.npsurf;
        const long long nb = P.nb[0];
        for (long long o = threadIdx.x; o < nb; o += blockDim.x) {
            const int p = (int)(o % nps);
            const int is = (int)((o / nps) % NF);
            const int side = (int)(o / ((long long)nps * NF));
            double s = 0.0;
            for (int m = 0; m < nd; m++) {
                const bool fw = P.cosv[m] >= 0.0;
                if ((side == 1) == fw) s += P.frow_d[(long long)nps * m + p] * L.fx[(long long)m * RB_SCAN_NF + is];
            }
            const long long k = P.off_b[0] + o;
            zout[k] = matvec ? zin[k] - s : s;
        }
    }
    __syncthreads();
}

template <typename R, typename PS>
__device__ bool sweep1d_local_fixed(ClusterTeam &t, const DevProblem &P, GroupShared &gs, Local1D &L,
                                    const double *zin, double *zout, int matvec, int np_source, const double *pE,
                                    double *phiE_out, int ig) {
    const int nm = P.nm5, nf = P.nmf[0], ne = P.nm4;
#define RB_LOCAL(NM_, NF_, NE_, CSD_) \
    sweep1d_local<R, NM_, NF_, NE_, CSD_, PS>(t, P, gs, L, zin, zout, matvec, np_source, pE, phiE_out, ig)
    if (!P.csd) {
        if (nm == 1 && nf == 1) { RB_LOCAL(1, 1, 1, false); return true; }
        if (nm == 2 && nf == 1) { RB_LOCAL(2, 1, 1, false); return true; }
        if (nm == 3 && nf == 1) { RB_LOCAL(3, 1, 1, false); return true; }
    } else {
        if (nm == 1 && nf == 1 && ne == 1) { RB_LOCAL(1, 1, 1, true); return true; }
        if (nm == 2 && nf == 1 && ne == 2) { RB_LOCAL(2, 1, 2, true); return true; }
        if (nm == 2 && nf == 2 && ne == 1) { RB_LOCAL(2, 2, 1, true); return true; }
        if (nm == 4 && nf == 2 && ne == 2) { RB_LOCAL(4, 2, 2, true); return true; }
    }
#undef RB_LOCAL
    return false;
}

// the products of the local pass, compiled as functions of their own so that their registers
// are allocated apart from the rest of the solve
template <typename T, typename PS>
__device__ __noinline__ void m2d_local(const DevProblem &P, GroupShared &gs, Local1D &L, const double *zin,
                                       int homog) {
    const int nd = P.nd, np = P.np, nm = P.nm5;
    const int nl = L.ce - L.cb;
    const long long col0 = (long long)nm * L.cb, ncl = (long long)nm * (nl > 0 ? nl : 0);
    PS *psi = reinterpret_cast<PS *>(L.psi);
    const long long ldp = L.ldp;
    CtaTeam ct;
    // M2D: ψ[n, col] = Mn·Qlout + Mn·(ys∘𝚽) + T·(Mn·ℳ)·𝚽 for the local columns
    if (ncl > 0) {
        const int *mat = L.mat;
        const double *ys = L.kmat;
        const double *add = homog ? nullptr : P.qnout;
        ProductArgs<double> a{P.mn, P.mnfp, nd, nd, np, zin + (long long)np * col0, np, ncl};
        auto sc = [=, &gs] __device__(int k, long long lc) {
            const int m = mat[lc / nm];
            return k < np ? ys[(long long)m * np + k] : gs.tg[m];
        };
        auto pre = [=] __device__(int i, long long lc) { return add ? add[(col0 + lc) * nd + i] : 0.0; };
        team_product<T>(ct, gs, a, sc, pre, [=] __device__(int i, long long lc, double v, double ad) {
            psi[i + ldp * lc] = (PS)(ad + v);
        });
    }
}

template <typename T, typename PS>
__device__ __noinline__ void d2m_local(const DevProblem &P, GroupShared &gs, Local1D &L, const double *zin,
                                       double *zout, int matvec) {
    const int nd = P.nd, np = P.np, nm = P.nm5;
    const int nl = L.ce - L.cb;
    const long long col0 = (long long)nm * L.cb, ncl = (long long)nm * (nl > 0 ? nl : 0);
    PS *psi = reinterpret_cast<PS *>(L.psi);
    const long long ldp = L.ldp;
    CtaTeam ct;
    // D2M: 𝚽[p, col] = Σ_n Dn[p,n]·ψ[n, col], direction order kept per output
    if (ncl > 0) {
        ProductArgs<PS> a{P.dn, nullptr, np, np, nd, psi, (int)ldp, ncl};
        auto one = [] __device__(int, long long) { return 1.0; };
        auto pre = [=] __device__(int i, long long lc) { return matvec ? zin[(col0 + lc) * np + i] : 0.0; };
        team_product<T>(ct, gs, a, one, pre, [=] __device__(int i, long long lc, double v, double z) {
            zout[(col0 + lc) * np + i] = matvec ? z - v : v;
        });
    }
}

// One pass T(z) = A·z + c (matvec: z − A·z) of a 1D problem whose local region fits. T is the
// arithmetic type of the products and the sweep, PS the storage type of ψ.
template <typename T, typename PS>
__device__ void pass1d_local_t(ClusterTeam &t, const DevProblem &P, GroupShared &gs, Local1D &L, const double *zin,
                               double *zout, int homog, int matvec, int ig, const double *phiE_in,
                               double *phiE_out) {
    m2d_local<T, PS>(P, gs, L, zin, homog);
    const int np_source = homog ? 0 : P.np_source;
    const double *pE = (P.csd && !homog) ? phiE_in : nullptr;
    sweep1d_local_fixed<T, PS>(t, P, gs, L, zin, zout, matvec, np_source, pE, phiE_out, ig);
    d2m_local<T, PS>(P, gs, L, zin, zout, matvec);
    t.sync();
}

__device__ __forceinline__ void pass1d_local(ClusterTeam &t, const DevProblem &P, GroupShared &gs, void *base,
                                             const double *zin, double *zout, int homog, int matvec, int ig,
                                             const double *phiE_in, double *phiE_out, int mixed) {
    Local1D L(P, t.crank, t.ncta, base);
    if (mixed) pass1d_local_t<float, float>(t, P, gs, L, zin, zout, homog, matvec, ig, phiE_in, phiE_out);
    else pass1d_local_t<double, double>(t, P, gs, L, zin, zout, homog, matvec, ig, phiE_in, phiE_out);
}

}  // namespace rb
