// rb_sweep_md.cuh -- the 2D and 3D sweeps (sn_sweep_2D.jl:54-183, sn_sweep_3D.jl:57-239) and
// their cell closures (flux_2D/3D_BTE/BFP, sn_2D_bte.jl:35-116, sn_2D_bfp.jl:45-154,
// sn_3D_bte.jl:42-152, sn_3D_bfp.jl:52-191).
//
// Ordering: a cell needs the outgoing faces of its upwind x, y (and z) neighbours. Planes are
// taken in z sweep order; inside a plane the rows form a skewed pipeline (KBA wavefront on
// ix + iy): at step s, the thread of row r solves column s − r, so its upwind x face is the one it
// produced at step s − 1 (kept in registers) and its upwind y face is the one row r − 1 produced
// at step s − 1 (handed over through shared memory, one slot per column). The z face comes from
// the previous plane (a per-direction scratch plane in global memory). Several directions share
// a CTA when the rows are fewer than its threads; directions are dealt to the team's CTAs.
// Results equal the reference's lexicographic order exactly in exact arithmetic, because every
// cell still sees the same upwind faces.
#pragma once
#include "rb_kernels.cuh"

namespace rb {

// Incoming face flux of direction n through the boundary face `face` at face cell `fcell`:
// surface source into moment 1 plus the lagged reflective / periodic in-moments of that face
// (sn_sweep_2D.jl:71-99, sn_sweep_3D.jl:80-163).
__device__ __forceinline__ void boundary_in_md(const DevProblem &P, int n, int axis, bool fwd, long long fcell,
                                               const double *zin, int np_source, int ig, double *f0, int nf) {
    const int face = 2 * axis + (fwd ? 0 : 1), side = fwd ? 0 : 1;
    const double *mrow = P.frow_m + ((long long)axis * P.nd + n) * P.npsurf;
    for (int f = 0; f < nf; f++) f0[f] = 0.0;
    const double *src = P.surf[face];
    if (src)
        for (int p = 0; p < np_source; p++)
            f0[0] += mrow[p] * src[ig + (long long)P.ng * (p + (long long)P.np_source * fcell)];
    const int bcv = P.bc[face];
    if (bcv != 0) {
        const int rside = (bcv == 1) ? side : 1 - side;
        const double *b = zin + P.off_b[axis];
        for (int p = 0; p < P.npsurf; p++)
            for (int is = 0; is < nf; is++)
                f0[is] += mrow[p] * b[p + (long long)P.npsurf * (is + (long long)nf * (rside + 2 * fcell))];
    }
}

// The closure of one cell with the run-time shapes of the problem (nm ≤ RB_MAXNM). F[a] holds the
// incoming face moments of axis a and receives the outgoing ones; FE likewise for the energy face.
struct CellMDrt {
    __device__ static void step(const DevProblem &P, const GroupShared &gs, int n, int nax, const double *h,
                                const bool *tang_unused, int m, double *Qn, double (*F)[RB_MAXFACE], double *FE) {
        const int nm = P.nm5;
        double S[RB_MAXNM * RB_MAXNM], q[RB_MAXNM];
#pragma unroll 1
        for (int e = 0; e < nm * nm; e++) S[e] = P.csd ? P.scsd[(long long)m * nm * nm + e] : 0.0;
#pragma unroll 1
        for (int i = 0; i < nm; i++) { S[i + nm * i] += gs.sigt[m]; q[i] = Qn[i]; }
#pragma unroll 1
        for (int a = 0; a < nax; a++) {
            const long long blk = (long long)n * 3 + a;
            const double *Gr = P.G + blk * nm * nm, *Gs = P.Gsrc + blk * nm * P.nfmax;
            const int nf = P.nmf[a];
#pragma unroll 1
            for (int e = 0; e < nm * nm; e++) S[e] += h[a] * Gr[e];
#pragma unroll 1
            for (int j = 0; j < nm; j++) {
                double s = 0.0;
#pragma unroll 1
                for (int f = 0; f < nf; f++) s += Gs[j + nm * f] * F[a][f];
                q[j] += h[a] * s;
            }
        }
        if (P.csd) {
            const int ne = P.nm4;
#pragma unroll 1
            for (int j = 0; j < nm; j++) {
                double s = 0.0;
#pragma unroll 1
                for (int e = 0; e < ne; e++) s += (P.EsA[j + nm * e] * gs.sp[m] - P.EsB[j + nm * e] * gs.sm[m]) * FE[e];
                q[j] -= s;
            }
        }
        lu_solve_rt<double>(S, q, nm);
#pragma unroll 1
        for (int a = 0; a < nax; a++) {
            const long long blk = (long long)n * 3 + a;
            const double *Go = P.Gout + blk * nm * P.nfmax;
            const int nf = P.nmf[a];
            double Fo[RB_MAXFACE];
#pragma unroll 1
            for (int f = 0; f < nf; f++) {
                double s = P.w1[a] * F[a][f];
#pragma unroll 1
                for (int j = 0; j < nm; j++) s += Go[f + nf * j] * q[j];
                Fo[f] = s;
            }
#pragma unroll 1
            for (int f = 0; f < nf; f++) F[a][f] = Fo[f];
        }
        if (P.csd) {
            const int ne = P.nm4;
            double Eo[RB_MAXFACE];
#pragma unroll 1
            for (int e = 0; e < ne; e++) {
                double s = P.w1[3] * FE[e];
#pragma unroll 1
                for (int j = 0; j < nm; j++) s += P.Eout[e + ne * j] * q[j];
                Eo[e] = s;
            }
#pragma unroll 1
            for (int e = 0; e < ne; e++) FE[e] = Eo[e];
        }
#pragma unroll 1
        for (int j = 0; j < nm; j++) Qn[j] = q[j];
    }
};

// The same closure with compile-time shapes (NM cell moments, NF face moments per axis, NE
// energy-face moments): everything stays in registers.
template <int NM, int NF, int NE, bool CSD, int NAX>
struct CellMDfix {
    __device__ static void step(const DevProblem &P, const GroupShared &gs, int n, const double *h, int m,
                                double (&Qn)[NM], double (&F)[3][NF], double (&FE)[NE]) {
        double S[NM * NM], q[1][NM];
#pragma unroll
        for (int e = 0; e < NM * NM; e++) S[e] = CSD ? P.scsd[(long long)m * NM * NM + e] : 0.0;
#pragma unroll
        for (int i = 0; i < NM; i++) { S[i + NM * i] += gs.sigt[m]; q[0][i] = Qn[i]; }
#pragma unroll
        for (int a = 0; a < NAX; a++) {
            const long long blk = (long long)n * 3 + a;
            const double *Gr = P.G + blk * NM * NM, *Gs = P.Gsrc + blk * NM * P.nfmax;
#pragma unroll
            for (int e = 0; e < NM * NM; e++) S[e] += h[a] * __ldg(Gr + e);
#pragma unroll
            for (int j = 0; j < NM; j++) {
                double s = 0.0;
#pragma unroll
                for (int f = 0; f < NF; f++) s += __ldg(Gs + j + NM * f) * F[a][f];
                q[0][j] += h[a] * s;
            }
        }
        if (CSD) {
#pragma unroll
            for (int j = 0; j < NM; j++) {
                double s = 0.0;
#pragma unroll
                for (int e = 0; e < NE; e++) s += (__ldg(P.EsA + j + NM * e) * gs.sp[m] - __ldg(P.EsB + j + NM * e) * gs.sm[m]) * FE[e];
                q[0][j] -= s;
            }
        }
        lu_solve<double, NM, 1>(S, q);
#pragma unroll
        for (int a = 0; a < NAX; a++) {
            const double *Go = P.Gout + ((long long)n * 3 + a) * NM * P.nfmax;
            double Fo[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) {
                double s = P.w1[a] * F[a][f];
#pragma unroll
                for (int j = 0; j < NM; j++) s += __ldg(Go + f + NF * j) * q[0][j];
                Fo[f] = s;
            }
#pragma unroll
            for (int f = 0; f < NF; f++) F[a][f] = Fo[f];
        }
        if (CSD) {
            double Eo[NE];
#pragma unroll
            for (int e = 0; e < NE; e++) {
                double s = P.w1[3] * FE[e];
#pragma unroll
                for (int j = 0; j < NM; j++) s += __ldg(P.Eout + e + NE * j) * q[0][j];
                Eo[e] = s;
            }
#pragma unroll
            for (int e = 0; e < NE; e++) FE[e] = Eo[e];
        }
#pragma unroll
        for (int j = 0; j < NM; j++) Qn[j] = q[0][j];
    }
};

// Run-time shapes routed through CellMDrt, with the arrays of the largest shapes.
struct CellMDgen {
    __device__ static void step(const DevProblem &P, const GroupShared &gs, int n, const double *h, int m,
                                double (&Qn)[RB_MAXNM], double (&F)[3][RB_MAXFACE], double (&FE)[RB_MAXFACE]) {
        CellMDrt::step(P, gs, n, P.ndims, h, nullptr, m, Qn, F, FE);
    }
};

// Scratch layout per direction (global): x exits [ny·nz], y exits [nx·nz], z exits [nx·ny],
// the z-face plane [nx·ny] and (3D) the y-face plane [nx·nz] handed between rows / tiles, then
// the incoming boundary fluxes of the x, y and z faces [ny·nz], [nx·nz], [nx·ny]; each × nfmax
// doubles. (rb_capi.cu allocates nd times this stride.)
__host__ __device__ __forceinline__ long long md_scratch_stride_n(long long nx, long long ny, long long nz, int nfm) {
    return (2 * ny * nz + 3 * nx * nz + 3 * nx * ny) * nfm;
}
__device__ __forceinline__ long long md_scratch_stride(const DevProblem &P) {
    return md_scratch_stride_n(P.nx, P.ny, P.nz, P.nfmax);
}
// offset of the incoming boundary fluxes of axis a inside a direction's scratch
__device__ __forceinline__ long long md_in_offset(const DevProblem &P, int a) {
    const long long nx = P.nx, ny = P.ny, nz = P.nz;
    const long long base = ny * nz + 2 * nx * nz + 2 * nx * ny;
    return (a == 0 ? base : (a == 1 ? base + ny * nz : base + ny * nz + nx * nz)) * P.nfmax;
}

// The incoming face flux of every direction on every boundary face cell it enters through
// (boundary_in_md: surface source plus the lagged reflective / periodic in-moments), as one
// team phase before the sweep, so that the sweep reads one value per face cell instead of a
// half-range sum per cell and direction.
template <class Team>
__device__ void boundary_in_phase(Team &t, const DevProblem &P, const double *zin, int np_source, int ig) {
    const long long sstride = md_scratch_stride(P);
    const int nfm = P.nfmax;
    for (int a = 0; a < P.ndims; a++) {
        const long long nfc = P.fcells[a];
        const int nf = P.nmf[a];
        const long long off = md_in_offset(P, a);
        for (long long o = t.rank(); o < (long long)P.nd * nfc; o += t.size()) {
            const int n = (int)(o / nfc);
            const long long fc = o % nfc;
            const bool fwd = P.cosv[(long long)a * P.nd + n] >= 0.0;
            double f0[RB_MAXFACE];
            boundary_in_md(P, n, a, fwd, fc, zin, np_source, ig, f0, nf);
            double *dst = P.fexit + (long long)n * sstride + off + fc * nfm;
            for (int f = 0; f < nf; f++) dst[f] = f0[f];
        }
    }
}

// 3D: pencils along x in tiles of TY×TZ (one thread per pencil). Inside a tile the cells form a
// hyperplane wavefront on ix + iy + iz: at step s the pencil (jy, jz) solves column s − jy − jz,
// reading the y face its lower neighbour wrote at step s − 1 and the z face its back neighbour
// wrote at step s − 1, both through per-direction face planes (L2-resident). Tiles are taken in
// an order that finishes both upwind tiles first (z-tiles outer, y-tiles inner, in sweep order).
template <class Cell, int AM, int AF, int AE, class Team>
__device__ void sweep_3d_tiles(Team &t, const DevProblem &P, GroupShared &gs, const double *zin, int np_source,
                               const double *phiE_in, double *phiE_out, int ig) {
    const int nd = P.nd, nx = P.nx, ny = P.ny, nz = P.nz, nfm = P.nfmax;
    const int nm = AM == 1 ? 1 : P.nm5, ne = AE == 1 ? 1 : P.nm4;  // compile-time 1 on the register path
    const int ncta = (int)t.ncta, crank = (int)t.crank;
    const int my_dirs = (nd - crank + ncta - 1) / ncta;
    const int TY = ny < 16 ? ny : 16, TZ = nz < 16 ? nz : 16;
    const int ntile_y = (ny + TY - 1) / TY, ntile_z = (nz + TZ - 1) / TZ;
    const int pen = TY * TZ;                               // pencils per tile
    int D = (int)blockDim.x / pen;                         // directions per round
    if (D < 1) D = 1;
    const long long sstride = md_scratch_stride(P);
    const int nfx = AF == 1 ? 1 : P.nmf[0], nfy = AF == 1 ? 1 : P.nmf[1], nfz = AF == 1 ? 1 : P.nmf[2];
    // one-moment cells and faces: inside a tile the y and z faces pass between neighbouring
    // pencils through shared memory, double-buffered by step parity (the pencil (jy, jz) reads at
    // step s what (jy−1, jz) and (jy, jz−1) wrote at step s − 1; tile edges use the global face
    // planes), and each pencil loads the source, material and width of its next cell while it
    // solves the current one
    constexpr bool PF = AM == 1 && AF == 1;
    const bool smf = PF && 4 * D * pen <= RB_TILE_DOUBLES;
    double *sfy = gs.tile, *sfz = gs.tile + 2 * D * pen;  // [2][D·pen] each
    for (int k0 = 0; k0 < my_dirs; k0 += D) {
        const int dl = threadIdx.x / pen, pl = threadIdx.x % pen;
        const int jy = pl % TY, jz = pl / TY;
        const bool active = dl < D && k0 + dl < my_dirs;
        const int n = crank + (k0 + dl) * ncta;
        const double mu = active ? P.cosv[n] : 0.0, eta = active ? P.cosv[nd + n] : 0.0;
        const double xi = active ? P.cosv[2 * nd + n] : 0.0;
        const bool fx = mu >= 0.0, fy = eta >= 0.0, fz = xi >= 0.0;
        double *scr = P.fexit + (active ? (long long)n * sstride : 0);
        double *exx = scr, *exy = exx + (long long)ny * nz * nfm, *exz = exy + (long long)nx * nz * nfm;
        double *zfc = exz + (long long)nx * ny * nfm, *yfc = zfc + (long long)nx * ny * nfm;
        for (int tz = 0; tz < ntile_z; tz++) {
            for (int ty = 0; ty < ntile_y; ty++) {
                const int iyy = ty * TY + jy, izz = tz * TZ + jz;
                const bool pcl = active && iyy < ny && izz < nz;
                const int iy = fy ? iyy : ny - 1 - iyy, iz = fz ? izz : nz - 1 - izz;
                double F[3][AF], FE[AE], Qn[AM];
                double qpre = 0.0, dxpre = 1.0;
                int mpre = 0;
                const int me = dl * pen + pl;  // this pencil's slot in the shared face buffers
                for (int s = 0; s < nx + TY + TZ - 2; s++) {
                    const int ixx = s - jy - jz;
                    const int rd = ((s + 1) & 1) * D * pen, wr = (s & 1) * D * pen;
                    if (pcl && ixx >= 0 && ixx < nx) {
                        const int ix = fx ? ixx : nx - 1 - ixx;
                        const long long c = ix + (long long)nx * (iy + (long long)ny * iz);
                        const long long yk = (ix + (long long)nx * iz) * nfm, zk = (ix + (long long)nx * iy) * nfm;
                        if (ixx == 0)
                            boundary_in_md(P, n, 0, fx, iy + (long long)ny * iz, zin, np_source, ig, F[0], nfx);
                        if (iyy == 0)
                            boundary_in_md(P, n, 1, fy, ix + (long long)nx * iz, zin, np_source, ig, F[1], nfy);
                        else if (smf && jy > 0)
                            F[1][0] = sfy[rd + me - 1];
                        else
                            for (int f = 0; f < nfy; f++) F[1][f] = yfc[yk + f];
                        if (izz == 0)
                            boundary_in_md(P, n, 2, fz, ix + (long long)nx * iy, zin, np_source, ig, F[2], nfz);
                        else if (smf && jz > 0)
                            F[2][0] = sfz[rd + me - TY];
                        else
                            for (int f = 0; f < nfz; f++) F[2][f] = zfc[zk + f];
                        double *pc = P.psi + n + (long long)nd * nm * c;
                        int m;
                        double dxc;
                        if (PF && ixx > 0) {
                            m = mpre;
                            dxc = dxpre;
                            Qn[0] = qpre;
                        } else {
                            m = P.mat[c];
                            dxc = P.dx[ix];
                            for (int j = 0; j < nm; j++) Qn[j] = pc[(long long)nd * j];
                        }
                        if (PF && ixx + 1 < nx) {  // the next cell of this pencil
                            const int ixn = fx ? ix + 1 : ix - 1;
                            const long long cn = fx ? c + 1 : c - 1;
                            qpre = P.psi[n + (long long)nd * cn];
                            mpre = P.mat[cn];
                            dxpre = P.dx[ixn];
                        }
                        double h[3] = {fabs(mu) / dxc, fabs(eta) / P.dy[iy], fabs(xi) / P.dz[iz]};
                        if (P.csd)
                            for (int e = 0; e < ne; e++)
                                FE[e] = phiE_in ? phiE_in[n + (long long)nd * (e + (long long)ne * c)] : 0.0;
                        Cell::step(P, gs, n, h, m, Qn, F, FE);
                        for (int j = 0; j < nm; j++) pc[(long long)nd * j] = Qn[j];
                        if (P.csd)
                            for (int e = 0; e < ne; e++) phiE_out[n + (long long)nd * (e + (long long)ne * c)] = FE[e];
                        if (smf) {
                            sfy[wr + me] = F[1][0];
                            sfz[wr + me] = F[2][0];
                        }
                        if (iyy < ny - 1) {
                            if (!smf || jy == TY - 1) for (int f = 0; f < nfy; f++) yfc[yk + f] = F[1][f];
                        } else {
                            for (int f = 0; f < nfy; f++) exy[yk + f] = F[1][f];
                        }
                        if (izz < nz - 1) {
                            if (!smf || jz == TZ - 1) for (int f = 0; f < nfz; f++) zfc[zk + f] = F[2][f];
                        } else {
                            for (int f = 0; f < nfz; f++) exz[zk + f] = F[2][f];
                        }
                        if (ixx == nx - 1) for (int f = 0; f < nfx; f++) exx[(iy + (long long)ny * iz) * nfm + f] = F[0][f];
                    }
                    __syncthreads();
                }
            }
        }
    }
}

template <class Cell, int AM, int AF, int AE, class Team>
__device__ void sweep_md(Team &t, const DevProblem &P, GroupShared &gs, const double *zin, int np_source,
                         const double *phiE_in, double *phiE_out, int ig) {
    const int nd = P.nd, nx = P.nx, ny = P.ny, nz = P.nz, nax = P.ndims, nfm = P.nfmax;
    const int nm = AM == 1 ? 1 : P.nm5, ne = AE == 1 ? 1 : P.nm4;  // compile-time 1 on the register path
    const int nfx = AF == 1 ? 1 : P.nmf[0], nfz = AF == 1 ? 1 : P.nmf[2];
    const int ncta = (int)t.ncta, crank = (int)t.crank;
    const int my_dirs = (nd - crank + ncta - 1) / ncta;
    const int R = ny < (int)blockDim.x ? ny : (int)blockDim.x;   // rows per direction
    int D = (int)blockDim.x / R;                                  // directions per round,
    const int dmax = RB_TILE_DOUBLES / (nx * P.nmf[1]);           // bounded by the y-face slots
    if (D > dmax) D = dmax;
    const int nrb = (ny + R - 1) / R;
    const long long sstride = md_scratch_stride(P);
    double *yface = gs.tile;  // [D][nx][nf_y]
    const int nfy = AF == 1 ? 1 : P.nmf[1];
    for (int k0 = 0; k0 < my_dirs; k0 += D) {
        const int dl = threadIdx.x / R, r = threadIdx.x % R;
        const bool active = dl < D && k0 + dl < my_dirs;
        const int n = crank + (k0 + dl) * ncta;
        const double mu = active ? P.cosv[n] : 0.0, eta = active ? P.cosv[nd + n] : 0.0;
        const double xi = (active && nax == 3) ? P.cosv[2 * nd + n] : 0.0;
        const bool fx = mu >= 0.0, fy = eta >= 0.0, fz = xi >= 0.0;
        double *scr = P.fexit + (active ? (long long)n * sstride : 0);
        double *exx = scr, *exy = exx + (long long)ny * nz * nfm, *exz = exy + (long long)nx * nz * nfm;
        double *zfc = exz + (long long)nx * ny * nfm;
        double *yf = yface + (long long)dl * nx * nfy;
        for (int izz = 0; izz < nz; izz++) {
            const int iz = fz ? izz : nz - 1 - izz;
            for (int rb = 0; rb < nrb; rb++) {
                const int iyy = rb * R + r;
                const bool row = active && iyy < ny;
                const int iy = fy ? iyy : ny - 1 - iyy;
                double F[3][AF], FE[AE], Qn[AM];
                for (int s = 0; s < nx + R - 1; s++) {
                    const int ixx = s - r;
                    if (row && ixx >= 0 && ixx < nx) {
                        const int ix = fx ? ixx : nx - 1 - ixx;
                        const long long c = ix + (long long)nx * (iy + (long long)ny * iz);
                        if (ixx == 0)  // X face of the row (sn_sweep_2D.jl:103-132)
                            boundary_in_md(P, n, 0, fx, iy + (long long)ny * iz, zin, np_source, ig, F[0], nfx);
                        if (iyy == 0)  // Y face of the column (sn_sweep_2D.jl:71-99)
                            boundary_in_md(P, n, 1, fy, ix + (long long)nx * iz, zin, np_source, ig, F[1], nfy);
                        else
                            for (int f = 0; f < nfy; f++) F[1][f] = yf[(long long)ixx * nfy + f];
                        if (nax == 3) {
                            if (izz == 0)  // Z face (sn_sweep_3D.jl:80-108)
                                boundary_in_md(P, n, 2, fz, ix + (long long)nx * iy, zin, np_source, ig, F[2], nfz);
                            else
                                for (int f = 0; f < nfz; f++) F[2][f] = zfc[(ix + (long long)nx * iy) * nfm + f];
                        }
                        const int m = P.mat[c];
                        double h[3];
                        h[0] = fabs(mu) / P.dx[ix];
                        h[1] = fabs(eta) / P.dy[iy];
                        h[2] = nax == 3 ? fabs(xi) / P.dz[iz] : 0.0;
                        double *pc = P.psi + n + (long long)nd * nm * c;
                        for (int j = 0; j < nm; j++) Qn[j] = pc[(long long)nd * j];
                        if (P.csd)
                            for (int e = 0; e < ne; e++)
                                FE[e] = phiE_in ? phiE_in[n + (long long)nd * (e + (long long)ne * c)] : 0.0;
                        Cell::step(P, gs, n, h, m, Qn, F, FE);
                        for (int j = 0; j < nm; j++) pc[(long long)nd * j] = Qn[j];
                        if (P.csd)
                            for (int e = 0; e < ne; e++) phiE_out[n + (long long)nd * (e + (long long)ne * c)] = FE[e];
                        for (int f = 0; f < nfy; f++) yf[(long long)ixx * nfy + f] = F[1][f];
                        if (nax == 3) {
                            if (izz < nz - 1)
                                for (int f = 0; f < nfz; f++) zfc[(ix + (long long)nx * iy) * nfm + f] = F[2][f];
                            else
                                for (int f = 0; f < nfz; f++) exz[(ix + (long long)nx * iy) * nfm + f] = F[2][f];
                        }
                        if (ixx == nx - 1)
                            for (int f = 0; f < nfx; f++) exx[(iy + (long long)ny * iz) * nfm + f] = F[0][f];
                        if (iyy == ny - 1)
                            for (int f = 0; f < nfy; f++) exy[(ix + (long long)nx * iz) * nfm + f] = F[1][f];
                    }
                    __syncthreads();
                }
            }
        }
    }
}

// Outgoing boundary moments of every face: b[p,is,side,cell] = Σ_n Dn_face[n][p]·exit[n][cell][is]
// over the directions leaving through that side (sn_sweep_2D.jl:146-179, accumulated over n in
// order as sn_inner_pass.jl:127-129 does).
//
// One thread per (face cell, face moment, side, block of PB half-range moments), neighbouring
// lanes on neighbouring face cells: the exit loads of a warp are contiguous and its cosine and
// half-range row loads are one address (one request, no divergence). The loads of 8 directions
// go out together; a direction leaving through the other side enters with weight 0, which adds
// exactly zero, so each moment is the sum over its side's directions in increasing n, as with one
// thread per output. PB trades exit re-reads against threads (boundary_out_md picks it).
template <int PB, class Team>
__device__ void boundary_out_pb(Team &t, const DevProblem &P, const double *zin, double *zout, int matvec) {
    const int nd = P.nd, nps = P.npsurf, nfm = P.nfmax;
    const int npb = (nps + PB - 1) / PB;
    const long long sstride = md_scratch_stride(P);
    for (int a = 0; a < P.ndims; a++) {
        const int nf = P.nmf[a];
        const long long nfc = P.nb[a] / ((long long)nps * nf * 2);
        const long long off = a == 0 ? 0 : (a == 1 ? (long long)P.ny * P.nz * nfm : ((long long)P.ny * P.nz + (long long)P.nx * P.nz) * nfm);
        const long long offb = P.off_b[a];
        const double *crow = P.cosv + (long long)a * nd;
        const double *frow = P.frow_d + (long long)a * nd * nps;
        const double *fex = P.fexit;
        const long long nitem = nfc * nf * 2 * npb;
        for (long long u = t.rank(); u < nitem; u += t.size()) {
            const long long cell = u % nfc;
            const long long rest = u / nfc;
            const int is = (int)(rest % nf);
            const int side = (int)((rest / nf) % 2);
            const int p0 = (int)(rest / (2LL * nf)) * PB;
            const double *ex = fex + off + cell * nfm + is;
            double acc[PB];
#pragma unroll
            for (int q = 0; q < PB; q++) acc[q] = 0.0;
            for (int n0 = 0; n0 < nd; n0 += 8) {
                double v[8];
                bool use[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int n = min(n0 + e, nd - 1);
                    v[e] = ex[(long long)n * sstride];
                    use[e] = n0 + e < nd && ((crow[n] >= 0.0) == (side == 1));
                }
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int n = min(n0 + e, nd - 1);
                    const double *fr = frow + (long long)n * nps;
#pragma unroll
                    for (int q = 0; q < PB; q++) {
                        const double w = fr[min(p0 + q, nps - 1)];
                        acc[q] = fma(use[e] ? w : 0.0, v[e], acc[q]);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < PB; q++) {
                if (p0 + q >= nps) continue;
                const long long k = offb + (p0 + q) + (long long)nps * (is + (long long)nf * (side + 2 * cell));
                zout[k] = matvec ? zin[k] - acc[q] : acc[q];
            }
        }
    }
}

// One thread per output, neighbouring lanes on neighbouring moments of one face cell (the exit
// loads of a warp are one address): the layout for faces too small to give the blocked form
// above a few items per thread.
template <class Team>
__device__ void boundary_out_rows(Team &t, const DevProblem &P, const double *zin, double *zout, int matvec) {
    const int nd = P.nd, nps = P.npsurf, nfm = P.nfmax;
    const long long sstride = md_scratch_stride(P);
    for (int a = 0; a < P.ndims; a++) {
        const int nf = P.nmf[a];
        const long long off = a == 0 ? 0 : (a == 1 ? (long long)P.ny * P.nz * nfm : ((long long)P.ny * P.nz + (long long)P.nx * P.nz) * nfm);
        for (long long o = t.rank(); o < P.nb[a]; o += t.size()) {
            const int p = (int)(o % nps);
            const int is = (int)((o / nps) % nf);
            const int side = (int)((o / ((long long)nps * nf)) % 2);
            const long long cell = o / ((long long)nps * nf * 2);
            double s = 0.0;
            for (int n = 0; n < nd; n++) {
                const bool fwd = P.cosv[(long long)a * nd + n] >= 0.0;
                if ((side == 1) == fwd)
                    s += P.frow_d[((long long)a * nd + n) * nps + p] * P.fexit[(long long)n * sstride + off + cell * nfm + is];
            }
            const long long k = P.off_b[a] + o;
            zout[k] = matvec ? zin[k] - s : s;
        }
    }
}

// Faces with many outputs per thread of the team take the blocked form with the largest moment
// block that still gives every thread about two items; small faces take one thread per output.
// Both forms give the same sums, in the same order.
template <class Team>
__device__ void boundary_out_md(Team &t, const DevProblem &P, const double *zin, double *zout, int matvec) {
    long long outs = 0;
    for (int a = 0; a < P.ndims; a++) outs += P.nb[a];
    const long long want = 2LL * t.size();
    if (outs / 16 >= want) boundary_out_pb<16>(t, P, zin, zout, matvec);
    else if (outs / 4 >= want) boundary_out_pb<4>(t, P, zin, zout, matvec);
    else boundary_out_rows(t, P, zin, zout, matvec);
}

}  // namespace rb
