// rb_sweep_oct.cuh -- 2D and 3D sweeps of one-moment cells (order-1 closures in every axis and
// in energy: the diamond-difference / DG0 cells of sn_2D_bte.jl:35-116, sn_2D_bfp.jl:45-154,
// sn_3D_bte.jl:42-152, sn_3D_bfp.jl:52-191), in FP64 (plain form) or FP32 (mixed form).
//
// 3D: directions are held grouped by octant, and all directions of one octant share one sweep
// order, so a thread owns one x-pencil (iy, iz) of a TY×TZ tile and solves up to DB directions
// of one octant at each cell it visits. Inside a tile the pencils form a hyperplane wavefront:
// at local step σ the pencil (jy, jz) solves column σ − jy − jz. The x face stays in registers;
// the y face of the pencil below comes by warp shuffle (it is the neighbouring lane); the z face
// of the pencil behind comes through shared memory, double-buffered by step parity. Tiles hand
// their outgoing y/z faces to the downstream tiles through per-direction face planes in global
// memory. Every (octant batch, tile) is one task on one CTA of the team; a tile is paced by its
// upwind tiles through per-CTA progress flags (a release after each pair of steps, an acquire
// before the faces of a step are staged), so it runs about one tile height behind them with no
// team barrier inside the sweep. The cell's inputs (angular source, material, incoming
// energy-face flux, and the faces entering the tile) are staged one step ahead with cp.async.
// Each cell sees the same upwind faces as in the reference's lexicographic order
// (sn_sweep_3D.jl:73-110), so the result equals it up to rounding.
//
// 2D: the KBA wavefront of sweep_md (rows of a direction skewed by one column per row, y faces
// handed between rows through shared memory), one direction per thread, with the next cell's
// inputs loaded one step ahead.
#pragma once
#include "rb_sweep_md.cuh"
#include "rb_tc.cuh"

#define RB_OCT_TILE 16   // tile edge in pencils (3D): 16×16 pencils, one per thread

namespace rb {

// octant batches: octant o's directions cut into ceil(count/db) batches of at most db
__device__ __forceinline__ int oct_groups(const DevProblem &P, int db) {
    int ng = 0;
    for (int o = 0; o < P.noct; o++) ng += (P.oct_start[o + 1] - P.oct_start[o] + db - 1) / db;
    return ng;
}
__device__ __forceinline__ int oct_group(const DevProblem &P, int db, int g, int &first, int &cnt) {
    for (int o = 0; o < P.noct; o++) {
        const int c = P.oct_start[o + 1] - P.oct_start[o], nb = (c + db - 1) / db;
        if (g < nb) {
            first = P.oct_start[o] + g * db;
            cnt = min(db, c - g * db);
            return o;
        }
        g -= nb;
    }
    first = 0;
    cnt = 0;
    return 0;
}

// The problem is a one-moment 2D/3D problem (every closure of order 1).
__device__ __forceinline__ bool one_moment_md(const DevProblem &P) {
    return P.nm5 == 1 && P.nmf[0] == 1 && P.nmf[1] == 1 && (P.ndims < 3 || P.nmf[2] == 1) && P.nm4 == 1;
}

template <typename R> struct OctDB { static constexpr int value = 10; };  // FP64: registers
template <> struct OctDB<float> { static constexpr int value = 12; };

// Stages of a step's inputs (cp.async, one step ahead): three, which lets a step write back the
// previous step's flux after its single barrier; two for FP64 with CSD (three do not fit beside
// the FP64 energy-face stages), with a second barrier per step.
template <typename R, bool CSD> struct OctNB { static constexpr int value = 3; };
template <> struct OctNB<double, true> { static constexpr int value = 2; };
#define RB_OCT_MAXNX 1024  // x widths whose inverses the sweep keeps in shared memory
#define RB_OCT_PUB 2       // a CTA publishes its progress every RB_OCT_PUB steps (and after its last)

// Shared-memory plan of the 3D octant sweep (byte offsets, each array 16-byte aligned): the
// staged upwind faces of the tile's first row and layer of pencils, OctNB stages of a step's
// angular source / flux, energy-face flux (CSD) and materials, the z-face hand-off between
// pencils (double-buffered by step parity), the direction constants of the octant batch, the
// inverse x widths and the per-material cell terms, and each pencil's cell base and coordinates.
template <typename R, bool CSD>
struct Oct3dSmem {
    static constexpr long long DB = OctDB<R>::value, T = RB_OCT_TILE, TP = T * T, NB = OctNB<R, CSD>::value;
    static constexpr long long RS = (long long)sizeof(R);
    static constexpr long long al(long long b) { return (b + 15) & ~15LL; }
    static constexpr long long fy = 0;                                      // double [NB][T][DB]
    static constexpr long long fz = fy + al(NB * T * DB * 8);               // double [NB][T][DB]
    static constexpr long long eb = fz + al(NB * T * DB * 8);               // double [NB][TP][DB]
    static constexpr long long pcb = eb + (CSD ? al(NB * TP * DB * 8) : 0); // long long [TP]
    static constexpr long long dc = pcb + al(TP * 8);                       // R [DB][9]
    static constexpr long long sfz = dc + al(DB * 9 * RS);                  // R [2][DB][TP]
    static constexpr long long qb = sfz + al(2 * DB * TP * RS);             // R [NB][TP][DB]
    static constexpr long long ix = qb + al(NB * TP * DB * RS);             // R [RB_OCT_MAXNX]
    static constexpr long long ms = ix + al(RB_OCT_MAXNX * RS);             // R [RB_MAXMAT]
    static constexpr long long mq = ms + al(RB_MAXMAT * RS);                // R [RB_MAXMAT]
    static constexpr long long mb = mq + al(RB_MAXMAT * RS);                // int [NB][TP]
    static constexpr long long pj = mb + al(NB * TP * 4);                   // int [TP]
    static constexpr long long py = pj + al(TP * 4);                        // int [TP]
    static constexpr long long pz = py + al(TP * 4);                        // int [TP]
    static constexpr long long bytes = pz + al(TP * 4);
};
template <typename R, bool CSD>
__host__ __device__ constexpr long long oct3d_smem() { return Oct3dSmem<R, CSD>::bytes; }
__host__ __device__ constexpr long long oct3d_smem_max() {
    return oct3d_smem<double, true>() > oct3d_smem<float, true>() ? oct3d_smem<double, true>()
                                                                  : oct3d_smem<float, true>();
}

// Tile height in y: a power of two up to RB_OCT_TILE, so that a pencil's lower neighbour is the
// previous lane of the same warp.
__device__ __forceinline__ int oct_ty(int ny) {
    int ty = 1;
    while (ty * 2 <= ny && ty * 2 <= RB_OCT_TILE) ty *= 2;
    return ty;
}

// The 3D octant sweep applies: one-moment cells, one octant batch's tiles fit in the team, every
// CTA of the team has a progress flag, and the step and round counts fit their bit fields.
__device__ __forceinline__ bool oct3d_ok(const DevProblem &P, int ncta, long long smem_bytes, int mixed) {
    if (P.ndims != 3 || !one_moment_md(P) || ncta > RB_OCT_MAXCTA) return false;
    if (P.nx + 2 * RB_OCT_TILE >= (1 << 20) || P.nd >= (1 << 12)) return false;
    const int TY = oct_ty(P.ny), TZ = min(P.nz, RB_OCT_TILE);
    const int ntiles = ((P.ny + TY - 1) / TY) * ((P.nz + TZ - 1) / TZ);
    const long long need = mixed ? (P.csd ? oct3d_smem<float, true>() : oct3d_smem<float, false>())
                                 : (P.csd ? oct3d_smem<double, true>() : oct3d_smem<double, false>());
    return ntiles <= ncta && smem_bytes >= need;
}

// asynchronous global -> shared copies (cp.async, L1-allocating), and their groups
template <int B>
__device__ __forceinline__ void cp_async(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src),
                 "n"(B)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// progress flags between the CTAs of a team (GPU-scope release / acquire)
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Waits until *f >= target; `seen` keeps the last value read. Gives up (false) after a bounded
// number of polls (about a second), so a wait can never hang the GPU.
__device__ __forceinline__ bool wait_progress(const unsigned long long *f, unsigned long long target,
                                              unsigned long long &seen) {
    if (seen >= target) return true;
    for (int it = 0; it < (1 << 24); it++) {
        seen = ld_acquire_u64(f);
        if (seen >= target) return true;
        if (it >= 32) __nanosleep(64);
    }
    return false;
}

// q / S of a cell: IEEE division in FP64 (the plain form), the fast reciprocal-based division
// in FP32 (the mixed form, whose FP64 defect correction absorbs its 2-ulp error)
__device__ __forceinline__ double oct_div(double q, double s) { return q / s; }
__device__ __forceinline__ float oct_div(float q, float s) { return __fdividef(q, s); }

// The sweep of one octant batch over one tile of pencils is a task; the tasks of a round (one per
// CTA) run concurrently, and a tile is paced by the tiles upwind of it in y and z: before it
// stages the faces of step s, thread 0 waits until the upwind tiles have published the steps that
// write them (s + TY − 1 and s + TZ − 1 of their own counts). A CTA publishes the number of steps
// it has completed, tagged with the sweep's epoch and the round, after a barrier that follows the
// face stores and a GPU-scope fence, so a downstream tile runs about TY steps behind its upwind
// tile with no team barrier inside the sweep.
template <typename R, typename PS, bool CSD, class Team>
__device__ __noinline__ void sweep3d_oct(Team &t, const DevProblem &P, GroupShared &gs, void *smem, const double *zin,
                                         int np_source, const double *phiE_in, double *phiE_out, int ig, PS *psi) {
    using L = Oct3dSmem<R, CSD>;
    static_assert(sizeof(PS) == sizeof(R), "angular buffer and arithmetic of one width");
    constexpr int DB = OctDB<R>::value, TT = RB_OCT_TILE, TP = TT * TT, NB = OctNB<R, CSD>::value;
    // one barrier per step: the write-back and the publication of step sg follow the barrier of
    // step sg + 1, which also orders the z-face hand-off; the stage being written back is then
    // neither the one being staged nor the one being solved
    constexpr bool ONEBAR = NB >= 3;
    const int nd = P.nd, nx = P.nx, ny = P.ny, nz = P.nz, nfm = P.nfmax;
    const int TY = oct_ty(ny), TZ = min(nz, RB_OCT_TILE);
    const int nty = (ny + TY - 1) / TY, ntz = (nz + TZ - 1) / TZ, ntiles = nty * ntz;
    const int ngrp = oct_groups(P, DB);
    const int gpr = (int)t.ncta / ntiles;  // octant batches per round (≥ 1: oct3d_ok)
    const int nround = (ngrp + gpr - 1) / gpr;
    const int nsteps = nx + TY + TZ - 2;
    // per-direction scratch (md_scratch_stride): exits x [ny·nz], y [nx·nz], z [nx·ny], the
    // z-face plane [nx·ny] and the y-face plane [nx·nz] handed between tiles, then the incoming
    // boundary fluxes (boundary_in_phase)
    const long long sstride = md_scratch_stride(P);
    const long long eyo = (long long)ny * nz * nfm, ezo = eyo + (long long)nx * nz * nfm;
    const long long zoff = ezo + (long long)nx * ny * nfm, yoff = zoff + (long long)nx * ny * nfm;
    const long long xin = md_in_offset(P, 0), yin = md_in_offset(P, 1), zin_ = md_in_offset(P, 2);
    unsigned char *base = reinterpret_cast<unsigned char *>(smem);
    double *fyb = reinterpret_cast<double *>(base + L::fy);
    double *fzb = reinterpret_cast<double *>(base + L::fz);
    double *eb = reinterpret_cast<double *>(base + L::eb);
    long long *pcb = reinterpret_cast<long long *>(base + L::pcb);
    R *dc = reinterpret_cast<R *>(base + L::dc);
    R *sfz = reinterpret_cast<R *>(base + L::sfz);
    PS *qb = reinterpret_cast<PS *>(base + L::qb);
    R *idxs = reinterpret_cast<R *>(base + L::ix);
    R *mS = reinterpret_cast<R *>(base + L::ms);
    R *mQ = reinterpret_cast<R *>(base + L::mq);
    int *mb = reinterpret_cast<int *>(base + L::mb);
    int *pjs = reinterpret_cast<int *>(base + L::pj);
    int *piy = reinterpret_cast<int *>(base + L::py);
    int *piz = reinterpret_cast<int *>(base + L::pz);
    const int me = threadIdx.x, jy = me % TY, jz = me / TY;
    const R w1x = (R)P.w1[0], w1y = (R)P.w1[1], w1z = (R)P.w1[2], w1e = (R)P.w1[3];
    const R esa = CSD ? (R)P.EsA[0] : R(0), esb = CSD ? (R)P.EsB[0] : R(0), eout = CSD ? (R)P.Eout[0] : R(0);
    // this sweep's tables: inverse x widths, and per material Σt (+ the CSD cell term) and the
    // factor of the incoming energy-face flux
    const bool xs_sm = nx <= RB_OCT_MAXNX;
    __syncthreads();
    if (xs_sm)
        for (int i = me; i < nx; i += blockDim.x) idxs[i] = (R)(1.0 / P.dx[i]);
    for (int m = me; m < P.nmat; m += blockDim.x) {
        const R sigt = (R)gs.sigt[m];
        R scs = R(0), sq = R(0);
        if (CSD) {
            scs = (R)P.scsd[m];
            sq = esa * (R)gs.sp[m] - esb * (R)gs.sm[m];
        }
        mS[m] = scs + sigt;
        mQ[m] = sq;
    }
    if (me == 0) gs.oct_epoch++;
    __syncthreads();
    const unsigned long long epoch = (unsigned long long)gs.oct_epoch;
    unsigned long long seen_y = 0, seen_z = 0;  // thread 0: the upwind flags as last read
    bool gave_up = false;
    for (int rnd = 0; rnd < nround; rnd++) {
        const int g = rnd * gpr + (int)t.crank / ntiles;
        const int tile = (int)t.crank % ntiles;
        int first = 0, cnt = 0, oc = 0;
        if ((int)t.crank < gpr * ntiles && g < ngrp) oc = oct_group(P, DB, g, first, cnt);
        if (cnt == 0) continue;  // uniform over the CTA
        const bool fx = !(oc & 1), fy = !(oc & 2), fz = !(oc & 4);
        const int tyq = tile % nty, tzq = tile / nty;  // tile coordinates in sweep order
        const int iyy = tyq * TY + jy, izz = tzq * TZ + jz;
        const bool pok = me < TY * TZ && iyy < ny && izz < nz;
        const int iy = fy ? iyy : ny - 1 - iyy, iz = fz ? izz : nz - 1 - izz;
        const unsigned long long tagr = (epoch << 32) | ((unsigned long long)rnd << 20);
        const unsigned long long *upy = tyq > 0 ? P.oct_flags + (t.crank - 1) : nullptr;
        const unsigned long long *upz = tzq > 0 ? P.oct_flags + (t.crank - nty) : nullptr;
        __syncthreads();  // the previous round's readers of the region are done
        if (me < DB) {
            const int n = first + me;
            for (int a = 0; a < 3; a++) {
                const long long blk = (long long)n * 3 + a;
                const double ac = me < cnt ? fabs(P.cosv[(long long)a * nd + n]) : 0.0;
                dc[me * 9 + a] = me < cnt ? (R)(ac * P.G[blk]) : R(0);
                dc[me * 9 + 3 + a] = me < cnt ? (R)(ac * P.Gsrc[blk * nfm]) : R(0);
                dc[me * 9 + 6 + a] = me < cnt ? (R)P.Gout[blk * nfm] : R(0);
            }
        }
        if (me < TP) {
            pcb[me] = pok ? (long long)nx * (iy + (long long)ny * iz) : -1;
            pjs[me] = jy + jz;
            piy[me] = iy;
            piz[me] = iz;
        }
        __syncthreads();
        // A step's cells are staged cooperatively: element e = me + TP·r (r < cnt) of the step is
        // direction k = e % cnt of pencil p = e / cnt, so consecutive lanes read consecutive
        // directions of a cell (one contiguous run of cnt values per cell).
        const int qd = TP / cnt, rm = TP % cnt, p0 = me / cnt, k0 = me % cnt;
        auto cell_of = [&](int p, int sg) -> long long {  // cell of pencil p at step sg, −1 if none
            const long long cb = pcb[p];
            const int ixx = sg - pjs[p];
            if (cb < 0 || ixx < 0 || ixx >= nx) return -1;
            return cb + (fx ? ixx : nx - 1 - ixx);
        };
        // thread 0: the upwind tiles have published the steps that write the faces of step s
        auto wait_up = [&](int s) {
            if (me != 0 || gave_up || s < 0 || s >= nsteps) return;
            bool ok = true;
            if (upy) ok = wait_progress(upy, tagr | (unsigned long long)(min(s + TY - 1, nsteps - 1) + 1), seen_y);
            if (ok && upz) ok = wait_progress(upz, tagr | (unsigned long long)(min(s + TZ - 1, nsteps - 1) + 1), seen_z);
            if (!ok) {
                gave_up = true;
                atomicOr(P.status, RB_DEV_TIMEOUT);
            }
        };
        // step s's inputs into stage s % NB (one commit group): angular source, energy-face flux,
        // materials, and the faces entering the tile's pencils (0, jz) and (jy, 0)
        auto issue = [&](int s) {
            if (s >= 0 && s < nsteps) {
                const int st = s % NB;
                int p = p0, k = k0;
#pragma unroll
                for (int r = 0; r < DB; r++) {
                    if (r < cnt) {
                        const long long c = cell_of(p, s);
                        if (c >= 0) {
                            const long long so = ((long long)st * TP + p) * DB + k;
                            const long long go = first + k + (long long)nd * c;
                            cp_async<sizeof(PS)>(qb + so, psi + go);
                            if (CSD && phiE_in) cp_async<8>(eb + so, phiE_in + go);
                        }
                    }
                    p += qd;
                    k += rm;
                    if (k >= cnt) { k -= cnt; p++; }
                }
                {
                    const long long c = cell_of(me, s);
                    if (c >= 0) cp_async<4>(mb + st * TP + me, P.mat + c);
                }
                const int nfy = TZ * cnt, nfz = TY * cnt;
                for (int e = me; e < nfy + nfz; e += blockDim.x) {
                    const bool isy = e < nfy;
                    const int e2 = isy ? e : e - nfy;
                    const int j = e2 / cnt, kk = e2 % cnt;  // pencil (0, j) for y faces, (j, 0) for z faces
                    const int pp = isy ? TY * j : j;
                    const int ixx = s - j;
                    if (pcb[pp] >= 0 && ixx >= 0 && ixx < nx) {
                        const int ix = fx ? ixx : nx - 1 - ixx;
                        const long long o = isy ? (tyq == 0 ? yin : yoff) + (ix + (long long)nx * piz[pp]) * nfm
                                                : (tzq == 0 ? zin_ : zoff) + (ix + (long long)nx * piy[pp]) * nfm;
                        cp_async<8>((isy ? fyb : fzb) + ((long long)st * TT + j) * DB + kk,
                                    P.fexit + (long long)(first + kk) * sstride + o);
                    }
                }
            }
            cp_async_commit();
        };
        const R idy = pok ? (R)(1.0 / P.dy[iy]) : R(0), idz = pok ? (R)(1.0 / P.dz[iz]) : R(0);
        R fxs[DB], fyl[DB];
        {
            const long long o = xin + (iy + (long long)ny * iz) * nfm;  // the domain's incoming x faces
#pragma unroll
            for (int k = 0; k < DB; k++) {
                fyl[k] = R(0);
                fxs[k] = (pok && k < cnt) ? (R)P.fexit[(long long)(first + k) * sstride + o] : R(0);
            }
        }
        // step s done by every thread: publish it (the barrier before this orders every thread's
        // face stores before thread 0's fence and release), then write its stage back, consecutive
        // lanes on consecutive directions of a cell
        auto finish = [&](int s) {
            if (me == 0 && ((s + 1) % RB_OCT_PUB == 0 || s == nsteps - 1)) {
                __threadfence();
                st_release_u64(P.oct_flags + t.crank, tagr | (unsigned long long)(s + 1));
            }
            const int ss = s % NB;
            int p = p0, k = k0;
#pragma unroll
            for (int r = 0; r < DB; r++) {
                if (r < cnt) {
                    const long long c = cell_of(p, s);
                    if (c >= 0) {
                        const long long so = ((long long)ss * TP + p) * DB + k;
                        const long long go = first + k + (long long)nd * c;
                        psi[go] = qb[so];
                        if (CSD) phiE_out[go] = eb[so];
                    }
                }
                p += qd;
                k += rm;
                if (k >= cnt) { k -= cnt; p++; }
            }
        };
        wait_up(0);
        __syncthreads();
        issue(0);
        for (int sg = 0; sg < nsteps; sg++) {
            wait_up(sg + 1);
            cp_async_wait<0>();  // this thread's copies of step sg have landed
            __syncthreads();     // everyone's; step sg − 1 solved; step sg + 1's faces are written
            if (ONEBAR && sg > 0) finish(sg - 1);
            issue(sg + 1);       // in flight while step sg is solved
            const int ixx = sg - jy - jz;
            const int rd = (sg + 1) & 1, wr = sg & 1, sb = sg % NB;
            R fyi[DB];
#pragma unroll
            for (int k = 0; k < DB; k++) fyi[k] = __shfl_up_sync(0xffffffffu, fyl[k], 1);
            if (pok && ixx >= 0 && ixx < nx) {
                const int ix = fx ? ixx : nx - 1 - ixx;
                const long long yk = (ix + (long long)nx * iz) * nfm, zk = (ix + (long long)nx * iy) * nfm;
                // every input of the cell first, then the arithmetic, then the stores (no shared
                // store sits between two loads, so the directions' chains overlap)
                R fzi[DB], qv[DB], fe[DB];
                PS *qc = qb + ((long long)sb * TP + me) * DB;
                double *ec = eb + ((long long)sb * TP + me) * DB;
                if (jy == 0) {
#pragma unroll
                    for (int k = 0; k < DB; k++) fyi[k] = (R)fyb[((long long)sb * TT + jz) * DB + k];
                }
                if (jz == 0) {
#pragma unroll
                    for (int k = 0; k < DB; k++) fzi[k] = (R)fzb[((long long)sb * TT + jy) * DB + k];
                } else {
#pragma unroll
                    for (int k = 0; k < DB; k++) fzi[k] = sfz[(rd * DB + k) * TP + me - TY];
                }
#pragma unroll
                for (int k = 0; k < DB; k++) {
                    qv[k] = (R)qc[k];
                    fe[k] = (CSD && phiE_in) ? (R)ec[k] : R(0);
                }
                const int m = mb[sb * TP + me];
                const R S0 = mS[m], sq = mQ[m];
                const R idx = xs_sm ? idxs[ix] : (R)(1.0 / P.dx[ix]);
                R v[DB];
#pragma unroll
                for (int k = 0; k < DB; k++) {
                    const R *d = dc + k * 9;
                    const R S = S0 + d[0] * idx + d[1] * idy + d[2] * idz;
                    R q = qv[k] + (d[3] * idx) * fxs[k] + (d[4] * idy) * fyi[k] + (d[5] * idz) * fzi[k];
                    if (CSD) q -= sq * fe[k];
                    v[k] = oct_div(q, S);
                    fxs[k] = w1x * fxs[k] + d[6] * v[k];
                    fyi[k] = w1y * fyi[k] + d[7] * v[k];
                    fzi[k] = w1z * fzi[k] + d[8] * v[k];
                }
#pragma unroll
                for (int k = 0; k < DB; k++) {
                    if (k >= cnt) continue;
                    qc[k] = (PS)v[k];
                    if (CSD) ec[k] = (double)(w1e * fe[k] + eout * v[k]);
                    sfz[(wr * DB + k) * TP + me] = fzi[k];
                }
                // faces leaving the tile or the domain
                if (jy == TY - 1 || iyy == ny - 1) {
                    const long long off = iyy < ny - 1 ? yoff : eyo;
#pragma unroll
                    for (int k = 0; k < DB; k++)
                        if (k < cnt) P.fexit[(long long)(first + k) * sstride + off + yk] = (double)fyi[k];
                }
                if (jz == TZ - 1 || izz == nz - 1) {
                    const long long off = izz < nz - 1 ? zoff : ezo;
#pragma unroll
                    for (int k = 0; k < DB; k++)
                        if (k < cnt) P.fexit[(long long)(first + k) * sstride + off + zk] = (double)fzi[k];
                }
                if (ixx == nx - 1) {
                    const long long o = (iy + (long long)ny * iz) * nfm;
#pragma unroll
                    for (int k = 0; k < DB; k++)
                        if (k < cnt) P.fexit[(long long)(first + k) * sstride + o] = (double)fxs[k];
                }
            }
#pragma unroll
            for (int k = 0; k < DB; k++) fyl[k] = fyi[k];
            if (!ONEBAR) {
                __syncthreads();
                finish(sg);
            }
        }
        if (ONEBAR && nsteps > 0) {
            __syncthreads();
            finish(nsteps - 1);
        }
        cp_async_wait<0>();
        __syncthreads();
    }
}

// 2D, one-moment cells: sweep_md's wavefront with the next cell's inputs loaded one step ahead
// and the arithmetic in R (FP64 or FP32) over an angular buffer of PS.
template <typename R, typename PS, bool CSD, class Team>
__device__ __noinline__ void sweep2d_pf(Team &t, const DevProblem &P, GroupShared &gs, const double *zin, int np_source,
                           const double *phiE_in, double *phiE_out, int ig, PS *psi) {
    const int nd = P.nd, nx = P.nx, ny = P.ny, nfm = P.nfmax;
    const int ncta = (int)t.ncta, crank = (int)t.crank;
    // directions dealt in contiguous blocks, so the directions of a CTA are neighbours in ψ
    const int dlo = (int)((long long)nd * crank / ncta), dhi = (int)((long long)nd * (crank + 1) / ncta);
    const int my_dirs = dhi - dlo;
    const int Rr = ny < (int)blockDim.x ? ny : (int)blockDim.x;  // rows per direction
    int D = (int)blockDim.x / Rr;
    const int dmax = RB_TILE_DOUBLES * (int)(sizeof(double) / sizeof(R)) / nx;  // y-face slots
    if (D > dmax) D = dmax;
    const int nrb = (ny + Rr - 1) / Rr;
    const long long sstride = md_scratch_stride(P);
    const long long xin = md_in_offset(P, 0), yin = md_in_offset(P, 1);
    R *yface = reinterpret_cast<R *>(gs.tile);  // [D][nx]
    const R w1x = (R)P.w1[0], w1y = (R)P.w1[1], w1e = (R)P.w1[3];
    const R esa = CSD ? (R)P.EsA[0] : R(0), esb = CSD ? (R)P.EsB[0] : R(0), eout = CSD ? (R)P.Eout[0] : R(0);
    for (int k0 = 0; k0 < my_dirs; k0 += D) {
        const int dl = threadIdx.x / Rr, r = threadIdx.x % Rr;
        const bool active = dl < D && k0 + dl < my_dirs;
        const int n = dlo + k0 + dl;
        const double mu = active ? P.cosv[n] : 0.0, eta = active ? P.cosv[nd + n] : 0.0;
        const bool fx = mu >= 0.0, fy = eta >= 0.0;
        R gx = R(0), gy = R(0), sx = R(0), sy = R(0), ox = R(0), oy = R(0);
        if (active) {
            gx = (R)(fabs(mu) * P.G[(long long)n * 3]);
            gy = (R)(fabs(eta) * P.G[(long long)n * 3 + 1]);
            sx = (R)(fabs(mu) * P.Gsrc[((long long)n * 3) * nfm]);
            sy = (R)(fabs(eta) * P.Gsrc[((long long)n * 3 + 1) * nfm]);
            ox = (R)P.Gout[((long long)n * 3) * nfm];
            oy = (R)P.Gout[((long long)n * 3 + 1) * nfm];
        }
        double *scr = P.fexit + (active ? (long long)n * sstride : 0);
        double *exx = scr, *exy = exx + (long long)ny * nfm;
        R *yf = yface + (long long)dl * nx;
        for (int rb = 0; rb < nrb; rb++) {
            const int iyy = rb * Rr + r;
            const bool row = active && iyy < ny;
            const int iy = fy ? iyy : ny - 1 - iyy;
            const R idy = row ? (R)(1.0 / P.dy[iy]) : R(0);
            R F0 = R(0), qp = R(0), fep = R(0), idxp = R(0);
            int mp = 0;
            if (row) {  // the inputs of the row's first cell; the later ones are loaded a step ahead
                const int ix0 = fx ? 0 : nx - 1;
                const long long c0 = ix0 + (long long)nx * iy;
                qp = (R)psi[n + (long long)nd * c0];
                if (CSD) fep = phiE_in ? (R)phiE_in[n + (long long)nd * c0] : R(0);
                mp = P.mat[c0];
                idxp = (R)(1.0 / P.dx[ix0]);
            }
            for (int s = 0; s < nx + Rr - 1; s++) {
                const int ixx = s - r;
                R qn = R(0), fen = R(0), idxn = R(0);
                int mn_ = 0;
                const bool nxt = row && ixx >= 0 && ixx + 1 < nx;
                if (nxt) {
                    const int ixn = fx ? ixx + 1 : nx - 2 - ixx;
                    const long long cn = ixn + (long long)nx * iy;
                    qn = (R)psi[n + (long long)nd * cn];
                    if (CSD) fen = phiE_in ? (R)phiE_in[n + (long long)nd * cn] : R(0);
                    mn_ = P.mat[cn];
                    idxn = (R)(1.0 / P.dx[ixn]);
                }
                if (row && ixx >= 0 && ixx < nx) {
                    const int ix = fx ? ixx : nx - 1 - ixx;
                    const long long c = ix + (long long)nx * iy;
                    // X face of the row and Y face of the column (sn_sweep_2D.jl:71-132): the
                    // incoming fluxes of boundary_in_phase
                    if (ixx == 0) F0 = (R)scr[xin + (long long)iy * nfm];
                    const R F1 = iyy == 0 ? (R)scr[yin + (long long)ix * nfm] : yf[ixx];
                    const int m = mp;
                    R S = (R)gs.sigt[m], srcE = R(0);
                    if (CSD) {
                        S = (R)P.scsd[m] + S;
                        srcE = esa * (R)gs.sp[m] - esb * (R)gs.sm[m];
                    }
                    const R idx = idxp;
                    S = S + gx * idx + gy * idy;
                    R q = qp + (sx * idx) * F0 + (sy * idy) * F1;
                    if (CSD) q -= srcE * fep;
                    const R v = q / S;
                    F0 = w1x * F0 + ox * v;
                    const R F1o = w1y * F1 + oy * v;
                    psi[n + (long long)nd * c] = (PS)v;
                    if (CSD) phiE_out[n + (long long)nd * c] = (double)(w1e * fep + eout * v);
                    yf[ixx] = F1o;
                    if (ixx == nx - 1) exx[(long long)iy * nfm] = (double)F0;
                    if (iyy == ny - 1) exy[(long long)ix * nfm] = (double)F1o;
                }
                if (nxt) { qp = qn; fep = fen; mp = mn_; idxp = idxn; }
                __syncthreads();
            }
        }
    }
}

// The pass for 2D and 3D problems. mixed: FP32 angular buffer, products and sweep where the
// cells are one-moment and (3D) the octant sweep fits the team; every other 2D/3D pass runs in
// FP64 (the result is then the plain form's).
template <class Team>
__device__ __noinline__ void pass_md(Team &t, const DevProblem &P, GroupShared &gs, void *smem, long long smem_bytes,
                        const double *zin, double *zout, int homog, int matvec, int ig, const double *phiE_in,
                        double *phiE_out, int mixed) {
    const bool one = one_moment_md(P);
    const bool oct = oct3d_ok(P, (int)t.ncta, smem_bytes, mixed);
    const int mx = (mixed && one && (P.ndims == 2 || oct)) ? 1 : 0;
    // the mixed form's products go to the tensor cores where the CTA holds TMEM and they fit
    if (!mx || !m2d_tc(t, P, gs, gs.tc, smem, smem_bytes, zin, homog ? nullptr : P.qnout))
        m2d_tiles(t, P, gs, zin, homog ? nullptr : P.qnout, 1, mx);
    const int np_source = homog ? 0 : P.np_source;
    const double *pE = (P.csd && !homog) ? phiE_in : nullptr;
    const bool newsweep = (P.ndims == 3 && oct) || (P.ndims == 2 && one);
    if (newsweep) boundary_in_phase(t, P, zin, np_source, ig);
    t.sync();
    if (P.ndims == 3 && oct) {
        if (mx) {
            if (P.csd) sweep3d_oct<float, float, true>(t, P, gs, smem, zin, np_source, pE, phiE_out, ig, P.psi32);
            else sweep3d_oct<float, float, false>(t, P, gs, smem, zin, np_source, pE, phiE_out, ig, P.psi32);
        } else {
            if (P.csd) sweep3d_oct<double, double, true>(t, P, gs, smem, zin, np_source, pE, phiE_out, ig, P.psi);
            else sweep3d_oct<double, double, false>(t, P, gs, smem, zin, np_source, pE, phiE_out, ig, P.psi);
        }
    } else if (P.ndims == 2 && one) {
        if (mx) {
            if (P.csd) sweep2d_pf<float, float, true>(t, P, gs, zin, np_source, pE, phiE_out, ig, P.psi32);
            else sweep2d_pf<float, float, false>(t, P, gs, zin, np_source, pE, phiE_out, ig, P.psi32);
        } else {
            if (P.csd) sweep2d_pf<double, double, true>(t, P, gs, zin, np_source, pE, phiE_out, ig, P.psi);
            else sweep2d_pf<double, double, false>(t, P, gs, zin, np_source, pE, phiE_out, ig, P.psi);
        }
    } else if (P.ndims == 3) {
        if (one && !P.csd) sweep_3d_tiles<CellMDfix<1, 1, 1, false, 3>, 1, 1, 1>(t, P, gs, zin, np_source, pE, phiE_out, ig);
        else if (one) sweep_3d_tiles<CellMDfix<1, 1, 1, true, 3>, 1, 1, 1>(t, P, gs, zin, np_source, pE, phiE_out, ig);
        else sweep_3d_tiles<CellMDgen, RB_MAXNM, RB_MAXFACE, RB_MAXFACE>(t, P, gs, zin, np_source, pE, phiE_out, ig);
    } else {
        sweep_md<CellMDgen, RB_MAXNM, RB_MAXFACE, RB_MAXFACE>(t, P, gs, zin, np_source, pE, phiE_out, ig);
    }
    t.sync();
    if (!mx || !d2m_tc(t, P, gs.tc, smem, smem_bytes, zin, zout, matvec)) d2m_tiles(t, P, gs, zin, zout, matvec, mx);
    boundary_out_md(t, P, zin, zout, matvec);
    t.sync();
}

}  // namespace rb
