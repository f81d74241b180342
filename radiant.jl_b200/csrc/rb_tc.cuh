// rb_tc.cuh -- the moment<->direction products of the mixed form of 2D/3D passes on the
// 5th-generation tensor cores: tcgen05.mma kind::tf32, accumulators in tensor memory (TMEM).
//
// The products are the M2D and D2M lines of sn_sweep_2D.jl:54-183 / sn_sweep_3D.jl:57-239
// (Qn = Mn[n,:]·Ql, 𝚽l += Dn[:,n]·𝚽n) with the in-group scattering (scattering_source.jl:25-30)
// and Fokker-Planck (fokker_planck_source.jl:29-33) sources folded in, as team_product does in
// FP64 (rb_kernels.cuh):
//   M2D  ψ[col,n] = pre + Σ_p ys[mat,p]·𝚽[col,p]·Mn[n,p] + Σ_p T[mat]·𝚽[col,p]·(Mn·ℳ)[n,p]
//   D2M  z[col,p] = pre ∓ Σ_n ψ[col,n]·Dn[p,n]
// A column ("col") is one cell moment of one cell; its values are contiguous in memory (the
// moments 𝚽[col·np + p], the directions ψ[col·nd + n]). The products run with the columns as
// the M side of the MMA (128 columns per tile, TMEM lane = column) and the operator as the N side
// (N = directions or moments, up to 256), so a thread stages and stores the contiguous run of one
// column. Operator parts are stacked along K (K = parts·nk): the Fokker-Planck part of M2D takes
// its per-cell factor T[mat] on the column side, and one accumulator holds the whole sum.
//
// Split precision: every FP32 value x is hi + lo with hi = tf32(x) and lo = x − hi, and a product
// is A_hi·B_hi + A_hi·B_lo + A_lo·B_hi (the dropped A_lo·B_lo is ~2^-22 of it), accumulated in
// FP32 in TMEM: about FP32 accuracy at tensor-core rate.
//
// Layout. Both operands are K-major, no swizzle, in the canonical layout of the UMMA
// descriptors: 8 rows × 16 bytes core matrices, K-adjacent core matrices 128 bytes apart (LBO),
// 8-row groups 1024 bytes apart (SBO): element (r, k) of a 32-deep K chunk at byte
// (r%8)·16 + (k%4)·4 + (k/4)·128 + (r/8)·1024. The operator is packed on the host
// (rb_capi.cu, pack_tc_operator): chunk kc of NJ rows (NJ = rows rounded up to 16), TF32 high
// block then low block, NJ·32 floats each. It is either copied into shared memory once per
// product (when it fits beside two column stages) or streamed chunk by chunk with the columns.
//
// Pipeline of one CTA over its column tiles: for each 32-deep K chunk the threads load the
// chunk of their column (two threads per column, 16 K each), wait until the MMAs that last read
// the stage are done (one mbarrier per stage, signalled by tcgen05.commit), write the split
// values into the stage, and one thread issues 4 K-steps × 3 split terms of tcgen05.mma; the
// two stages alternate, so a chunk's loads overlap the previous chunk's MMAs. After a tile's last
// chunk the epilogue reads the accumulators with tcgen05.ld (warp w reads TMEM lanes
// 32·(w%4)..+31, i.e. 32 columns, and half of the 8-wide output groups), adds the pre term and
// stores each column's contiguous run. Every wait is bounded (RB_DEV_TIMEOUT on expiry).
// This code runs on one GPU only and reads only this GPU's memory; it issues no TMA copies.
#pragma once
#include "rb_kernels.cuh"

#define RB_TC_KC 32          // K per staged chunk
#define RB_TC_M 128          // columns per tile (MMA M)
#define RB_TC_TMEM_COLS 512  // tensor-memory columns a CTA allocates for the accumulators

namespace rb {
namespace tc {

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0), version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: kind::tf32 (A, B TF32), FP32 accumulator, both K-major, M×N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(mbar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *m) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(m)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the phase with the given parity to complete; gives up (false) after a bounded
// number of polls, so a wait can never hang the GPU.
__device__ __forceinline__ bool mbar_wait(uint64_t *m, uint32_t parity) {
    const uint32_t a = saddr(m);
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One whole warp: allocate / free `ncols` TMEM columns (the address is written to *dst).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 8 consecutive FP32 columns of the warp's 32 TMEM lanes (one value per lane and column).
__device__ __forceinline__ void tmem_ld8(uint32_t addr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// 16-byte asynchronous copy global -> shared, L2 only
__device__ __forceinline__ void cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit_wait_all() {
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Bytes of one column stage (hi and lo of 128 columns × 32 K) and of one operator chunk.
__host__ __device__ constexpr long long col_stage_bytes() { return 2LL * RB_TC_M * RB_TC_KC * 4; }
__host__ __device__ constexpr long long op_chunk_bytes(int nj) { return 2LL * nj * RB_TC_KC * 4; }
// Shared memory of a product whose operator has nj rows (rounded to 16) and K = nk: resident
// operator (all chunks) plus two column stages, or two stages of (column chunk + operator chunk).
__host__ __device__ constexpr long long bytes_resident(int nj, int nk) {
    return ((nk + RB_TC_KC - 1) / RB_TC_KC) * op_chunk_bytes(nj) + 2 * col_stage_bytes();
}
__host__ __device__ constexpr long long bytes_streamed(int nj) { return 2 * (col_stage_bytes() + op_chunk_bytes(nj)); }
__host__ __device__ constexpr int round16(int n) { return (n + 15) & ~15; }

}  // namespace tc

// One 16-K half chunk of a column into registers: k0 = first K (stacked over the parts: part
// k / nkp, index k % nkp), X[col·ldx + index], times scale(part, col, index); zero past K.
template <class TX, class Scale>
__device__ __forceinline__ void tc_load_half(float (&xv)[16], const TX *X, long long ldx, long long col, bool colok,
                                             int k0, int nk, int nkp, bool vec, Scale scale) {
    const int part = k0 / nkp, kk0 = k0 % nkp;
    if (colok && vec && (kk0 * (int)sizeof(TX)) % 16 == 0 && kk0 + 16 <= nkp && k0 + 16 <= nk) {
        // one part, aligned: 16-byte loads of the contiguous run
        const TX *src = X + col * ldx + kk0;
        double v[16];
        if constexpr (sizeof(TX) == 8) {
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const double2 d = *reinterpret_cast<const double2 *>(src + 2 * q);
                v[2 * q] = d.x;
                v[2 * q + 1] = d.y;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 f = *reinterpret_cast<const float4 *>(src + 4 * q);
                v[4 * q] = f.x; v[4 * q + 1] = f.y; v[4 * q + 2] = f.z; v[4 * q + 3] = f.w;
            }
        }
#pragma unroll
        for (int e = 0; e < 16; e++) xv[e] = (float)(scale(part, col, kk0 + e) * v[e]);
        return;
    }
#pragma unroll
    for (int e = 0; e < 16; e++) {
        const int k = k0 + e;
        float x = 0.0f;
        if (colok && k < nk) {
            const int p = k / nkp, kk = k % nkp;
            x = (float)(scale(p, col, kk) * (double)X[col * ldx + kk]);
        }
        xv[e] = x;
    }
}

// D[col, j] = Σ_k Xs[col, k]·Op[j, k] over the team's column tiles (tiles dealt round robin to
// the CTAs), k over the stacked parts (K = parts·nkp), Xs[col, k] = scale(k / nkp, col, k % nkp)·
// X[col·ldx + k % nkp]; then epi(col, j0, acc[8]) stores the outputs j0..j0+7 of a column.
// opA: the packed operator (NJ = round16(nj) rows). Returns false (no output touched) where it
// does not fit.
template <class TX, class Team, class Scale, class Epi>
__device__ bool tc_product(Team &t, TcState &ts, unsigned char *sm, long long sm_bytes, const float *opA, int nj,
                           int nkp, int parts, const TX *X, long long ldx, long long ncol, Scale scale, Epi epi,
                           int *status) {
    const int NJ = tc::round16(nj), nk = nkp * parts, kch = (nk + RB_TC_KC - 1) / RB_TC_KC;
    if (!ts.ready || NJ > 256 || NJ > RB_TC_TMEM_COLS) return false;
    const bool resident = tc::bytes_resident(NJ, nk) <= sm_bytes;
    if (!resident && tc::bytes_streamed(NJ) > sm_bytes) return false;
    const long long opc = tc::op_chunk_bytes(NJ) / 4, cst = tc::col_stage_bytes() / 4;  // floats
    // regions: [operator: all chunks (resident) | one chunk per stage][column stages]
    float *sOp = reinterpret_cast<float *>(sm);
    float *sCol = sOp + (resident ? kch * opc : 2 * opc);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int half = tid >> 7, cm = tid & 127;  // this thread's half chunk and column of a tile
    const bool vec = ((ldx * (long long)sizeof(TX)) % 16 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    const uint32_t IDESC = tc::idesc_tf32(RB_TC_M, NJ);
    if (resident) {  // the whole operator, once
        const float4 *src = reinterpret_cast<const float4 *>(opA);
        for (long long e = tid; e < kch * opc / 4; e += blockDim.x) tc::cp16(reinterpret_cast<float4 *>(sOp) + e, src + e);
        tc::cp_commit_wait_all();
    }
    uint32_t ph = ts.phase;  // bit s: parity of the next completion of stage s (same in all threads)
    int pend = 0;            // bit s: stage s has MMAs not yet waited for
    int g = 0;               // chunks issued in this call (stage = g & 1)
    const long long ntile = (ncol + RB_TC_M - 1) / RB_TC_M;
    for (long long tl = t.crank; tl < ntile; tl += t.ncta) {
        const long long c0 = tl * RB_TC_M;
        const long long col = c0 + cm;
        const bool colok = col < ncol;
        for (int kc = 0; kc < kch; kc++, g++) {
            const int s = g & 1;
            float xv[16];
            tc_load_half(xv, X, ldx, col, colok, kc * RB_TC_KC + 16 * half, nk, nkp, vec, scale);
            // the stage's previous MMAs are done
            if (pend & (1 << s)) {
                if (!tc::mbar_wait(&ts.mbar[s], (ph >> s) & 1) && tid == 0) atomicOr(status, RB_DEV_TIMEOUT);
                ph ^= 1u << s;
                pend &= ~(1 << s);
            }
            float *sO = resident ? sOp + kc * opc : sOp + s * opc;
            if (!resident) {
                const float4 *src = reinterpret_cast<const float4 *>(opA + kc * opc);
                for (long long e = tid; e < opc / 4; e += blockDim.x) tc::cp16(reinterpret_cast<float4 *>(sO) + e, src + e);
            }
            // the column's 16 K, hi and lo, as four 16-byte rows of core matrices
            float *hi = sCol + s * cst, *lo = hi + cst / 2;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float h[4], l[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    h[e] = tc::tf32_hi(xv[4 * q + e]);
                    l[e] = xv[4 * q + e] - h[e];
                }
                const int k4 = 4 * half + q;
                const int off = ((cm & 7) * 16 + (cm >> 3) * 1024 + k4 * 128) / 4;
                *reinterpret_cast<float4 *>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<float4 *>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
            }
            if (!resident) tc::cp_commit_wait_all();
            tc::fence_async_smem();
            tc::fence_before();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after();
                const uint32_t ah = tc::saddr(hi), al = tc::saddr(lo);
                const uint32_t bh = tc::saddr(sO), bl = bh + (uint32_t)(opc / 2) * 4;
#pragma unroll
                for (int st = 0; st < RB_TC_KC / 8; st++) {
                    const uint32_t o = st * 256;
                    const uint32_t acc = (kc > 0 || st > 0) ? 1u : 0u;
                    tc::mma_tf32(ts.tmem, tc::sdesc(ah + o, 128, 1024), tc::sdesc(bh + o, 128, 1024), IDESC, acc);
                    tc::mma_tf32(ts.tmem, tc::sdesc(ah + o, 128, 1024), tc::sdesc(bl + o, 128, 1024), IDESC, 1u);
                    tc::mma_tf32(ts.tmem, tc::sdesc(al + o, 128, 1024), tc::sdesc(bh + o, 128, 1024), IDESC, 1u);
                }
                tc::commit(&ts.mbar[s]);
            }
            pend |= 1 << s;
        }
        // the tile's accumulators: wait for its last chunk's MMAs
        {
            const int s = (g - 1) & 1;
            if (!tc::mbar_wait(&ts.mbar[s], (ph >> s) & 1) && tid == 0) atomicOr(status, RB_DEV_TIMEOUT);
            ph ^= 1u << s;
            pend &= ~(1 << s);
        }
        tc::fence_after();
        const int lq = warp & 3;  // TMEM lane quarter of this warp: columns c0 + 32·lq + lane
        const long long ecol = c0 + 32 * lq + lane;
        for (int j0 = 8 * (warp >> 2); j0 < NJ; j0 += 16) {
            float a[8];
            tc::tmem_ld8(ts.tmem + ((uint32_t)(32 * lq) << 16) + (uint32_t)j0, a);
            if (ecol < ncol) epi(ecol, j0, a);
        }
        tc::fence_before();
        __syncthreads();  // every accumulator read before the next tile's MMAs overwrite them
    }
    // no MMA left unwaited, so the next call starts from settled barriers
    for (int s = 0; s < 2; s++)
        if (pend & (1 << s)) {
            if (!tc::mbar_wait(&ts.mbar[s], (ph >> s) & 1) && tid == 0) atomicOr(status, RB_DEV_TIMEOUT);
            ph ^= 1u << s;
        }
    __syncthreads();
    if (tid == 0) ts.phase = ph;
    __syncthreads();
    return true;
}

// The M2D product of a mixed-form 2D/3D pass on the tensor cores (into the FP32 angular buffer);
// false when the shapes do not fit (the caller then uses team_product).
template <class Team>
__device__ bool m2d_tc(Team &t, const DevProblem &P, GroupShared &gs, TcState &ts, void *smem, long long smem_bytes,
                       const double *zin, const double *add) {
    if (!P.tc_m2d) return false;
    const int nd = P.nd, np = P.np, nm = P.nm5;
    const int parts = P.mnfp ? 2 : 1;
    const int *mat = P.mat;
    const double *ys = P.kmat;
    const double *tg = gs.tg;
    float *psi = P.psi32;
    const long long ncol = (long long)nm * P.ncell;
    // part 0: ys[mat, p]·𝚽 against Mn; part 1: T[mat]·𝚽 against Mn·ℳ
    auto sc = [=] __device__(int part, long long col, int k) -> double {
        const int m = mat[col / nm];
        return part == 0 ? ys[(long long)m * np + k] : tg[m];
    };
    const bool v4 = (nd % 4) == 0, v2 = (nd % 2) == 0;
    auto epi = [=] __device__(long long col, int j0, const float (&a)[8]) {
        float *dst = psi + col * nd + j0;
        const double *pre = add ? add + col * nd + j0 : nullptr;
        float o[8];
        if (pre && v2 && j0 + 8 <= nd) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const double2 p2 = *reinterpret_cast<const double2 *>(pre + 2 * q);
                o[2 * q] = (float)(p2.x + (double)a[2 * q]);
                o[2 * q + 1] = (float)(p2.y + (double)a[2 * q + 1]);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++) o[q] = (j0 + q < nd) ? (float)((pre ? pre[q] : 0.0) + (double)a[q]) : 0.0f;
        }
        if (v4 && j0 + 8 <= nd) {
            *reinterpret_cast<float4 *>(dst) = make_float4(o[0], o[1], o[2], o[3]);
            *reinterpret_cast<float4 *>(dst + 4) = make_float4(o[4], o[5], o[6], o[7]);
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (j0 + q < nd) dst[q] = o[q];
        }
    };
    return tc_product(t, ts, reinterpret_cast<unsigned char *>(smem), smem_bytes, P.tc_m2d, nd, np, parts, zin,
                      (long long)np, ncol, sc, epi, P.status);
}

// The D2M product of a mixed-form 2D/3D pass on the tensor cores (FP32 angular buffer in, FP64
// state out; matvec: zout = zin − Dn·ψ).
template <class Team>
__device__ bool d2m_tc(Team &t, const DevProblem &P, TcState &ts, void *smem, long long smem_bytes, const double *zin,
                       double *zout, int matvec) {
    if (!P.tc_d2m) return false;
    const int nd = P.nd, np = P.np, nm = P.nm5;
    const long long ncol = (long long)nm * P.ncell;
    auto one = [] __device__(int, long long, int) -> double { return 1.0; };
    const bool v2 = (np % 2) == 0;
    auto epi = [=] __device__(long long col, int j0, const float (&a)[8]) {
        double *dst = zout + col * np + j0;
        const double *pre = zin + col * np + j0;
        if (v2 && j0 + 8 <= np) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                double2 r;
                if (matvec) {
                    const double2 p2 = *reinterpret_cast<const double2 *>(pre + 2 * q);
                    r = make_double2(p2.x - (double)a[2 * q], p2.y - (double)a[2 * q + 1]);
                } else {
                    r = make_double2((double)a[2 * q], (double)a[2 * q + 1]);
                }
                *reinterpret_cast<double2 *>(dst + 2 * q) = r;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (j0 + q < np) dst[q] = matvec ? pre[q] - (double)a[q] : (double)a[q];
        }
    };
    return tc_product(t, ts, reinterpret_cast<unsigned char *>(smem), smem_bytes, P.tc_d2m, np, nd, 1, P.psi32,
                      (long long)nd, ncol, one, epi, P.status);
}

}  // namespace rb
