// rb_tc.cuh -- the moment<->direction products of the mixed form of 2D/3D passes on the
// 5th-generation tensor cores: tcgen05.mma kind::tf32, accumulators in tensor memory (TMEM).
//
// The products are the M2D and D2M lines of sn_sweep_2D.jl:54-183 / sn_sweep_3D.jl:57-239
// (Qn = Mn[n,:]·Ql, 𝚽l += Dn[:,n]·𝚽n) with the in-group scattering (scattering_source.jl:25-30)
// and Fokker-Planck (fokker_planck_source.jl:29-33) sources folded in, as team_product does in
// FP64 (rb_kernels.cuh):
//   M2D  ψ[n,col] = pre + Σ_p Mn[n,p]·ys[mat,p]·𝚽[p,col] + T[mat]·Σ_p (Mn·ℳ)[n,p]·𝚽[p,col]
//   D2M  z[p,col] = pre ∓ Σ_n Dn[p,n]·ψ[n,col]
// The operator (Mn, Mn·ℳ or Dn, "A") is small and fixed per problem; the columns (cells × cell
// moments, "B") are many. Split precision: every FP32 value x is hi + lo with hi = tf32(x) and
// lo = x − hi, and a product is A_hi·B_hi + A_hi·B_lo + A_lo·B_hi (the dropped A_lo·B_lo is
// ~2^-22 of it), accumulated in FP32 in TMEM: about FP32 accuracy at tensor-core rate.
//
// Layout. A is packed on the host (rb_capi.cu, pack_tc_operator) into blocks of 128 rows × 32 K,
// hi block then lo block, each in the K-major no-swizzle canonical layout of the UMMA
// descriptors: element (r, k) at byte (r%8)·16 + (r/8)·1024 + (k%4)·4 + (k/4)·128, i.e. 8×16-byte
// core matrices, K-adjacent core matrices 128 bytes apart (LBO) and 8-row groups 1024 bytes apart
// (SBO). B is staged by the CTA's threads into the same layout (N columns × 32 K): each thread
// reads 4 consecutive K of a column (32 contiguous bytes) and writes one 16-byte row of a core
// matrix, so a quarter-warp writes 128 contiguous bytes (no bank conflict).
//
// Per CTA and column tile of N columns: for each 32-deep K chunk the threads load the next
// chunk's B values into registers, wait for the MMAs of the previous chunk (mbarrier signalled
// by tcgen05.commit), stage A and B in shared memory, and one thread issues 4 K-steps × 3 split
// terms of tcgen05.mma per (part, 128-row tile). The epilogue reads the accumulators back with
// tcgen05.ld (warp w reads TMEM lanes 32·(w%4)..+31, i.e. 32 consecutive output rows, so the
// stores of a column are coalesced) and applies the scale, the pre-added term and the store.
// This code runs on one GPU only and reads only this GPU's memory; it issues no TMA copies.
#pragma once
#include "rb_kernels.cuh"

#define RB_TC_KC 32          // K per staged chunk
#define RB_TC_BLOCK 4096     // floats in one 128×32 operator block
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
// 16 consecutive FP32 columns of the warp's 32 TMEM lanes (one value per lane and column).
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Shared memory (bytes) a product with `parts` operator parts of `mtiles` 128-row tiles, `nb` B
// operands and N columns per tile stages per K chunk.
__host__ __device__ constexpr long long stage_bytes(int parts, int mtiles, int nb, int N) {
    return (long long)parts * mtiles * 2 * RB_TC_BLOCK * 4 + (long long)nb * 2 * N * RB_TC_KC * 4;
}

}  // namespace tc

// C[i, col] = Σ_k A_p[i,k]·B_b(p)[k,col] for every operator part p (b(p) = min(p, nb−1)) over
// column tiles of N columns dealt to the team's CTAs; B_0[k,col] = scale0(k,col)·X[k + ldx·col],
// B_1[k,col] = X[k + ldx·col]. The epilogue object provides pre(i, col) (the term added to the
// product), scale(col) (the factor of part 1) and store(i, col, acc0 + scale·acc1, pre).
// opA: packed operator, block (p, mtile, kchunk) at ((p·mtiles + m)·kchunks + kc)·2·RB_TC_BLOCK
// floats (hi block, then lo). Returns false (without touching any output) if it does not fit.
template <int N, class TX, class Team, class Scale, class Epi>
__device__ bool tc_product(Team &t, TcState &ts, unsigned char *sm, long long sm_bytes, const float *opA, int parts,
                           int ni, int nk, int nb, const TX *X, int ldx, long long ncol, Scale scale0, Epi epi,
                           int *status) {
    const int mtiles = (ni + 127) / 128, kchunks = (nk + RB_TC_KC - 1) / RB_TC_KC;
    if (!ts.ready || ni > 256 || parts * mtiles * N > RB_TC_TMEM_COLS || tc::stage_bytes(parts, mtiles, nb, N) > sm_bytes)
        return false;
    constexpr int CPT = N / 32;                 // columns per thread in the B staging
    constexpr uint32_t IDESC = tc::idesc_tf32(128, N);
    float *sA = reinterpret_cast<float *>(sm);  // [parts·mtiles][hi,lo][RB_TC_BLOCK]
    float *sB = sA + (long long)parts * mtiles * 2 * RB_TC_BLOCK;  // [nb][hi,lo][N·32]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // B staging: a warp covers 8 columns × 16 K of each 32 columns (lanes 8·q..8·q+7 take the
    // 4-deep K group k4 of 8 neighbouring columns), so a load instruction touches 8 columns'
    // contiguous K runs and a quarter-warp stores 128 contiguous bytes
    const int k4 = (lane >> 3) + 4 * (warp & 1);  // this thread's 4-deep K group of the chunk (0..7)
    const int cw = (lane & 7) + 8 * (warp >> 1);   // its column inside each group of 32
    const long long ntile = (ncol + N - 1) / N;
    uint32_t ph = ts.phase;  // parity of the next MMA completion (identical in every thread)
    for (long long tl = t.crank; tl < ntile; tl += t.ncta) {
        const long long c0 = tl * N;
        for (int kc = 0; kc < kchunks; kc++) {
            // this chunk's B values: CPT columns × 4 K
            float xv[CPT][4], x0[CPT][4];
#pragma unroll
            for (int j = 0; j < CPT; j++) {
                const long long col = c0 + cw + 32 * j;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int k = kc * RB_TC_KC + 4 * k4 + e;
                    const bool in = col < ncol && k < nk;
                    const double x = in ? (double)X[k + (long long)ldx * col] : 0.0;
                    xv[j][e] = (float)x;
                    x0[j][e] = in ? (float)(scale0(k, col) * x) : 0.0f;
                }
            }
            // the previous chunk's MMAs have read shared memory
            if (kc > 0) {
                if (!tc::mbar_wait(&ts.mbar, ph & 1) && tid == 0) atomicOr(status, RB_DEV_TIMEOUT);
                ph++;
            }
            // stage A: every (part, mtile) block of this chunk, hi and lo (16-byte copies)
            {
                const int nblk = parts * mtiles * 2;
                const float4 *src4 = reinterpret_cast<const float4 *>(opA);
                float4 *dst4 = reinterpret_cast<float4 *>(sA);
                for (int e = tid; e < nblk * (RB_TC_BLOCK / 4); e += blockDim.x) {
                    const int b = e / (RB_TC_BLOCK / 4), w = e % (RB_TC_BLOCK / 4);
                    const int pm = b >> 1, hl = b & 1;
                    const long long gb = ((long long)pm * kchunks + kc) * 2 + hl;
                    dst4[e] = src4[gb * (RB_TC_BLOCK / 4) + w];
                }
            }
            // stage B: hi/lo of each operand in the canonical layout (one 16-byte row per store)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                if (b >= nb) break;
                float *hi = sB + (long long)b * 2 * N * RB_TC_KC, *lo = hi + N * RB_TC_KC;
#pragma unroll
                for (int j = 0; j < CPT; j++) {
                    const int cl = cw + 32 * j;
                    float h[4], l[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const float x = b == 0 ? x0[j][e] : xv[j][e];
                        h[e] = tc::tf32_hi(x);
                        l[e] = x - h[e];
                    }
                    const int off = ((cl & 7) * 16 + (cl >> 3) * 1024 + k4 * 128) / 4;
                    *reinterpret_cast<float4 *>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<float4 *>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
                }
            }
            tc::fence_async_smem();
            tc::fence_before();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after();
                for (int p = 0; p < parts; p++) {
                    const int b = p < nb ? p : nb - 1;
                    const uint32_t bh = tc::saddr(sB + (long long)b * 2 * N * RB_TC_KC), bl = bh + N * RB_TC_KC * 4;
                    for (int m = 0; m < mtiles; m++) {
                        const uint32_t ah = tc::saddr(sA + (long long)(p * mtiles + m) * 2 * RB_TC_BLOCK);
                        const uint32_t al = ah + RB_TC_BLOCK * 4;
                        const uint32_t d = ts.tmem + (uint32_t)((p * mtiles + m) * N);
#pragma unroll
                        for (int s = 0; s < RB_TC_KC / 8; s++) {
                            const uint32_t o = s * 256;
                            const uint32_t acc = (kc > 0 || s > 0) ? 1u : 0u;
                            tc::mma_tf32(d, tc::sdesc(ah + o, 128, 1024), tc::sdesc(bh + o, 128, 1024), IDESC, acc);
                            tc::mma_tf32(d, tc::sdesc(ah + o, 128, 1024), tc::sdesc(bl + o, 128, 1024), IDESC, 1u);
                            tc::mma_tf32(d, tc::sdesc(al + o, 128, 1024), tc::sdesc(bh + o, 128, 1024), IDESC, 1u);
                        }
                    }
                }
                tc::commit(&ts.mbar);
            }
        }
        // epilogue: the accumulators of this column tile
        if (!tc::mbar_wait(&ts.mbar, ph & 1) && tid == 0) atomicOr(status, RB_DEV_TIMEOUT);
        ph++;
        tc::fence_after();
        const int lg = warp & 3;                   // TMEM lane quarter of this warp
        const int cbase = (warp >> 2) * (N / 2);   // its half of the columns
#pragma unroll 1
        for (int m = 0; m < mtiles; m++) {
            const int i = 128 * m + 32 * lg + lane;
#pragma unroll 1
            for (int cc = 0; cc < N / 2; cc += 16) {
                float a0[16], a1[16];
                const uint32_t lanes = (uint32_t)(32 * lg) << 16;
                tc::tmem_ld16(ts.tmem + lanes + (uint32_t)(m * N + cbase + cc), a0);
                if (parts > 1)
                    tc::tmem_ld16(ts.tmem + lanes + (uint32_t)((mtiles + m) * N + cbase + cc), a1);
                else
#pragma unroll
                    for (int q = 0; q < 16; q++) a1[q] = 0.0f;
                if (i < ni) {
                    // every load the epilogue makes for the 16 outputs first, then the stores
                    // (a store may alias those loads, so they are not interleaved)
                    double pv[16], sv[16];
#pragma unroll
                    for (int q = 0; q < 16; q++) {
                        const long long col = c0 + cbase + cc + q;
                        pv[q] = col < ncol ? epi.pre(i, col) : 0.0;
                        sv[q] = col < ncol ? epi.scale(col) : 0.0;
                    }
#pragma unroll
                    for (int q = 0; q < 16; q++) {
                        const long long col = c0 + cbase + cc + q;
                        if (col < ncol) epi.store(i, col, (double)a0[q] + sv[q] * (double)a1[q], pv[q]);
                    }
                }
            }
        }
        tc::fence_before();
        __syncthreads();  // every accumulator read before the next tile's MMAs overwrite them
    }
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
    auto sc = [=] __device__(int k, long long col) { return ys[(long long)mat[col / nm] * np + k]; };
    struct {
        const double *add, *tg;
        const int *mat;
        float *psi;
        int nd, nm, parts;
        __device__ double pre(int i, long long col) const { return add ? add[col * nd + i] : 0.0; }
        __device__ double scale(long long col) const { return parts > 1 ? tg[mat[col / nm]] : 0.0; }
        __device__ void store(int i, long long col, double v, double p) const { psi[col * nd + i] = (float)(p + v); }
    } epi{add, tg, mat, psi, nd, nm, parts};
    unsigned char *sm = reinterpret_cast<unsigned char *>(smem);
    if (tc_product<128>(t, ts, sm, smem_bytes, P.tc_m2d, parts, nd, np, parts, zin, np, ncol, sc, epi, P.status))
        return true;
    return tc_product<64>(t, ts, sm, smem_bytes, P.tc_m2d, parts, nd, np, parts, zin, np, ncol, sc, epi, P.status);
}

// The D2M product of a mixed-form 2D/3D pass on the tensor cores (FP32 angular buffer in, FP64
// state out; matvec: zout = zin − Dn·ψ).
template <class Team>
__device__ bool d2m_tc(Team &t, const DevProblem &P, TcState &ts, void *smem, long long smem_bytes, const double *zin,
                       double *zout, int matvec) {
    if (!P.tc_d2m) return false;
    const int nd = P.nd, np = P.np, nm = P.nm5;
    const long long ncol = (long long)nm * P.ncell;
    auto one = [] __device__(int, long long) { return 1.0; };
    struct {
        const double *zin;
        double *zout;
        int np, matvec;
        __device__ double pre(int i, long long col) const { return matvec ? zin[col * np + i] : 0.0; }
        __device__ double scale(long long) const { return 0.0; }
        __device__ void store(int i, long long col, double v, double p) const { zout[col * np + i] = matvec ? p - v : v; }
    } epi{zin, zout, np, matvec};
    unsigned char *sm = reinterpret_cast<unsigned char *>(smem);
    if (tc_product<128>(t, ts, sm, smem_bytes, P.tc_d2m, 1, np, nd, 1, P.psi32, nd, ncol, one, epi, P.status))
        return true;
    return tc_product<64>(t, ts, sm, smem_bytes, P.tc_d2m, 1, np, nd, 1, P.psi32, nd, ncol, one, epi, P.status);
}

}  // namespace rb
