// rb_capi.cu -- the C ABI of include/radiant_b200.h.
//
// The persistent solve kernels it launches are defined in rb_kernel_{batch,local1d,grid}.cu
// (declared in rb_solve.cuh); this file holds the host side and the small layout kernels.
// Host side of the library: validates a problem description, derives the per-direction
// closure tables once per solve, lays every table and work buffer out in one device
// allocation per problem, launches the persistent solve kernel on a stream and copies the
// results back in the reference's array layouts. No exception crosses the ABI: every entry
// point returns a status and records a message for rb_last_error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/radiant_b200.h"
#include "rb_solve.cuh"


namespace rb {
// [ng][nphi] (group-major) -> [ng, nphi] (group fastest, the reference's layout)
__global__ void to_reference_layout(const double *__restrict__ src, double *__restrict__ dst, int ng,
                                    long long nphi) {
    __shared__ double tile[32][33];
    const long long k0 = (long long)blockIdx.x * 32;
    const int g0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int g = g0 + j;
        const long long k = k0 + threadIdx.x;
        if (g < ng && k < nphi) tile[j][threadIdx.x] = src[(long long)g * nphi + k];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long long k = k0 + j;
        const int g = g0 + threadIdx.x;
        if (g < ng && k < nphi) dst[(long long)ng * k + g] = tile[threadIdx.x][j];
    }
}
// [ng, nphi] (group fastest, the reference's layout) -> [ng][nphi] (group-major)
__global__ void from_reference_layout(const double *__restrict__ src, double *__restrict__ dst, int ng,
                                      long long nphi) {
    __shared__ double tile[32][33];
    const long long k0 = (long long)blockIdx.x * 32;
    const int g0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long long k = k0 + j;
        const int g = g0 + threadIdx.x;
        if (g < ng && k < nphi) tile[threadIdx.x][j] = src[(long long)ng * k + g];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int g = g0 + j;
        const long long k = k0 + threadIdx.x;
        if (g < ng && k < nphi) dst[(long long)g * nphi + k] = tile[j][threadIdx.x];
    }
}

// ---- fixed sources built on the device (rb_upload_sources) -----------------------------------
struct DevBeam {
    int group, face;  // 0-based group; face 0..5
    double intensity;
    double dir[3], lo[3], hi[3];
};

// Volume_Source boxes into the group-major volume sources (zeroed before): angular moment 1,
// cell moment 1 of every voxel whose centre lies inside a box gets the box's intensity, boxes
// added in order (volume_source.jl:42-110 builds Q, Source.jl:129-133 adds it). pos holds the
// voxel centres [nx | ny | nz].
__global__ void assemble_volume(double *__restrict__ vol, long long nphi, long long npm, int nx, int ny, int nz,
                                int ndims, const double *__restrict__ pos, const rb_volume_box *__restrict__ boxes,
                                int nbox) {
    const long long ncell = (long long)nx * ny * nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(c % nx);
        const long long r = c / nx;
        const int iy = (int)(r % ny), iz = (int)(r / ny);
        const double px = pos[ix], py = ndims >= 2 ? pos[nx + iy] : 0.0, pz = ndims >= 3 ? pos[nx + ny + iz] : 0.0;
        for (int b = 0; b < nbox; b++) {
            const rb_volume_box B = boxes[b];
            bool in = B.lo[0] <= px && B.hi[0] >= px;
            if (ndims >= 2) in = in && B.lo[1] <= py && B.hi[1] >= py;
            if (ndims >= 3) in = in && B.lo[2] <= pz && B.hi[2] >= pz;
            if (in) {
                double *v = vol + (long long)(B.energy_group - 1) * nphi + npm * c;
                *v = *v + B.intensity;
            }
        }
    }
}

// Surface_Source beams of one face into its surface sources [ng, np_source, face cells] (zeroed
// before): intensity · basis[p] · (face-cell widths, in-plane axes in increasing order) on the
// face cells inside the aperture, when the beam enters through the face (surface_source.jl:
// 89-96 in 1D, 158-187 in 2D, 216-275 in 3D), beams added in order (Source.jl:196-201). The
// face cells are column-major over the in-plane axes a (fastest) and b.
__global__ void assemble_surface(double *__restrict__ surf, int ng, int nps, int ndims, int face, int na, int nb,
                                 const double *__restrict__ pos_a, const double *__restrict__ pos_b,
                                 const double *__restrict__ d_a, const double *__restrict__ d_b, int ax_a, int ax_b,
                                 const DevBeam *__restrict__ beams, const double *__restrict__ basis, int nbeam) {
    const long long ncf = (long long)na * nb;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncf;
         c += (long long)gridDim.x * blockDim.x) {
        const int ia = (int)(c % na), ib = (int)(c / na);
        for (int b = 0; b < nbeam; b++) {
            const DevBeam &B = beams[b];
            if (B.face != face) continue;
            const double cosv = B.dir[face / 2];
            if (!((face % 2 == 0 && cosv > 0.0) || (face % 2 == 1 && cosv < 0.0))) continue;
            if (ndims >= 2 && (pos_a[ia] < B.lo[ax_a] || pos_a[ia] > B.hi[ax_a])) continue;
            if (ndims >= 3 && (pos_b[ib] < B.lo[ax_b] || pos_b[ib] > B.hi[ax_b])) continue;
            for (int p = 0; p < nps; p++) {
                double q = B.intensity * basis[(long long)b * nps + p];
                if (ndims >= 2) q = q * d_a[ia];
                if (ndims >= 3) q = q * d_b[ib];
                double *v = surf + B.group + (long long)ng * (p + (long long)nps * c);
                *v = __dadd_rn(*v, q);  // the beam's value rounded on its own, then added (no FMA)
            }
        }
    }
}

// ---- coupled transport (rb_transport) ------------------------------------------------------
// tot += gen over [ng][nphi]; for the entries of angular moment 1, cell moment 1 also the
// largest |tot_new − tot_old| / max(|tot_new|, eps) (the reference's flux criterion,
// transport.jl:114-118), as the bits of a non-negative double in *maxrel.
__global__ void accumulate_generation(double *__restrict__ tot, const double *__restrict__ gen, long long n,
                                      long long nphi, int np, int nm5, unsigned long long *maxrel) {
    __shared__ double red[32];
    double m = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double t0 = tot[e], t1 = t0 + gen[e];
        tot[e] = t1;
        if (maxrel) {
            const long long o = e % nphi;
            if (o % ((long long)np * nm5) == 0) {  // p = 1 and is = 1 of a cell
                const double r = fabs(t1 - t0) / fmax(fabs(t1), 2.220446049250313e-16);
                m = fmax(m, r);
            }
        }
    }
    if (!maxrel) return;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x + 31) / 32; w++) m = fmax(m, red[w]);
        atomicMax(maxrel, (unsigned long long)__double_as_longlong(m));
    }
}

// particle_source (particle_source.jl:23-79) of one cell and one cell moment k of the outgoing
// particle, added to its particle source: one CTA per (cell, k). Shared memory: the incoming
// flux of the cell [ng_i][np_i] and the group-transferred source [ng_o][np_i].
__global__ void particle_source_kernel(const double *__restrict__ flux_i, int ng_i, int np_i, int nm_i,
                                       const int *__restrict__ mat, int nmat, const double *__restrict__ sigma_s,
                                       int ls, const int *__restrict__ pl_i, const double *__restrict__ transfer,
                                       const int *__restrict__ moment_map, double *__restrict__ pvol_o, int ng_o,
                                       int np_o, int nm_o, long long ncell) {
    extern __shared__ double sm[];
    double *phi = sm;                        // [ng_i][np_i]
    double *ql = sm + (long long)ng_i * np_i;  // [ng_o][np_i]
    const long long c = blockIdx.x;
    const int k = blockIdx.y;
    const int kin = moment_map[k] - 1;
    if (kin < 0 || c >= ncell) return;
    const long long nphi_i = (long long)np_i * nm_i * ncell, nphi_o = (long long)np_o * nm_o * ncell;
    const int m = mat[c];
    for (int e = threadIdx.x; e < ng_i * np_i; e += blockDim.x) {
        const int gi = e / np_i, p = e % np_i;
        phi[e] = flux_i[(long long)gi * nphi_i + p + (long long)np_i * (kin + (long long)nm_i * c)];
    }
    __syncthreads();
    // Ql_in[gf,p] = Σ_gi Σs[m,gi,gf,pl[p]]·𝚽[gi,p], gi in increasing order (particle_sources)
    for (int e = threadIdx.x; e < ng_o * np_i; e += blockDim.x) {
        const int gf = e / np_i, p = e % np_i;
        const double *ss = sigma_s + m + (long long)nmat * (long long)ng_i * (gf + (long long)ng_o * pl_i[p]);
        double q = 0.0;
        for (int gi = 0; gi < ng_i; gi++) q += ss[(long long)nmat * gi] * phi[(long long)gi * np_i + p];
        ql[e] = q;
    }
    __syncthreads();
    // Ql_out[gf,q] = Σ_p T[q,p]·Ql_in[gf,p] over the non-zero T, p in increasing order, then added
    // to the particle source
    for (int e = threadIdx.x; e < ng_o * np_o; e += blockDim.x) {
        const int gf = e / np_o, qo = e % np_o;
        double v = 0.0;
        for (int p = 0; p < np_i; p++) {
            const double tq = transfer[qo + (long long)np_o * p];
            if (tq != 0.0) v += tq * ql[(long long)gf * np_i + p];
        }
        double *dst = pvol_o + (long long)gf * nphi_o + qo + (long long)np_o * (k + (long long)nm_o * c);
        *dst = *dst + v;
    }
}

// ---- deposition (rb_deposition, rb_transport) ------------------------------------------------
// energy_deposition.jl:65-77 / charge_deposition.jl:67-79 for one particle, per voxel c:
// d = (Σ_g sig[g,mat]·𝚽[g,1,1,c] + sig[ng,mat]·𝚽cutoff[1,1,c]) / (ρ[mat]·norm), sig [ng+1, nmat]
// (Σe or Σc) and mat 0-based; dep[c] = d, or dep[c] + d to sum particles (Dtot += D).
__global__ void deposition_kernel(const double *__restrict__ flux, int ng, long long nphi, long long cstride,
                                  const double *__restrict__ cutoff, const int *__restrict__ mat,
                                  const double *__restrict__ sig, const double *__restrict__ rho, double norm,
                                  long long ncell, double *__restrict__ dep, int accumulate) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const int m = mat[c];
        const double *sg = sig + (long long)(ng + 1) * m;
        double d = 0.0;
        for (int g = 0; g < ng; g++) d += sg[g] * flux[(long long)g * nphi + cstride * c];
        if (cutoff) d += sg[ng] * cutoff[cstride * c];
        d = d / (rho[m] * norm);
        dep[c] = accumulate ? dep[c] + d : d;
    }
}
// max over c of |cur − prev| / max(|cur|, eps) (transport.jl:125, 131), as the bits of a
// non-negative double in *maxrel
__global__ void max_rel_change(const double *__restrict__ cur, const double *__restrict__ prev, long long n,
                               unsigned long long *maxrel) {
    __shared__ double red[32];
    double m = 0.0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(cur[c] - prev[c]) / fmax(fabs(cur[c]), 2.220446049250313e-16));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x + 31) / 32; w++) m = fmax(m, red[w]);
        atomicMax(maxrel, (unsigned long long)__double_as_longlong(m));
    }
}
}  // namespace rb

namespace {

thread_local std::string g_create_error;

struct ProblemRec {
    DevProblem h;            // host copy of the device record
    DevProblem *d = nullptr; // device copy
    DevProblem **own_list = nullptr;  // one-entry launch list inside the problem's block
    int *own_queue = nullptr;         // its work-queue counter
    cudaEvent_t done = nullptr;       // serving: completion of the request's launch
    char *block = nullptr;   // the problem's single device allocation
    size_t bytes = 0;
    int ng = 0, np = 0, nm5 = 0, csd = 0;
    long long ncell = 0, nphi = 0;
    cudaStream_t stream = nullptr;  // stream of the last solve
    cudaEvent_t solve_done = nullptr;  // recorded behind the last solve on `stream`
    bool solved = false;
    // rb_download_async: copies in flight into `dl_res` (flux, cutoff) and into `dl_small`, a
    // page-locked buffer from the context's list: [passes, status, rho, resid, iters, conv]
    bool dl_pending = false;
    rb_sn_result *dl_res = nullptr;
    char *dl_small = nullptr;
    size_t dl_small_cap = 0;
};

}  // namespace

struct rb_context {
    int device = 0;
    int nsm = 0;
    int cluster = 0;  // CTAs per problem team (0 = sized per batch); RB_CLUSTER_SIZE overrides
    int md_cluster = 0;  // 2D/3D problems on cluster teams instead of the whole GPU (RB_MD_TEAM=cluster)
    int local1d = 1;     // 1D problems take the cell-split local pass where it fits (RB_LOCAL1D=0: never)
    double *d_gpart = nullptr;  // grid-team reduction partials
    uint64_t budget = 0;
    uint64_t used = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;  // problem blocks (stream-ordered allocation)
    std::string err;
    std::map<int64_t, std::unique_ptr<ProblemRec>> probs;
    int64_t next_handle = 1;
    // launch scratch: problem pointer array + queue counter, staging for the layout change
    DevProblem **d_list = nullptr;
    int list_cap = 0;
    int *d_queue = nullptr;
    double *d_stage = nullptr;
    size_t stage_cap = 0;
    // serving: stream pool for concurrently running requests
    std::vector<cudaStream_t> serve_streams;
    size_t next_stream = 0;
    // measured launch rules (rb_set_launch_rules): team size by problem class
    std::vector<rb_launch_rule> rules;
    // rb_download_async: its own staging buffer, copy stream and events
    double *d_dstage = nullptr;
    size_t dstage_cap = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t dl_ready = nullptr, dl_done = nullptr;
    bool dl_busy = false;
    // page-locked small buffers of the async downloads, reused (cudaFreeHost would wait for the
    // whole device, so they are given back only by rb_destroy)
    std::vector<std::pair<char *, size_t>> small_free;
    std::vector<char *> small_all;
};

namespace {

int fail(rb_context *ctx, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf; else g_create_error = buf;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(ctx, RB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------------------------
// moment bookkeeping of the closures (same flattening as sn_{1,2,3}D_{bte,bfp}.jl)
// ---------------------------------------------------------------------------------------------
struct Moments {
    int nax = 0, ax[4] = {0}, ord[4] = {0}, nm = 0;
    int tup[RB_MAXNM][4];
    int face[4][RB_MAXNM];
    int nface[4] = {1, 1, 1, 1};
};

int flat_index(int nax, const int *ord, const int *t, int fc) {
    if (fc) {
        int idx = 0, stride = 1;
        for (int a = 0; a < nax; a++) { idx += (t[a] - 1) * stride; stride *= ord[a]; }
        return idx;
    }
    int off = 1;
    for (int a = 0; a < nax; a++) {
        if (t[a] > 1) return off + (t[a] - 2);
        off += ord[a] - 1;
    }
    return 0;
}
int count_of(int nax, const int *ord, int fc) {
    int c = 1;
    if (fc) { for (int a = 0; a < nax; a++) c *= ord[a]; return c; }
    for (int a = 0; a < nax; a++) c += ord[a] - 1;
    return c;
}
bool build_moments(Moments &M, int ndims, int csd, const int32_t *order, int fc) {
    M.nax = 0;
    if (csd) { M.ax[M.nax] = 3; M.ord[M.nax] = order[3]; M.nax++; }
    for (int d = 0; d < ndims; d++) { M.ax[M.nax] = d; M.ord[M.nax] = order[d]; M.nax++; }
    M.nm = count_of(M.nax, M.ord, fc);
    if (M.nm > RB_MAXNM) return false;
    int total = 1;
    for (int a = 0; a < M.nax; a++) total *= M.ord[a];
    for (int c = 0; c < total; c++) {
        int t[4], r = c, nbig = 0;
        for (int a = 0; a < M.nax; a++) { t[a] = r % M.ord[a] + 1; r /= M.ord[a]; if (t[a] > 1) nbig++; }
        if (!fc && nbig >= 2) continue;
        int j = flat_index(M.nax, M.ord, t, fc);
        for (int k = 0; k < 4; k++) M.tup[j][k] = 1;
        for (int a = 0; a < M.nax; a++) M.tup[j][M.ax[a]] = t[a];
        for (int a = 0; a < M.nax; a++) {
            int sub[4], so[4], ns = 0;
            for (int b = 0; b < M.nax; b++) if (b != a) { sub[ns] = t[b]; so[ns] = M.ord[b]; ns++; }
            M.face[M.ax[a]][j] = flat_index(ns, so, sub, fc);
            M.nface[M.ax[a]] = count_of(ns, so, fc);
        }
    }
    return true;
}

double ipow(double s, int k) { double r = 1.0; for (int i = 0; i < k; i++) r *= s; return r; }
double m1pow(int k) { return (k % 2 == 0) ? 1.0 : -1.0; }
double jsign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

long long face_cells(int ndims, const int *ns, int axis) {
    if (ndims == 1) return 1;
    if (ndims == 2) return axis == 0 ? ns[1] : ns[0];
    if (axis == 0) return (long long)ns[1] * ns[2];
    if (axis == 1) return (long long)ns[0] * ns[2];
    return (long long)ns[0] * ns[1];
}

// Layout of one problem's device block.
struct Layout {
    size_t off = 0;
    template <class T>
    size_t take(size_t count) {
        size_t o = (off + 255) & ~size_t(255);
        off = o + sizeof(T) * (count > 0 ? count : 1);
        return o;
    }
};

int nvec_for(const rb_sn_problem *P) {
    switch (P->accel) {
        case RB_ACCEL_NONE:
        case RB_ACCEL_LIVOLANT: return 5;
        case RB_ACCEL_ANDERSON: return 5 + 2 * (P->anderson_depth > 1 ? P->anderson_depth : 1);
        // the mixed form's defect correction keeps two more vectors (δ and the residual)
        case RB_ACCEL_GMRES: return 5 + (P->gmres_restart > 1 ? P->gmres_restart : 1) + (P->precision == 1 ? 2 : 0);
        case RB_ACCEL_BICGSTAB: return 8 + (P->precision == 1 ? 2 : 0);
    }
    return 8;
}

// TF32 rounding of the tensor cores' input conversion (cvt.rna.tf32.f32: to nearest, ties away
// from zero, 10 mantissa bits kept).
float tf32_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    u = (u + 0x1000u) & 0xFFFFE000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

// Packs operator parts A_p[i + lda·k] (ni rows, nk columns each) for tc_product (rb_tc.cuh), the
// parts stacked along K (K = parts·nk, k' = p·nk + k): NJ = ni rounded up to 16 rows, chunks of 32
// K, chunk kc at kc·2·NJ·32 floats holding the TF32 high block then the low block v − hi, element
// (r, k') at byte (r%8)·16 + (r/8)·1024 + (k'%4)·4 + ((k'%32)/4)·128 of its block (the K-major,
// no-swizzle canonical layout). Zero outside the operator.
std::vector<float> pack_tc_operator(const std::vector<const double *> &parts, int lda, int ni, int nk) {
    const int NJ = (ni + 15) & ~15, K = (int)parts.size() * nk, kch = (K + 31) / 32;
    const size_t blk = (size_t)NJ * 32;
    std::vector<float> out((size_t)kch * 2 * blk, 0.0f);
    for (int kc = 0; kc < kch; kc++)
        for (int r = 0; r < ni; r++)
            for (int kk = 0; kk < 32; kk++) {
                const int k = 32 * kc + kk;
                if (k >= K) continue;
                const double v = parts[k / nk][r + (size_t)lda * (k % nk)];
                const float hi = tf32_round((float)v);
                const float lo = (float)(v - (double)hi);
                const size_t e = (size_t)((r % 8) * 16 + (r / 8) * 1024 + (kk % 4) * 4 + (kk / 4) * 128) / 4;
                out[(size_t)kc * 2 * blk + e] = hi;
                out[(size_t)kc * 2 * blk + blk + e] = lo;
            }
    return out;
}

// Everything derived from the description before it goes to the device.
struct Derived {
    Moments M;
    int ns[3];
    long long ncell, nphi, nstate, off_b[3], nb[3], fcells[3];
    int csd;
    std::vector<int> mat0;
    std::vector<double> cosv, mn, dn, mnfp, frow_m, frow_d, G, Gsrc, Gout, Kcsd, Bcsd, EsA, EsB, Eout;
    std::vector<int> tang;
    // 2D/3D: the device holds the directions grouped by octant (quadrant in 2D), each group in
    // the reference's order; perm[k] is the reference index of device direction k, and
    // oct_start[o] .. oct_start[o+1] the device directions of octant o (bit 0: μ < 0,
    // bit 1: η < 0, bit 2: ξ < 0). 1D keeps the reference's order.
    std::vector<int> perm;
    int noct = 1, oct_start[9] = {0};
    // mixed form, 2D/3D: Mn (and Mn·ℳ) and Dn packed for the tensor-core products (rb_tc.cuh)
    std::vector<float> tc_m2d, tc_d2m;
    double w1[4];
    int nfmax = 1;
};

int validate_and_derive(rb_context *ctx, const rb_sn_problem *P, Derived &D) {
    if (!P) return fail(ctx, RB_ERR_INVALID, "null problem");
    if (P->ndims < 1 || P->ndims > 3) return fail(ctx, RB_ERR_INVALID, "ndims must be 1, 2 or 3 (got %d)", P->ndims);
    if (P->is_adaptive) return fail(ctx, RB_ERR_UNSUPPORTED, "adaptive (AWD) closures are not built");
    if (P->is_em) return fail(ctx, RB_ERR_UNSUPPORTED, "external electromagnetic fields are not built");
    if (P->solver_type < 1 || P->solver_type > 6) return fail(ctx, RB_ERR_INVALID, "solver_type %d", P->solver_type);
    if (P->accel < 0 || P->accel > 4) return fail(ctx, RB_ERR_INVALID, "accel %d", P->accel);
    if (P->accel == RB_ACCEL_GMRES && P->gmres_restart > RB_MAXRESTART)
        return fail(ctx, RB_ERR_INVALID, "gmres_restart %d exceeds %d", P->gmres_restart, RB_MAXRESTART);
    if (P->accel == RB_ACCEL_ANDERSON && P->anderson_depth > RB_MAXDEPTH)
        return fail(ctx, RB_ERR_INVALID, "anderson_depth %d exceeds %d", P->anderson_depth, RB_MAXDEPTH);
    if (P->nmat < 1 || P->nmat > RB_MAXMAT) return fail(ctx, RB_ERR_INVALID, "nmat %d out of [1,%d]", P->nmat, RB_MAXMAT);
    if (P->nd < 1 || P->np < 1 || P->ng < 1) return fail(ctx, RB_ERR_INVALID, "empty angular or energy grid");
    if (!P->mat || !P->mn || !P->dn || !P->pl || !P->sigma_t || !P->sigma_s || !P->mu || !P->dx)
        return fail(ctx, RB_ERR_INVALID, "a required table is NULL");
    if (P->max_iter < 1) return fail(ctx, RB_ERR_INVALID, "max_iter must be >= 1");
    if (P->precision != 0 && P->precision != 1) return fail(ctx, RB_ERR_INVALID, "precision %d", P->precision);
    if (!(P->tol > 0)) return fail(ctx, RB_ERR_INVALID, "tol must be > 0");
    D.csd = P->solver_type >= 2;
    if (D.csd && (!P->s_minus || !P->s_plus || !P->s_mom || !P->e_width || !P->ww))
        return fail(ctx, RB_ERR_INVALID, "CSD solver without stopping powers / energy widths");
    if ((P->solver_type == 2 || P->solver_type == 4) && (!P->t_mom || !P->fp))
        return fail(ctx, RB_ERR_INVALID, "Fokker-Planck solver without momentum transfer / matrix");
    if (P->order[3] > RB_MAXORD || P->order[0] > RB_MAXORD) return fail(ctx, RB_ERR_INVALID, "scheme order too high");
    D.ns[0] = P->nx; D.ns[1] = P->ndims >= 2 ? P->ny : 1; D.ns[2] = P->ndims >= 3 ? P->nz : 1;
    if (D.ns[0] < 1 || D.ns[1] < 1 || D.ns[2] < 1) return fail(ctx, RB_ERR_INVALID, "empty geometry");
    if (!build_moments(D.M, P->ndims, D.csd, P->order, P->is_fc))
        return fail(ctx, RB_ERR_UNSUPPORTED, "cell system larger than %d moments", RB_MAXNM);
    if (D.M.nm != P->nm[4]) return fail(ctx, RB_ERR_INVALID, "nm[4]=%d but the closures give %d moments", P->nm[4], D.M.nm);
    for (int d = 0; d < P->ndims; d++)
        if (D.M.nface[d] != P->nm[d]) return fail(ctx, RB_ERR_INVALID, "nm[%d]=%d but the closures give %d", d, P->nm[d], D.M.nface[d]);
    if (D.csd && D.M.nface[3] != P->nm[3]) return fail(ctx, RB_ERR_INVALID, "nm[3] inconsistent");
    if (P->nm[0] > RB_MAXFACE || P->nm[3] > RB_MAXFACE) return fail(ctx, RB_ERR_INVALID, "too many face moments");
    for (int k = 0; k < P->np; k++)
        if (P->pl[k] < 0 || P->pl[k] > P->ls) return fail(ctx, RB_ERR_INVALID, "pl[%d]=%d outside [0,ls=%d]", k, P->pl[k], P->ls);
    D.ncell = (long long)D.ns[0] * D.ns[1] * D.ns[2];
    const int nm5 = D.M.nm, np = P->np, nd = P->nd, nps = P->np_surf;
    D.nphi = (long long)np * nm5 * D.ncell;
    long long off = D.nphi;
    for (int d = 0; d < 3; d++) {
        D.nb[d] = d < P->ndims ? (long long)nps * P->nm[d] * 2 * face_cells(P->ndims, D.ns, d) : 0;
        D.off_b[d] = off;
        off += D.nb[d];
    }
    D.nstate = off;
    // materials
    D.mat0.resize(D.ncell);
    for (long long c = 0; c < D.ncell; c++) {
        int m = P->mat[c];
        if (m < 1 || m > P->nmat) return fail(ctx, RB_ERR_INVALID, "mat[%lld]=%d outside 1..%d", c, m, P->nmat);
        D.mat0[c] = m - 1;
    }
    for (long long c = 0; c < D.ns[0]; c++)
        if (!(P->dx[c] > 0)) return fail(ctx, RB_ERR_INVALID, "dx[%lld] must be > 0", c);
    if (P->ndims >= 2) {
        if (!P->dy || !P->eta) return fail(ctx, RB_ERR_INVALID, "2D problem without dy / eta");
        for (long long c = 0; c < D.ns[1]; c++)
            if (!(P->dy[c] > 0)) return fail(ctx, RB_ERR_INVALID, "dy[%lld] must be > 0", c);
        if ((long long)D.ns[0] * P->nm[1] > RB_TILE_DOUBLES)
            return fail(ctx, RB_ERR_UNSUPPORTED, "nx x face moments = %lld exceeds the wavefront's shared slots (%d)",
                        (long long)D.ns[0] * P->nm[1], RB_TILE_DOUBLES);
    }
    if (P->ndims == 3) {
        if (!P->dz || !P->xi) return fail(ctx, RB_ERR_INVALID, "3D problem without dz / xi");
        for (long long c = 0; c < D.ns[2]; c++)
            if (!(P->dz[c] > 0)) return fail(ctx, RB_ERR_INVALID, "dz[%lld] must be > 0", c);
    }
    for (int d = 0; d < 3; d++) D.fcells[d] = d < P->ndims ? face_cells(P->ndims, D.ns, d) : 0;
    // directions, grouped by octant on 2D/3D problems (stable: the reference's order inside)
    D.perm.resize(nd);
    D.noct = P->ndims == 1 ? 1 : (P->ndims == 2 ? 4 : 8);
    {
        auto oct = [&](int n) {
            if (P->ndims == 1) return 0;
            int o = (P->mu[n] < 0.0 ? 1 : 0) + (P->eta[n] < 0.0 ? 2 : 0);
            if (P->ndims == 3) o += P->xi[n] < 0.0 ? 4 : 0;
            return o;
        };
        int k = 0;
        for (int o = 0; o < D.noct; o++) {
            D.oct_start[o] = k;
            for (int n = 0; n < nd; n++)
                if (oct(n) == o) D.perm[k++] = n;
        }
        for (int o = D.noct; o <= 8; o++) D.oct_start[o] = nd;
    }
    const std::vector<int> &pm = D.perm;
    D.cosv.assign(3 * (size_t)nd, 0.0);
    D.mn.resize((size_t)nd * np);
    D.dn.resize((size_t)np * nd);
    for (int n = 0; n < nd; n++) {
        D.cosv[n] = P->mu[pm[n]];
        D.cosv[nd + n] = P->eta ? P->eta[pm[n]] : 0.0;
        D.cosv[2 * nd + n] = P->xi ? P->xi[pm[n]] : 0.0;
        for (int p = 0; p < np; p++) {
            D.mn[n + (size_t)nd * p] = P->mn[pm[n] + (long long)nd * p];
            D.dn[p + (size_t)np * n] = P->dn[p + (long long)np * pm[n]];
        }
    }
    // Mn·ℳ
    if (P->solver_type == 2 || P->solver_type == 4) {
        D.mnfp.assign((size_t)nd * np, 0.0);
        for (int n = 0; n < nd; n++)
            for (int p = 0; p < np; p++) {
                double s = 0.0;
                for (int q = 0; q < np; q++) s += D.mn[n + (size_t)nd * q] * P->fp[q + (long long)np * p];
                D.mnfp[n + (size_t)nd * p] = s;
            }
    }
    // the mixed form's tensor-core operators (2D/3D, up to 256 rows)
    if (P->precision == 1 && P->ndims >= 2 && nd <= 256 && np <= 256) {
        std::vector<const double *> pm2d{D.mn.data()};
        if (!D.mnfp.empty()) pm2d.push_back(D.mnfp.data());
        D.tc_m2d = pack_tc_operator(pm2d, nd, nd, np);
        D.tc_d2m = pack_tc_operator({D.dn.data()}, np, np, nd);
    }
    // half-range rows per direction and axis (sn_inner_pass.jl:47-58)
    D.frow_m.assign((size_t)3 * nd * (nps > 0 ? nps : 1), 0.0);
    D.frow_d.assign((size_t)3 * nd * (nps > 0 ? nps : 1), 0.0);
    for (int a = 0; a < P->ndims; a++) {
        int fm = 2 * a, fp = 2 * a + 1;
        for (int n = 0; n < nd; n++) {
            int k1 = P->n_to_nplus[fm] ? P->n_to_nplus[fm][pm[n]] : 0;
            int k2 = P->n_to_nplus[fp] ? P->n_to_nplus[fp][pm[n]] : 0;
            int f = -1, k = 0;
            if (k1 != 0) { f = fm; k = k1; } else if (k2 != 0) { f = fp; k = k2; }
            if (f < 0) continue;
            if (k > P->nd_plus[f]) return fail(ctx, RB_ERR_INVALID, "n_to_nplus[%d][%d]=%d > nd_plus", f, n, k);
            for (int p = 0; p < nps; p++) {
                D.frow_m[((size_t)a * nd + n) * nps + p] = P->mn_surf[f][(k - 1) + (long long)P->nd_plus[f] * p];
                D.frow_d[((size_t)a * nd + n) * nps + p] = P->dn_surf[f][p + (long long)nps * (k - 1)];
            }
        }
    }
    // closure coefficient tables (the terms of flux_xD_BTE / flux_xD_BFP, factored by h)
    const Moments &M = D.M;
    const double *C = P->cc;
    for (int a = 0; a < 4; a++) D.w1[a] = P->w_axis[a] ? P->w_axis[a][0] : 0.0;
    int nfmax = 1;
    for (int a = 0; a < P->ndims; a++) nfmax = P->nm[a] > nfmax ? P->nm[a] : nfmax;
    D.nfmax = nfmax;
    D.G.assign((size_t)nd * 3 * nm5 * nm5, 0.0);
    D.Gsrc.assign((size_t)nd * 3 * nm5 * nfmax, 0.0);
    D.Gout.assign((size_t)nd * 3 * nm5 * nfmax, 0.0);
    D.tang.assign(nd, 0);
    for (int n = 0; n < nd; n++) {
        for (int a = 0; a < P->ndims; a++) {
            double cosa = D.cosv[(size_t)a * nd + n];
            double s = jsign(cosa);
            if (P->ndims == 1 && std::fabs(cosa) <= 1e-10) { s = 1.0; D.tang[n] = 1; }  // sn_1D_bte.jl:30-32
            const double *w = P->w_axis[a];
            const int nfa = P->nm[a];
            const size_t blk = (size_t)n * 3 + a;
            double *Gb = &D.G[blk * nm5 * nm5];
            for (int i = 0; i < nm5; i++)
                for (int j = 0; j < nm5; j++) {
                    bool same = true;
                    for (int k = 0; k < 4; k++) if (k != a && M.tup[i][k] != M.tup[j][k]) same = false;
                    if (!same) continue;
                    int ia = M.tup[i][a], ja = M.tup[j][a];
                    double v = 0.0;
                    if (ia >= ja + 1) v -= C[ia - 1] * s * C[ja - 1] * (1.0 - m1pow(ia - ja));
                    v += C[ia - 1] * ipow(s, ia - 1) * C[ja - 1] * ipow(s, ja - 1) * w[ja];
                    Gb[i + nm5 * j] = v;
                }
            for (int j = 0; j < nm5; j++) {
                int ja = M.tup[j][a], f = M.face[a][j];
                D.Gsrc[blk * nm5 * nfmax + j + (size_t)nm5 * f] = -C[ja - 1] * (ipow(s, ja - 1) * w[0] - ipow(-s, ja - 1));
                D.Gout[blk * nm5 * nfmax + f + (size_t)nfa * j] = C[ja - 1] * ipow(s, ja - 1) * w[ja];
            }
        }
    }
    const int oE = P->order[3];
    const int nE = D.csd ? P->nm[3] : 1;
    D.Kcsd.assign((size_t)oE * nm5 * nm5, 0.0);
    D.Bcsd.assign((size_t)nm5 * nm5, 0.0);
    D.EsA.assign((size_t)nm5 * nE, 0.0); D.EsB.assign((size_t)nm5 * nE, 0.0); D.Eout.assign((size_t)nm5 * nE, 0.0);
    if (D.csd) {
        const double *wE = P->w_axis[3];
        for (int i = 0; i < nm5; i++)
            for (int j = 0; j < nm5; j++) {
                bool same = true;
                for (int d = 0; d < P->ndims; d++) if (M.tup[i][d] != M.tup[j][d]) same = false;
                if (!same) continue;
                int iE = M.tup[i][3], jE = M.tup[j][3];
                for (int kE = 1; kE <= iE - 1; kE++)
                    for (int wi = 1; wi <= oE; wi++)
                        D.Kcsd[(size_t)(wi - 1) * nm5 * nm5 + i + nm5 * j] +=
                            C[iE - 1] * C[jE - 1] * C[kE - 1] * C[wi - 1] * (1.0 - m1pow(iE - kE)) *
                            P->ww[(jE - 1) + oE * ((kE - 1) + oE * (wi - 1))];
                D.Bcsd[i + nm5 * j] = C[iE - 1] * m1pow(iE - 1) * C[jE - 1] * m1pow(jE - 1) * wE[jE];
            }
        for (int j = 0; j < nm5; j++) {
            int jE = M.tup[j][3], e = M.face[3][j];
            D.EsA[j + (size_t)nm5 * e] = C[jE - 1] * m1pow(jE - 1) * wE[0];
            D.EsB[j + (size_t)nm5 * e] = C[jE - 1];
            D.Eout[e + (size_t)nE * j] = C[jE - 1] * m1pow(jE - 1) * wE[jE];
        }
    }
    return RB_OK;
}

template <class T>
int put(rb_context *ctx, char *block, size_t off, const T *src, size_t count, cudaStream_t s) {
    if (count == 0 || !src) return RB_OK;
    CK(cudaMemcpyAsync(block + off, src, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    return RB_OK;
}

int required(const rb_sn_problem *P, const Derived &D, Layout &L, size_t offs[64]) {
    const int nd = P->nd, np = P->np, nm5 = D.M.nm, ng = P->ng, nmat = P->nmat;
    const long long nq = (long long)nd * nm5 * D.ncell;
    const long long nE = (long long)nd * P->nm[3] * D.ncell;
    int k = 0;
    offs[k++] = L.take<DevProblem>(1);
    offs[k++] = L.take<double>(D.ns[0]);                  // 1 dx
    offs[k++] = L.take<int>(D.ncell);                     // 2 mat
    offs[k++] = L.take<double>(3 * (size_t)nd);           // 3 cosv
    offs[k++] = L.take<double>((size_t)nd * np);          // 4 mn
    offs[k++] = L.take<double>((size_t)np * nd);          // 5 dn
    offs[k++] = L.take<int>(np);                          // 6 pl
    offs[k++] = L.take<double>(D.mnfp.size());            // 7 mnfp
    offs[k++] = L.take<double>(D.frow_m.size());          // 8
    offs[k++] = L.take<double>(D.frow_d.size());          // 9
    offs[k++] = L.take<double>(D.G.size());               // 10
    offs[k++] = L.take<double>(D.Gsrc.size());            // 11
    offs[k++] = L.take<double>(D.Gout.size());            // 12
    offs[k++] = L.take<int>(D.tang.size());               // 13
    offs[k++] = L.take<double>(3 * D.EsA.size());         // 14 EsA, EsB, Eout
    offs[k++] = L.take<double>(D.Kcsd.size());            // 15
    offs[k++] = L.take<double>(D.Bcsd.size());            // 16
    offs[k++] = L.take<unsigned long long>(RB_OCT_MAXCTA); // 17 progress flags of the 3D octant sweep
    offs[k++] = L.take<double>((size_t)ng * nmat);        // 18 sigma_t
    offs[k++] = L.take<double>((size_t)nmat * ng * ng * (P->ls + 1)); // 19 sigma_s
    offs[k++] = L.take<double>(D.csd ? (size_t)ng * nmat : 0);        // 20 s_minus
    offs[k++] = L.take<double>(D.csd ? (size_t)ng * nmat : 0);        // 21 s_plus
    offs[k++] = L.take<double>(D.csd ? (size_t)ng * nmat * P->order[3] : 0); // 22 s_mom
    offs[k++] = L.take<double>(P->t_mom ? (size_t)ng * nmat : 0);     // 23 t_mom
    offs[k++] = L.take<double>(D.csd ? (size_t)ng : 0);               // 24 e_width
    offs[k++] = L.take<double>(P->volume_sources ? (size_t)P->ng * D.nphi : 0);  // 25 vol (group-major)
    for (int f = 0; f < 6; f++)                                       // 26..31 surface
        offs[k++] = L.take<double>((f < 2 * P->ndims && P->surface_sources[f])
                                       ? (size_t)ng * P->np_source * face_cells(P->ndims, D.ns, f / 2) : 0);
    offs[k++] = L.take<double>((size_t)ng * D.nphi);      // 32 flux
    offs[k++] = L.take<double>((size_t)nvec_for(P) * ((D.nstate + 1) & ~1LL)); // 33 vecs (even stride)
    offs[k++] = L.take<double>(D.nphi);                   // 34 qlout
    offs[k++] = L.take<double>(nq);                       // 35 qnout
    offs[k++] = L.take<double>(nq);                       // 36 psi
    offs[k++] = L.take<double>((size_t)nmat * np);        // 37 kmat (in-group Σs per material and moment)
    offs[k++] = L.take<double>((size_t)nmat * nm5 * nm5); // 38 scsd
    {
        const long long md = (long long)nd * rb::md_scratch_stride_n(D.ns[0], D.ns[1], D.ns[2], D.nfmax);
        const long long one = (long long)nd * RB_MAXFACE;
        offs[k++] = L.take<double>(P->ndims == 1 ? one : md);  // 39 fexit / multi-D face scratch
    }
    offs[k++] = L.take<double>(D.csd ? nE : 0);           // 40 phiE_a
    offs[k++] = L.take<double>(D.csd ? nE : 0);           // 41 phiE_b
    offs[k++] = L.take<double>(D.csd ? D.nphi : 0);       // 42 cutoff
    offs[k++] = L.take<double>(2 * (size_t)ng);           // 43 rho, resid
    offs[k++] = L.take<int>(2 * (size_t)ng);              // 44 iters, conv
    offs[k++] = L.take<long long>(1);                     // 45 passes
    offs[k++] = L.take<int>(1);                           // 46 status
    offs[k++] = L.take<double>(D.ns[1]);                  // 47 dy
    offs[k++] = L.take<double>(D.ns[2]);                  // 48 dz
    offs[k++] = L.take<float>(P->precision == 1 ? (size_t)nq : 0);  // 49 psi32 (mixed form)
    offs[k++] = L.take<DevProblem *>(1);                  // 50 own launch list (one entry)
    offs[k++] = L.take<int>(1);                           // 51 own work-queue counter
    offs[k++] = L.take<float>(D.tc_m2d.size());           // 52 tensor-core M2D operator (mixed 2D/3D)
    offs[k++] = L.take<float>(D.tc_d2m.size());           // 53 tensor-core D2M operator
    return k;
}

// Cluster size and shared memory of a launch (one CTA per SM): GroupShared plus, when some 1D
// problem can take the local pass, a local region of all the shared memory left. The cluster:
//   LAUNCH_FIXED   the caller's size;
//   LAUNCH_SERVE   the caller's size, doubled (up to 4×) until the local pass fits;
//   LAUNCH_BATCH   from 4 CTAs up, the smallest size that still gives no more teams than
//                  problems (a large batch runs many small teams, a small one a few large
//                  teams), among the sizes at which every 1D problem fits the local pass with its
//                  Gram-Schmidt slice in shared memory (else, fits it at all). Below 4 CTAs a team
//                  is slower per pass than the extra teams gain, measured on B200.
// Problems that do not fit take the team-wide pass.
enum { LAUNCH_FIXED = 0, LAUNCH_SERVE = 1, LAUNCH_BATCH = 2 };
struct LaunchShape {
    int cluster;
    long long local_bytes;
    size_t smem;
};

static LaunchShape choose_shape(const std::vector<const DevProblem *> &hs, int cluster, int mode, int nsm) {
    int dev = 0, per_sm = 0, reserved = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const long long gsz = (long long)sizeof(rb::GroupShared);
    const long long b1 = (std::min<long long>(optin, (long long)per_sm - reserved) - gsz) & ~15LL;
    LaunchShape sh{cluster, 0, (size_t)gsz};
    bool any = false;  // some problem takes the local 1D pass or the 3D octant sweep
    for (const DevProblem *h : hs) any = any || rb::local1d_ok(*h, 1 << 4, 1LL << 40) || h->ndims == 3;
    if (!any || b1 <= 0) return sh;
    auto fits = [&](int C, bool w) {  // every local-shaped 1D problem fits the local pass at cluster C
        for (const DevProblem *h : hs)
            if (rb::local1d_ok(*h, C, 1LL << 40) && !(w ? rb::local1d_w(*h, C, b1) : rb::local1d_ok(*h, C, b1)))
                return false;
        return true;
    };
    int C = cluster;
    if (mode == LAUNCH_SERVE) {
        for (int c = cluster; c <= std::min(RB_MAXCLUSTER, 4 * cluster); c *= 2)
            if (fits(c, false)) { C = c; break; }
    } else if (mode == LAUNCH_BATCH) {
        const int n = (int)hs.size();
        for (int w = 1; w >= 0 && C == cluster; w--) {
            int best = -1, largest = -1;
            for (int c = 4; c <= RB_MAXCLUSTER; c *= 2) {
                if (!fits(c, w != 0)) continue;
                largest = c;
                if (best < 0 && nsm / c <= n + n / 20) best = c;
            }
            if (best < 0) best = largest;
            if (best > 0) { C = best; break; }
        }
    }
    sh.cluster = C;
    sh.local_bytes = b1;
    sh.smem = (size_t)(gsz + b1);
    return sh;
}

// Launches the persistent solve kernel as clusters of `cluster` CTAs (one team per problem),
// as many clusters as fit on the device at once, capped by the number of problems. `hs` holds
// host copies of the problems' records (sizes only) for the shared-memory plan.
int launch_solve(rb_context *ctx, DevProblem **list, int n, int *queue, int nsm, int cluster, cudaStream_t s,
                 const std::vector<const DevProblem *> &hs, int mode) {
    if (cluster < 1) cluster = 1;
    if (cluster > RB_MAXCLUSTER) cluster = RB_MAXCLUSTER;
    const LaunchShape sh =
        choose_shape((ctx && !ctx->local1d) ? std::vector<const DevProblem *>() : hs, cluster, mode, nsm);
    cluster = sh.cluster;
    const size_t smem = sh.smem;
    const int local_bytes = (int)sh.local_bytes;
    // a batch whose every problem takes the local 1D pass runs on the kernel carrying only it
    bool all_local = !hs.empty() && local_bytes > 0;
    for (const DevProblem *h : hs) all_local = all_local && rb::local1d_ok(*h, cluster, local_bytes);
    void (*kern)(DevProblem *const *, int, int *, int) = all_local ? rb::solve_local1d_kernel : rb::solve_batch_kernel;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (cluster > 8) CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(RB_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int max_clusters = 0;
    cfg.gridDim = dim3(cluster * (nsm / cluster > 0 ? nsm / cluster : 1), 1, 1);
    CK(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg));
    if (max_clusters < 1) return fail(ctx, RB_ERR_CUDA, "no cluster of %d CTAs fits on the device", cluster);
    int nclusters = max_clusters < n ? max_clusters : n;
    cfg.gridDim = dim3(cluster * nclusters, 1, 1);
    CK(cudaLaunchKernelEx(&cfg, kern, (DevProblem *const *)list, n, queue, local_bytes));
    return RB_OK;
}

// One 2D/3D problem on every SM: a cooperative launch of one CTA per SM (the team is the grid),
// with the shared memory of the 3D octant sweep after GroupShared.
int launch_grid(rb_context *ctx, DevProblem *prob, const DevProblem &hp, cudaStream_t s) {
    // the region after GroupShared serves the 3D octant sweep and the tensor-core products; it is
    // sized to what this problem uses, since the rest of the SM's 256 KB stays L1 cache
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const long long avail = (optin - (long long)sizeof(rb::GroupShared)) & ~1023LL;
    const DevProblem &h = hp;
    const bool mixed = h.precision == 1;
    long long need = 0;
    if (h.ndims == 3 && h.nm5 == 1 && h.nm4 == 1 && h.nmf[0] == 1 && h.nmf[1] == 1 && h.nmf[2] == 1)
        need = mixed ? (h.csd ? rb::oct3d_smem<float, true>() : rb::oct3d_smem<float, false>())
                     : (h.csd ? rb::oct3d_smem<double, true>() : rb::oct3d_smem<double, false>());
    if (mixed && h.tc_m2d) {  // the products: operator resident where it fits, else streamed
        const int parts = h.mnfp ? 2 : 1;
        auto plan = [&](int nj, int nk) {
            const long long r = rb::tc::bytes_resident(rb::tc::round16(nj), nk);
            return r <= avail ? r : rb::tc::bytes_streamed(rb::tc::round16(nj));
        };
        need = std::max(need, std::max(plan(h.nd, parts * h.np), plan(h.np, h.nd)));
    }
    if (need > avail) need = 0;  // the problem then takes the paths that need no region
    const int local_bytes = (int)((need + 1023) & ~1023LL);
    const size_t smem = sizeof(rb::GroupShared) + local_bytes;
    CK(cudaFuncSetAttribute(rb::solve_grid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rb::solve_grid_kernel, RB_THREADS, smem));
    if (per_sm < 1) return fail(ctx, RB_ERR_CUDA, "the grid solve kernel does not fit on an SM");
    if (per_sm > 1) per_sm = 1;
    const int grid = ctx->nsm * per_sm;
    if (!ctx->d_gpart) CK(cudaMalloc(&ctx->d_gpart, sizeof(double) * 2 * 4 * 4096));
    void *args[] = {(void *)&prob, (void *)&ctx->d_gpart, (void *)&local_bytes};
    CK(cudaLaunchCooperativeKernel((void *)rb::solve_grid_kernel, dim3(grid), dim3(RB_THREADS), args, smem, s));
    return RB_OK;
}

int ensure_launch_scratch(rb_context *ctx, int n) {
    if (n > ctx->list_cap) {
        if (ctx->d_list) cudaFree(ctx->d_list);
        int cap = n < 64 ? 64 : n;
        CK(cudaMalloc(&ctx->d_list, sizeof(DevProblem *) * cap));
        ctx->list_cap = cap;
    }
    if (!ctx->d_queue) CK(cudaMalloc(&ctx->d_queue, sizeof(int) * 64));
    return RB_OK;
}

// The work estimate of a problem (the work queue's order and the launch rules' classes):
// groups × directions × cells × cell moments, doubled for the CSD solvers.
static double problem_work(const DevProblem &h) {
    return (double)h.ng * h.nd * (double)h.ncell * h.nm5 * (h.csd ? 2.0 : 1.0);
}

// The team size the launch rules give a batch: for each problem the first rule of its dimension
// whose direction, work and batch-size bounds cover it; the largest of the problems' sizes; 0
// when some problem has no rule (the built-in shape choice then applies).
static int rule_cluster(const rb_context *ctx, const std::vector<const DevProblem *> &hs) {
    if (!ctx || ctx->rules.empty() || hs.empty()) return 0;
    int c = 0;
    for (const DevProblem *h : hs) {
        int got = 0;
        for (const rb_launch_rule &r : ctx->rules)
            if (r.ndims == h->ndims && h->nd <= r.nd_max && problem_work(*h) <= (double)r.work_max &&
                (long long)hs.size() <= (long long)r.batch_max) {
                got = r.cluster;
                break;
            }
        if (got <= 0) return 0;
        c = std::max(c, got);
    }
    return c;
}

int launch(rb_context *ctx, const std::vector<ProblemRec *> &recs, cudaStream_t s) {
    int n = (int)recs.size();
    if (n == 0) return RB_OK;
    int st = ensure_launch_scratch(ctx, n);
    if (st) return st;
    CK(cudaMemsetAsync(ctx->d_queue, 0, sizeof(int), s));
    for (auto *r : recs) CK(cudaMemsetAsync(r->h.status, 0, sizeof(int), s));
    // 1D problems (and 2D/3D ones when RB_MD_TEAM=cluster) share one persistent cluster launch;
    // 2D/3D problems otherwise get the whole GPU each, one cooperative launch after another
    std::vector<DevProblem *> small;
    std::vector<const DevProblem *> small_h;
    std::vector<ProblemRec *> large;
    std::vector<ProblemRec *> qs;
    for (auto *r : recs) {
        if (r->h.ndims == 1 || ctx->md_cluster) qs.push_back(r);
        else large.push_back(r);
    }
    // the work queue hands problems out heaviest first (longest-processing-time order), so the
    // light ones fill the teams' last slots; the estimate is groups × directions × cells × cell
    // moments, doubled for the CSD solvers
    auto work = [](const DevProblem &h) { return problem_work(h); };
    std::stable_sort(qs.begin(), qs.end(), [&](const ProblemRec *a, const ProblemRec *b) { return work(a->h) > work(b->h); });
    for (auto *r : qs) { small.push_back(r->d); small_h.push_back(&r->h); }
    if (!small.empty()) {
        CK(cudaMemcpyAsync(ctx->d_list, small.data(), sizeof(DevProblem *) * small.size(), cudaMemcpyHostToDevice, s));
        int cluster = ctx->cluster;
        const int ruled = cluster > 0 ? 0 : rule_cluster(ctx, small_h);
        if (ruled > 0) cluster = ruled;  // a measured launch rule
        if (cluster <= 0) {  // one cluster per problem, sized to the problem's directions
            const DevProblem &h0 = recs[0]->h;
            cluster = h0.nd >= 32 ? 4 : (h0.nd >= 16 ? 4 : (h0.nd >= 8 ? 2 : 1));
        }
        int st2 = launch_solve(ctx, ctx->d_list, (int)small.size(), ctx->d_queue, ctx->nsm, cluster, s, small_h,
                               (ctx->cluster > 0 || ruled > 0) ? LAUNCH_FIXED : LAUNCH_BATCH);
        if (st2) return st2;
    }
    for (auto *r : large) {
        int st3 = launch_grid(ctx, r->d, r->h, s);
        if (st3) return st3;
    }
    for (auto *r : recs) {
        if (!r->solve_done) CK(cudaEventCreateWithFlags(&r->solve_done, cudaEventDisableTiming));
        CK(cudaEventRecord(r->solve_done, s));
        r->stream = s;
        r->solved = true;
    }
    return RB_OK;
}

ProblemRec *find(rb_context *ctx, rb_handle h) {
    auto it = ctx->probs.find(h);
    return it == ctx->probs.end() ? nullptr : it->second.get();
}

// Lays one problem out in the device block `b` (offsets `o` from required()): fills the
// device record `h`, queues the table copies on `s` and writes the record to *dptr.
// Source definitions of rb_upload_sources and where their device copies sit in the block.
struct SourceDefs {
    const rb_source_set *src;
    size_t off_pos, off_box, off_beam, off_basis;
};

int place_sources(rb_context *ctx, const rb_sn_problem *P, const Derived &D, const SourceDefs &S, char *b,
                  cudaStream_t s, const DevProblem &h);

int place_problem(rb_context *ctx, const rb_sn_problem *P, const Derived &D, const size_t *o, char *b,
                  cudaStream_t s, DevProblem &h, DevProblem **dptr, double *stage, const SourceDefs *defs = nullptr) {
    memset(&h, 0, sizeof(h));
    const int nd = P->nd, np = P->np, nm5 = D.M.nm, ng = P->ng, nmat = P->nmat;
    h.ndims = P->ndims; h.nx = D.ns[0]; h.ny = D.ns[1]; h.nz = D.ns[2]; h.ncell = D.ncell;
    h.nd = nd; h.np = np; h.nm5 = nm5;
    for (int d = 0; d < 3; d++) h.nmf[d] = d < P->ndims ? P->nm[d] : 1;
    h.nm4 = D.csd ? P->nm[3] : 1;
    h.npsurf = P->np_surf; h.ng = ng; h.nmat = nmat; h.ls = P->ls; h.oE = P->order[3]; h.csd = D.csd;
    h.solver_type = P->solver_type; h.accel = P->accel; h.maxit = P->max_iter; h.restart = P->gmres_restart;
    h.depth = P->anderson_depth; h.precision = P->precision; h.tol = P->tol; h.np_source = P->np_source;
    h.nphi = D.nphi; h.nstate = D.nstate;
    for (int d = 0; d < 3; d++) { h.off_b[d] = D.off_b[d]; h.nb[d] = D.nb[d]; }
    h.nvec = nvec_for(P);
    h.vstride = (D.nstate + 1) & ~1LL;
    for (int a = 0; a < 4; a++) h.w1[a] = D.w1[a];
    for (int f = 0; f < 6; f++) h.bc[f] = P->bc[f];
    h.noct = D.noct;
    for (int o = 0; o <= 8; o++) h.oct_start[o] = D.oct_start[o];
#define DP(T, k) (reinterpret_cast<T *>(b + o[k]))
    h.dx = DP(double, 1); h.mat = DP(int, 2); h.cosv = DP(double, 3); h.mn = DP(double, 4); h.dn = DP(double, 5);
    h.pl = DP(int, 6); h.mnfp = D.mnfp.empty() ? nullptr : DP(double, 7); h.frow_m = DP(double, 8);
    h.frow_d = DP(double, 9); h.G = DP(double, 10); h.Gsrc = DP(double, 11); h.Gout = DP(double, 12);
    h.tang = DP(int, 13); h.Kcsd = DP(double, 15); h.Bcsd = DP(double, 16);
    h.oct_flags = DP(unsigned long long, 17);
    h.EsA = DP(double, 14); h.EsB = h.EsA + D.EsA.size(); h.Eout = h.EsA + 2 * D.EsA.size();
    h.nfmax = D.nfmax;
    h.sigma_t = DP(double, 18); h.sigma_s = DP(double, 19);
    h.s_minus = D.csd ? DP(double, 20) : nullptr; h.s_plus = D.csd ? DP(double, 21) : nullptr;
    h.s_mom = D.csd ? DP(double, 22) : nullptr; h.t_mom = P->t_mom ? DP(double, 23) : nullptr;
    h.e_width = D.csd ? DP(double, 24) : nullptr; h.vol = P->volume_sources ? DP(double, 25) : nullptr;
    for (int f = 0; f < 6; f++) h.surf[f] = (f < 2 * P->ndims && P->surface_sources[f]) ? DP(double, 26 + f) : nullptr;
    h.flux = DP(double, 32); h.vecs = DP(double, 33); h.qlout = DP(double, 34); h.qnout = DP(double, 35);
    h.psi = DP(double, 36); h.kmat = DP(double, 37); h.scsd = DP(double, 38); h.fexit = DP(double, 39);
    h.phiE_a = D.csd ? DP(double, 40) : nullptr; h.phiE_b = D.csd ? DP(double, 41) : nullptr;
    h.cutoff = D.csd ? DP(double, 42) : nullptr;
    h.rho = DP(double, 43); h.resid = h.rho + ng; h.iters = DP(int, 44); h.conv = h.iters + ng;
    h.passes = DP(long long, 45); h.status = DP(int, 46);
    h.dy = P->ndims >= 2 ? DP(double, 47) : nullptr; h.dz = P->ndims >= 3 ? DP(double, 48) : nullptr;
    h.psi32 = P->precision == 1 ? DP(float, 49) : nullptr;
    h.tc_m2d = D.tc_m2d.empty() ? nullptr : DP(float, 52);
    h.tc_d2m = D.tc_d2m.empty() ? nullptr : DP(float, 53);
    // mixed form: its contract is 1e-5 relative L2 against the FP64 solution; the FP32
    // operator's noise floor is near 1e-7, so its in-group criterion is held at 1e-7 or looser
    // (the energy-face chain of a CSD solve amplifies the in-group error about tenfold)
    for (int d = 0; d < 3; d++) h.fcells[d] = D.fcells[d];
    int r = RB_OK;
#define PUT(T, k, src, n) if ((r = put<T>(ctx, b, o[k], src, n, s)) != RB_OK) return r;
    PUT(double, 1, P->dx, D.ns[0]);
    if (P->ndims >= 2) PUT(double, 47, P->dy, D.ns[1]);
    if (P->ndims >= 3) PUT(double, 48, P->dz, D.ns[2]);
    PUT(int, 2, D.mat0.data(), D.mat0.size());
    PUT(double, 3, D.cosv.data(), D.cosv.size());
    PUT(double, 4, D.mn.data(), (size_t)nd * np);
    PUT(double, 5, D.dn.data(), (size_t)np * nd);
    PUT(int, 6, P->pl, np);
    PUT(double, 7, D.mnfp.data(), D.mnfp.size());
    PUT(double, 8, D.frow_m.data(), D.frow_m.size());
    PUT(double, 9, D.frow_d.data(), D.frow_d.size());
    PUT(double, 10, D.G.data(), D.G.size());
    PUT(double, 11, D.Gsrc.data(), D.Gsrc.size());
    PUT(double, 12, D.Gout.data(), D.Gout.size());
    PUT(int, 13, D.tang.data(), D.tang.size());
    std::vector<double> eabo;
    eabo.insert(eabo.end(), D.EsA.begin(), D.EsA.end());
    eabo.insert(eabo.end(), D.EsB.begin(), D.EsB.end());
    eabo.insert(eabo.end(), D.Eout.begin(), D.Eout.end());
    PUT(double, 14, eabo.data(), eabo.size());
    PUT(double, 15, D.Kcsd.data(), D.Kcsd.size());
    PUT(double, 16, D.Bcsd.data(), D.Bcsd.size());
    PUT(double, 18, P->sigma_t, (size_t)ng * nmat);
    PUT(double, 19, P->sigma_s, (size_t)nmat * ng * ng * (P->ls + 1));
    if (D.csd) {
        PUT(double, 20, P->s_minus, (size_t)ng * nmat);
        PUT(double, 21, P->s_plus, (size_t)ng * nmat);
        PUT(double, 22, P->s_mom, (size_t)ng * nmat * P->order[3]);
        PUT(double, 24, P->e_width, ng);
    }
    if (P->t_mom) PUT(double, 23, P->t_mom, (size_t)ng * nmat);
    if (defs) {
        if ((r = place_sources(ctx, P, D, *defs, b, s, h)) != RB_OK) return r;
    } else if (P->volume_sources) {
        // the volume sources arrive in the reference's layout [ng, np, nm5, cells] (group
        // fastest): copied to the staging buffer and turned group-major on the device
        CK(cudaMemcpyAsync(stage, P->volume_sources, sizeof(double) * (size_t)ng * D.nphi, cudaMemcpyHostToDevice, s));
        dim3 blk(32, 8), grd((unsigned)((D.nphi + 31) / 32), (unsigned)((ng + 31) / 32));
        rb::from_reference_layout<<<grd, blk, 0, s>>>(stage, const_cast<double *>(h.vol), ng, D.nphi);
        CK(cudaGetLastError());
    }
    PUT(float, 52, D.tc_m2d.data(), D.tc_m2d.size());
    PUT(float, 53, D.tc_d2m.data(), D.tc_d2m.size());
    for (int f = 0; f < 2 * P->ndims; f++)
        if (P->surface_sources[f] && !defs)
            PUT(double, 26 + f, P->surface_sources[f], (size_t)ng * P->np_source * face_cells(P->ndims, D.ns, f / 2));
#undef PUT
    *dptr = DP(DevProblem, 0);
#undef DP
    CK(cudaMemcpyAsync(*dptr, &h, sizeof(DevProblem), cudaMemcpyHostToDevice, s));
    return RB_OK;
}

// The in-plane axes of a face (increasing order; -1 where the geometry has fewer axes).
void face_axes(int ndims, int face, int &a, int &b) {
    const int ax = face / 2;
    int k = 0, o[2] = {-1, -1};
    for (int d = 0; d < ndims; d++)
        if (d != ax) o[k++] = d;
    a = o[0];
    b = o[1];
}

// Copies the definitions into the block and builds the volume and surface sources from them.
int place_sources(rb_context *ctx, const rb_sn_problem *P, const Derived &D, const SourceDefs &S, char *b,
                  cudaStream_t s, const DevProblem &h) {
    const rb_source_set *src = S.src;
    const int ndims = P->ndims, ng = P->ng, nps = P->np_source;
    double *pos = reinterpret_cast<double *>(b + S.off_pos);
    const long long na = D.ns[0], nb = D.ns[1], nc = D.ns[2];
    CK(cudaMemcpyAsync(pos, src->position[0], sizeof(double) * na, cudaMemcpyHostToDevice, s));
    if (ndims >= 2) CK(cudaMemcpyAsync(pos + na, src->position[1], sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    if (ndims >= 3) CK(cudaMemcpyAsync(pos + na + nb, src->position[2], sizeof(double) * nc, cudaMemcpyHostToDevice, s));
    const int threads = 256;
    auto blocks = [&](long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 4096)); };
    if (h.vol) {
        auto *boxes = reinterpret_cast<rb_volume_box *>(b + S.off_box);
        CK(cudaMemcpyAsync(boxes, src->volume, sizeof(rb_volume_box) * src->nvolume, cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(const_cast<double *>(h.vol), 0, sizeof(double) * (size_t)ng * D.nphi, s));
        rb::assemble_volume<<<blocks(D.ncell), threads, 0, s>>>(const_cast<double *>(h.vol), D.nphi,
                                                                 (long long)P->np * D.M.nm, D.ns[0], D.ns[1], D.ns[2],
                                                                 ndims, pos, boxes, src->nvolume);
        CK(cudaGetLastError());
    }
    if (src->nsurface > 0) {
        std::vector<rb::DevBeam> beams(src->nsurface);
        std::vector<double> basis((size_t)src->nsurface * nps);
        for (int k = 0; k < src->nsurface; k++) {
            const rb_surface_beam &B = src->surface[k];
            rb::DevBeam &d = beams[k];
            d.group = B.energy_group - 1;
            d.face = B.face;
            d.intensity = B.intensity;
            for (int a = 0; a < 3; a++) { d.dir[a] = B.direction[a]; d.lo[a] = B.lo[a]; d.hi[a] = B.hi[a]; }
            for (int p = 0; p < nps; p++) basis[(size_t)k * nps + p] = B.basis[p];
        }
        auto *dbeams = reinterpret_cast<rb::DevBeam *>(b + S.off_beam);
        auto *dbasis = reinterpret_cast<double *>(b + S.off_basis);
        CK(cudaMemcpyAsync(dbeams, beams.data(), sizeof(rb::DevBeam) * beams.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dbasis, basis.data(), sizeof(double) * basis.size(), cudaMemcpyHostToDevice, s));
        const double *widths[3] = {h.dx, h.dy, h.dz};
        const long long off_axis[3] = {0, na, na + nb};
        for (int f = 0; f < 2 * ndims; f++) {
            if (!h.surf[f]) continue;
            int a, c;
            face_axes(ndims, f, a, c);
            const int la = a >= 0 ? D.ns[a] : 1, lc = c >= 0 ? D.ns[c] : 1;
            CK(cudaMemsetAsync(const_cast<double *>(h.surf[f]), 0, sizeof(double) * (size_t)ng * nps * la * lc, s));
            rb::assemble_surface<<<blocks((long long)la * lc), threads, 0, s>>>(
                const_cast<double *>(h.surf[f]), ng, nps, ndims, f, la, lc, a >= 0 ? pos + off_axis[a] : pos,
                c >= 0 ? pos + off_axis[c] : pos, a >= 0 ? widths[a] : h.dx, c >= 0 ? widths[c] : h.dx,
                a >= 0 ? a : 0, c >= 0 ? c : 0, dbeams, dbasis, src->nsurface);
            CK(cudaGetLastError());
        }
    }
    return RB_OK;
}

// Checks the definitions against the problem and writes each source's normalization factor:
// volume_source.jl:42-110 (Σ intensity · voxel volume over the voxels inside, x outermost) and
// surface_source.jl:89 (1D: the intensity), :158-187 (2D), :216-275 (3D: Σ intensity · face-cell
// area over the face cells inside, the first in-plane axis outermost).
int check_sources(rb_context *ctx, const rb_sn_problem *P, const rb_source_set *src, double *norms) {
    if (P->volume_sources) return fail(ctx, RB_ERR_INVALID, "volume_sources must be NULL with source definitions");
    for (int f = 0; f < 6; f++)
        if (P->surface_sources[f]) return fail(ctx, RB_ERR_INVALID, "surface_sources must be NULL with source definitions");
    if (src->nvolume < 0 || src->nsurface < 0 || (src->nvolume > 0 && !src->volume) || (src->nsurface > 0 && !src->surface))
        return fail(ctx, RB_ERR_INVALID, "bad source counts or NULL source arrays");
    const int ndims = P->ndims;
    const int n[3] = {P->nx, ndims >= 2 ? P->ny : 1, ndims >= 3 ? P->nz : 1};
    const double *w[3] = {P->dx, P->dy, P->dz};
    for (int a = 0; a < ndims; a++)
        if (!src->position[a]) return fail(ctx, RB_ERR_INVALID, "voxel positions of axis %d are NULL", a);
    if (src->nsurface > 0 && (P->np_source < 1 || P->np_source > P->np_surf))
        return fail(ctx, RB_ERR_INVALID, "np_source %d out of [1, np_surf=%d] with surface beams", P->np_source, P->np_surf);
    for (int k = 0; k < src->nvolume; k++) {
        const rb_volume_box &B = src->volume[k];
        if (B.energy_group < 1 || B.energy_group > P->ng)
            return fail(ctx, RB_ERR_INVALID, "volume source %d: energy group %d out of [1, %d]", k, B.energy_group, P->ng);
        double norm = 0.0;
        for (int ix = 0; ix < n[0]; ix++) {
            const double x = src->position[0][ix];
            if (!(B.lo[0] <= x && B.hi[0] >= x)) continue;
            for (int iy = 0; iy < n[1]; iy++) {
                if (ndims >= 2) { const double y = src->position[1][iy]; if (!(B.lo[1] <= y && B.hi[1] >= y)) continue; }
                for (int iz = 0; iz < n[2]; iz++) {
                    if (ndims >= 3) { const double z = src->position[2][iz]; if (!(B.lo[2] <= z && B.hi[2] >= z)) continue; }
                    if (ndims == 1) norm = norm + B.intensity * w[0][ix];
                    else if (ndims == 2) norm = norm + B.intensity * w[0][ix] * w[1][iy];
                    else norm = norm + B.intensity * w[0][ix] * w[1][iy] * w[2][iz];
                }
            }
        }
        if (norms) norms[k] = norm;
    }
    for (int k = 0; k < src->nsurface; k++) {
        const rb_surface_beam &B = src->surface[k];
        if (B.energy_group < 1 || B.energy_group > P->ng)
            return fail(ctx, RB_ERR_INVALID, "surface source %d: energy group %d out of [1, %d]", k, B.energy_group, P->ng);
        if (B.face < 0 || B.face >= 2 * ndims)
            return fail(ctx, RB_ERR_INVALID, "surface source %d: face %d out of [0, %d)", k, B.face, 2 * ndims);
        if (!B.basis) return fail(ctx, RB_ERR_INVALID, "surface source %d: NULL basis", k);
        double norm = 0.0;
        if (ndims == 1) {
            norm = B.intensity;
        } else {
            int a, c;
            face_axes(ndims, B.face, a, c);
            const int nc = c >= 0 ? n[c] : 1;
            for (int ia = 0; ia < n[a]; ia++) {
                const double pa = src->position[a][ia];
                if (pa < B.lo[a] || pa > B.hi[a]) continue;
                for (int ic = 0; ic < nc; ic++) {
                    if (c < 0) { norm += B.intensity * w[a][ia]; continue; }
                    const double pc = src->position[c][ic];
                    if (pc < B.lo[c] || pc > B.hi[c]) continue;
                    norm += B.intensity * w[a][ia] * w[c][ic];
                }
            }
        }
        if (norms) norms[src->nvolume + k] = norm;
    }
    return RB_OK;
}

const double k_built_on_device = 0.0;  // marks the source slots rb_upload_sources fills

int upload_impl(rb_context *ctx, const rb_sn_problem *P0, const rb_source_set *src, rb_handle *out, double *norms) {
    if (!ctx || !out) return fail(ctx, RB_ERR_INVALID, "null context or handle");
    if (!P0) return fail(ctx, RB_ERR_INVALID, "null problem");
    CK(cudaSetDevice(ctx->device));
    rb_sn_problem Pm = *P0;
    const rb_sn_problem *P = P0;
    if (src) {
        int st = check_sources(ctx, P0, src, norms);
        if (st) return st;
        if (src->nvolume > 0) Pm.volume_sources = &k_built_on_device;
        for (int k = 0; k < src->nsurface; k++) Pm.surface_sources[src->surface[k].face] = &k_built_on_device;
        P = &Pm;
    }
    Derived D;
    int st = validate_and_derive(ctx, P, D);
    if (st) return st;
    Layout L;
    size_t o[64];
    required(P, D, L, o);
    SourceDefs defs{};
    if (src) {
        defs.src = src;
        defs.off_pos = L.take<double>((size_t)D.ns[0] + D.ns[1] + D.ns[2]);
        defs.off_box = L.take<rb_volume_box>(src->nvolume);
        defs.off_beam = L.take<rb::DevBeam>(src->nsurface);
        defs.off_basis = L.take<double>((size_t)src->nsurface * P->np_source);
    }
    if (ctx->used + L.off > ctx->budget)
        return fail(ctx, RB_ERR_BUDGET, "problem needs %zu bytes, %llu of %llu budget bytes in use", L.off,
                    (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
    if (P->volume_sources && !src) {  // staging for the volume sources' layout change
        const size_t need = (size_t)P->ng * D.nphi;
        if (need > ctx->stage_cap) {
            if (ctx->d_stage) cudaFree(ctx->d_stage);
            ctx->d_stage = nullptr;
            ctx->stage_cap = 0;
            CK(cudaMalloc(&ctx->d_stage, need * sizeof(double)));
            ctx->stage_cap = need;
        }
    }
    auto rec = std::make_unique<ProblemRec>();
    cudaStream_t s = ctx->stream;
    // stream-ordered allocation from the context's pool: unlike cudaMalloc / cudaFree it does not
    // wait for kernels running on other streams, so an upload overlaps a solve in flight and a
    // release does not stall the requests still running
    CK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&rec->block), L.off, ctx->pool, s));
    rec->bytes = L.off;
    DevProblem &h = rec->h;
    st = place_problem(ctx, P, D, o, rec->block, s, h, &rec->d, ctx->d_stage, src ? &defs : nullptr);
    if (st) { cudaStreamSynchronize(s); cudaFreeAsync(rec->block, s); cudaStreamSynchronize(s); return st; }
    rec->own_list = reinterpret_cast<DevProblem **>(rec->block + o[50]);
    rec->own_queue = reinterpret_cast<int *>(rec->block + o[51]);
    CK(cudaMemcpyAsync(rec->own_list, &rec->d, sizeof(DevProblem *), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    rec->ng = P->ng; rec->np = P->np; rec->nm5 = D.M.nm; rec->csd = D.csd; rec->ncell = D.ncell; rec->nphi = D.nphi;
    ctx->used += L.off;
    rb_handle hd = ctx->next_handle++;
    ctx->probs[hd] = std::move(rec);
    *out = hd;
    return RB_OK;
}

}  // namespace

// =============================================================================================
// ABI
// =============================================================================================
extern "C" {

const char *rb_version(void) { return "radiant_b200 0.1 (sm_100a)"; }

int32_t rb_create(int32_t device, uint64_t hbm_budget_bytes, rb_context **out) {
    if (!out) return fail(nullptr, RB_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(nullptr, RB_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(nullptr, RB_ERR_INVALID, "device %d out of range", device);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, RB_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    auto *c = new rb_context();
    c->device = device;
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)(fr * 0.9);
    if (const char *cs = getenv("RB_CLUSTER_SIZE")) c->cluster = atoi(cs);
    if (const char *mt = getenv("RB_MD_TEAM")) c->md_cluster = strcmp(mt, "cluster") == 0;
    if (const char *lo = getenv("RB_LOCAL1D")) c->local1d = atoi(lo) != 0;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return fail(nullptr, RB_ERR_CUDA, "stream: %s", cudaGetErrorString(e)); }
    // problem blocks come from the context's own stream-ordered pool: it keeps what is freed for
    // the next upload instead of unmapping it at every synchronisation, and gives everything back
    // when the context is destroyed (the device's default pool, which other code in the process
    // may use, is left as it is)
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&c->pool, &props);
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return fail(nullptr, RB_ERR_CUDA, "memory pool: %s", cudaGetErrorString(e));
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    *out = c;
    return RB_OK;
}

int32_t rb_destroy(rb_context *ctx) {
    if (!ctx) return RB_ERR_INVALID;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    for (auto &kv : ctx->probs) {
        cudaFreeAsync(kv.second->block, ctx->stream);
        if (kv.second->solve_done) cudaEventDestroy(kv.second->solve_done);
    }
    for (char *p : ctx->small_all) cudaFreeHost(p);
    ctx->probs.clear();
    cudaStreamSynchronize(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->d_list) cudaFree(ctx->d_list);
    if (ctx->d_queue) cudaFree(ctx->d_queue);
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    if (ctx->d_gpart) cudaFree(ctx->d_gpart);
    for (auto ss : ctx->serve_streams) cudaStreamDestroy(ss);
    if (ctx->d_dstage) cudaFree(ctx->d_dstage);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->dl_ready) cudaEventDestroy(ctx->dl_ready);
    if (ctx->dl_done) cudaEventDestroy(ctx->dl_done);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return RB_OK;
}

int32_t rb_last_error(const rb_context *ctx, char *buf, uint64_t len) {
    if (!buf || len == 0) return RB_ERR_INVALID;
    const std::string &s = ctx ? ctx->err : g_create_error;
    size_t n = s.size() < len - 1 ? s.size() : (size_t)(len - 1);
    memcpy(buf, s.data(), n);
    buf[n] = 0;
    return RB_OK;
}

int32_t rb_required_bytes(const rb_sn_problem *prob, uint64_t *bytes) {
    Derived D;
    int st = validate_and_derive(nullptr, prob, D);
    if (st) return st;
    Layout L;
    size_t offs[64];
    required(prob, D, L, offs);
    if (bytes) *bytes = L.off;
    return RB_OK;
}

int32_t rb_upload(rb_context *ctx, const rb_sn_problem *P, rb_handle *out) {
    return upload_impl(ctx, P, nullptr, out, nullptr);
}

int32_t rb_upload_sources(rb_context *ctx, const rb_sn_problem *P, const rb_source_set *src, rb_handle *out,
                          double *norms) {
    if (!src) return fail(ctx, RB_ERR_INVALID, "null source set");
    return upload_impl(ctx, P, src, out, norms);
}

int32_t rb_solve(rb_context *ctx, rb_handle hd, void *stream) {
    return rb_solve_batch(ctx, &hd, 1, stream);
}

int32_t rb_solve_batch(rb_context *ctx, const rb_handle *hs, int32_t n, void *stream) {
    if (!ctx || (!hs && n > 0) || n < 0) return fail(ctx, RB_ERR_INVALID, "bad arguments");
    CK(cudaSetDevice(ctx->device));
    std::vector<ProblemRec *> recs;
    for (int i = 0; i < n; i++) {
        ProblemRec *r = find(ctx, hs[i]);
        if (!r) return fail(ctx, RB_ERR_NOT_FOUND, "unknown problem handle %lld", (long long)hs[i]);
        recs.push_back(r);
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return launch(ctx, recs, s);
}

int32_t rb_download(rb_context *ctx, rb_handle hd, rb_sn_result *res) {
    if (!ctx || !res) return fail(ctx, RB_ERR_INVALID, "null context or result");
    CK(cudaSetDevice(ctx->device));
    ProblemRec *r = find(ctx, hd);
    if (!r) return fail(ctx, RB_ERR_NOT_FOUND, "unknown problem handle %lld", (long long)hd);
    if (!r->solved) return fail(ctx, RB_ERR_INVALID, "problem %lld was not solved", (long long)hd);
    cudaStream_t s = r->stream;
    const DevProblem &h = r->h;
    if (res->flux) {
        size_t need = (size_t)r->ng * r->nphi;
        if (need > ctx->stage_cap) {
            if (ctx->d_stage) cudaFree(ctx->d_stage);
            ctx->d_stage = nullptr;
            CK(cudaMalloc(&ctx->d_stage, need * sizeof(double)));
            ctx->stage_cap = need;
        }
        dim3 blk(32, 8), grd((unsigned)((r->nphi + 31) / 32), (unsigned)((r->ng + 31) / 32));
        rb::to_reference_layout<<<grd, blk, 0, s>>>(h.flux, ctx->d_stage, r->ng, r->nphi);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(res->flux, ctx->d_stage, need * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (res->flux_cutoff && r->csd)
        CK(cudaMemcpyAsync(res->flux_cutoff, h.cutoff, r->nphi * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res->rho) CK(cudaMemcpyAsync(res->rho, h.rho, r->ng * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res->group_resid) CK(cudaMemcpyAsync(res->group_resid, h.resid, r->ng * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res->group_iters) CK(cudaMemcpyAsync(res->group_iters, h.iters, r->ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (res->group_converged) CK(cudaMemcpyAsync(res->group_converged, h.conv, r->ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    long long passes = 0;
    int status = 0;
    CK(cudaMemcpyAsync(&passes, h.passes, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&status, h.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    res->passes = passes;
    if (status & RB_DEV_TIMEOUT) return fail(ctx, RB_ERR_TIMEOUT, "a device wait gave up");
    if (status & RB_DEV_BAD_TABLE) return fail(ctx, RB_ERR_INVALID, "singular cell system or bad table");
    return RB_OK;
}

int32_t rb_download_async(rb_context *ctx, rb_handle hd, rb_sn_result *res) {
    if (!ctx || !res) return fail(ctx, RB_ERR_INVALID, "null context or result");
    CK(cudaSetDevice(ctx->device));
    ProblemRec *r = find(ctx, hd);
    if (!r) return fail(ctx, RB_ERR_NOT_FOUND, "unknown problem handle %lld", (long long)hd);
    if (!r->solved) return fail(ctx, RB_ERR_INVALID, "problem %lld was not solved", (long long)hd);
    if (r->dl_pending) return fail(ctx, RB_ERR_INVALID, "problem %lld already has a download in flight", (long long)hd);
    if (!ctx->copy_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->dl_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->dl_done, cudaEventDisableTiming));
    }
    // one staging buffer per context: the copies of the previous download must be done with it
    if (ctx->dl_busy) CK(cudaEventSynchronize(ctx->dl_done));
    const size_t need = (size_t)r->ng * r->nphi;
    if (res->flux && need > ctx->dstage_cap) {
        if (ctx->d_dstage) cudaFree(ctx->d_dstage);
        ctx->d_dstage = nullptr;
        ctx->dstage_cap = 0;
        CK(cudaMalloc(&ctx->d_dstage, need * sizeof(double)));
        ctx->dstage_cap = need;
    }
    const size_t small = 16 + (size_t)r->ng * (8 + 8 + 4 + 4);
    if (!r->dl_small) {
        for (size_t i = 0; i < ctx->small_free.size(); i++)
            if (ctx->small_free[i].second >= small) {
                r->dl_small = ctx->small_free[i].first;
                r->dl_small_cap = ctx->small_free[i].second;
                ctx->small_free.erase(ctx->small_free.begin() + i);
                break;
            }
        if (!r->dl_small) {
            const size_t cap = std::max<size_t>(small, 4096);
            CK(cudaHostAlloc(reinterpret_cast<void **>(&r->dl_small), cap, cudaHostAllocPortable));
            ctx->small_all.push_back(r->dl_small);
            r->dl_small_cap = cap;
        }
    }
    char *sm = r->dl_small;
    double *s_rho = reinterpret_cast<double *>(sm + 16), *s_resid = s_rho + r->ng;
    int *s_iters = reinterpret_cast<int *>(s_resid + r->ng), *s_conv = s_iters + r->ng;
    cudaStream_t s = r->stream, c = ctx->copy_stream;
    const DevProblem &h = r->h;
    // the layout change runs on the solve's stream, right behind the solve (before whatever is
    // launched there next); the copies wait for it on the copy stream and overlap later work
    if (res->flux) {
        dim3 blk(32, 8), grd((unsigned)((r->nphi + 31) / 32), (unsigned)((r->ng + 31) / 32));
        rb::to_reference_layout<<<grd, blk, 0, s>>>(h.flux, ctx->d_dstage, r->ng, r->nphi);
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(ctx->dl_ready, s));
    CK(cudaStreamWaitEvent(c, ctx->dl_ready, 0));
    if (res->flux) CK(cudaMemcpyAsync(res->flux, ctx->d_dstage, need * sizeof(double), cudaMemcpyDeviceToHost, c));
    if (res->flux_cutoff && r->csd)
        CK(cudaMemcpyAsync(res->flux_cutoff, h.cutoff, r->nphi * sizeof(double), cudaMemcpyDeviceToHost, c));
    // the per-group record lands in the page-locked small buffer (a copy into pageable memory
    // would make this call wait for the flux copy queued before it); rb_download_wait hands it on
    CK(cudaMemcpyAsync(s_rho, h.rho, r->ng * sizeof(double), cudaMemcpyDeviceToHost, c));
    CK(cudaMemcpyAsync(s_resid, h.resid, r->ng * sizeof(double), cudaMemcpyDeviceToHost, c));
    CK(cudaMemcpyAsync(s_iters, h.iters, r->ng * sizeof(int), cudaMemcpyDeviceToHost, c));
    CK(cudaMemcpyAsync(s_conv, h.conv, r->ng * sizeof(int), cudaMemcpyDeviceToHost, c));
    memset(sm, 0, 16);
    CK(cudaMemcpyAsync(sm, h.passes, sizeof(long long), cudaMemcpyDeviceToHost, c));
    CK(cudaMemcpyAsync(sm + 8, h.status, sizeof(int), cudaMemcpyDeviceToHost, c));
    CK(cudaEventRecord(ctx->dl_done, c));
    ctx->dl_busy = true;
    r->dl_pending = true;
    r->dl_res = res;
    return RB_OK;
}

int32_t rb_download_wait(rb_context *ctx, rb_handle hd) {
    if (!ctx) return RB_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    ProblemRec *r = find(ctx, hd);
    if (!r) return fail(ctx, RB_ERR_NOT_FOUND, "unknown problem handle %lld", (long long)hd);
    if (!r->dl_pending) return fail(ctx, RB_ERR_INVALID, "problem %lld has no download in flight", (long long)hd);
    // the copy stream runs in order: the last download's event covers every earlier one
    CK(cudaEventSynchronize(ctx->dl_done));
    r->dl_pending = false;
    const char *sm = r->dl_small;
    const double *s_rho = reinterpret_cast<const double *>(sm + 16), *s_resid = s_rho + r->ng;
    const int *s_iters = reinterpret_cast<const int *>(s_resid + r->ng), *s_conv = s_iters + r->ng;
    rb_sn_result *res = r->dl_res;
    if (res->rho) memcpy(res->rho, s_rho, r->ng * sizeof(double));
    if (res->group_resid) memcpy(res->group_resid, s_resid, r->ng * sizeof(double));
    if (res->group_iters) memcpy(res->group_iters, s_iters, r->ng * sizeof(int));
    if (res->group_converged) memcpy(res->group_converged, s_conv, r->ng * sizeof(int));
    long long passes = 0;
    int status = 0;
    memcpy(&passes, sm, sizeof(long long));
    memcpy(&status, sm + 8, sizeof(int));
    res->passes = passes;
    if (status & RB_DEV_TIMEOUT) return fail(ctx, RB_ERR_TIMEOUT, "a device wait gave up");
    if (status & RB_DEV_BAD_TABLE) return fail(ctx, RB_ERR_INVALID, "singular cell system or bad table");
    return RB_OK;
}

int32_t rb_release(rb_context *ctx, rb_handle hd) {
    if (!ctx) return RB_ERR_INVALID;
    auto it = ctx->probs.find(hd);
    if (it == ctx->probs.end()) return fail(ctx, RB_ERR_NOT_FOUND, "unknown problem handle %lld", (long long)hd);
    // wait for this problem's own work only (later launches on the same stream may still run)
    if (it->second->done) cudaEventSynchronize(it->second->done);
    else if (it->second->solve_done) cudaEventSynchronize(it->second->solve_done);
    else if (it->second->stream) cudaStreamSynchronize(it->second->stream);
    if (it->second->solve_done) cudaEventDestroy(it->second->solve_done);
    if (it->second->dl_pending && ctx->dl_done) cudaEventSynchronize(ctx->dl_done);
    if (it->second->dl_small) ctx->small_free.push_back({it->second->dl_small, it->second->dl_small_cap});
    // the problem's stream is idle (synchronised above): the block goes back to the pool in the
    // context stream's order, without waiting for other streams' work
    cudaFreeAsync(it->second->block, ctx->stream);
    ctx->used -= it->second->bytes;
    ctx->probs.erase(it);
    return RB_OK;
}

int32_t rb_host_alloc(uint64_t bytes, void **out) {
    if (!out || bytes == 0) return fail(nullptr, RB_ERR_INVALID, "null output or zero size");
    *out = nullptr;
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        *out = nullptr;
        return fail(nullptr, RB_ERR_CUDA, "cudaHostAlloc(%llu): %s", (unsigned long long)bytes, cudaGetErrorString(e));
    }
    return RB_OK;
}

int32_t rb_host_free(void *p) {
    if (!p) return RB_OK;
    cudaError_t e = cudaFreeHost(p);
    return e == cudaSuccess ? RB_OK : fail(nullptr, RB_ERR_CUDA, "cudaFreeHost: %s", cudaGetErrorString(e));
}

int32_t rb_host_register(void *p, uint64_t bytes) {
    if (!p || bytes == 0) return fail(nullptr, RB_ERR_INVALID, "null pointer or zero size");
    cudaError_t e = cudaHostRegister(p, bytes, cudaHostRegisterPortable);
    return e == cudaSuccess ? RB_OK : fail(nullptr, RB_ERR_CUDA, "cudaHostRegister: %s", cudaGetErrorString(e));
}

int32_t rb_host_unregister(void *p) {
    if (!p) return fail(nullptr, RB_ERR_INVALID, "null pointer");
    cudaError_t e = cudaHostUnregister(p);
    return e == cudaSuccess ? RB_OK : fail(nullptr, RB_ERR_CUDA, "cudaHostUnregister: %s", cudaGetErrorString(e));
}

int32_t rb_compute_flux(int32_t device, const rb_sn_problem *prob, rb_sn_result *res) {
    rb_context *ctx = nullptr;
    int st = rb_create(device, 0, &ctx);
    if (st) return st;
    rb_handle h = 0;
    st = rb_upload(ctx, prob, &h);
    if (!st) st = rb_solve(ctx, h, nullptr);
    if (!st) st = rb_download(ctx, h, res);
    if (st) g_create_error = ctx->err;
    rb_destroy(ctx);
    return st;
}

int32_t rb_submit(rb_context *ctx, const rb_sn_problem *prob, rb_handle *out) {
    // Continuous batching: a request is admitted when its device state fits the remaining HBM
    // budget (RB_ERR_BUDGET otherwise, nothing allocated); an admitted request is uploaded and
    // launched at once on its own stream from a pool, as one cluster team, so it runs beside the
    // requests already on the device and its results never depend on them.
    if (!ctx || !prob || !out) return fail(ctx, RB_ERR_INVALID, "null argument");
    CK(cudaSetDevice(ctx->device));
    uint64_t need = 0;
    int st = rb_required_bytes(prob, &need);
    if (st) { char buf[512]; rb_last_error(nullptr, buf, sizeof(buf)); return fail(ctx, st, "%s", buf); }
    if (ctx->used + need > ctx->budget)
        return fail(ctx, RB_ERR_BUDGET, "request needs %llu bytes; %llu of %llu budget bytes in use",
                    (unsigned long long)need, (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
    if (ctx->serve_streams.empty()) {
        for (int i = 0; i < 32; i++) {
            cudaStream_t ss;
            CK(cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking));
            ctx->serve_streams.push_back(ss);
        }
    }
    cudaStream_t s = ctx->serve_streams[ctx->next_stream++ % ctx->serve_streams.size()];
    cudaStream_t saved = ctx->stream;
    ctx->stream = s;  // upload on the request's stream
    st = rb_upload(ctx, prob, out);
    ctx->stream = saved;
    if (st) return st;
    ProblemRec *r = find(ctx, *out);
    CK(cudaMemsetAsync(r->own_queue, 0, sizeof(int), s));
    CK(cudaMemsetAsync(r->h.status, 0, sizeof(int), s));
    int cluster = ctx->cluster > 0 ? ctx->cluster : (r->h.ndims > 1 ? 16 : (r->h.nd >= 16 ? 4 : 2));
    st = launch_solve(ctx, r->own_list, 1, r->own_queue, ctx->nsm, cluster, s, {&r->h},
                      ctx->cluster > 0 ? LAUNCH_FIXED : LAUNCH_SERVE);
    if (st) return st;
    CK(cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming));
    CK(cudaEventRecord(r->done, s));
    r->stream = s;
    r->solved = true;
    return RB_OK;
}

int32_t rb_poll(rb_context *ctx, rb_handle hd, rb_sn_result *res) {
    if (!ctx) return RB_ERR_INVALID;
    ProblemRec *r = find(ctx, hd);
    if (!r) return fail(ctx, RB_ERR_NOT_FOUND, "unknown request %lld", (long long)hd);
    cudaError_t q = r->done ? cudaEventQuery(r->done) : cudaStreamQuery(r->stream);
    if (q == cudaErrorNotReady) return RB_ERR_NOT_READY;
    if (q != cudaSuccess) return fail(ctx, RB_ERR_CUDA, "request %lld: %s", (long long)hd, cudaGetErrorString(q));
    int st = rb_download(ctx, hd, res);
    if (r->done) cudaEventDestroy(r->done);
    r->done = nullptr;
    rb_release(ctx, hd);
    return st;
}

int32_t rb_energy_deposition(int32_t ng, int32_t np, int32_t nm5, int64_t ncell, int32_t nmat,
                             const int32_t *mat, const double *flux, const double *flux_cutoff,
                             const double *sigma_e, const double *density, double norm, double *dep) {
    // energy_deposition.jl:58-76: a reduction over groups per voxel; small, done on the host
    // from the downloaded flux (it is outside the transport solve).
    if (!mat || !flux || !sigma_e || !density || !dep) return fail(nullptr, RB_ERR_INVALID, "null argument");
    for (int64_t c = 0; c < ncell; c++) {
        int m = mat[c] - 1;
        if (m < 0 || m >= nmat) return fail(nullptr, RB_ERR_INVALID, "mat[%lld] out of range", (long long)c);
        double d = 0.0;
        for (int g = 0; g < ng; g++) d += sigma_e[g + (int64_t)(ng + 1) * m] * flux[g + (int64_t)ng * ((int64_t)np * nm5 * c)];
        if (flux_cutoff) d += sigma_e[ng + (int64_t)(ng + 1) * m] * flux_cutoff[(int64_t)np * nm5 * c];
        dep[c] = d / (density[m] * norm);
    }
    return RB_OK;
}

int32_t rb_set_launch_rules(rb_context *ctx, const rb_launch_rule *rules, int32_t n) {
    if (!ctx || n < 0 || (n > 0 && !rules)) return fail(ctx, RB_ERR_INVALID, "bad launch rules");
    for (int i = 0; i < n; i++)
        if (rules[i].ndims < 1 || rules[i].ndims > 3 || rules[i].cluster < 1 || rules[i].cluster > RB_MAXCLUSTER ||
            (rules[i].cluster & (rules[i].cluster - 1)) != 0)
            return fail(ctx, RB_ERR_INVALID, "launch rule %d: dimension 1-3 and a power-of-two team of 1-%d CTAs",
                        i, RB_MAXCLUSTER);
    ctx->rules.assign(rules, rules + n);
    return RB_OK;
}

int32_t rb_deposition(rb_context *ctx, int32_t npart, const rb_handle *handles, const double *const *sigma_dep,
                      const double *density, double norm, double *dep) {
    // energy_deposition.jl:24-87 / charge_deposition.jl:26-89 over resident, solved problems: a
    // device reduction over groups per voxel, summed over the particles in the order given; only
    // the voxel array comes back
    if (!ctx || npart < 1 || !handles || !sigma_dep || !density || !dep)
        return fail(ctx, RB_ERR_INVALID, "null argument");
    CK(cudaSetDevice(ctx->device));
    std::vector<ProblemRec *> recs;
    size_t nsig = 0;
    for (int i = 0; i < npart; i++) {
        ProblemRec *r = find(ctx, handles[i]);
        if (!r) return fail(ctx, RB_ERR_NOT_FOUND, "unknown problem handle %lld", (long long)handles[i]);
        if (!r->solved) return fail(ctx, RB_ERR_INVALID, "problem %lld was not solved", (long long)handles[i]);
        if (!sigma_dep[i]) return fail(ctx, RB_ERR_INVALID, "no deposition cross sections for particle %d", i);
        if (i > 0 && (r->ncell != recs[0]->ncell || r->h.nmat != recs[0]->h.nmat))
            return fail(ctx, RB_ERR_INVALID, "particle %d is not on the geometry of particle 1", i);
        recs.push_back(r);
        nsig += (size_t)(r->ng + 1) * r->h.nmat;
    }
    const int nmat = recs[0]->h.nmat;
    const long long ncell = recs[0]->ncell;
    for (auto *r : recs)
        if (r->stream) CK(cudaStreamSynchronize(r->stream));
    cudaStream_t s = ctx->stream;
    double *buf = nullptr;
    CK(cudaMalloc(&buf, (nsig + nmat + ncell) * sizeof(double)));
    double *dsig = buf, *drho = buf + nsig, *ddep = drho + nmat;
    int st = RB_OK;
    auto run = [&]() -> int {
        CK(cudaMemcpyAsync(drho, density, nmat * sizeof(double), cudaMemcpyHostToDevice, s));
        size_t o = 0;
        for (int i = 0; i < npart; i++) {
            const ProblemRec *r = recs[i];
            const size_t n = (size_t)(r->ng + 1) * nmat;
            CK(cudaMemcpyAsync(dsig + o, sigma_dep[i], n * sizeof(double), cudaMemcpyHostToDevice, s));
            const int blocks = (int)std::min<long long>((ncell + 255) / 256, (long long)ctx->nsm * 8);
            rb::deposition_kernel<<<blocks, 256, 0, s>>>(r->h.flux, r->ng, r->nphi, (long long)r->np * r->nm5,
                                                         r->csd ? r->h.cutoff : nullptr, r->h.mat, dsig + o, drho,
                                                         norm, ncell, ddep, i > 0);
            CK(cudaGetLastError());
            o += n;
        }
        CK(cudaMemcpyAsync(dep, ddep, ncell * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return RB_OK;
    };
    st = run();
    cudaFree(buf);
    return st;
}

}  // extern "C"

// =============================================================================================
// Entry point that allocates no device memory
// =============================================================================================
// Some callers cannot call cudaMalloc: a host process whose device memory is owned by another
// allocator (a Julia CUDA.jl pool or a PyTorch caching allocator that has reserved the HBM)
// must not see cudaMalloc/cudaFree, which synchronise the whole device and can fail or
// fragment that pool mid-run. rb_compute_flux_static serves them: every byte of device memory
// it touches -- the problem's tables, its work buffers and the result staging -- lives in the
// file-scope array below, reserved once when the library is loaded and held by every GPU
// that loads it until the process exits.
#define RB_STATIC_SCRATCH_BYTES (16ull << 20)  // 16 MiB per device
static __device__ __align__(256) unsigned char rb_static_scratch[RB_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
char *g_static_scratch[kMaxDevices] = {nullptr};  // device address of rb_static_scratch, per device
std::mutex g_static_mu;

// Host code cannot use `rb_static_scratch` as a device address: look it up once per device,
// with that device current.
int static_scratch_address(int dev, char **out) {
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (dev < 0 || dev >= kMaxDevices) return fail(nullptr, RB_ERR_INVALID, "device %d out of range", dev);
    if (!g_static_scratch[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, rb_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(nullptr, RB_ERR_CUDA, "cudaGetSymbolAddress(rb_static_scratch): %s", cudaGetErrorString(e));
        g_static_scratch[dev] = static_cast<char *>(p);
    }
    *out = g_static_scratch[dev];
    return RB_OK;
}
}  // namespace

extern "C" int32_t rb_compute_flux_static(const rb_sn_problem *prob, rb_sn_result *res, void *stream) {
    rb_context *ctx = nullptr;  // errors go to rb_last_error(NULL, ...)
    if (!prob || !res) return fail(nullptr, RB_ERR_INVALID, "null problem or result");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    char *base = nullptr;
    int st = static_scratch_address(dev, &base);
    if (st) return st;
    Derived D;
    st = validate_and_derive(nullptr, prob, D);
    if (st) return st;
    Layout L;
    size_t o[64];
    required(prob, D, L, o);
    const size_t off_list = L.take<DevProblem *>(1);
    const size_t off_queue = L.take<int>(1);
    const size_t off_stage = L.take<double>((size_t)prob->ng * D.nphi);
    if (L.off > RB_STATIC_SCRATCH_BYTES)
        return fail(nullptr, RB_ERR_BUDGET, "problem needs %zu bytes of device memory; the static scratch of "
                    "rb_compute_flux_static holds %llu", L.off, (unsigned long long)RB_STATIC_SCRATCH_BYTES);
    cudaStream_t s = (cudaStream_t)stream;
    DevProblem h;
    DevProblem *d = nullptr;
    double *d_stage = reinterpret_cast<double *>(base + off_stage);
    st = place_problem(nullptr, prob, D, o, base, s, h, &d, d_stage);
    if (st) return st;
    DevProblem **d_list = reinterpret_cast<DevProblem **>(base + off_list);
    int *d_queue = reinterpret_cast<int *>(base + off_queue);
    // the array keeps the previous call's contents: zero the queue counter and status word
    CK(cudaMemcpyAsync(d_list, &d, sizeof(DevProblem *), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(d_queue, 0, sizeof(int), s));
    CK(cudaMemsetAsync(h.status, 0, sizeof(int), s));
    // one team of one CTA (one SM): the array holds no grid-team reduction slots, and the entry
    // point serves small problems
    st = launch_solve(nullptr, d_list, 1, d_queue, 1, 1, s, {&h}, LAUNCH_FIXED);
    if (st) return st;
    const int ng = prob->ng;
    if (res->flux) {
        dim3 blk(32, 8), grd((unsigned)((D.nphi + 31) / 32), (unsigned)((ng + 31) / 32));
        rb::to_reference_layout<<<grd, blk, 0, s>>>(h.flux, d_stage, ng, D.nphi);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(res->flux, d_stage, (size_t)ng * D.nphi * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (res->flux_cutoff && D.csd)
        CK(cudaMemcpyAsync(res->flux_cutoff, h.cutoff, D.nphi * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res->rho) CK(cudaMemcpyAsync(res->rho, h.rho, ng * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res->group_resid) CK(cudaMemcpyAsync(res->group_resid, h.resid, ng * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res->group_iters) CK(cudaMemcpyAsync(res->group_iters, h.iters, ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (res->group_converged) CK(cudaMemcpyAsync(res->group_converged, h.conv, ng * sizeof(int), cudaMemcpyDeviceToHost, s));
    long long passes = 0;
    int status = 0;
    CK(cudaMemcpyAsync(&passes, h.passes, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&status, h.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    res->passes = passes;
    if (status & RB_DEV_TIMEOUT) return fail(nullptr, RB_ERR_TIMEOUT, "a device wait gave up");
    if (status & RB_DEV_BAD_TABLE) return fail(nullptr, RB_ERR_INVALID, "singular cell system or bad table");
    return RB_OK;
}

// =============================================================================================
// Coupled particles: the generation loop of transport() on the device
// =============================================================================================
namespace {
struct CoupledPart {
    rb_handle h = 0;
    ProblemRec *r = nullptr;
    double *tot = nullptr, *tot_cut = nullptr, *pvol = nullptr;  // summed flux, summed cutoff, particle source
    unsigned long long *maxrel = nullptr;                          // ϵ of the last generation (double bits)
    DevProblem with_fixed{}, without_fixed{};                      // records of generation 1 / later ones
    long long passes = 0;
};
struct CoupledPair {
    double *sigma_s = nullptr, *transfer = nullptr;
    int *map = nullptr;
    int ls = 0;
};
}  // namespace

extern "C" int32_t rb_transport(int32_t device, int32_t npart, const rb_sn_problem *const *probs,
                                const rb_coupling *couplings, int32_t ngen_max, double eps_gen, int32_t conv_type,
                                const double *const *sigma_dep, const double *density, double norm,
                                rb_sn_result *const *results, double *deposition, int32_t *generations,
                                double *eps_final) {
    rb_context *ctx = nullptr;
    if (npart < 1 || !probs || !results) return fail(nullptr, RB_ERR_INVALID, "bad particle list");
    if (ngen_max < 1) return fail(nullptr, RB_ERR_INVALID, "ngen_max must be >= 1");
    if (conv_type < 0 || conv_type > 2) return fail(nullptr, RB_ERR_INVALID, "Unknown convergence type.");
    const bool use_dep = conv_type != 0 || deposition != nullptr;
    if (use_dep) {
        if (!sigma_dep || !density) return fail(nullptr, RB_ERR_INVALID, "deposition cross sections or densities missing");
        for (int i = 0; i < npart; i++)
            if (!sigma_dep[i]) return fail(nullptr, RB_ERR_INVALID, "no deposition cross sections for particle %d", i);
    }
    for (int i = 0; i < npart; i++) {
        const rb_sn_problem *a = probs[i], *b = probs[0];
        if (!a || !results[i]) return fail(nullptr, RB_ERR_INVALID, "null problem or result %d", i);
        if (a->ndims != b->ndims || a->nx != b->nx || (a->ndims > 1 && a->ny != b->ny) ||
            (a->ndims > 2 && a->nz != b->nz) || a->nmat != b->nmat)
            return fail(nullptr, RB_ERR_INVALID, "particle %d is not on the geometry of particle 1", i);
    }
    // the first particle with fixed sources leads the order (transport.jl:60-73)
    int i0 = -1;
    for (int i = 0; i < npart && i0 < 0; i++) {
        bool any = probs[i]->volume_sources != nullptr;
        for (int f = 0; f < 6; f++) any = any || probs[i]->surface_sources[f] != nullptr;
        if (any) i0 = i;
    }
    if (i0 < 0) return fail(nullptr, RB_ERR_INVALID, "No fixed sources are defined.");
    std::vector<int> order;
    for (int i = i0; i < npart; i++) order.push_back(i);
    for (int i = 0; i < i0; i++) order.push_back(i);
    int st = rb_create(device, 0, &ctx);
    if (st) return st;
    std::vector<CoupledPart> parts(npart);
    std::vector<CoupledPair> pairs((size_t)npart * npart);
    // deposition buffers (the energy- and charge-deposition criteria, and the summed deposition)
    std::vector<double *> dsig(npart, nullptr);
    double *drho = nullptr, *dep_cur = nullptr, *dep_prev = nullptr;
    unsigned long long *dmax = nullptr;
    auto cleanup = [&](int code) {
        cudaStreamSynchronize(ctx->stream);
        for (auto q : dsig) if (q) cudaFree(q);
        if (drho) cudaFree(drho);
        if (dep_cur) cudaFree(dep_cur);
        if (dep_prev) cudaFree(dep_prev);
        if (dmax) cudaFree(dmax);
        for (auto &p : parts) {
            if (p.tot) cudaFree(p.tot);
            if (p.tot_cut) cudaFree(p.tot_cut);
            if (p.pvol) cudaFree(p.pvol);
            if (p.maxrel) cudaFree(p.maxrel);
        }
        for (auto &q : pairs) {
            if (q.sigma_s) cudaFree(q.sigma_s);
            if (q.transfer) cudaFree(q.transfer);
            if (q.map) cudaFree(q.map);
        }
        if (code != RB_OK) g_create_error = ctx->err;  // the message outlives the context
        rb_destroy(ctx);
        return code;
    };
#define CKT(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return cleanup(fail(ctx, RB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_))); \
    } while (0)
    cudaStream_t s = ctx->stream;
    for (int i = 0; i < npart; i++) {
        CoupledPart &P = parts[i];
        st = rb_upload(ctx, probs[i], &P.h);
        if (st) return cleanup(st);
        P.r = find(ctx, P.h);
        const size_t n = (size_t)P.r->ng * P.r->nphi;
        CKT(cudaMalloc(&P.tot, n * sizeof(double)));
        CKT(cudaMalloc(&P.pvol, n * sizeof(double)));
        CKT(cudaMalloc(&P.maxrel, sizeof(unsigned long long)));
        CKT(cudaMemsetAsync(P.tot, 0, n * sizeof(double), s));
        CKT(cudaMemsetAsync(P.pvol, 0, n * sizeof(double), s));
        if (P.r->csd) {
            CKT(cudaMalloc(&P.tot_cut, P.r->nphi * sizeof(double)));
            CKT(cudaMemsetAsync(P.tot_cut, 0, P.r->nphi * sizeof(double), s));
        }
        P.with_fixed = P.r->h;
        P.with_fixed.pvol = P.pvol;
        P.without_fixed = P.with_fixed;  // later generations: the particle source alone
        P.without_fixed.vol = nullptr;
        P.without_fixed.np_source = 0;
        for (int f = 0; f < 6; f++) P.without_fixed.surf[f] = nullptr;
    }
    for (int i = 0; i < npart; i++)
        for (int j = 0; j < npart; j++) {
            const rb_coupling *c = couplings ? &couplings[(size_t)i * npart + j] : nullptr;
            if (i == j || !c || !c->sigma_s) continue;
            const DevProblem &a = parts[i].r->h, &b = parts[j].r->h;
            if (!c->transfer || !c->moment_map || c->ls < 0)
                return cleanup(fail(ctx, RB_ERR_INVALID, "coupling %d->%d without transfer matrix or moment map", i, j));
            for (int k = 0; k < b.nm5; k++)
                if (c->moment_map[k] < 0 || c->moment_map[k] > a.nm5)
                    return cleanup(fail(ctx, RB_ERR_INVALID, "moment_map[%d] of coupling %d->%d out of range", k, i, j));
            for (int p = 0; p < a.np; p++)
                if (probs[i]->pl[p] > c->ls)
                    return cleanup(fail(ctx, RB_ERR_INVALID, "coupling %d->%d: ls below the incoming Legendre orders", i, j));
            const long long smem = 8LL * ((long long)a.ng * a.np + (long long)b.ng * a.np);
            if (smem > 200 * 1024)
                return cleanup(fail(ctx, RB_ERR_UNSUPPORTED, "coupling %d->%d: groups x moments too large (%lld B)", i, j, smem));
            CoupledPair &q = pairs[(size_t)i * npart + j];
            q.ls = c->ls;
            const size_t nss = (size_t)a.nmat * a.ng * b.ng * (c->ls + 1);
            CKT(cudaMalloc(&q.sigma_s, nss * sizeof(double)));
            CKT(cudaMalloc(&q.transfer, (size_t)b.np * a.np * sizeof(double)));
            CKT(cudaMalloc(&q.map, (size_t)b.nm5 * sizeof(int)));
            CKT(cudaMemcpyAsync(q.sigma_s, c->sigma_s, nss * sizeof(double), cudaMemcpyHostToDevice, s));
            CKT(cudaMemcpyAsync(q.transfer, c->transfer, (size_t)b.np * a.np * sizeof(double), cudaMemcpyHostToDevice, s));
            CKT(cudaMemcpyAsync(q.map, c->moment_map, (size_t)b.nm5 * sizeof(int), cudaMemcpyHostToDevice, s));
        }
    // deposition (the energy- and charge-deposition criteria, and the summed deposition out):
    // per-particle cross sections [ng+1, nmat], densities, this and the last generation's map
    const long long ncell = parts[0].r->ncell;
    const int nmat = parts[0].r->h.nmat;
    if (use_dep) {
        int e = RB_OK;
        for (int i = 0; i < npart && e == RB_OK; i++) {
            const size_t n = (size_t)(parts[i].r->ng + 1) * nmat;
            if (cudaMalloc(&dsig[i], n * sizeof(double)) != cudaSuccess ||
                cudaMemcpyAsync(dsig[i], sigma_dep[i], n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
                e = RB_ERR_CUDA;
        }
        if (e == RB_OK && (cudaMalloc(&drho, nmat * sizeof(double)) != cudaSuccess ||
                           cudaMalloc(&dep_cur, ncell * sizeof(double)) != cudaSuccess ||
                           cudaMalloc(&dep_prev, ncell * sizeof(double)) != cudaSuccess ||
                           cudaMalloc(&dmax, sizeof(unsigned long long)) != cudaSuccess ||
                           cudaMemcpyAsync(drho, density, nmat * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess))
            e = RB_ERR_CUDA;
        if (e != RB_OK) return cleanup(fail(ctx, RB_ERR_CUDA, "deposition buffers"));
    }
    // the summed deposition of the running totals into dep_cur, particles in the solve order (the
    // order the reference's Flux holds them in)
    auto deposit = [&]() -> int {
        const int blocks = (int)std::min<long long>((ncell + 255) / 256, (long long)ctx->nsm * 8);
        for (int p = 0; p < npart; p++) {
            const int i = order[p];
            const CoupledPart &P = parts[i];
            rb::deposition_kernel<<<blocks, 256, 0, s>>>(P.tot, P.r->ng, P.r->nphi, (long long)P.r->np * P.r->nm5,
                                                         P.r->csd ? P.tot_cut : nullptr, P.r->h.mat, dsig[i], drho,
                                                         norm, ncell, dep_cur, p > 0);
            if (cudaGetLastError() != cudaSuccess) return RB_ERR_CUDA;
        }
        return RB_OK;
    };
    CKT(cudaFuncSetAttribute(rb::particle_source_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CKT(cudaStreamSynchronize(s));
    double eps_last = NAN;
    int ngen = 0;
    for (int n = 1; n <= ngen_max; n++) {
        ngen = n;
        for (int p = 0; p < npart; p++) {
            const int i = order[p];
            CoupledPart &P = parts[i];
            const DevProblem &hv = n == 1 ? P.with_fixed : P.without_fixed;
            P.r->h = hv;
            CKT(cudaMemcpyAsync(P.r->d, &hv, sizeof(DevProblem), cudaMemcpyHostToDevice, s));
            std::vector<ProblemRec *> one{P.r};
            st = launch(ctx, one, s);
            if (st) return cleanup(st);
            // the solution of this generation into the particle's sum, with its change
            const long long nall = (long long)P.r->ng * P.r->nphi;
            CKT(cudaMemsetAsync(P.maxrel, 0, sizeof(unsigned long long), s));
            const int blocks = (int)std::min<long long>((nall + 255) / 256, (long long)ctx->nsm * 8);
            rb::accumulate_generation<<<blocks, 256, 0, s>>>(P.tot, hv.flux, nall, P.r->nphi, hv.np, hv.nm5, P.maxrel);
            CKT(cudaGetLastError());
            if (P.r->csd) {
                rb::accumulate_generation<<<blocks, 256, 0, s>>>(P.tot_cut, hv.cutoff, P.r->nphi, P.r->nphi, hv.np,
                                                                 hv.nm5, nullptr);
                CKT(cudaGetLastError());
            }
            long long ps = 0;
            int status = 0;
            CKT(cudaMemcpyAsync(&ps, hv.passes, sizeof(long long), cudaMemcpyDeviceToHost, s));
            CKT(cudaMemcpyAsync(&status, hv.status, sizeof(int), cudaMemcpyDeviceToHost, s));
            CKT(cudaStreamSynchronize(s));
            P.passes += ps;
            if (status & RB_DEV_TIMEOUT) return cleanup(fail(ctx, RB_ERR_TIMEOUT, "a device wait gave up"));
            if (status & RB_DEV_BAD_TABLE) return cleanup(fail(ctx, RB_ERR_INVALID, "singular cell system or bad table"));
            // the sources this solution produces (transport.jl:96-107)
            if (n == ngen_max && p == npart - 1) continue;
            for (int qq = 0; qq < npart; qq++) {
                const int j = order[qq];
                if (n == ngen_max && qq <= p) continue;
                if (i == j) {
                    CKT(cudaMemsetAsync(P.pvol, 0, (size_t)nall * sizeof(double), s));
                    continue;
                }
                const CoupledPair &q = pairs[(size_t)i * npart + j];
                if (!q.sigma_s) continue;
                const DevProblem &a = hv, &b = parts[j].with_fixed;
                const size_t smem = 8 * ((size_t)a.ng * a.np + (size_t)b.ng * a.np);
                dim3 grd((unsigned)a.ncell, (unsigned)b.nm5);
                rb::particle_source_kernel<<<grd, 256, smem, s>>>(hv.flux, a.ng, a.np, a.nm5, a.mat, a.nmat, q.sigma_s,
                                                                 q.ls, a.pl, q.transfer, q.map, parts[j].pvol, b.ng, b.np,
                                                                 b.nm5, a.ncell);
                CKT(cudaGetLastError());
            }
        }
        if (conv_type == 0 && n > 1) {  // the flux criterion (transport.jl:116-121)
            int px = 0;
            double emax = 0.0;
            for (int i = 0; i < npart; i++) {
                unsigned long long bits = 0;
                CKT(cudaMemcpyAsync(&bits, parts[i].maxrel, sizeof(bits), cudaMemcpyDeviceToHost, s));
                CKT(cudaStreamSynchronize(s));
                double e;
                memcpy(&e, &bits, sizeof(e));
                emax = std::max(emax, e);
                if (e < eps_gen) px++;
            }
            eps_last = emax;
            if (px == npart) break;
        }
        if (conv_type != 0) {  // energy / charge deposition criterion (transport.jl:122-133)
            const int e = deposit();
            if (e != RB_OK) return cleanup(fail(ctx, e, "deposition kernel"));
            if (n > 1) {
                unsigned long long bits = 0;
                CKT(cudaMemsetAsync(dmax, 0, sizeof(bits), s));
                const int blocks = (int)std::min<long long>((ncell + 255) / 256, (long long)ctx->nsm * 8);
                rb::max_rel_change<<<blocks, 256, 0, s>>>(dep_cur, dep_prev, ncell, dmax);
                CKT(cudaGetLastError());
                CKT(cudaMemcpyAsync(&bits, dmax, sizeof(bits), cudaMemcpyDeviceToHost, s));
                CKT(cudaStreamSynchronize(s));
                memcpy(&eps_last, &bits, sizeof(eps_last));
            }
            std::swap(dep_cur, dep_prev);  // dep_prev: the deposition of this generation's totals
            if (n > 1 && eps_last < eps_gen) break;
        }
    }
    if (deposition) {  // the summed deposition of the final totals
        if (conv_type != 0) std::swap(dep_cur, dep_prev);
        else {
            const int e = deposit();
            if (e != RB_OK) return cleanup(fail(ctx, e, "deposition kernel"));
        }
        CKT(cudaMemcpyAsync(deposition, dep_cur, ncell * sizeof(double), cudaMemcpyDeviceToHost, s));
        CKT(cudaStreamSynchronize(s));
    }
    // the summed solutions out, in the reference's layouts
    for (int i = 0; i < npart; i++) {
        CoupledPart &P = parts[i];
        rb_sn_result *res = results[i];
        const DevProblem &h = P.r->h;
        if (res->flux) {
            const size_t need = (size_t)P.r->ng * P.r->nphi;
            if (need > ctx->stage_cap) {
                if (ctx->d_stage) cudaFree(ctx->d_stage);
                ctx->d_stage = nullptr;
                ctx->stage_cap = 0;
                CKT(cudaMalloc(&ctx->d_stage, need * sizeof(double)));
                ctx->stage_cap = need;
            }
            dim3 blk(32, 8), grd((unsigned)((P.r->nphi + 31) / 32), (unsigned)((P.r->ng + 31) / 32));
            rb::to_reference_layout<<<grd, blk, 0, s>>>(P.tot, ctx->d_stage, P.r->ng, P.r->nphi);
            CKT(cudaGetLastError());
            CKT(cudaMemcpyAsync(res->flux, ctx->d_stage, need * sizeof(double), cudaMemcpyDeviceToHost, s));
            CKT(cudaStreamSynchronize(s));
        }
        if (res->flux_cutoff && P.r->csd)
            CKT(cudaMemcpyAsync(res->flux_cutoff, P.tot_cut, P.r->nphi * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (res->rho) CKT(cudaMemcpyAsync(res->rho, h.rho, P.r->ng * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (res->group_resid) CKT(cudaMemcpyAsync(res->group_resid, h.resid, P.r->ng * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (res->group_iters) CKT(cudaMemcpyAsync(res->group_iters, h.iters, P.r->ng * sizeof(int), cudaMemcpyDeviceToHost, s));
        if (res->group_converged)
            CKT(cudaMemcpyAsync(res->group_converged, h.conv, P.r->ng * sizeof(int), cudaMemcpyDeviceToHost, s));
        CKT(cudaStreamSynchronize(s));
        res->passes = P.passes;
    }
#undef CKT
    if (generations) *generations = ngen;
    if (eps_final) *eps_final = eps_last;
    return cleanup(RB_OK);
}
