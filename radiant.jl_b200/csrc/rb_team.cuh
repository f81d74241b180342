// rb_team.cuh -- the team that owns one problem: one thread-block cluster.
//
// Every phase of a transport pass and every vector operation of the in-group accelerators is
// spread over all threads of the cluster; team barriers are hardware cluster barriers.
// Reductions are deterministic and give the same bits in every thread of every CTA: each warp
// reduces by xor butterfly (commutative pairs, identical in all lanes), each CTA sums its warps
// in a fixed order and stores that partial into its own slot in every CTA of the cluster
// (distributed shared memory), and after one cluster barrier every thread adds the slots in
// rank order from its own shared memory. Slot sets alternate between two buffers, so a
// reduction costs one cluster barrier. All threads run the same control flow, which the
// identical reduction bits guarantee, so no CTA can leave a barrier sequence early.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

namespace rb {
namespace cg = cooperative_groups;

struct TeamShared {
    double part[2][16][4];  // partial sums of each CTA, double-buffered, up to 4 values per reduction
    double warp[32][4];
    int idx;            // problem index broadcast by the cluster leader
};

struct ClusterTeam {
    TeamShared *sh;
    unsigned crank;   // CTA rank in the cluster
    unsigned ncta;    // CTAs in the cluster
    int phase;        // reduction counter (selects the slot)

    __device__ void init(TeamShared *s) {
        sh = s;
        cg::cluster_group cl = cg::this_cluster();
        crank = cl.block_rank();
        ncta = cl.num_blocks();
        phase = 0;
    }
    __device__ __forceinline__ int rank() const { return (int)(crank * blockDim.x + threadIdx.x); }
    __device__ __forceinline__ int size() const { return (int)(ncta * blockDim.x); }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }  // one per CTA
    __device__ __forceinline__ void sync() const { cg::this_cluster().sync(); }

    // Sum of K values over the team (K <= 4); every thread gets identical bits.
    template <int K>
    __device__ void sumk(double (&v)[K]) {
#pragma unroll
        for (int k = 0; k < K; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int k = 0; k < K; k++) sh->warp[w][k] = v[k];
        __syncthreads();
        const int slot = phase & 1;
        phase++;
        cg::cluster_group cl = cg::this_cluster();
        if (threadIdx.x < ncta) {  // thread q stores this CTA's partial into CTA q
            double s[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                s[k] = 0.0;
                for (int i = 0; i < nw; i++) s[k] += sh->warp[i][k];
            }
            double *dst = cl.map_shared_rank(&sh->part[slot][crank][0], threadIdx.x);
#pragma unroll
            for (int k = 0; k < K; k++) dst[k] = s[k];
        }
        cl.sync();
#pragma unroll
        for (int k = 0; k < K; k++) v[k] = 0.0;
        for (unsigned r = 0; r < ncta; r++)
#pragma unroll
            for (int k = 0; k < K; k++) v[k] += sh->part[slot][r][k];
    }
    __device__ double sum(double v) {
        double a[1] = {v};
        sumk<1>(a);
        return a[0];
    }
    __device__ int any(int flag) { return sum(flag ? 1.0 : 0.0) > 0.0; }
    // Index handed out by the cluster leader (CTA 0, thread 0) to the whole cluster.
    __device__ int broadcast_from_leader(int v) {
        cg::cluster_group cl = cg::this_cluster();
        if (crank == 0 && threadIdx.x == 0) sh->idx = v;
        cl.sync();
        const int r = *cl.map_shared_rank(&sh->idx, 0);
        cl.sync();
        return r;
    }
};


// A team of every CTA of a cooperative launch (one problem on the whole GPU, for 2D and 3D
// solves). Barriers are grid barriers; a reduction writes one partial per CTA into a
// double-buffered global slot, and after the barrier every CTA adds all partials in CTA order,
// so every thread of the grid sees the same bits.
struct GridTeam {
    TeamShared *sh;
    double *gpart;    // [2][ncta][4] partial sums
    unsigned crank;
    unsigned ncta;
    int phase;

    __device__ void init(TeamShared *s, double *gp) {
        sh = s;
        gpart = gp;
        crank = blockIdx.x;
        ncta = gridDim.x;
        phase = 0;
    }
    __device__ __forceinline__ int rank() const { return (int)(crank * blockDim.x + threadIdx.x); }
    __device__ __forceinline__ int size() const { return (int)(ncta * blockDim.x); }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
    __device__ __forceinline__ void sync() const { cg::this_grid().sync(); }

    template <int K>
    __device__ void sumk(double (&v)[K]) {
#pragma unroll
        for (int k = 0; k < K; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int k = 0; k < K; k++) sh->warp[w][k] = v[k];
        __syncthreads();
        const int slot = phase & 1;
        phase++;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < K; k++) {
                double s = 0.0;
                for (int i = 0; i < nw; i++) s += sh->warp[i][k];
                gpart[((long long)slot * ncta + crank) * 4 + k] = s;
            }
        }
        cg::this_grid().sync();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < K; k++) {
                double s = 0.0;
                for (unsigned r = 0; r < ncta; r++) s += gpart[((long long)slot * ncta + r) * 4 + k];
                sh->part[slot][0][k] = s;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; k++) v[k] = sh->part[slot][0][k];
    }
    __device__ double sum(double v) {
        double a[1] = {v};
        sumk<1>(a);
        return a[0];
    }
    __device__ int any(int flag) { return sum(flag ? 1.0 : 0.0) > 0.0; }
};

}  // namespace rb
