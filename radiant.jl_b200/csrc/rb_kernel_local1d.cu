// rb_kernel_local1d.cu -- the persistent loop for batches whose every problem takes the local
// (cell-split) 1D pass: the kernel carries no other pass, so its registers go to that path
// alone. Its own translation unit so that the persistent kernels compile in parallel.
#include "rb_solve.cuh"

namespace rb {

__global__ void __launch_bounds__(RB_THREADS, 1) solve_local1d_kernel(DevProblem *const *probs, int nprob, int *queue,
                                                                   int local_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupShared &gs = *reinterpret_cast<GroupShared *>(smem_raw);
    void *local = (void *)(smem_raw + sizeof(GroupShared));
    if (threadIdx.x == 0) gs.tc.ready = 0;  // no tensor memory in this kernel
    __syncthreads();
    ClusterTeam t;
    t.init(&gs.team);
    while (true) {
        int idx = 0;
        if (t.crank == 0 && threadIdx.x == 0) idx = atomicAdd(queue, 1);
        idx = t.broadcast_from_leader(idx);
        if (idx >= nprob) break;
        solve_problem<ClusterTeam, true>(t, *probs[idx], gs, local, local_bytes);
    }
}

}  // namespace rb
