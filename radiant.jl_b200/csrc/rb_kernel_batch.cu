// rb_kernel_batch.cu -- the persistent batch kernel: thread-block clusters (one team per
// problem) pull problems of any shape from a device work queue and run each one's whole group
// loop (solve_problem, rb_solve.cuh). Its own translation unit so that the three persistent
// kernels compile in parallel.
#include "rb_solve.cuh"

namespace rb {

__global__ void __launch_bounds__(RB_THREADS, 1) solve_batch_kernel(DevProblem *const *probs, int nprob, int *queue,
                                                                 int local_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupShared &gs = *reinterpret_cast<GroupShared *>(smem_raw);
    void *local = local_bytes > 0 ? (void *)(smem_raw + sizeof(GroupShared)) : nullptr;
    if (threadIdx.x == 0) gs.tc.ready = 0;  // no tensor memory in this kernel
    __syncthreads();
    ClusterTeam t;
    t.init(&gs.team);
    while (true) {
        int idx = 0;
        if (t.crank == 0 && threadIdx.x == 0) idx = atomicAdd(queue, 1);
        idx = t.broadcast_from_leader(idx);
        if (idx >= nprob) break;
        solve_problem(t, *probs[idx], gs, local, local_bytes);
    }
}

}  // namespace rb
