// rb_kernel_grid.cu -- one large (2D/3D) problem on the whole GPU: a cooperative launch whose
// CTAs form one team (grid barriers) and run the problem's whole group loop. Its own
// translation unit so that the persistent kernels compile in parallel.
#include "rb_solve.cuh"

namespace rb {

// Dynamic shared memory: GroupShared, then `local_bytes` for the 3D octant sweep.
__global__ void __launch_bounds__(RB_THREADS, 1) solve_grid_kernel(DevProblem *prob, double *gpart, int local_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupShared &gs = *reinterpret_cast<GroupShared *>(smem_raw);
    void *local = local_bytes > 0 ? (void *)(smem_raw + sizeof(GroupShared)) : nullptr;
    GridTeam t;
    t.init(&gs.team, gpart);
    // the mixed form's 2D/3D products run on the tensor cores: every CTA holds TMEM columns for
    // their accumulators and the mbarriers of MMA completion for the whole launch
    const bool use_tc = prob->precision == 1 && prob->ndims >= 2 && prob->tc_m2d != nullptr;
    if (threadIdx.x == 0) {
        gs.tc.ready = 0;
        gs.tc.phase = 0;
    }
    if (use_tc) {
        if (threadIdx.x < 32) tc::tmem_alloc(&gs.tc.tmem, RB_TC_TMEM_COLS);
        if (threadIdx.x == 0) {
            tc::mbar_init(&gs.tc.mbar[0]);
            tc::mbar_init(&gs.tc.mbar[1]);
        }
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (threadIdx.x == 0) gs.tc.ready = 1;
    }
    __syncthreads();
    solve_problem(t, *prob, gs, local, local_bytes);
    if (use_tc) {
        tc::fence_before();
        __syncthreads();
        if (threadIdx.x < 32) {
            tc::fence_after();
            tc::tmem_dealloc(gs.tc.tmem, RB_TC_TMEM_COLS);
        }
    }
}

}  // namespace rb
