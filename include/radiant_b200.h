/*
 * radiant_b200.h -- C ABI of the B200-native discrete-ordinates (SN) transport solve.
 *
 * This library replaces one Julia method of Radiant.jl:
 *     compute_flux(cross_sections::Cross_Sections, geometry::Geometry, solver::SN,
 *                  source::Source, electromagnetic_field::Electromagnetic_Field)
 *   (src/particle_transport/sn_flux.jl:22-233)
 * together with everything it calls: the in-group solve (sn_one_speed.jl:81-195), the
 * source-iteration pass (sn_inner_pass.jl:17-137), the 1D/2D/3D sweeps
 * (sn_sweep_1D.jl:51-123, sn_sweep_2D.jl:54-183, sn_sweep_3D.jl:57-239), the cell closures
 * (sn_{1,2,3}D_{bte,bfp}.jl), the scattering and Fokker-Planck sources
 * (scattering_source.jl:25-68, fokker_planck_source.jl:26-35) and the in-group solvers
 * (src/tools/{livolant,anderson,gmres,bicgstab,krylov_state}.jl).
 *
 * Conventions (chosen so that a Julia `ccall` can pass its arrays unchanged):
 *   - every array is column-major (first index fastest), exactly the shape the reference
 *     holds it in; shapes are written [a,b,c] in that order;
 *   - material ids are 1-based (Julia's `mat`), converted from Int64 to int32 by the caller;
 *   - every entry point returns an int32 status, 0 = RB_OK; no exception crosses the ABI;
 *   - host buffers belong to the caller; device memory belongs to the context.
 *   - one host thread per context; calls on one context are serialised by the caller.
 */
#ifndef RADIANT_B200_H
#define RADIANT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RB_API __attribute__((visibility("default")))
#else
#define RB_API
#endif

/* ---- status codes -------------------------------------------------------------------- */
#define RB_OK 0
#define RB_ERR_INVALID 1     /* bad argument or inconsistent problem description          */
#define RB_ERR_UNSUPPORTED 2 /* valid in the reference but not built here (AWD, EM field)  */
#define RB_ERR_CUDA 3        /* a CUDA runtime call failed                                 */
#define RB_ERR_BUDGET 4      /* admission refused: the solve does not fit the HBM budget   */
#define RB_ERR_TIMEOUT 5     /* a bounded device wait gave up (never a hang)               */
#define RB_ERR_NOT_READY 6   /* rb_poll: the request is still on the device                */
#define RB_ERR_NOT_FOUND 7   /* unknown problem / request handle                           */

/* ---- enumerations (values follow the reference) -------------------------------------- */
/* solver_type, src/structures/SN.jl:478-500 */
#define RB_SOLVER_BTE 1
#define RB_SOLVER_BFP 2
#define RB_SOLVER_BCSD 3
#define RB_SOLVER_FP 4
#define RB_SOLVER_CSD 5
#define RB_SOLVER_BFP_EF 6
/* boundary conditions, src/structures/Geometry.jl:604-631 */
#define RB_BC_VOID 0
#define RB_BC_REFLECTIVE 1
#define RB_BC_PERIODIC 2
/* in-group acceleration, src/structures/SN.jl:348-362 */
#define RB_ACCEL_NONE 0
#define RB_ACCEL_LIVOLANT 1
#define RB_ACCEL_ANDERSON 2
#define RB_ACCEL_GMRES 3
#define RB_ACCEL_BICGSTAB 4
/* arithmetic form */
#define RB_PRECISION_FP64 0  /* plain form: FP64 throughout (the drop-in)                   */
#define RB_PRECISION_MIXED 1 /* sweeps in FP32; Krylov / outer update / tests in FP64       */

/*
 * Everything compute_flux(::SN) holds when it enters its group loop (sn_flux.jl:27-147),
 * i.e. the tables the reference's own host functions build: quadrature, angular bases,
 * scheme weights, cross sections after the Fokker-Planck and elastic-free corrections
 * (sn_flux.jl:69-113), and the fixed sources.
 */
typedef struct rb_sn_problem {
    /* geometry (Geometry getters, sn_flux.jl:27-33) */
    int32_t ndims;                /* 1, 2 or 3                                              */
    int32_t nx, ny, nz;           /* voxels per axis (1 on unused axes)                     */
    const double *dx, *dy, *dz;   /* voxel widths [nx], [ny], [nz] (NULL on unused axes)    */
    const int32_t *mat;           /* [nx,ny,nz] 1-based material id per voxel               */
    int32_t nmat;
    int32_t bc[6];                /* X-,X+,Y-,Y+,Z-,Z+ : RB_BC_*                            */

    /* angular discretisation (sn_flux.jl:44-48) */
    int32_t nd;                   /* number of directions                                   */
    const double *mu, *eta, *xi;  /* direction cosines [nd] (eta/xi may be NULL in 1D)      */
    int32_t np;                   /* number of angular moments                              */
    const double *mn;             /* moment-to-discrete  Mn [nd,np]                         */
    const double *dn;             /* discrete-to-moment  Dn [np,nd]                         */
    const int32_t *pl;            /* Legendre order of each moment [np]                     */
    int32_t np_surf;              /* moments of the half-range surface bases                */
    int32_t nd_plus[6];           /* incoming directions through each face                 */
    const double *mn_surf[6];     /* per face [nd_plus[f], np_surf]                         */
    const double *dn_surf[6];     /* per face [np_surf, nd_plus[f]]                         */
    const int32_t *n_to_nplus[6]; /* per face [nd], 1-based half-range index, 0 = none      */

    /* spatial / energy closures (sn_flux.jl:62-64, SN.jl:520-544, scheme_weights.jl) */
    int32_t order[4];             /* scheme order 𝒪 along x, y, z, E                        */
    int32_t nm[5];                /* Nm: face moments x,y,z, energy-face moments, cell moments */
    int32_t is_fc;                /* full coupling of the high-order moments                */
    const double *w_axis[4];      /* closure weights ω along x,y,z,E, length order[a]+1     */
    const double *cc;             /* 𝒞 [ncc], 𝒞_i = sqrt(2i-1)                              */
    int32_t ncc;
    const double *ww;             /* 𝒲 [order[3],order[3],order[3]]                         */
    int32_t is_adaptive;          /* AWD closures: rejected with RB_ERR_UNSUPPORTED         */
    int32_t is_em;                /* external EM field: rejected with RB_ERR_UNSUPPORTED    */

    /* cross sections of one particle (sn_flux.jl:53-113) */
    int32_t solver_type;          /* RB_SOLVER_*                                            */
    int32_t ng;                   /* energy groups                                          */
    const double *sigma_t;        /* Σtot [ng,nmat] (with T·λ₀ / elastic-free corrections)  */
    int32_t ls;                   /* highest Legendre order carried (maximum(pl))           */
    const double *sigma_s;        /* Σs [nmat,ng,ng,ls+1]  (gi, gf)                         */
    const double *s_minus;        /* S⁻ [ng,nmat]  (CSD only, else NULL)                   */
    const double *s_plus;         /* S⁺ [ng,nmat]                                           */
    const double *s_mom;          /* S  [ng,nmat,order[3]]                                  */
    const double *t_mom;          /* T  [ng,nmat]  (solver 2 and 4, else NULL)              */
    const double *fp;             /* ℳ  [np,np]    (solver 2 and 4, else NULL)              */
    const double *e_width;        /* ΔE [ng]       (CSD only)                               */

    /* fixed sources (Source getters, sn_flux.jl:138-140) */
    const double *volume_sources; /* [ng,np,nm5,nx,ny,nz] or NULL                          */
    int32_t np_source;            /* moments of the surface sources actually used           */
    const double *surface_sources[6]; /* per face [ng,np_source,face cells] or NULL;
                                         face cells: 1 (1D); ny or nx (2D); (ny,nz),(nx,nz),
                                         (nx,ny) column-major (3D)                           */

    /* in-group solver (SN getters, sn_flux.jl:130-147) */
    int32_t accel;                /* RB_ACCEL_*                                             */
    double tol;                   /* convergence criterion ϵ_max                            */
    int32_t max_iter;             /* I_max                                                  */
    int32_t gmres_restart;
    int32_t anderson_depth;

    int32_t precision;            /* RB_PRECISION_*                                         */
} rb_sn_problem;

/* What compute_flux returns in its Flux_Per_Particle (sn_flux.jl:226-232), plus the
 * per-group record sn_one_speed prints (sn_one_speed.jl:422-426). NULL pointers are skipped. */
typedef struct rb_sn_result {
    double *flux;            /* 𝚽l [ng,np,nm5,nx,ny,nz]                                     */
    double *flux_cutoff;     /* 𝚽cutoff [np,nm5,nx,ny,nz] (CSD solvers)                     */
    double *rho;             /* spectral-radius estimate per group [ng] (NaN where none)    */
    int32_t *group_iters;    /* solver iterations per group [ng]                            */
    double *group_resid;     /* final relative residual per group [ng]                      */
    int32_t *group_converged;/* 1 if the group met tol [ng]                                 */
    int64_t passes;          /* total source-iteration passes (the reference's Ntot)        */
} rb_sn_result;

typedef struct rb_context rb_context;
typedef int64_t rb_handle;

/* ---- context ------------------------------------------------------------------------- */
/* Replaces nothing in the reference (which owns no device); the context holds the device,
 * its stream pool and the HBM budget that admission control checks against. Problem memory
 * comes from a stream-ordered memory pool the context owns: uploads and releases do not wait
 * for kernels on other streams, freed blocks are kept for later uploads, and rb_destroy gives
 * everything back. */
RB_API int32_t rb_create(int32_t device, uint64_t hbm_budget_bytes, rb_context **ctx);
RB_API int32_t rb_destroy(rb_context *ctx);
/* Copies the message of the last failed call on ctx (or of the last rb_create failure when
 * ctx is NULL) into buf, truncated to len bytes including the terminating zero. */
RB_API int32_t rb_last_error(const rb_context *ctx, char *buf, uint64_t len);

/* ---- one problem at a time: the compute_flux(::SN) drop-in ---------------------------- */
/* Validates the description and copies every table to the device (the arrays
 * compute_flux builds in sn_flux.jl:27-147). */
RB_API int32_t rb_upload(rb_context *ctx, const rb_sn_problem *prob, rb_handle *out);
/* Runs the full group loop of sn_flux.jl:162-224 on the device, asynchronously on
 * `stream` (a cudaStream_t; NULL = the context's own stream). */
RB_API int32_t rb_solve(rb_context *ctx, rb_handle h, void *stream);
/* Solves several uploaded problems in one persistent launch (one work queue). */
RB_API int32_t rb_solve_batch(rb_context *ctx, const rb_handle *hs, int32_t n, void *stream);
/* Waits for the problem's stream and copies the results into caller-owned host buffers. */
RB_API int32_t rb_download(rb_context *ctx, rb_handle h, rb_sn_result *res);
/* rb_download in two halves, for a caller that launches more work meanwhile: rb_download_async
 * queues the layout change of the flux on the problem's solve stream (right behind the solve,
 * before anything launched there later) and the copies on a copy stream of the context, and
 * returns; rb_download_wait waits for them and reports the solve's status. `res` and its buffers
 * must stay alive until the wait (page-locked buffers let the copies overlap later solves). The
 * context holds one staging buffer for these downloads: a second rb_download_async first waits
 * for the copies of the one before. */
RB_API int32_t rb_download_async(rb_context *ctx, rb_handle h, rb_sn_result *res);
RB_API int32_t rb_download_wait(rb_context *ctx, rb_handle h);
RB_API int32_t rb_release(rb_context *ctx, rb_handle h);
/* Bytes of device memory rb_upload would reserve for `prob` (admission control). */
RB_API int32_t rb_required_bytes(const rb_sn_problem *prob, uint64_t *bytes);

/* upload + solve + download + release on a private context: the one-call drop-in. */
RB_API int32_t rb_compute_flux(int32_t device, const rb_sn_problem *prob, rb_sn_result *res);

/* rb_compute_flux without any device allocation. No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- a process whose device memory belongs to another
 * allocator (a Julia CUDA.jl pool, a PyTorch caching allocator) that must not see
 * cudaMalloc/cudaFree, which synchronise the device and can fail or fragment that pool.
 * All device memory it uses (tables, work buffers, result staging) is one file-scope static
 * device array of 16 MiB that every GPU loading the library holds until the process exits;
 * a problem needing more returns RB_ERR_BUDGET with the sizes in rb_last_error(NULL, ...).
 * Runs on the current device and `stream` (NULL = the legacy default stream) and returns once
 * the results are in the caller's host buffers. The first call on a device looks the array's
 * device address up (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. Every call shares the one array and overwrites it: calls that
 * overlap on the GPU (other host threads, other streams) race and must be serialised.
 * The solve runs as one team of a single CTA (one SM of the GPU), whatever the dimension: the
 * entry point is meant for the small problems that fit its array, not for throughput (larger
 * or throughput-bound work belongs on rb_compute_flux / rb_solve_batch). */
RB_API int32_t rb_compute_flux_static(const rb_sn_problem *prob, rb_sn_result *res, void *stream);

/* ---- coupled particles: transport() ----------------------------------------------------- */
/* The coupling of particle i into particle j in the generation loop of transport()
 * (transport.jl:79-143): the source of j produced by i's flux, particle_source(flux_i, ...)
 * (particle_source.jl:23-79) =
 *   Ql_in[gf,p,is,c]  = sum_gi sigma_s[mat,gi,gf,pl_i[p]] * flux_i[gi,p,is,c]   (particle_sources,
 *                       scattering_source.jl:97-104)
 *   Ql_out[gf,q,k,c]  = sum_p transfer[q,p] * Ql_in[gf,p,moment_map[k]-1,c]      (map_moments.jl:21-56)
 * added to j's volume source. */
typedef struct rb_coupling {
    const double *sigma_s;      /* [nmat, ng_i, ng_j, ls+1]: get_scattering(particle_i, particle_j, maximum(pl_i));
                                   NULL = i produces no j                                      */
    int32_t ls;
    const double *transfer;     /* [np_j, np_i]: angular_transfer_matrix(basis_i, basis_j)      */
    const int32_t *moment_map;  /* [nm5_j]: 1-based cell moment of i feeding each moment of j, 0 = none */
} rb_coupling;

/* Replaces transport(cross_sections, geometry, solvers, sources) (transport.jl:21-147) for a
 * set of SN particles on one geometry: every particle's problem, its accumulated particle source
 * and its running total flux stay on the device for the whole generation loop; a generation
 * solves the particles in order (starting from the first one with fixed sources), each solve
 * followed by the sources it produces for the others (device kernels), and the fixed sources
 * count in the first generation only. couplings[i*npart + j] couples i into j (the diagonal is
 * ignored). conv_type (transport.jl:112-137): 0 = "flux" (after generation n > 1, every
 * particle's max |Φ_n − Φ_(n−1)| / max(|Φ_n|, eps) over groups and cells, moment 1 and cell
 * moment 1, below eps_gen), 1 = "energy-deposition", 2 = "charge-deposition" (the summed
 * deposition's max relative change below eps_gen); other values: RB_ERR_INVALID.
 * sigma_dep[i] [ng_i+1, nmat] (Σe for energy, Σc for charge deposition: the same formula),
 * density [nmat] and norm (the sources' normalization factor) are needed by criteria 1 and 2 and
 * by `deposition` (else NULL). results[i]: flux and flux_cutoff summed over the generations
 * (the reference's Flux_Per_Particle sums its solutions), rho / iterations / residuals /
 * converged of the last generation's solve, passes summed over all solves. deposition (NULL =
 * skip): [nx,ny,nz], the summed deposition of the final fluxes (energy_deposition.jl:24-87 with
 * sigma_dep). *generations: generations run; *eps_final: the last ϵ (NaN after one). */
RB_API int32_t rb_transport(int32_t device, int32_t npart, const rb_sn_problem *const *probs,
                            const rb_coupling *couplings, int32_t ngen_max, double eps_gen, int32_t conv_type,
                            const double *const *sigma_dep, const double *density, double norm,
                            rb_sn_result *const *results, double *deposition, int32_t *generations,
                            double *eps_final);

/* ---- launch rules (the autotuner's table) --------------------------------------------- */
/* No counterpart in the reference (a Julia solve has no launch shape). A rule gives the team size
 * (CTAs per problem, a power of two up to 16) for the problems of a class in batches of a size:
 * dimension `ndims`, at most nd_max directions, at most work_max work (groups × directions ×
 * cells × cell moments, doubled for the CSD solvers), in a batch of at most batch_max problems.
 * rb_solve / rb_solve_batch of problems that all match a rule (the first matching rule of each;
 * the largest team among them) launch with that team size, which a tuning run measured as the
 * fastest for the class at that batch size (radiant_b200/autotune.py); other batches keep the
 * built-in shape choice. Serving requests (rb_submit) do not use the rules. n = 0 clears them. */
typedef struct rb_launch_rule {
    int32_t ndims;
    int32_t nd_max;
    int64_t work_max;
    int32_t batch_max;
    int32_t cluster;
} rb_launch_rule;
RB_API int32_t rb_set_launch_rules(rb_context *ctx, const rb_launch_rule *rules, int32_t n);

/* ---- fixed sources built on the device ------------------------------------------------- */
/* A Volume_Source (src/structures/Volume_Source.jl) as volume_source() reads it
 * (volume_source.jl:21-122): `intensity` in group `energy_group` on every voxel whose centre lies
 * inside [lo, hi] on each axis of the geometry (bounds inclusive; axes beyond ndims unused). */
typedef struct rb_volume_box {
    int32_t energy_group;   /* 1-based */
    int32_t reserved;       /* 0 */
    double intensity;
    double lo[3], hi[3];
} rb_volume_box;

/* A Surface_Source (src/structures/Surface_Source.jl) of an SN solve as surface_source() reads it
 * (surface_source.jl:22-330): a beam of `intensity` in group `energy_group` through `face`
 * (0..5 = X-, X+, Y-, Y+, Z-, Z+) with direction (mu, eta, xi), on the face cells whose centres lie
 * inside [lo, hi] on the face's in-plane axes. `basis` holds the np_source values of the beam's
 * half-range basis in the order of the surface moments: the shifted Legendre polynomials
 * P_l(|mu|) (1D, Qdims 1: surface_source.jl:103) or the half-range real spherical harmonics at
 * (|mu|, atan(xi, eta)) (surface_source.jl:137, :195, :284), zero beyond the source's own
 * Legendre order. */
typedef struct rb_surface_beam {
    int32_t energy_group;   /* 1-based */
    int32_t face;
    double intensity;
    double direction[3];
    double lo[3], hi[3];
    const double *basis;    /* [np_source] */
} rb_surface_beam;

/* The sources of one problem, added in this order as Source.add_source does
 * (src/structures/Source.jl:129-203), and the voxel centres they are tested against
 * (geometry.voxels_position, particle_transport/geometry.jl:68,147-148,252-254). */
typedef struct rb_source_set {
    const double *position[3];  /* [nx], [ny], [nz] voxel centres (axes beyond ndims NULL) */
    int32_t nvolume;
    int32_t nsurface;
    const rb_volume_box *volume;
    const rb_surface_beam *surface;
} rb_source_set;

/* rb_upload for a problem whose fixed sources come as definitions instead of dense arrays: the
 * library builds the volume sources [ng, np, nm5, cells] and the per-face surface sources
 * [ng, np_source, face cells] on the device (what volume_source / surface_source and
 * Source.add_source build on the host), so only the definitions cross the host link.
 * prob->volume_sources and prob->surface_sources must be NULL. norms (NULL allowed) receives the
 * normalization factor of each source, volume boxes first, then beams, summed in the
 * reference's order. No counterpart in the reference: it exists to take the dense source arrays
 * off the host (the volume sources of a 64^3 S8 problem with 40 groups are 6.7 GB). */
RB_API int32_t rb_upload_sources(rb_context *ctx, const rb_sn_problem *prob, const rb_source_set *src,
                                 rb_handle *out, double *norms);

/* ---- serving: continuous batching ---------------------------------------------------- */
/* Admits a request (one particle solve) when its state fits the remaining HBM budget
 * (RB_ERR_BUDGET otherwise, nothing allocated). An admitted request is uploaded and launched at
 * once as its own cluster team (one persistent-kernel launch on a stream of a pool of 32), so it
 * runs beside the requests already on the device and its result never depends on them. */
RB_API int32_t rb_submit(rb_context *ctx, const rb_sn_problem *prob, rb_handle *out);
/* RB_OK when the request finished (results copied into res and the request released),
 * RB_ERR_NOT_READY while it is still running. */
RB_API int32_t rb_poll(rb_context *ctx, rb_handle h, rb_sn_result *res);

/* ---- post-processing ------------------------------------------------------------------- */
/* energy_deposition.jl:24-87 for one particle: D[c] = (Σ_g Σe[g,mat]·𝚽l[g,1,1,c]
 * + Σe[ng+1,mat]·𝚽cutoff[1,1,c]) / (ρ[mat]·norm). flux_cutoff may be NULL (no CSD). */
RB_API int32_t rb_energy_deposition(int32_t ng, int32_t np, int32_t nm5, int64_t ncell,
                             int32_t nmat, const int32_t *mat, const double *flux,
                             const double *flux_cutoff, const double *sigma_e,
                             const double *density, double norm, double *dep);
/* energy_deposition.jl:24-87 (sigma_dep = Σe) or charge_deposition.jl:26-89 (sigma_dep = Σc;
 * the same formula) of problems already solved in the context (rb_solve / rb_solve_batch), on
 * the device: dep[c] = Σ_particles (Σ_g sig_i[g,mat]·𝚽l_i[g,1,1,c] + sig_i[ng_i+1,mat]·
 * 𝚽cutoff_i[1,1,c]) / (ρ[mat]·norm), particles summed in the order of `handles`; sigma_dep[i]
 * [ng_i+1, nmat], dep [nx,ny,nz]. Only the voxel array crosses to the host. */
RB_API int32_t rb_deposition(rb_context *ctx, int32_t npart, const rb_handle *handles, const double *const *sigma_dep,
                             const double *density, double norm, double *dep);

/* ---- page-locked host buffers ------------------------------------------------------------ */
/* No counterpart in the reference (Julia arrays are pageable). The upload and download copies
 * run at the host link's speed only from page-locked memory: from pageable memory the driver
 * stages every copy through its own buffer at a fraction of it. rb_host_alloc returns `bytes`
 * of page-locked memory usable by every device (free with rb_host_free); rb_host_register locks
 * an existing allocation in place (a Julia Array's storage) until rb_host_unregister. Both cost
 * time per byte (the pages are locked one by one): lock the buffers a caller reuses, once. */
RB_API int32_t rb_host_alloc(uint64_t bytes, void **out);
RB_API int32_t rb_host_free(void *p);
RB_API int32_t rb_host_register(void *p, uint64_t bytes);
RB_API int32_t rb_host_unregister(void *p);

/* Library version string. */
RB_API const char *rb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RADIANT_B200_H */
