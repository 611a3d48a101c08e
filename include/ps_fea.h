/*
 * psfea — B200 (sm_100a) matrix-free voxel elasticity solver behind a C ABI.
 *
 * Drop-in for Parts Sim's linear-static solve: the reference's C++ class
 *   ps::VoxelFEA(dims, density, nu, bc, coarsestMaxDof = 1100, diagAdd = nullptr)
 *       native/src/fea/voxel_fea.hpp:136-137
 *   SolveResult VoxelFEA::solve(const std::vector<double>& f, const SolveOptions&)
 *       native/src/fea/voxel_fea.hpp:112-124, :153
 *   void VoxelFEA::precondition(const double* r, double* z)      native/src/fea/voxel_fea.hpp:151
 *   void VoxelFEA::apply(int l, const double* x, double* y, bool raw) native/src/fea/voxel_fea.hpp:143
 *   NodalStresses VoxelFEA::stresses(u, E, h, principals)        native/src/fea/voxel_fea.hpp:157
 *   std::array<double,3> VoxelFEA::reactions(u, f)              native/src/fea/voxel_fea.hpp:154
 * and of its GPU sibling ps::GpuFeaSolver (native/src/gpu/gpu_fea.hpp:17-35), which has the same
 * solve/precondition contract.
 *
 * Layout (identical to the reference): voxel e = i + nx*(j + ny*k); node n = i + NX*(j + NY*k)
 * with NX = nx+1 etc.; DOF 3n + d. Units are the solver's normalised ones (E = 1, voxel size 1):
 * u_physical = u / (E*h) for forces in N.
 *
 * All pointers are plain host pointers unless the name says _dev (device pointers on the
 * handle's CUDA device). Errors are status codes (the reference throws std::invalid_argument for
 * the PS_EINVAL / PS_ENONFINITE cases). ps_last_error() gives the message of the calling thread's
 * last failure. A handle may be used from one thread at a time.
 */
#ifndef PS_FEA_H
#define PS_FEA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_FEA_ABI_VERSION 1

typedef enum ps_status {
    PS_OK = 0,              /* converged: true relative residual <= 10 * tol (voxel_fea.cpp:925) */
    PS_NOT_CONVERGED = 1,   /* iteration cap reached; u and residual are still returned */
    PS_BREAKDOWN = 2,       /* p.Kp <= 0 (a mechanism; voxel_fea.cpp:904); u is returned */
    PS_CANCELLED = 3,       /* the cancel flag was raised; u is returned */
    PS_TIMEOUT = 4,         /* the time limit ran out; u is returned */
    PS_PENDING = 5,         /* a served request has not finished yet */
    PS_EINVAL = 10,         /* bad dims, sizes, density or nu (voxel_fea.cpp:141-146, hex8.cpp:9) */
    PS_ENONFINITE = 11,     /* non-finite f or x0 (voxel_fea.cpp:866-868) */
    PS_EOOM = 12,           /* device memory or admission budget exhausted */
    PS_ECUDA = 13,          /* CUDA runtime failure */
    PS_ENODEV = 14          /* no usable CUDA device */
} ps_status;

typedef enum ps_precision {
    /* The drop-in: FP64 flexible CG (Polak-Ribiere beta) preconditioned by the FP32 multigrid
     * V-cycle with r scaled to order one, exactly the reference's VoxelFEA::solve
     * (voxel_fea.cpp:835-927). */
    PS_PREC_FP64 = 0,
    /* The same FP64 flexible CG with a reduced-precision preconditioner: the FP32 V-cycle reads
     * every own (Galerkin) element matrix as FP16 times a power-of-two level scale, halving the
     * HBM traffic of the coarse levels' operators. The Krylov recurrence and its iteration count
     * are those of PS_PREC_FP64. */
    PS_PREC_MIXED = 1,
    /* FP32 CG and FP32 V-cycle with FP16 element matrices, kept to FP64 accuracy by reliable
     * updates: whenever the FP32 residual has dropped tenfold the FP32 iterate is folded into the
     * FP64 solution and the FP64 defect f - K u replaces the FP32 residual. On ill-conditioned
     * models the FP32 recurrence needs markedly more iterations than the FP64 one. */
    PS_PREC_FP32 = 2,
    /* FP64 iterative refinement around an FP32 flexible PCG whose V-cycle keeps every level below
     * the finest in FP16 vectors: the outer FP64 step forms the defect f - K u, rescales it to
     * max |r| = 1 and restarts the inner FP32 recurrence on it, which runs until its residual has
     * fallen by the refinement factor (0.1; PSFEA_REFINE_ETA), when its iterate is added to u in
     * FP64. Levels >= 1 store residuals r * 8^-l and iterates x * 8^-l * delta_l (delta_l a
     * power of two near the level's median diagonal over 16), so that both sit near order one in
     * FP16 with headroom; every scale is a power of two and the operator sums run in FP32.
     * FP16 element matrices as in PS_PREC_MIXED. One scale per level cannot hold graded
     * stiffness: where a level's diagonal spans more than a factor 256 (SIMP densities), the
     * coarse vectors stay FP32 and only the refinement remains. */
    PS_PREC_HALF = 3
} ps_precision;

typedef struct ps_fea ps_fea_t;

typedef struct ps_solve_opts {
    double tol;                       /* relative residual target (reference default 1e-6) */
    int32_t max_iter;                 /* reference default 500 */
    int32_t precision;                /* ps_precision */
    const double* x0;                 /* warm start, nDof values, or NULL (voxel_fea.hpp:115) */
    const volatile int32_t* cancel;   /* polled between iteration batches; nonzero cancels (the
                                         onProgress-returns-true contract, voxel_fea.cpp:910) */
    double time_limit_s;              /* 0 = none */
    int32_t smoother_degree;          /* Chebyshev smoother degree per V-cycle half (0 = the
                                         reference's 2, voxel_fea.cpp:692-725); 1..8 */
} ps_solve_opts;

typedef struct ps_solve_result {
    int32_t iterations;   /* CG iterations (voxel_fea.hpp:121) */
    int32_t converged;    /* residual <= 10 * tol */
    int32_t status;       /* ps_status of the outcome */
    int32_t folds;        /* PS_PREC_FP32: number of FP64 reliable updates */
    double residual;      /* true relative residual ||f - K u|| / ||f_free||, in FP64 */
    double seconds;       /* wall time of the call */
    int64_t kernels;      /* device kernels this call launched */
} ps_solve_result;

/* tol 1e-6, max_iter 500, PS_PREC_FP64, no warm start, no cancel flag, no time limit, smoother
 * degree 2 */
void ps_solve_opts_default(ps_solve_opts* opts);

/* Builds the multigrid hierarchy (2:1 coarsening with exact Galerkin coarse elements until the
 * free DOFs are <= coarsest_max_dof or 12 levels; dense FP64 factor of the coarsest level) and
 * uploads it to the current CUDA device. Replaces VoxelFEA::VoxelFEA (voxel_fea.cpp:138-183).
 * density: nx*ny*nz floats in [0, 1]; bc: 3*NX*NY*NZ bytes (1 = held); diag_add: nDof doubles
 * added to K's diagonal, or NULL. */
ps_status ps_fea_create(const int32_t dims[3], const float* density, double nu, const uint8_t* bc,
                        int64_t coarsest_max_dof, const double* diag_add, ps_fea_t** out);

/* K u = f (voxel_fea.cpp:863-927 / gpu_fea.cpp:452-574). f and u_out: nDof doubles on the host.
 * Returns the outcome status; u_out and *result are filled for PS_OK .. PS_TIMEOUT.
 * result may be NULL; opts may be NULL (defaults). */
ps_status ps_fea_solve(ps_fea_t* h, const double* f, const ps_solve_opts* opts, double* u_out,
                       ps_solve_result* result);

/* The same solve with f, x0 (opts->x0 is then a device pointer) and u already in device memory. */
ps_status ps_fea_solve_dev(ps_fea_t* h, const double* f_dev, const ps_solve_opts* opts, double* u_dev,
                           ps_solve_result* result);

/* nrhs solves on one hierarchy (the multi-load-case form: the sizing study's load groups,
 * study_runner.cpp:453-465, run as one batch). f and u_out: nrhs consecutive nDof vectors.
 * results: nrhs entries or NULL. opts->x0 (if set) holds nrhs warm starts. Returns the worst
 * outcome status. The FP64-Krylov forms run in blocks of up to 32 right-hand sides whose kernels
 * take the whole block (each element matrix and voxel word read once per block); every right-hand
 * side keeps its own CG scalars and stops on its own. PS_PREC_FP32 runs as concurrent single
 * solves. */
ps_status ps_fea_solve_batch(ps_fea_t* h, int32_t nrhs, const double* f, const ps_solve_opts* opts,
                             double* u_out, ps_solve_result* results);

/* One V-cycle as a preconditioner, z ~ K^-1 r (voxel_fea.cpp:830-861; gpu_fea.cpp:431-450). */
ps_status ps_fea_precondition(ps_fea_t* h, const double* r, double* z);

/* The same preconditioner applied to a block of nvec vectors at once, as LOBPCG applies it to its
 * block of residuals (eigen.cpp:508-513): r_dev, z_dev are nvec consecutive nDof-vectors in device
 * memory; each z_k = V-cycle(r_k / max|r_k|) * max|r_k|. The V-cycle kernels take up to 32 vectors
 * per launch. Stream-ordered on cuda_stream (NULL = the handle's stream); returns without waiting
 * for the GPU. */
ps_status ps_fea_precondition_block(ps_fea_t* h, int32_t nvec, const double* r_dev, double* z_dev, void* cuda_stream);

/* y = K x on level `level` in FP64; held/inactive DOFs of y zeroed unless raw
 * (voxel_fea.cpp:388). */
ps_status ps_fea_apply(ps_fea_t* h, int32_t level, const double* x, double* y, int32_t raw);

/* Nodal von Mises and (if principals) first/third principal stresses in Pa from physical
 * displacements u [m] (voxel_fea.cpp:968-1037). vm, p1, p3: NX*NY*NZ floats; p1/p3 may be NULL
 * when principals == 0. */
ps_status ps_fea_stresses(ps_fea_t* h, const double* u, double E, double vox, int32_t principals,
                          float* vm, float* p1, float* p3);

/* Support reactions: sum over held DOFs of active nodes of (K u - f); f may be NULL
 * (voxel_fea.cpp:929-940). */
ps_status ps_fea_reactions(ps_fea_t* h, const double* u, const double* f, double reaction[3]);

/* Routes all of the handle's device work to a caller-owned cudaStream_t (NULL = its own stream). */
ps_status ps_fea_set_stream(ps_fea_t* h, void* cuda_stream);

/* Mean device time in ms (CUDA events, `reps` back-to-back launches on the handle's stream) of the
 * finest level's operator kernel: which = 0 the FP32 Chebyshev smoothing step of the V-cycle,
 * 1 the FP64 product of the CG. Diagnostics for roofline reports. */
ps_status ps_fea_time_kernel(ps_fea_t* h, int32_t which, int32_t reps, double* ms);

/* No counterpart in the reference. y = K x (FP64, held DOFs of y zero) on the finest level and
 * *dot_dev = x . y, with x_dev, y_dev (nDof doubles) and dot_dev (one double) in device memory, for
 * callers that cannot allocate device memory during a call: code whose device memory belongs to
 * another allocator or a fixed budget, and loops that must not stall on the device-wide
 * synchronisation a cudaMalloc can cause. The call allocates nothing: the reduction's scratch
 * is a static 32.25 KiB device array in the library (at most 4096 reduction blocks; a device whose
 * launch shape needs more gets PS_EINVAL). The first call on each device looks up that array's
 * address and should come before any stream capture. All calls on a device share the array, so
 * calls that overlap on the GPU race. Stream-ordered on `cuda_stream` (NULL = the handle's own
 * stream; pass cudaStreamLegacy, (void*)1, for the legacy default stream, which is the stream
 * PyTorch reports as 0): a caller's stream is made to wait for the handle's uploads, but not for
 * other work the caller left queued on the handle's own stream. Call it with the handle's device
 * current (PS_EINVAL otherwise). Returns without waiting for the GPU. */
ps_status ps_fea_apply_dot_noalloc(ps_fea_t* h, const double* x_dev, double* y_dev, double* dot_dev, void* cuda_stream);

/* ---- Autotuning (no counterpart in the reference, which fixes a degree-2 Chebyshev smoother,
 * voxel_fea.cpp:692-725, and the coarsest size, voxel_fea.cpp:174-180) */
typedef struct ps_tune_result {
    int32_t smoother_degree;   /* chosen Chebyshev degree per V-cycle half (1-4) */
    int32_t inner64;           /* the finest level's FP64 tiles compute their boundary nodes in the tile */
    int64_t split_levels;      /* bit l: level l's FP32 tiles leave boundary nodes to the list kernel */
    int64_t coarsest_max_dof;  /* ps_fea_create_tuned: the chosen coarsening depth (else 0) */
    int32_t trials;            /* solves timed (0: taken from the process's cache of tuned models) */
    int32_t cached;
    double best_seconds;       /* solve time of the chosen configuration */
    double default_seconds;    /* solve time of the configuration before tuning */
} ps_tune_result;

#define PS_TUNE_FORCE 1        /* ignore the cache of tuned models */

/* Times complete solves of f (host, nDof values) to opts->tol over smoother degrees 1-4 and the
 * tile-path choices of the tiled levels, keeps the fastest configuration on the handle (solves whose
 * smoother_degree is 0 use the tuned degree) and caches it for models with the same voxel words,
 * masks and depth. opts->precision and max_iter apply to the trials. */
ps_status ps_fea_autotune(ps_fea_t* h, const double* f, const ps_solve_opts* opts, int32_t flags, ps_tune_result* out);

/* ps_fea_create for several coarsening depths (coarsest_max_dof 300, 1100 and 3000, the last the
 * largest dense coarsest solve the hierarchy takes), each autotuned on f; keeps the fastest handle. */
ps_status ps_fea_create_tuned(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, const double* diag_add,
                              const double* f, const ps_solve_opts* opts, int32_t flags, ps_tune_result* out, ps_fea_t** handle);

/* Device kernels the handle has launched since it was created. */
int64_t ps_fea_kernel_launches(const ps_fea_t* h);

int64_t ps_fea_ndof(const ps_fea_t* h);
int32_t ps_fea_num_levels(const ps_fea_t* h);
/* info[9] = nx, ny, nz, nNodes, nDof, freeDof, nElems, nOwn (own coarse matrices), coarsest m */
ps_status ps_fea_level_info(const ps_fea_t* h, int32_t level, int64_t info[9]);
/* the level's fixed-DOF mask (1 = held, inactive or zero diagonal; voxel_fea.cpp:227-232) */
ps_status ps_fea_level_fixed(const ps_fea_t* h, int32_t level, uint8_t* out);
/* the smoother's eigenvalue estimate of D^-1 K on a level (0 until the first solve) */
double ps_fea_level_lmax(const ps_fea_t* h, int32_t level);
/* bytes of device memory the handle holds */
int64_t ps_fea_device_bytes(const ps_fea_t* h);

void ps_fea_destroy(ps_fea_t* h);

/* The host-side hierarchy alone (no device memory, no GPU needed): the same build as
 * ps_fea_create, for inspecting levels, masks and coarse matrices (the reference exposes them as
 * the public member VoxelFEA::levels, voxel_fea.hpp:164). */
typedef struct ps_hierarchy ps_hierarchy_t;
ps_status ps_hierarchy_create(const int32_t dims[3], const float* density, double nu, const uint8_t* bc,
                              int64_t coarsest_max_dof, const double* diag_add, ps_hierarchy_t** out);
/* The same hierarchy with the Galerkin coarse matrices (voxel_fea.cpp:268-386, the coarsen step of
 * the VoxelFEA constructor) computed on the current CUDA device wherever a level's classes of
 * equal child patterns number at least PSFEA_DEVICE_GALERKIN_MIN (default 4096: graded grids),
 * bitwise equal to the host build; ps_fea_create builds this way when PSFEA_DEVICE_GALERKIN=1.
 * The result holds no device memory. PS_ENODEV without a device. */
ps_status ps_hierarchy_create_dev(const int32_t dims[3], const float* density, double nu, const uint8_t* bc,
                                  int64_t coarsest_max_dof, const double* diag_add, ps_hierarchy_t** out);
int32_t ps_hierarchy_num_levels(const ps_hierarchy_t* h);
ps_status ps_hierarchy_level_info(const ps_hierarchy_t* h, int32_t level, int64_t info[9]);
ps_status ps_hierarchy_level_fixed(const ps_hierarchy_t* h, int32_t level, uint8_t* out);
/* own coarse matrices in increasing coarse-voxel order: nOwn * 576 floats */
ps_status ps_hierarchy_level_own(const ps_hierarchy_t* h, int32_t level, float* out);
/* the level's uniform element Kb (576 doubles) */
ps_status ps_hierarchy_level_kb(const ps_hierarchy_t* h, int32_t level, double* out);
void ps_hierarchy_destroy(ps_hierarchy_t* h);

/* Condensed 24x24 unit-cube element (E = 1) with 9 Wilson incompatible modes, and its corner
 * stress matrices D*Bbar (8 x 6 x 24); corner_stress may be NULL (hex8.cpp:104-155). */
ps_status ps_element_matrix(double nu, double K[576], double* corner_stress);

/* Voxels not face-connected to a voxel touching a held node become empty
 * (pruneFloating, voxel_fea.cpp:1086-1119). held_node: NX*NY*NZ bytes. */
ps_status ps_prune_floating(const int32_t dims[3], const float* density, const uint8_t* held_node,
                            float* out, int32_t* removed);

/* ---- Study loops on the device: the solve of every iteration warm-started from the previous
 * displacements in device memory, the loops' per-voxel work (density filter, element energies,
 * optimality-criteria update and its volume bisection, failure measure) as kernels beside it. */

typedef struct ps_topology_opts {
    double vol_frac;     /* volume budget, fraction of the design domain (0.4) */
    double penal;        /* SIMP penalty p (3) */
    double rmin;         /* density-filter radius in voxels (1.5) */
    double move;         /* optimality-criteria move limit (0.2) */
    double tol;          /* stop once the largest design change is below it, after 5 iterations (0.01) */
    int32_t max_iter;    /* 40 */
    double solve_tol;    /* relative residual of each iteration's solve (1e-5, study_runner.cpp:413) */
    int32_t precision;   /* ps_precision of the solves */
} ps_topology_opts;

typedef struct ps_topology_step {
    int32_t it;
    int32_t solve_iterations;
    int32_t solve_status;  /* ps_status of the iteration's solve */
    double compliance;     /* f . u */
    double volume;         /* used volume / design volume */
    double change;         /* largest design change of the previous update */
    double seconds;
} ps_topology_step;

/* defaults of native/src/fea/topology.hpp:38-48 */
void ps_topology_opts_default(ps_topology_opts* opts);

/* SIMP compliance minimisation (optimizeTopology, native/src/fea/topology.cpp:103-183): design
 * voxels are those with fill > 0 (fill: nx ny nz values in (0, 1]); keep (or NULL) marks voxels
 * that stay solid; bc and f as for ps_fea_create / ps_fea_solve. density_out: nx ny nz final
 * physical densities; history: opts->max_iter entries, *n_steps of them filled. */
ps_status ps_topology_run(const int32_t dims[3], const float* fill, const uint8_t* keep, double nu, const uint8_t* bc, const double* f,
                          const ps_topology_opts* opts, float* density_out, ps_topology_step* history, int32_t* n_steps);

typedef enum ps_break_reason {
    PS_BREAK_STEP_LIMIT = 0, PS_BREAK_SEPARATED = 1, PS_BREAK_UNSUPPORTED = 2, PS_BREAK_NOT_CONVERGED = 3, PS_BREAK_NO_STRESS = 4
} ps_break_reason;

typedef struct ps_break_step {
    int32_t step;
    int32_t voxels;            /* solved voxels */
    int32_t solve_iterations;
    int32_t cracked;           /* voxels removed as failed in this step */
    int32_t detached;          /* voxels that fell off with them (pruned) */
    double lambda;             /* load factor at which the most stressed voxel reaches the strength */
    double max_disp;           /* largest displacement magnitude at that load factor [m] */
    double seconds;
} ps_break_step;

/* Progressive failure (breakTest, native/src/fea/static_study.cpp:199-279): solve (warm-started),
 * nodal von Mises (principal = 0) or first principal stress, voxel measure = worst corner stress,
 * the most stressed voxels (within 5 % of the peak, at most 2 % of n^(2/3)) removed, floating parts
 * pruned, repeat for max_steps. steps: max_steps entries, *n_steps filled; cracked (or NULL): the
 * removed voxels of all steps in order, room for cracked_cap; density_out: the density left;
 * *peak: the largest load factor; *reason: ps_break_reason. E [Pa] and h [m] scale the stresses. */
ps_status ps_break_test(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, const double* f, double E, double h,
                        double strength, int32_t principal, int32_t max_steps, ps_break_step* steps, int32_t* n_steps, int32_t* cracked,
                        int64_t cracked_cap, float* density_out, double* peak, int32_t* reason);

/* pruneFloating (voxel_fea.cpp:1086-1119) on device arrays, for callers that keep their voxel grid
 * on the GPU (the break test prunes this way after every step): out_dev = density_dev where the
 * voxel's face-connected solid component touches a held node (held_dev: NX NY NZ bytes), else 0;
 * *removed = solid voxels dropped. Components by lock-free union-find; the kept set is unique, so
 * the result equals the reference's breadth-first search. Stream-ordered on cuda_stream (NULL = the
 * legacy default stream); returns once the result is written. */
ps_status ps_prune_floating_dev(const int32_t dims[3], const float* density_dev, const uint8_t* held_dev, float* out_dev, int32_t* removed,
                                void* cuda_stream);

/* ---- Serving: many independent solves on one GPU with continuous batching (no counterpart in the
 * reference, which runs one job at a time behind a GPU lock, native/src/gpu/gpu.hpp:43).
 * Requests are submitted at any time; host threads build their hierarchies; a scheduler admits
 * them in arrival order as device memory (estimated footprint against the budget) and active
 * slots allow, runs them concurrently on separate streams, retires finished ones and back-fills. */
typedef struct ps_server ps_server_t;

typedef struct ps_request {
    int32_t dims[3];
    const float* density;      /* copied at submit */
    double nu;
    const uint8_t* bc;         /* copied at submit */
    const double* f;           /* copied at submit */
    int64_t coarsest_max_dof;  /* 0 = 300 */
    double tol;                /* 0 = 1e-8 */
    int32_t max_iter;          /* 0 = 5000 */
    int32_t precision;         /* ps_precision */
    int32_t smoother_degree;   /* 0 = 2 */
} ps_request;

typedef struct ps_request_result {
    int64_t id;
    int32_t status;            /* ps_status of the solve (or the error that ended the request) */
    int32_t iterations;
    int32_t converged;
    double residual;
    int64_t n_dof;
    const double* u;           /* n_dof displacements, valid until ps_server_release */
    double build_s;            /* submit -> hierarchy built (host) */
    double wait_s;             /* built -> admitted to the GPU */
    double solve_s;            /* admitted -> finished */
    double total_s;            /* submit -> finished */
} ps_request_result;

typedef struct ps_server_stats {
    int64_t queued, active, completed;
    int64_t device_bytes_in_use, peak_device_bytes, budget_bytes;
    int64_t peak_active;
} ps_server_stats;

/* budget_bytes 0 = 80 % of the free device memory; max_active 0 = 4 (measured best for the
 * serving stream: each small-grid solve already spreads over the whole GPU); build_threads 0 = half
 * the host cores. */
ps_status ps_server_create(int64_t device_budget_bytes, int32_t max_active, int32_t build_threads, ps_server_t** out);
ps_status ps_server_submit(ps_server_t* s, const ps_request* req, int64_t* id);
/* PS_PENDING until the request has finished, then PS_OK with *out filled */
ps_status ps_server_poll(ps_server_t* s, int64_t id, ps_request_result* out);
ps_status ps_server_wait(ps_server_t* s, int64_t id, ps_request_result* out);
/* frees a finished request's result */
ps_status ps_server_release(ps_server_t* s, int64_t id);
ps_status ps_server_get_stats(ps_server_t* s, ps_server_stats* out);
void ps_server_destroy(ps_server_t* s);

/* Message of the calling thread's last error ("" if none). */
const char* ps_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PS_FEA_H */
