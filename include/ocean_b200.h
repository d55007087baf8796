/*
 * ocean_b200.h - C ABI of the B200 (sm_100a) hydrostatic ocean-core time step.
 *
 * Plain C types only: the library owns its device state and workspace, the
 * caller hands in host or device pointers with their sizes. Every function
 * returns an int status (OC_OK = 0); oc_last_error() gives the message.
 * A handle is not thread-safe; all GPU work of a handle is issued on the
 * stream passed to oc_step (or the default stream) in issue order.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - the backend process boundary `<binary> <prefix>.nml` ->
 *     `<prefix>_state3d5.bin` + `<prefix>_metrics.json`
 *     (tools/compare_backends3d5.py:69-78, libs/cuda/src/cfd_exp3d5_cuda.cu:1104-1237)
 *     -> oc_run_namelist() and the `ocean3d5_b200` executable;
 *   - the stepper object `Stepper3DV05(domain, physics, params, dt)` with
 *     `.step` / `.integrate` and its counters (libs/core/model3d_v05.py:78-545;
 *     CUDA twin Stepper5, cfd_exp3d5_cuda.cu:915-1097)
 *     -> oc_create / oc_set_domain / oc_set_forcing / oc_set_state / oc_step /
 *        oc_get_state / oc_get_stats / oc_destroy;
 *   - the variable-coefficient Helmholtz solve `HelmholtzVar.solve`
 *     (libs/core/solvers_var.py:162-197; HelmVar::solve, cfd_exp3d5_cuda.cu:374-412)
 *     -> oc_helmholtz_solve;
 *   - the batched column solve `thomas_batched` (libs/core/vertical.py:17-44;
 *     k_thomas, cfd_exp3d5_cuda.cu:450-461) -> oc_thomas;
 *   - the equation of state `buoyancy` (libs/core/eos.py:130-133; k3_eos,
 *     cfd_exp3d5_cuda.cu:818-850) -> oc_buoyancy.
 */
#ifndef OCEAN_B200_H
#define OCEAN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    OC_OK = 0,
    OC_ERR_ARG = 1,         /* invalid argument or configuration */
    OC_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    OC_ERR_UNSUPPORTED = 3, /* option the step refuses (open boundaries, moving coordinates) */
    OC_ERR_STATE = 4,       /* call out of order (no domain / no state yet) */
    OC_ERR_TIMEOUT = 5,     /* a device-side wait ran out its bound */
    OC_ERR_IO = 6,          /* file missing or of the wrong size */
    OC_ERR_TOO_LARGE = 7    /* request larger than a fixed-size buffer of the library */
};

/* option codes (the namelist strings of tools/toml2nml.py:209-264) */
enum { OC_SCHEME_FB = 0, OC_SCHEME_THETA = 1, OC_SCHEME_SPLIT = 2 };
enum { OC_SOLVER_PCG_JACOBI = 0, OC_SOLVER_PCG_RBGS = 1, OC_SOLVER_RBGS = 2, OC_SOLVER_MULTIGRID = 3 };
/* no reference counterpart: FP32 inner PCG-Jacobi inside FP64 iterative
 * refinement, for the standalone solver (oc_helm_*) and the mixed-precision step
 * (fp64 handles refuse it); the stopping test stays |b - A x| <= rtol |b| in FP64 */
enum { OC_SOLVER_PCG_REFINED = 4 };
/* no reference counterpart: CG preconditioned by one symmetric V(2,2) cycle of
 * the multigrid hierarchy, fp64, for the step (either precision, through the C
 * ABI and Python; the namelist protocol keeps the reference's four) and the
 * standalone solver. */
enum { OC_SOLVER_PCG_MG = 5 };
enum { OC_BC_PERIODIC = 0, OC_BC_CLOSED = 1 };
enum { OC_FACE_MIN = 0, OC_FACE_MEAN = 1, OC_FACE_HARMONIC = 2 };
enum { OC_EOS_LINEAR = 0, OC_EOS_SEOS = 1, OC_EOS_TEOS10 = 2 };
enum { OC_PGF_REMOVE = 0, OC_PGF_KEEP = 1 };
enum { OC_ADV_NONE = 0, OC_ADV_CENTERED2 = 1, OC_ADV_UPWIND1 = 2, OC_ADV_UP3 = 3, OC_ADV_UP3_TVD = 4 };
enum { OC_TRACERS_BUOYANCY = 0, OC_TRACERS_TS = 1 };
enum { OC_CLOSURE_NONE = 0, OC_CLOSURE_TKE = 1 };
enum { OC_MXL_INTEGRAL = 0, OC_MXL_RECURSIVE = 1 };
enum { OC_BTAVG_NONE = 0, OC_BTAVG_MEAN = 1 };
/* precision of the step (no reference counterpart: the reference's precision
 * variants are whole-program fp32 builds, libs/cuda/Makefile:77-113).
 * OC_PRECISION_FP64: every field fp64, bit-identical to the reference.
 * OC_PRECISION_MIXED: the 3D state (u, v, T, S, e, K_m, K_h) and the 3D
 * stencils and column solves in FP32; the buoyancy, its potential, the
 * pressure-gradient and EOS arithmetic, the surface elevation and every 2D
 * field (transports, the Helmholtz system and its solve) in fp64. Schemes theta
 * and fb with TS tracers. */
enum { OC_PRECISION_FP64 = 0, OC_PRECISION_MIXED = 1 };

/* Every scalar of the step; field meaning and units as the reference namelist keys. */
typedef struct oc_config {
    int32_t nx, ny, nz;
    double lx, ly;
    double g, f0, h0, n2, nu, kappa, rho0, tau_x, tau_y, bottom_drag;
    int32_t scheme;
    double theta, theta_cor, theta_v;
    int32_t n_picard, n_split, barotropic_average;
    int32_t solver;
    double rtol;
    int32_t max_iter;
    double dt;
    int32_t bc_x, bc_y, face_rule;
    double min_partial;
    int32_t eos, pgf, pgf_correction, advection, tracers;
    double alpha_t, beta_s, t0, s0, cp, a_h, k_h, q_heat, q_salt;
    int32_t closure, mxl;
    double c_k, c_eps, pr_t, z_0, e_min, l_min, e_bb, n2_min;
    int32_t device;
    int32_t precision;  /* OC_PRECISION_*; 0 (fp64) when zero-initialised */
} oc_config;

/* Pointers to one model state. eta [ny][nx]; u, v, b, T, S [nz][ny][nx];
 * e, km, kh on interfaces [nz+1][ny][nx]. T and S are ignored when
 * tracers = buoyancy. On oc_set_state a NULL e means the reference's start
 * value e_min (State3D.e is None, model3d_v05.py:175); a NULL km/kh keeps the
 * handle's current viscosity/diffusivity, which persist across steps like the
 * reference stepper's self.nu/self.kappa (nu/kappa after oc_set_domain or
 * oc_reset_mixing); a NULL b with TS tracers means "diagnose b from T and S
 * with the EOS". On oc_get_state NULL entries are skipped. */
typedef struct oc_state_view {
    double *eta, *u, *v, *b, *T, *S, *e, *km, *kh;
} oc_state_view;

/* Counters of the reference stepper (model3d_v05.py:89-94) plus run status. */
typedef struct oc_stats {
    int64_t steps;
    int64_t solver_iterations;
    int64_t solver_failures;
    int64_t solver_rebuilds;
    int64_t tridiagonal_solves;
    int64_t barotropic_substeps;
    int64_t solves;
    int32_t n_split;
    int32_t n_levels;          /* multigrid levels (1 for the other solvers) */
    int32_t diverged;          /* max|eta| >= 1e6 or NaN at the last check */
    int32_t device_status;     /* 0, or the OC_ERR_* a device-side check raised */
    int64_t device_bytes;      /* device memory held by the handle */
    int64_t kernel_launches;   /* kernels this library launched since creation / reset */
} oc_stats;

/* Accumulated device time of one kernel class (oc_set_profiling). */
typedef struct oc_kernel_time {
    char name[32];
    int64_t launches;
    double total_ms;
} oc_kernel_time;

typedef struct oc_handle oc_handle;

const char* oc_version(void);

/* Validate the configuration and bind the handle to cfg->device. */
int oc_create(const oc_config* cfg, oc_handle** out);

/* Bathymetry H and land mask [ny][nx] (host, fp64); dzr [nz] optional level
 * thicknesses (NULL = uniform max(H)/nz as the reference). Builds masks,
 * partial cells, face thicknesses and the static coefficients. */
int oc_set_domain(oc_handle* h, const double* H, const double* mask, const double* dzr);

/* One y-slab of a larger domain, for a multi-GPU run of the fb scheme
 * (reference libs/cuda/src/cfd_exp3d5_cuda_multi.cu:96-118: static arrays built
 * once on the whole domain and cut by rows, the whole domain's spacing kept).
 * H, mask, mask_u, mask_v are the larger domain's arrays at the handle's ny rows
 * (owned rows plus halo rows, wrapped periodically); the face masks carry the
 * larger domain's walls, so a wall at a slab edge stays a wall. dzr (required)
 * is the larger domain's level table, dx and dy its spacing. The handle's
 * configuration has ny = the slab's rows and scheme fb; other schemes are
 * refused (OC_ERR_UNSUPPORTED): theta needs a global elliptic solve and
 * split_explicit a halo exchange per substep. */
int oc_set_domain_slab(oc_handle* h, const double* H, const double* mask, const double* dzr,
                       const double* mask_u, const double* mask_v, double dx, double dy);

/* Halo exchange of a slab (reference cfd_exp3d5_cuda_multi.cu:133-172: k_pack /
 * k_unpack over u, v, b, T, S, eta and, with TKE, e, K_m, K_h). The exchanged
 * fields, in this order: eta, u, v, b, T and S (TS tracers), e, km, kh (TKE
 * closure). oc_halo_values_per_row gives the doubles one row of all of them
 * takes; oc_pack_rows copies rows [j0, j0 + nrows) of each field, level after
 * level, into the device buffer `buf` (values_per_row * nrows doubles), and
 * oc_unpack_rows writes such a buffer into those rows and recomputes w for the
 * velocities now in the state. Asynchronous on `stream`. */
/* Levels one CTA marches in the explicit-momentum and tracer right-hand-side
 * kernels (1..nz; 10 or nz by default). Every value gives the same results bit
 * for bit; only the speed depends on it. oc_set_tiling sets both; oc_autotune
 * times each kernel on the current state over a candidate list, keeps the
 * fastest and returns the choice (synchronous; on a mixed-precision handle it
 * times the FP32 kernels). No reference counterpart: the tile shapes of the
 * batched-ensemble form. */
int oc_set_tiling(oc_handle* h, int32_t mom_levels, int32_t tracer_levels);
int oc_autotune(oc_handle* h, int32_t* mom_levels, int32_t* tracer_levels);

/* An ensemble: several handles (members of any grid size, on one device, each
 * with its state set) advanced together. oc_ensemble_step records two steps of
 * every member into one CUDA graph -- each member on a branch of its own, its
 * kernels free to overlap the other members', the cooperative Helmholtz solves
 * of all members ordered one after another -- and replays it n_steps / 2 times
 * on `stream`; an odd last step, or any step while a member profiles, runs
 * member after member. Every member's results and counters equal those of the
 * member stepped alone. The graph is recorded again when a member's buffers,
 * forcing, tiling or solve-log capacity changed. No reference counterpart: the
 * batched-ensemble form. */
typedef struct oc_ensemble oc_ensemble;
int oc_ensemble_create(oc_handle* const* members, int32_t n_members, oc_ensemble** out);
int oc_ensemble_step(oc_ensemble* e, int32_t n_steps, void* stream);
const char* oc_ensemble_last_error(const oc_ensemble* e);
int oc_ensemble_destroy(oc_ensemble* e);

int oc_halo_values_per_row(oc_handle* h, int64_t* count);
int oc_pack_rows(oc_handle* h, int32_t j0, int32_t nrows, double* buf, void* stream);
int oc_unpack_rows(oc_handle* h, int32_t j0, int32_t nrows, const double* buf, void* stream);

/* Optional surface stress field at cell centres [ny][nx] in N m-2 (host);
 * NULL for both keeps the scalar tau_x/tau_y of the configuration. */
int oc_set_forcing(oc_handle* h, const double* taux_c, const double* tauy_c);

/* Copy a state in (on_device = 0: host pointers, 1: device pointers). */
int oc_set_state(oc_handle* h, const oc_state_view* s, int32_t on_device);

/* The same, enqueued on `stream` (cudaStream_t; NULL = legacy default stream)
 * without waiting: the source buffers must stay unchanged until the stream has
 * passed the copies, and host buffers must be pinned for the copies to overlap
 * other work. A following oc_step on the same stream sees the state. No
 * reference counterpart: the reference steps host arrays synchronously. */
int oc_set_state_async(oc_handle* h, const oc_state_view* s, int32_t on_device, void* stream);

/* Take caller-owned device buffers as the state, without a copy (fp64
 * handles; the mixed-precision step keeps FP32 fields and refuses). `a` holds
 * the state to start from: eta, u, v, b and, with TS tracers, T and S are
 * required; e, km and kh are optional (NULL keeps the handle's own arrays, e
 * then reset to e_min as oc_set_state does). `b` names a second set of eta, u,
 * v, b (and T, S) that the step writes into: the state alternates between the
 * two sets, one step each (oc_state_parity says which holds it). Every buffer
 * is device memory of this handle's device, 8-byte aligned, of the size
 * oc_set_state reads, and no two of them overlap. The handle never frees
 * them; they must outlive the handle or the next oc_bind_state. Recorded
 * graphs are dropped. Both NULL: back to the handle's own buffers (the state
 * must then be set again). Synchronises. No reference counterpart: the
 * reference's stepper returns new arrays from every step. */
int oc_bind_state(oc_handle* h, const oc_state_view* a, const oc_state_view* b);

/* Which bound set holds the current state: 0 = a, 1 = b (0 when unbound). */
int oc_state_parity(oc_handle* h, int32_t* which);

/* Restore the constant viscosity nu and diffusivity kappa of the
 * configuration (the stepper's state at construction). */
int oc_reset_mixing(oc_handle* h);

/* Copy the current state out (host or device pointers). Synchronises the stream. */
int oc_get_state(oc_handle* h, const oc_state_view* s, int32_t on_device);

/* The same, enqueued on `stream` after the work already on it, without
 * waiting; the destination is complete once the stream has passed the copies.
 * A device-side error of the steps before it is reported by the next
 * synchronous call (oc_get_state, oc_get_stats). No reference counterpart. */
int oc_get_state_async(oc_handle* h, const oc_state_view* s, int32_t on_device, void* stream);

/* Advance n_steps on `stream` (a cudaStream_t, or NULL for the legacy default stream).
 * Asynchronous: returns once the work is enqueued. */
int oc_step(oc_handle* h, int32_t n_steps, void* stream);

/* The same through CUDA graphs: two steps (one period of the state's ping-pong
 * buffers) are recorded once per starting buffer, on first use, and replayed;
 * an odd last step runs as oc_step. Results and counters are those of
 * oc_step. The first call for each buffer records (and must not itself be
 * inside a stream capture); a grown solve log, new forcing or enabled per-kernel
 * profiling make it record again or fall back to oc_step. This is the
 * graph-captured step of the reference's proposed oc_graph_capture /
 * oc_graph_launch pair, folded into one call. */
int oc_step_graph(oc_handle* h, int32_t n_steps, void* stream);

/* Wait for the handle's work, then fill the counters (synchronises). */
int oc_get_stats(oc_handle* h, oc_stats* out);

/* Per-kernel device timing: when enabled, every launch of oc_step is bracketed
 * by CUDA events on its stream. oc_get_kernel_times synchronises, returns the
 * accumulated times per kernel class and clears them. */
int oc_set_profiling(oc_handle* h, int32_t enable);
int oc_get_kernel_times(oc_handle* h, oc_kernel_time* out, int32_t capacity, int32_t* n_out);

/* Per-solve Helmholtz iteration counts since creation (or the last reset). */
int oc_get_solve_log(oc_handle* h, int32_t* iterations, int32_t capacity, int32_t* n_out);

/* Zero the counters and the solve log (the state is kept). */
int oc_reset_stats(oc_handle* h);

/* Bound of the step's device-side waits (the grid barriers of its Helmholtz
 * solve) in SM clock cycles; the default, 2e9, is about 1 s. A wait that runs
 * out sets OC_ERR_TIMEOUT in the handle's status, every CTA leaves the solve and
 * the next synchronous call (oc_get_state, oc_get_stats) returns it; the status
 * stays set. A bound of a few hundred cycles makes the waits run out, which is
 * how the failure path is tested. Recorded graphs are dropped. No reference
 * counterpart: the reference's solves have no device-side waits. */
int oc_set_wait_bound(oc_handle* h, int64_t cycles);

/* One Helmholtz solve with the current face coefficients: x = A^-1 rhs on
 * device buffers [ny][nx]. *iterations receives the count (synchronises). */
int oc_helmholtz_solve(oc_handle* h, const double* rhs, double* x, int32_t* iterations,
                       void* stream);

/* Batched tridiagonal solve on device buffers laid out [n][ncols]: one system
 * of n rows per column, sub[0] and sup[n-1] ignored. */
int oc_thomas(const double* sub, const double* diag, const double* sup, const double* rhs,
              double* x, int32_t n, int32_t ncols, void* stream);

/* The batched tridiagonal solve of oc_thomas for callers that cannot allocate
 * device memory (a host that fixes its device footprint at start-up, or an
 * asynchronous pipeline that cannot afford the device-wide synchronisation of
 * cudaMalloc/cudaFree). No counterpart in the reference. Its scratch is a fixed
 * array of OC_THOMAS_NOALLOC_MAX_CELLS doubles (8 MiB); n * ncols above that
 * returns OC_ERR_TOO_LARGE. It calls no allocator, but CUDA loads the array
 * lazily: the first call on a device commits the 8 MiB there (held until exit)
 * and looks up the array's device address, so a host with a fixed footprint
 * makes one warm-up call per device at start-up, before any stream capture.
 * The address is kept per device: do not use the library again after
 * cudaDeviceReset. An error already pending on the calling thread is returned
 * as OC_ERR_CUDA and left pending. Work is enqueued on `stream` and not waited
 * for; calls that can overlap on the GPU share the array and race, so the
 * caller serialises them. */
#define OC_THOMAS_NOALLOC_MAX_CELLS 1048576
int oc_thomas_noalloc(const double* sub, const double* diag, const double* sup, const double* rhs,
                      double* x, int32_t n, int32_t ncols, void* stream);

/* b = -g rho'(T, S, z) / rho0 on device buffers of `count` cells, with the EOS
 * and constants of the handle's configuration. */
int oc_buoyancy(oc_handle* h, const double* T, const double* S, const double* z, double* b,
                int64_t count, void* stream);

/* ---- Standalone kernels (the reference's standalone benches) --------------
 *
 * A Helmholtz solver on given depth-integrated face coefficients, replacing
 * the solver of the reference's standalone bench (libs/cuda/src/
 * helmholtz_bench.cu) on the system tools/write_helmholtz_case.py writes:
 * A = I - coef D[K G .] on an nx x ny periodic-index grid with spacings dx,
 * dy, solved by HelmholtzVar's four methods (libs/core/solvers_var.py:162-197).
 * It is the step's own solver, so the iteration counts equal NumPy's. */
typedef struct oc_helm oc_helm;
typedef struct oc_helm_config {
    int32_t nx, ny;
    double dx, dy;     /* fine-grid spacing [m]; level l uses dx * 2^l */
    double coef;       /* g theta^2 dt^2 */
    int32_t solver;    /* OC_SOLVER_* */
    double rtol;
    int32_t max_iter;
    int32_t device;
} oc_helm_config;

/* ku, kv, mask: host fp64 [ny][nx] (ku.bin, kv.bin, mask.bin of a case). */
int oc_helm_create(const oc_helm_config* cfg, const double* ku, const double* kv, const double* mask,
                   oc_helm** out);
/* x = A^-1 rhs (on_device = 0: host arrays, 1: device arrays), synchronising;
 * *iterations and *converged as HelmholtzVar's SolveReport. */
int oc_helm_solve(oc_helm* h, const double* rhs, double* x, int32_t on_device, int32_t* iterations,
                  int32_t* converged, void* stream);
const char* oc_helm_last_error(oc_helm* h);
int oc_helm_destroy(oc_helm* h);

/* Mixed-precision form of the standalone solver (cfg->solver =
 * OC_SOLVER_PCG_REFINED; no reference counterpart, the reference's precision
 * variants being whole-program fp32 builds, Makefile:77-113). The operator and
 * the Krylov vectors of an inner PCG-Jacobi are FP32; the residual b - A x, the
 * norms, the dot-product sums and the correction x += d are FP64, and the
 * stopping test is HelmholtzVar's |b - A x|_2 <= rtol |b|_2 evaluated in FP64.
 * oc_helm_solve then reports the inner iterations summed over the refinement.
 * oc_helm_refine_report gives the last solve's refinement steps and FP64
 * relative residual; oc_helm_set_inner_rtol sets the inner solves' relative
 * tolerance (default 1e-3). Both return OC_ERR_UNSUPPORTED for other solvers. */
int oc_helm_refine_report(oc_helm* h, int32_t* refinement_steps, double* relative_residual);
int oc_helm_set_inner_rtol(oc_helm* h, double inner_rtol);

/* The reference EOS bench's per-cell quantity (libs/cuda/src/eos_bench.cu over
 * libs/core/eos.py:68-127) on device buffers of `count` cells: rho' for
 * OC_EOS_LINEAR (with rho0, alpha_t, beta_s, t0, s0) and OC_EOS_SEOS, the full
 * in-situ density rho for OC_EOS_TEOS10. Asynchronous on `stream`. */
int oc_density(int32_t eos, double rho0, double alpha_t, double beta_s, double t0, double s0,
               const double* T, const double* S, const double* z, double* rho, int64_t count, void* stream);

/* Copy a static geometry or coefficient field to host memory: names "dz3",
 * "mask3", "mask3u", "mask3v", "dz3u", "dz3v", "zc" ([nz][ny][nx]), "q"
 * ([nz][ny][nx]), "ku", "kv", "mask_u", "mask_v" ([ny][nx]). */
int oc_get_field(oc_handle* h, const char* name, double* host_out, int64_t count);

/* The full backend protocol of the reference binaries: read the namelist and
 * its bundle files, run n_warmup + n_repeat repeats of n_steps, write
 * <out_prefix>_state3d5.bin and <out_prefix>_metrics.json. */
int oc_run_namelist(const char* nml_path);

/* Adjoint of one fp64 step (no reference counterpart: the reference has no
 * adjoint). Given the state before the step (x0: eta, u, v, b, T, S), the
 * state after it (x1: u, v, T, S; the step's output from x0) and the
 * cotangents of the step's outputs (x1_b: eta, u, v, b, T, S), it writes the
 * cotangents of the step's inputs into x0_b (eta, u, v, b, T, S; overwritten)
 * and adds the cotangent of the surface x-stress field at cell centres to
 * taux_b (and of the y-stress to tauy_b, when not NULL), all [ny][nx] or
 * [nz][ny][nx] fp64 device arrays. It is the transpose of the step's Jacobian:
 * the transposed column solves, a second Helmholtz solve with the same
 * (symmetric) operator, and the advection with the limiter branches the
 * forward values select. Covered: the theta scheme with TS tracers, the
 * closure off and pgf keep (OC_ERR_UNSUPPORTED otherwise). Asynchronous on
 * `stream`; its first call makes its work buffers and solver. */
int oc_adjoint_step(oc_handle* h, const oc_state_view* x0, const oc_state_view* x1, const oc_state_view* x1_b,
                    oc_state_view* x0_b, double* taux_b, double* tauy_b, void* stream);
/* The EOS's part of an initial state whose b is diagnosed from T and S:
 * T_b += b_b m3 db/dT, S_b += b_b m3 db/dS (device arrays [nz][ny][nx]). */
int oc_adjoint_eos(oc_handle* h, const double* T, const double* S, const double* b_b, double* T_b, double* S_b,
                   void* stream);

const char* oc_last_error(const oc_handle* h);

void oc_destroy(oc_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* OCEAN_B200_H */
