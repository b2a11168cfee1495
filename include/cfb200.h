/*
 * cfb200.h -- C ABI of the B200 CNRK2 engine for ChannelFlow.jl's time step.
 *
 * The engine replaces the device path of the reference's CNRK2 `step!`
 * (src/timesteppers/cnrk2.jl:149-207): the nonlinear term in any of its
 * three forms (src/nonlinear.jl:113-199), the batched influence/tau Stokes
 * solve (src/solvers/stokes.jl:81-108, batchedinfluence.jl:101-160,
 * meanmode.jl:103-150) and the padded Fourier-Chebyshev transforms
 * (src/ffts.jl:65-82, 151-166, 242-312; src/transforms/chebyshev.jl:45-66).
 * The reference reaches that path through Julia dispatch on CuArray storage
 * (ext/ChannelFlowCUDAExt.jl:7-32); a Julia host calls these functions with
 * `ccall` instead.  All functions returning int return 0 on success and a
 * negative CF_E_* code on failure; cf_last_error() describes the last failure
 * of the calling thread.
 *
 * Field layout (identical to Julia's ComplexF64 arrays of size (Nx/2+1, Nz, Ny)):
 * complex128 interleaved (re, im), k fastest, then l (FFT order), then the
 * Chebyshev degree n.  A velocity is three such fields back to back.
 * One handle owns its device memory and one CUDA stream; it is not reentrant
 * (the reference's workspaces "must not be used concurrently", cnrk2.jl:147).
 * A handle belongs to the device that was current at cf_create; every entry
 * point makes that device current for its duration and restores the caller's.
 */
#ifndef CFB200_H
#define CFB200_H
#ifdef __cplusplus
extern "C" {
#endif

#define CF_OK 0
#define CF_E_ARG -1       /* invalid argument: ArgumentError/DimensionMismatch (cnrk2.jl:60, 157-164; stokes.jl:35-38) */
#define CF_E_SINGULAR -2  /* singular influence matrix (batchedinfluence.jl:75-76) */
#define CF_E_NOMEM -3     /* device allocation failed */
#define CF_E_CUDA -4      /* CUDA runtime error, or a bounded kernel wait that gave up */
#define CF_E_UNSUPPORTED -5 /* size outside the engine's transform limits */
#define CF_E_NONFINITE -6 /* the state went non-finite (the abort of examples/mkm590/run.jl:225-226) */

#define CF_PROFILE_COUETTE 0    /* Ub(y) = y        (CouetteFlow, problem.jl:122-123) */
#define CF_PROFILE_POISEUILLE 1 /* Ub(y) = 1 - y^2  (PoiseuilleFlow, problem.jl:137-144) */
#define CF_PROFILE_VALUES 2     /* Ub given at the Ny Lobatto points y_j = cos(pi j/(Ny-1)) (grids.jl:27-30) */

#define CF_CONSTRAINT_PRESSUREGRADIENT 0 /* (dPdx, dPdz) prescribed */
#define CF_CONSTRAINT_BULKVELOCITY 1     /* total bulk velocities (Ubulk, Wbulk) prescribed */

/* Precision of the step.  FP64: the plain form, every operation in double
 * precision (parity with the reference's step!).  MIXED: the nonlinear term's
 * periodic transforms and products in FP32 (its nodal fields stored in FP32);
 * Chebyshev transforms, right-hand side, tau Helmholtz solves,
 * influence-matrix and tau corrections, mean mode and flux constraint stay
 * FP64, as does the state.  MIXED_TC: as MIXED with the Chebyshev transforms
 * as tensor-core contractions (TF32 heads and remainders, FP32 accumulation)
 * between FP32 coefficient and nodal fields; Ny <= 512.  MIXED_BF16: as
 * MIXED_TC with the contractions on the BF16 tensor cores, each operand
 * split into three BF16 pieces (24 significant bits) and the six products of
 * order >= 2^-16 accumulated in FP32.  MIXED_F32STATE: as MIXED with the
 * state (velocity, pressure and the RK history) stored in FP32 in device
 * memory; every stage widens it to FP64 for the right-hand side, the tau
 * Helmholtz solves, the influence-matrix and tau corrections, the mean mode
 * and the flux constraint, and rounds the new state to FP32.  The state
 * crosses the C ABI in FP64 as for every precision (cf_set_state rounds it,
 * cf_get_state widens it); cf_step_host runs as cf_set_state + cf_step +
 * cf_get_state, and cf_step_dt is not supported (CF_E_UNSUPPORTED). */
#define CF_PRECISION_FP64 0
#define CF_PRECISION_MIXED 1
#define CF_PRECISION_MIXED_TC 2
#define CF_PRECISION_MIXED_BF16 3
#define CF_PRECISION_MIXED_F32STATE 4

/* Nonlinear form of NonLinearTerm(...; form) (src/nonlinear.jl:11-17, 113-199).
 * ROTATIONAL: u x curl(u) with the modified pressure (the default);
 * CONVECTIVE: -(u.grad)u; DIVERGENCE: -div(u u).  The last two carry the
 * ordinary pressure (pressure.jl:86-93).  The mixed precision and ensembles
 * run the rotational form only. */
#define CF_FORM_ROTATIONAL 0
#define CF_FORM_CONVECTIVE 1
#define CF_FORM_DIVERGENCE 2

typedef struct cf_config {
    int Nx, Ny, Nz;      /* Grid(Nx, Ny, Nz, Lx, Lz): grids.jl:27-30 */
    double Lx, Lz;
    double nu, dt;       /* CNRK2(grid, baseflow, nu, dt): cnrk2.jl:58-82 */
    int profile;         /* CF_PROFILE_* */
    const double* base_values; /* Ny values when profile == CF_PROFILE_VALUES */
    int constraint;      /* CF_CONSTRAINT_* (problem.jl:81-87) */
    double c1, c2;       /* gradients or bulk velocities */
    int precision;       /* CF_PRECISION_* (0: FP64 plain form) */
    int form;            /* CF_FORM_* (0: rotational) */
} cf_config;

typedef struct cf_engine cf_handle;

/* ChannelFlowProblem(grid, profile, nu, dt; constraint) + adapt(CuArray, problem)
 * (problem.jl:69-107, ext/ChannelFlowCUDAExt.jl:18-32). */
int cf_create(const cf_config* cfg, cf_handle** out);
void cf_destroy(cf_handle* h);

/* Replace the constraint used by later steps (the step! keywords
 * pressuregradient / bulkvelocity, cnrk2.jl:149-158). */
int cf_set_constraint(cf_handle* h, int kind, double c1, double c2);

/* adapt(CuArray, state) / Array(...) (src/adapt.jl:6-11): host buffers of
 * 3*Nr and Nr complex128 values, Nr = (Nx/2+1)*Nz*Ny.  P may be NULL in get. */
int cf_set_state(cf_handle* h, const double* U, const double* P);
int cf_get_state(cf_handle* h, double* U, double* P);
/* The same with device pointers (no host copy). */
int cf_set_state_device(cf_handle* h, const void* U, const void* P);
int cf_get_state_device(cf_handle* h, void* U, void* P);

/* step!(scheme, nlterm, U, P, t; constraint...) repeated nsteps times on the
 * engine state (cnrk2.jl:149-207).  *t_out = t + nsteps*dt; grads_out
 * (may be NULL) receives the last stage's (dPdx, dPdz), the value solve!
 * returns (stokes.jl:100-107).  Only NoForcing is supported (forcing.jl:9-11).
 * Asynchronous when grads_out is NULL; with grads_out the call waits and
 * reports CF_E_NONFINITE if the state went non-finite in any stage since the
 * last check (the flag is then cleared; cf_sync reports it as well). */
int cf_step(cf_handle* h, double t, int nsteps, double* t_out, double* grads_out);

/* One step! of duration dt from t: the Flows adapter's step
 * (ext/ChannelFlowFlowsExt.jl:36-52), which Flows calls with a shortened dt to
 * end an interval between nominal steps.  dt equal to the nominal step is
 * cf_step(h, t, 1, ...); any other dt runs with Stokes factors built for it
 * (the adapter's temporary CNRK2, :45) on the first call with that dt and kept
 * for repeated calls, while the nominal factors stay in place.
 * *t_out = t + dt. */
int cf_step_dt(cf_handle* h, double t, double dt, double* t_out, double* grads_out);

/* step!(scheme, nlterm, U, P, t; ...) on host fields (CPU arrays of the
 * layout of cf_set_state; cnrk2.jl:149-207): the engine state becomes U, P,
 * nsteps steps run, and the new state is written back into U, P.  Equal to
 * cf_set_state + cf_step + cf_get_state, with the transfers overlapped with
 * the first and last column kernels (kz-plane chunks on a copy stream).
 * Pinned buffers give full PCIe bandwidth.  *t_out, grads_out as cf_step. */
int cf_step_host(cf_handle* h, double* U, double* P, double t, int nsteps, double* t_out, double* grads_out);

/* NonLinearTerm(t, U, N) of the handle's form on host buffers
 * (nonlinear.jl:113-199, _store_rhs! :200-208). */
int cf_nonlinear(cf_handle* h, const double* U, double* N);

/* Chebyshev transform of many FP32 columns on the tensor cores (the kernel of
 * the mixed-precision path), on host buffers: X and Y hold nfields arrays of
 * Ny rows of C floats (a complex field read as real columns).  inverse != 0:
 * coefficients -> values at the Lobatto nodes (plan_icheb with doubled
 * endpoints, chebyshev.jl:32-66, and the 1/2 of copy_to_padded!,
 * ffts.jl:162); inverse == 0: nodal values -> coefficients times `scale`
 * with the endpoint halving (plan_cheb and normalize_forward!,
 * ffts.jl:254-269).  TF32 operands split in heads and remainders (three
 * products), FP32 accumulation: ~FP32 accuracy.  2 <= Ny <= 512, nfields <= 6. */
int cf_cheb_transform(const float* X, float* Y, int Ny, long C, int nfields, int inverse, double scale);
/* The same with a chosen operand split: 0 TF32 heads and remainders (as
 * cf_cheb_transform), 1 three BF16 pieces with six BF16 products; both
 * accumulate in FP32 and reach ~FP32 accuracy. */
int cf_cheb_transform_split(const float* X, float* Y, int Ny, long C, int nfields, int inverse, double scale,
                            int split);

/* ---- Ensembles: many independent channels advanced together ----------------
 * The reference advances one channel per step! call (cnrk2.jl:149-207); an
 * ensemble of N instances (each its own grid, nu, dt, constraint and state)
 * is stepped here with one CUDA graph per step.  The instances are ordinary
 * handles owned by the ensemble: set and read their state, random_state,
 * diagnostics and (one at a time) cf_step through cf_batch_instance().  Work
 * queued through an instance handle completes before the next cf_step_batch;
 * later instance calls wait for the ensemble. */
typedef struct cf_batch cf_batch;
int cf_create_batch(const cf_config* cfgs, int n, cf_batch** out);
void cf_destroy_batch(cf_batch* b);
int cf_batch_size(cf_batch* b);
/* borrowed handle of instance i (owned by the ensemble; NULL if out of range) */
cf_handle* cf_batch_instance(cf_batch* b, int i);
/* nsteps CNRK2 steps of every instance (step! per instance, cnrk2.jl:149-207); asynchronous */
int cf_step_batch(cf_batch* b, int nsteps);
/* kernel launches issued by the last cf_step_batch */
int cf_batch_last_launch_count(cf_batch* b);
/* the ensemble's CUDA stream (cudaStream_t) */
void* cf_batch_stream(cf_batch* b);
/* The launch schedule the ensemble's autotuner chose at cf_create_batch, as
 * text: per size class the z kernels' transforms per block, the x-pass rows
 * per block, the column kernel's variant (columns per block, register bound)
 * and its schedule (one block per column block of every instance, or a
 * persistent grid claiming the items in order), with the timings of every
 * candidate.  Writes at most cap - 1 characters and a NUL; returns
 * the number written. */
int cf_batch_schedule(cf_batch* b, char* buf, int cap);

/* cf_nonlinear without allocating: U and N are staged in a fixed
 * module-scope device array of CF_NOALLOC_SCRATCH_BYTES (16 MiB) instead of
 * buffers that cf_nonlinear allocates on its first call.  No counterpart in
 * the reference: an addition of this library for callers that must not
 * allocate device memory once they run (a host whose allocator is frozen or
 * accounted, e.g. inside another framework's memory pool or a
 * graph-replayed loop).  Limit: 3 * Nr * 16 bytes <= 16 MiB, i.e.
 * Nr = (Nx/2+1) * Nz * Ny <= 349525; larger grids return CF_E_ARG.  The
 * array is one per device for the whole process, held from module load until
 * exit, and its address is looked up by cf_create with the handle's device
 * current.  Every call shares the array and leaves its contents behind: calls
 * through different handles (or streams) on one device must not overlap; the
 * caller serialises them. */
#define CF_NOALLOC_SCRATCH_BYTES (16u << 20)
int cf_nonlinear_noalloc(cf_handle* h, const double* U, double* N);

/* project!(U, problem) on a host velocity, in place (pressure.jl:36-54). */
int cf_project(cf_handle* h, double* U);
/* pressure(U, problem) (pressure.jl:95-104): modified pressure of U. */
int cf_pressure(cf_handle* h, const double* U, double* P);

/* random_state(problem, epsilon) analogue (initialization.jl:32-51): seeded
 * spectral Gaussian perturbation with amplitude amp and spectrum `shape` (0:
 * exp(-(|k|+|l|)/4) exp(-n/4); 1: (1+k^2+l^2)^-1 rho^n), conjugate symmetric
 * on k = 0, then project! and pressure.  Sets the engine state. */
int cf_random_state(cf_handle* h, unsigned long long seed, double amp, int shape, double rho);

/* Diagnostics of the engine's perturbation velocity, computed on the device
 * (one column team per Fourier mode; five doubles come back): out[0]
 * kinetic_energy (postprocessing.jl:80), out[1] dissipation_rate nu<|curl
 * u|^2> (:91-111), out[2] max |div u| coefficient, out[3] nu du/dy(+1) and
 * out[4] nu du/dy(-1) of the (0,0) mode. */
int cf_diagnostics(cf_handle* h, double* out);

/* power_input(U, nu; pressuregradient=(dPdx, dPdz)) (postprocessing.jl:113-128)
 * of the engine's velocity: nu/2 [u . du/dy] between the walls minus the
 * gradient's work on the bulk velocity, from the (0,0) mode.  with_base != 0
 * adds the base profile to the streamwise mean first (the total-flow input,
 * laminar_power_input at :175-181 for a zero perturbation). */
int cf_power_input(cf_handle* h, int with_base, double dPdx, double dPdz, double* out);

/* step! repeated nsteps times (as cf_step) with the flow's diagnostics
 * recorded on the device after every `every` steps, with no host
 * synchronisation until the end: the monitoring a production run does
 * between steps (`record`, examples/mkm590/run.jl:221-256, with the quantities of
 * postprocessing.jl:80-128).  series receives nsteps/every rows of 9
 * doubles: t, kinetic energy, dissipation rate, max |div u|, nu du/dy(+1) and
 * nu du/dy(-1) of the (0,0) mode (cf_diagnostics' five values), the step's
 * last mean gradients (dPdx, dPdz) and the total-flow power input with those
 * gradients (cf_power_input with the base profile).  Waits for the steps;
 * reports CF_E_NONFINITE as cf_step with grads_out does. */
int cf_step_record(cf_handle* h, double t, int nsteps, int every, double* series, double* t_out,
                   double* grads_out);

/* step! like cf_step without the CUDA graph, with CUDA events around every
 * kernel class; kernel_ms[0..5] receives the summed device time of the
 * z-inverse, x-pass, z-forward and column kernels and (mixed precision) the
 * forward and inverse tensor-core Chebyshev transforms over the nsteps steps. */
int cf_step_profiled(cf_handle* h, double t, int nsteps, double* t_out, double* kernel_ms);

/* Block until the handle's stream is idle; reports a non-finite state or a
 * kernel wait that gave up since the last check (then clears it). */
int cf_sync(cf_handle* h);
/* Number of kernel launches issued by the most recent cf_step call. */
int cf_last_launch_count(cf_handle* h);
/* Device stream of the handle (cudaStream_t), for callers that time on it. */
void* cf_stream(cf_handle* h);
/* Device memory held by the handle, in bytes (every allocation it made). */
long long cf_device_bytes(cf_handle* h);

/* Test hook: the number of polls after which the first bounded wait of a
 * TMA or tensor-core kernel gives up (negative: the default, 2^22).  A wait
 * that gives up makes the call return CF_E_CUDA instead of hanging; the
 * kernel still lets its own copies in flight land before it exits, so the
 * handle stays usable.  Not for production use. */
int cf_set_wait_limit(cf_handle* h, long spins);

const char* cf_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
