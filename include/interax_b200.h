/*
 * interax_b200.h -- C ABI of the B200 (sm_100a) kernels for the InteraxFF short-range path.
 *
 * The reference plugin reaches its GPU path through OpenMM's platform-kernel interface: the abstract kernels
 * CalcInteraxDispersionForceKernel, CalcInteraxExchangeForceKernel, CalcInteraxShortRangeForceKernel and
 * CalcInteraxThreeBodyForceKernel (openmmapi/include/InteraxKernels.h:51-189), each with
 *   initialize(const System&, const <Force>&)
 *   double execute(ContextImpl&, bool includeForces, bool includeEnergy)
 *   copyParametersToContext(ContextImpl&, const <Force>&)
 * implemented for CUDA by platforms/common/src/CommonInteraxKernels.cpp:139-646 and registered by
 * platforms/cuda/src/CudaInteraxKernelFactory.cpp:45-87.  This header is the flat boundary those classes (or any
 * FFI: ctypes, cgo, JNI) bind: plain pointers and sizes, no C++ or torch types.
 *
 * Conventions
 *   - Every function returns IX_OK (0) or an error code; ix_last_error() returns the message, which repeats the
 *     reference's OpenMMException text where the reference throws one.
 *   - Lengths nm, energies kJ/mol, forces kJ/mol/nm, positions double precision, row-major N x 3.
 *   - Box vectors: 9 doubles a, b, c in OpenMM's reduced form (a = (ax,0,0), b = (bx,by,0), c = (cx,cy,cz)).
 *   - A context is used from one host thread at a time; independent contexts may run concurrently.
 *   - The context owns all device memory it allocates; no caller pointer is kept after a call returns.
 */
#ifndef INTERAX_B200_H
#define INTERAX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IX_OK 0
#define IX_ERR_INVALID 1     /* illegal settings or arguments (OpenMMException in the reference) */
#define IX_ERR_CUDA 2        /* a CUDA runtime error; the message names the call */
#define IX_ERR_STATE 3       /* call made in the wrong order (e.g. compute before positions) */
#define IX_ERR_NO_DEVICE 4   /* no CUDA device, or the requested device is missing */
#define IX_ERR_MEMORY 5      /* a server's device memory budget cannot hold the allocation */

/* Nonbonded methods (InteraxPairForce.h:79-96) */
#define IX_NO_CUTOFF 0
#define IX_CUTOFF_NON_PERIODIC 1
#define IX_CUTOFF_PERIODIC 2

/* Overlap methods (InteraxExchangeForce.h:66-79) */
#define IX_OVERLAP_EXACT 0
#define IX_OVERLAP_INTERAX_ORDER2 2

/* Three-body damping methods (InteraxThreeBodyForce.h:85-96) */
#define IX_NO_DAMPING 0
#define IX_TANG_TOENNIES 1

/* Term indices of the per-term energy array */
#define IX_TERM_DISPERSION 0
#define IX_TERM_EXCHANGE 1
#define IX_TERM_SHORT_RANGE 2
#define IX_TERM_THREE_BODY 3
#define IX_NUM_TERMS 4

typedef struct ix_ctx ix_ctx;

/* Settings every pair force has (InteraxPairForce.h:70-239).  The three pair forces of one context are evaluated
 * in one fused pass over one neighbor list, so, as on the reference's CUDA platform (InteraxPairForce.h:50-53,
 * CommonInteraxKernels.h:42-46), they must have identical nonbonded methods, cutoffs and exclusions. */
typedef struct {
    int nonbonded_method;          /* IX_NO_CUTOFF, IX_CUTOFF_NON_PERIODIC, IX_CUTOFF_PERIODIC */
    double cutoff;                 /* nm */
    int use_switching_function;
    double switching_distance;     /* nm */
    double softcore_radius;        /* nm, 0 disables the soft core */
    int force_group;               /* 0..31 */
    const char* alchemical_parameter;   /* name of the context parameter; NULL = "lambda_sterics" */
    int num_exclusions;
    const int32_t* exclusions;     /* 2 x num_exclusions particle indices */
} ix_pair_settings;

/* Create a context for a System of num_particles particles on CUDA device `device`.  `box` (9 doubles) is the
 * System's default periodic box, used to validate CutoffPeriodic cutoffs as checkPairForce does
 * (openmmapi/src/InteraxPairForce.cpp:113-136); it may be NULL for non-periodic systems. */
int ix_ctx_create(int num_particles, int device, const double* default_box, ix_ctx** out);

/* Destroy a context and free its device memory. */
void ix_ctx_destroy(ix_ctx* ctx);

/* Message of the last error of `ctx`, or of the last failed ix_ctx_create when ctx is NULL. */
const char* ix_last_error(const ix_ctx* ctx);

/* Add the pair forces.  Replaces CalcInterax{Dispersion,Exchange,ShortRange}ForceKernel::initialize
 * (InteraxKernels.h:64-67, 99-102, 134-137; CUDA: CommonInteraxKernels.cpp:221-249, 304-313, 345-354).
 *   dispersion params: num_particles x 5 (m1, m2, m3, alpha, width)       InteraxDispersionForce.h:103
 *   exchange params:   num_particles x 2 (amplitude, width)                InteraxExchangeForce.h:108
 *   short range:       num_particles x 3 (k, l, width)                     InteraxShortRangeForce.h:109
 *   is_alchemical:     num_particles bytes (0/1) */
int ix_add_dispersion(ix_ctx* ctx, const ix_pair_settings* settings, const double* params,
                      const uint8_t* is_alchemical, double damping_scale, int use_long_range_correction);
int ix_add_exchange(ix_ctx* ctx, const ix_pair_settings* settings, const double* params,
                    const uint8_t* is_alchemical, int overlap_method);
int ix_add_short_range(ix_ctx* ctx, const ix_pair_settings* settings, const double* params,
                       const uint8_t* is_alchemical, int overlap_method);

/* Add the three-body force.  Replaces CalcInteraxThreeBodyForceKernel::initialize (InteraxKernels.h:169-172;
 * CUDA: CommonInteraxKernels.cpp:437-571).  Site s is the unweighted centroid of
 * site_particles[site_offsets[s] .. site_offsets[s+1]); site_params is num_sites x 3 (alpha, frequency, width);
 * molecule < 0 puts a site in a molecule of its own (InteraxThreeBodyForce.h:116-130). */
int ix_add_three_body(ix_ctx* ctx, int num_sites, const int32_t* site_offsets, const int32_t* site_particles,
                      const double* site_params, const int32_t* molecule, const uint8_t* is_alchemical,
                      double cutoff, double scale_factor, int damping_method, double damping_scale,
                      double centroid_damping_radius, int periodic, const char* alchemical_parameter,
                      int force_group);

/* Replace copyParametersToContext (InteraxKernels.h:84-85, 119-120, 154-155, 187-188; Reference semantics
 * ReferenceInteraxKernels.cpp:98-198, CUDA CommonInteraxKernels.cpp:261-375, 618-629).  The particle count, the
 * alchemical flags, the exclusions, the nonbonded method, the cutoff and the overlap method cannot change. */
int ix_update_dispersion(ix_ctx* ctx, const double* params, double damping_scale);
int ix_update_exchange(ix_ctx* ctx, const double* params, int overlap_method);
int ix_update_short_range(ix_ctx* ctx, const double* params, int overlap_method);
int ix_update_three_body(ix_ctx* ctx, const double* site_params, double scale_factor, double damping_scale,
                         double centroid_damping_radius);

/* Long-range dispersion correction coefficients of a dispersion force, as
 * InteraxDispersionForceImpl::calcLongRangeCorrection (openmmapi/src/InteraxDispersionForceImpl.cpp:86-149): the
 * correction energy is (coefficient + lambda alchemical_coefficient) / V.  Both are 0 unless the method is
 * IX_CUTOFF_PERIODIC and use_long_range_correction is set.  params and is_alchemical as in ix_add_dispersion.  Host
 * only (FP64); needs no GPU. */
int ix_dispersion_long_range_correction(int num_particles, const double* params, const uint8_t* is_alchemical,
                                        const ix_pair_settings* settings, double damping_scale,
                                        int use_long_range_correction, double* coefficient,
                                        double* alchemical_coefficient);

/* Set a context parameter (the alchemical parameters; ContextImpl::setParameter in OpenMM).  Parameters that no
 * force uses are accepted and ignored. */
int ix_set_parameter(ix_ctx* ctx, const char* name, double value);

/* Copy positions (num_particles x 3, host memory) and, for periodic systems, the box (9 doubles, may be NULL to keep
 * the previous box) to the device. */
int ix_set_positions(ix_ctx* ctx, const double* positions, const double* box);

/* Evaluate the forces whose force group is in the bit mask `groups` (execute() of every selected kernel,
 * InteraxPairForceImpl.h:84-88, InteraxThreeBodyForceImpl.cpp:64-68).  `term_energies` (may be NULL) receives the
 * energy of each term (IX_TERM_*, 0 for terms not evaluated), `energy` (may be NULL) their sum, and `forces`
 * (num_particles x 3 host doubles, may be NULL) the total force of the selected terms (overwritten). */
int ix_compute(ix_ctx* ctx, int groups, int include_forces, int include_energy, double* term_energies,
               double* energy, double* forces);

/* Device-resident variant for integration into a GPU engine: evaluate on the context's stream using the positions
 * already on the device (ix_set_positions), and ADD the forces to d_force_fixed, an int64 fixed-point buffer (scale
 * 2^32, layout x[0..stride), y[stride..2 stride), z[...]) as OpenMM's CUDA platform keeps them
 * (platforms/common/src/kernels/interaxThreeBody.cc:644-652), in original particle order.  d_term_energies
 * (device, IX_NUM_TERMS doubles, may be NULL) receives the term energies.  Nothing is copied to the host and the
 * call does not synchronize; its list-overflow status is read with ix_get_device_status. */
int ix_compute_device(ix_ctx* ctx, int groups, long long* d_force_fixed, int force_stride,
                      double* d_term_energies);

/* Device positions in and device forces out, for callers that keep their state on the GPU: d_positions is
 * num_particles x 3 doubles on the device (copied device-to-device on the context's stream), d_forces receives
 * num_particles x 3 doubles (overwritten) and d_term_energies IX_NUM_TERMS doubles.  `box` (host, 9 doubles, may be
 * NULL to keep the previous box).  Does not synchronize; status as ix_compute_device. */
int ix_compute_device_f64(ix_ctx* ctx, int groups, const double* d_positions, const double* box,
                          double* d_forces, double* d_term_energies);

/* Position formats of ix_compute_device_posq: OpenMM's posq array in single precision (float4 x, y, z, charge), in
 * mixed precision (float4 posq plus the float4 posqCorrection that holds the rounding, x = posq.x + correction.x) and
 * in double precision (double4). */
#define IX_POSQ_FLOAT4 0
#define IX_POSQ_FLOAT4_CORRECTED 1
#define IX_POSQ_DOUBLE4 2

/* The drop-in for OpenMM's CUDA platform: what CalcInterax*ForceKernel::execute does there
 * (platforms/common/src/CommonInteraxKernels.cpp:251-259 for the pair forces, 631-646 for the three-body force), with
 * positions and forces in the platform's own device arrays and nothing copied through the host.
 *   d_posq, d_posq_correction: the platform's position array(s) in its slot order (posq_format above); slot k holds
 *       particle d_atom_index[k] (the platform's atom index array; NULL: slot k holds particle k).
 *   box: host, 9 doubles, NULL to keep the previous box (the platform's periodic box vectors).
 *   d_force_fixed: the platform's int64 force buffer (scale 2^32, x/y/z rows of force_stride, the padded atom count):
 *       the forces are ADDED at each particle's slot.
 *   d_energy: a device double to which the total energy of the selected terms is ADDED (may be NULL).
 *   d_status: a device int (may be NULL) written with the list status of this call: bit 0 = the pair list
 *       overflowed and the forces and energy are incomplete; bit 1 = a three-body list overflowed (the results are
 *       complete).  After bit 0, call again: the next call (or ix_get_device_status) grows the list first.
 * Asynchronous on the context's stream (order the caller's own work with ix_get_stream).  The box, the parameter
 * values and the force-group mask are read on the host at each call. */
int ix_compute_device_posq(ix_ctx* ctx, int groups, int posq_format, const void* d_posq,
                           const void* d_posq_correction, const int32_t* d_atom_index, const double* box,
                           long long* d_force_fixed, int force_stride, double* d_energy, int* d_status);

/* Wait for the last device call of `ctx` (ix_compute_device, ix_compute_device_f64, ix_compute_device_posq) and
 * return its list status (the bits of d_status above); lists that overflowed are grown, so a repeated call is
 * complete. */
int ix_get_device_status(ix_ctx* ctx, int* status);

/* Capacities of the neighbor lists at their next allocation: pair_tiles tiles of the pair list and site_neighbors
 * entries per site of the three-body list (0: estimated from the density, the default).  Lists grow when they
 * overflow; a small capacity forces that path (the tests use it).  ix_get_list_stats returns the current capacities
 * and how many times MD steps were rerun after a pair-list overflow.  No counterpart in the reference. */
int ix_set_list_capacity(ix_ctx* ctx, long long pair_tiles, int site_neighbors);
int ix_get_list_stats(ix_ctx* ctx, long long* pair_tiles, int* site_neighbors, long long* md_reruns);

/* Counts of the last evaluation: interacting pairs (non-excluded, within the cutoff, gate true, counted once) and
 * interacting triples.  Counting costs an extra reduction, so it is done only after ix_set_counting(ctx, 1). */
int ix_set_counting(ix_ctx* ctx, int enable);
int ix_get_counts(ix_ctx* ctx, long long* num_pairs, long long* num_triples);

/* Velocity-Verlet MD on the device with the context's forces (all groups): `num_steps` steps of `dt` ps, masses
 * in amu.  Velocities (N x 3, nm/ps) are read from and written back to `velocities`; positions are written back
 * to `positions` (both may be NULL to keep the state on the device; the first call must pass both).  Returns the
 * final potential energy in *energy if not NULL. */
int ix_md_set_masses(ix_ctx* ctx, const double* masses);
int ix_md_run(ix_ctx* ctx, int num_steps, double dt, double* positions, double* velocities, double* energy);

/* Distance constraints of the MD loop (OpenMM's System::addConstraint; the rigid 3-site waters of the benchmark):
 * particles pairs[2k], pairs[2k+1] kept at distances[k] nm.  Each connected cluster of constrained particles (at most
 * 8 particles and 12 constraints) is solved by SHAKE after the drift (Newton on all of the cluster's multipliers) and
 * by RATTLE's velocity stage after the second half kick (a direct linear solve), to the relative tolerance given (on
 * the squared distance, and on the stretching rate per ps).  num_constraints = 0 removes them.  A step whose constraints did not converge makes ix_md_finish return IX_ERR_STATE. */
int ix_md_set_constraints(ix_ctx* ctx, int num_constraints, const int32_t* pairs, const double* distances,
                          double tolerance);

/* The same split in two: ix_md_steps_async enqueues `num_steps` steps on the context's stream and returns at once
 * (ix_md_run or ix_md_set_masses plus a first ix_md_run must have set the masses and velocities); ix_md_finish
 * synchronizes, checks the neighbor lists and copies the state out (any pointer may be NULL).  When the pair list
 * overflowed during the steps, ix_md_finish grows it, restores the state saved before the first unfinished
 * ix_md_steps_async and runs the steps again, so the trajectory is the one a large enough list gives. */
int ix_md_steps_async(ix_ctx* ctx, int num_steps, double dt);
int ix_md_finish(ix_ctx* ctx, double* positions, double* velocities, double* energy);

/* Kernel timing for measurement: with profiling enabled (1), CUDA events bracket the pair and three-body kernels of
 * each evaluation; ix_get_kernel_times returns the durations (ms) of the last evaluation's kernels.  Level 2 also runs
 * the three-body chain after the pair chain instead of concurrently with it, so that each bracket times its kernels
 * alone.  A measurement tool with no counterpart in the reference. */
int ix_set_profiling(ix_ctx* ctx, int enable);
int ix_get_kernel_times(ix_ctx* ctx, double* pair_ms, double* three_body_ms);

/* Number of kernels of this library launched on the context so far (a measurement aid; no counterpart in the
 * reference). */
int ix_get_launch_count(ix_ctx* ctx, long long* launches);

/* Evaluations and MD steps are captured into CUDA graphs on first use and replayed with one launch until a parameter,
 * the box, a setting or a buffer changes (default: enabled).  enable = 0 launches every kernel directly; the results
 * are identical.  No counterpart in the reference (OpenMM launches kernels one by one). */
int ix_set_graphs(ix_ctx* ctx, int enable);

/* The context evaluated at several values of one alchemical parameter (lambda windows; the other parameters keep
 * their values, and the parameter's own value is restored).  energies: num_windows x 4 term energies; forces:
 * num_windows x num_particles x 3 (may be NULL).  Host buffers, synchronous.  Every term is linear in the parameter
 * when no force that uses it has a soft core: then two evaluations (at 0 and 1) give all windows; with a soft core
 * every window is evaluated in full.  The reference evaluates one value per Context::setParameter and getState. */
int ix_compute_windows(ix_ctx* ctx, const char* parameter, int num_windows, const double* values, double* energies,
                       double* forces);

/* ix_compute_windows with the forces written to device memory: d_forces (FP64, num_windows x num_particles x 3, on
 * the context's device, or NULL).  energies stay a host buffer; returns after the forces are written. */
int ix_compute_windows_device(ix_ctx* ctx, const char* parameter, int num_windows, const double* values,
                              double* energies, double* d_forces);

/* The CUDA stream the context launches on (as a void*), so callers can order their own work around it. */
void* ix_get_stream(ix_ctx* ctx);

/* Synchronize the context's stream and report any asynchronous error. */
int ix_synchronize(ix_ctx* ctx);

/* FP32 issue peak of CUDA device `device` in TFLOP/s (an FMA counts two operations), measured by a kernel of
 * independent FMA chains on every SM: the roofline denominator of the pair and three-body kernels.  A measurement
 * tool with no counterpart in the reference. */
int ix_measure_fp32_peak(int device, double* tflops);

/* Three-body (ATM) energy and forces with no allocation at all; this entry point has no counterpart in the
 * reference.  It is for callers that cannot call cudaMalloc where they need the forces: code running while a CUDA
 * graph is being captured (allocation is not allowed inside stream capture), engines whose device memory belongs to
 * their own pool, and step loops that must not allocate.  All working memory is one fixed file-scope __device__
 * array (about 2.7 MB on every GPU that loads the library, held until the process exits) that every call shares:
 * calls that overlap on the GPU race on it, so the caller must serialize them (one stream per device, or an event
 * between them).  Limits: 16384 particles and 4096 sites (larger inputs are rejected with IX_ERR_INVALID); a site
 * with more than 128 sites above it within the cutoff does not fit its neighbor list and is evaluated by scanning
 * every later site instead (slower, same result), which ix_three_body_noalloc_overflow reports.
 * Inputs and outputs are device pointers on the current CUDA device: d_positions (num_particles x 3 doubles), the
 * sites as in ix_add_three_body (site particle indices outside [0, num_particles) are ignored), d_forces
 * (num_particles x 3 doubles, overwritten with the three-body forces) and d_energy (one double).  `box` is a host
 * pointer (9 doubles, may be NULL when not periodic) and `stream` a cudaStream_t (NULL: the default stream).  The box
 * and the scalar arguments (cutoff, lambda, ...) are passed to the kernels by value when the call is made: a call
 * captured into a CUDA graph keeps them, and a graph replayed after the box or lambda changed uses the old values,
 * so capture it again after such a change.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) once and keeps it for the life of the process; make that first call before any stream
 * capture, and make no call after a cudaDeviceReset of that device.  The call is asynchronous on `stream`. */
int ix_three_body_noalloc(int num_particles, const double* d_positions, const double* box, int num_sites,
                          const int32_t* d_site_offsets, const int32_t* d_site_particles,
                          const double* d_site_params, const int32_t* d_molecule, const uint8_t* d_is_alchemical,
                          double cutoff, double scale_factor, int damping_method, double damping_scale,
                          double centroid_damping_radius, int periodic, double lambda, double* d_forces,
                          double* d_energy, void* stream);

/* Whether a site of the last ix_three_body_noalloc call on the current device had more neighbors than its list holds
 * (its triples were found by a full scan, so the results are complete).  Waits for the whole device
 * (cudaDeviceSynchronize), so that the flag of a call made on any stream has been written. */
int ix_three_body_noalloc_overflow(int* overflow);

/* Library version string. */
const char* ix_version(void);

/* ---- Batches of independent small systems -------------------------------------------------------------------------
 * Many non-periodic systems (clusters, dimer scans, copies at several lambda values) evaluated together: one static
 * launch sequence over all of them, captured once into a CUDA graph.  The systems are described like contexts (the
 * ix_batch_add_* functions take the arguments of the ix_add_* functions plus the system index and validate them the
 * same way); every system must carry the same forces with the same settings, and only particle parameters,
 * exclusions and three-body sites may differ.  Positions and forces are the systems' particles concatenated in system
 * order (3 doubles each); energies are 4 per system (dispersion, exchange, short range, three-body, kJ/mol).  Each
 * system's results are the same alone or in any batch.  The reference evaluates one System per Context; this is the
 * batched form of that evaluation, with no counterpart there. */
typedef struct ix_batch ix_batch;

int ix_batch_create(int device, ix_batch** out);
void ix_batch_destroy(ix_batch* batch);
const char* ix_batch_last_error(const ix_batch* batch);
int ix_batch_add_system(ix_batch* batch, int num_particles, int* system);
int ix_batch_add_dispersion(ix_batch* batch, int system, const ix_pair_settings* settings, const double* params,
                            const uint8_t* is_alchemical, double damping_scale, int use_long_range_correction);
int ix_batch_add_exchange(ix_batch* batch, int system, const ix_pair_settings* settings, const double* params,
                          const uint8_t* is_alchemical, int overlap_method);
int ix_batch_add_short_range(ix_batch* batch, int system, const ix_pair_settings* settings, const double* params,
                             const uint8_t* is_alchemical, int overlap_method);
int ix_batch_add_three_body(ix_batch* batch, int system, int num_sites, const int32_t* site_offsets,
                            const int32_t* site_particles, const double* site_params, const int32_t* molecule,
                            const uint8_t* is_alchemical, double cutoff, double scale_factor, int damping_method,
                            double damping_scale, double centroid_damping_radius, int periodic,
                            const char* alchemical_parameter, int force_group);
int ix_batch_set_parameter(ix_batch* batch, const char* name, double value);
int ix_batch_num_particles(const ix_batch* batch, int* num_particles, int* num_systems);
/* Host buffers; synchronous.  The first call (and the first after a change) builds the device arrays and the graph. */
int ix_batch_compute(ix_batch* batch, const double* positions, double* forces, double* energies);
/* Device buffers (any may be NULL), asynchronous on the batch's stream. */
int ix_batch_compute_device(ix_batch* batch, const double* d_positions, double* d_forces, double* d_energies);
int ix_batch_get_counts(ix_batch* batch, long long* num_pairs, long long* num_triples);
void* ix_batch_get_stream(ix_batch* batch);
/* Velocity-Verlet MD of every system at once (host buffers, synchronous): system s takes steps[s] steps of dt ps and
 * then stays put.  masses: one per particle (amu); positions and velocities (NULL = at rest) are updated in place;
 * forces and energies (may be NULL) are those of the final positions.  Each system's trajectory is the same alone or
 * in any batch. */
int ix_batch_md_run(ix_batch* batch, const int* steps, double dt, const double* masses, double* positions,
                    double* velocities, double* forces, double* energies);

/* ---- Served requests -----------------------------------------------------------------------------------------------
 * A request server for a stream of independent energy+force / MD requests of mixed sizes on one GPU.  A native worker
 * thread admits requests while their estimated device memory fits the budget (an arena of that size holds every
 * admitted request's state, so a request that does not fit waits until others finish), keeps each admitted request's
 * positions, parameters and neighbor lists resident on the device until its last step, and overlaps the work of all
 * admitted requests: periodic systems run as contexts on their own streams, small non-periodic systems with the same
 * force settings are gathered into batched cohorts (one CUDA graph per MD step for the whole cohort).  Requests
 * admitted while others run join as soon as memory and a slot are free (continuous batching).  A request's result is
 * the same as that of the request run alone.  No counterpart in the reference, which evaluates one Context at a time.
 *
 * A request is described like a context, on the host only: ix_request_create, the ix_add_* functions on it,
 * ix_request_set_state, then ix_server_submit (which takes ownership). */
typedef struct ix_server ix_server;

typedef struct {
    long long submitted, admitted, completed, failed;
    long long contexts, cohorts;              /* units launched: single-request contexts and batched cohorts */
    long long pending, running;               /* requests waiting for admission, requests admitted and not done */
    double budget_bytes, reserved_bytes, peak_reserved_bytes, arena_bytes, peak_arena_bytes;
    /* worker thread seconds: context set-up, context enqueue, cohort build, cohort enqueue, unit teardown, event
     * checks, admission scans, idle waits; within set-up and enqueue: pinned staging, device set-up, state uploads,
     * the steps' launches */
    double worker_seconds[12];
    long long contexts_reused;                /* contexts taken from the pool of finished requests' contexts */
} ix_server_stats;

/* A host-only request description of num_particles particles (box: 9 doubles, NULL for non-periodic). */
int ix_request_create(int num_particles, const double* box, ix_ctx** out);
/* Starting state: positions (n x 3, required), velocities (n x 3, NULL = at rest), masses (n, required for MD). */
int ix_request_set_state(ix_ctx* request, const double* positions, const double* velocities, const double* masses);
/* threads: native worker threads (1..64) that launch and collect requests in parallel; max_running: requests
 * admitted at once, over all threads. */
int ix_server_create(int device, double budget_bytes, int max_running, int threads, ix_server** out);
/* Cohorts: non-periodic requests of at most small_atoms particles are batched, up to max_cohort per cohort; a cohort
 * starts when it is full, when its oldest request has waited window_seconds, or when the GPU is idle. */
int ix_server_set_batching(ix_server* server, int small_atoms, int max_cohort, double window_seconds);
void ix_server_destroy(ix_server* server);
const char* ix_server_last_error(const ix_server* server);
/* Queue a request for `steps` velocity-Verlet steps of dt ps (0 steps: one energy+force evaluation).  On success the
 * server owns `request` and *id identifies it. */
int ix_server_submit(ix_server* server, ix_ctx* request, int steps, double dt, long long* id);
/* Ids of requests completed since the last poll or wait (up to max_ids); wait blocks until one completes or the
 * timeout passes. */
int ix_server_poll(ix_server* server, int max_ids, long long* ids, int* count);
int ix_server_wait(ix_server* server, double timeout_seconds, int max_ids, long long* ids, int* count);
/* Result of a completed request, then released: final positions, velocities, forces (n x 3 each, may be NULL),
 * term energies (4, may be NULL) and the seconds from submission to completion.  Returns the request's own status
 * (its error message in ix_server_last_error). */
int ix_server_result(ix_server* server, long long id, double* positions, double* velocities, double* forces,
                     double* term_energies, double* latency_seconds);
int ix_server_stats_get(ix_server* server, ix_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* INTERAX_B200_H */
