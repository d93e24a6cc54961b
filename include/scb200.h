/* scb200.h -- C ABI of the B200 SuperConga self-consistency engine.
 *
 * One handle is one self-consistency context: the grain, the Fermi surface,
 * the Ozaki energies and all iteration state live on one GPU.  Host buffers use
 * the reference's planar layout (GridData.h:276-291): every field is an N0 x N0
 * row-major plane (index y*N0 + x); a complex field is its real plane followed
 * by its imaginary plane; order-parameter components are ordered as the
 * reference driver adds them (dx2-y2, dxy, g, s; src/simulation.cu:213-290).
 * The induced vector potential is in the reference's internal units, i.e.
 * multiplied by lambda^2 (src/simulation.cu:368-373).
 *
 * Every function returns 0 on success and a negative status on error; the
 * message is available from sc_last_error().  Nothing here exits or throws.
 * A handle is not thread-safe; all its work is issued on one CUDA stream.
 */
#ifndef SCB200_H_
#define SCB200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sc_ctx sc_ctx;

#define SC_OK 0
#define SC_ERR_ARG -1     /* invalid argument or configuration */
#define SC_ERR_CUDA -2    /* CUDA runtime error (allocation, launch) */
#define SC_ERR_STATE -3   /* call not valid in the current state */
#define SC_ERR_SIZE -4    /* problem larger than the fixed scratch of sc_poisson_noalloc */

#define SC_MODE_FP64 0    /* complex FP64 end to end */
#define SC_MODE_MIXED 1   /* FP32 Riccati stepping, FP64 accumulation */

/* Creates a context from a reference JSON configuration (the file
 * simulation_f64 reads; src/simulation.cu:64-463 builds the same objects).
 * Replaces: the Context, Parameters, GeometryGroup, IntegrationIteratorOzaki,
 * OrderParameter, compute-object and RiccatiSolverConfined set-up of
 * src/simulation.cu:95-463 and Context::initialize (include/conga/Context.h:285-375).
 * The order parameter starts at zero; set it with sc_set_state. */
int sc_create(const char *config_json, int mode, sc_ctx **out);

/* Frees the context and all its device memory. */
int sc_destroy(sc_ctx *ctx);

/* Last error message of ctx (or of the last failed sc_create if ctx is NULL). */
const char *sc_last_error(const sc_ctx *ctx);

/* Lattice sizes: N0 (reference grid), N1 (trajectory frame), Fermi angles,
 * Ozaki energies, order-parameter components
 * (Parameters.h:48-50, IntegrationIteratorOzaki.h:207-210). */
int sc_get_dims(const sc_ctx *ctx, int *n0, int *n1, int *n_angles, int *n_energies,
                int *n_comp);

/* In-grain Riccati site-updates per iteration: 2 * Ne * sum_angles #{label > 0}. */
int sc_site_updates(const sc_ctx *ctx, long long *per_iteration);

/* Sets x = (order parameter [Nc][2][N0][N0], vector potential [2][N0][N0]),
 * host buffers.  a may be NULL (zero).  The order parameter is zeroed outside
 * the grain as OrderParameter::initialize does (OrderParameter.h:180-199).
 * Replaces the load_path injection of src/simulation.cu:300-377. */
int sc_set_state(sc_ctx *ctx, const double *delta, const double *a_internal);

/* Reads x back (host buffers, same layout). */
int sc_get_state(sc_ctx *ctx, double *delta, double *a_internal);

/* Runs n self-consistency iterations (Context::compute, Context.h:391-447):
 * accelerator step (from the second iteration on), Riccati sweep and Green
 * accumulation for all angles, boundary condition, vector potential.  On
 * return *residual holds Context::getResidual and *converged
 * Context::isPartiallyConverged of the last iteration.  Either may be NULL.
 * Under a stream capture by the caller (ctx's stream, sc_set_stream, is being
 * captured into a CUDA graph) the n iterations are only recorded into the
 * caller's graph; nothing is read back or synchronised, so *residual and
 * *converged are left unchanged (read them with sc_get_scalars after the graph
 * has run).  Only a steady iteration can be recorded: at least one iteration
 * must have run outside the capture, with profiling off and not on a batch
 * grain; otherwise SC_ERR_STATE is returned and nothing is recorded.  Every
 * other call that returns host data synchronises and is not available under
 * capture (sc_burn_in returns SC_ERR_STATE). */
int sc_compute(sc_ctx *ctx, int n, double *residual, int *converged);

/* Runs n burn-in iterations (Context::burnIn, Context.h:377-389): boundary
 * coherence functions only.  *residual is the boundary residual. */
int sc_burn_in(sc_ctx *ctx, int n, double *residual, int *converged);

/* g(x) of the last iteration: new order parameter [Nc][2][N0][N0], current
 * density [2][N0][N0] (ComputeCurrent::getResult), new vector potential
 * [2][N0][N0] (internal units).  Any pointer may be NULL. */
int sc_get_results(sc_ctx *ctx, double *delta_new, double *j, double *a_new);

/* out[0..10]: free energy, free energy per area, magnetic free energy,
 * magnetic free energy per area, residuals of order parameter, current, free
 * energy, vector potential and boundary, total residual, grain lattice sites
 * (ComputeFreeEnergy.h:281-414, Context.h:462-483). */
int sc_get_scalars(sc_ctx *ctx, double *out);

/* Sets the CUDA stream (cudaStream_t) all work of ctx is issued on. */
int sc_set_stream(sc_ctx *ctx, void *stream);

/* Device-pointer variants of sc_set_state / sc_get_state for callers whose
 * data already lives on the context's GPU (same layouts, FP64). */
int sc_set_state_device(sc_ctx *ctx, const double *d_delta, const double *d_a_internal);
int sc_get_state_device(sc_ctx *ctx, double *d_delta, double *d_a_internal);

/* ---- frozen-boundary evaluation and its adjoint --------------------------- */

/* No counterpart in the reference (its drivers have no derivative); these
 * replace a finite-difference loop around Context::compute (Context.h:391-447).
 * The functional is one pass of the self-consistency map with the incoming
 * boundary values held fixed (IntegrationIteratorOzaki.h:302-404 without the
 * boundary update):
 *   L(Delta, A, B_ext) = w_omega * Omega + sum_r beta(r) . j(r)
 * with Omega the free energy of ComputeFreeEnergy.h:281-414 and j the current
 * of ComputeCurrent.h:175-222.  FP64 self-consistency contexts only (others
 * return SC_ERR_STATE); the boundary values must be set (an iteration, a
 * burn-in or sc_boundary_initial). */

/* Sets the external field B_ext in units of B0 (the reference's
 * external_flux_quanta Phi = B_ext * area / pi, RiccatiSolver.h:137-139). */
int sc_set_external_field(sc_ctx *ctx, double b_ext);
int sc_get_external_field(const sc_ctx *ctx, double *b_ext);

/* One frozen-boundary pass at the current state: *free_energy = Omega;
 * sc_get_results then returns that pass's Delta, j and A. */
int sc_evaluate(sc_ctx *ctx, double *free_energy);

/* Reverse-mode derivative of L at the current state (checkpointed adjoint
 * Riccati sweeps, gamma kept every 16 sites).  beta_j [2][N0][N0] host (NULL:
 * no current term); outputs, host, any may be NULL: g_delta [Nc][2][N0][N0]
 * = dL/dRe Delta, dL/dIm Delta; g_a [2][N0][N0] = dL/dA (internal units);
 * *g_b = dL/dB_ext. */
int sc_adjoint(sc_ctx *ctx, double w_omega, const double *beta_j, double *g_delta, double *g_a,
               double *g_b);

/* ---- probes used by the parity tests ------------------------------------ */

/* Frame geometry of one angle: labels [N1*N1] (0 out, 1 in, 2 entry, 3 exit)
 * and the trajectory box {x0, x1, y0, y1}
 * (GeometryGroup::create(-theta), BoundaryStorage.h:265-350). */
int sc_get_frame_labels(const sc_ctx *ctx, int angle, signed char *labels, int *box);

/* Reference-frame domain [N0*N0] (GeometryGroup::createDomain). */
int sc_get_domain(const sc_ctx *ctx, signed char *domain);

/* Sizes of the sparse boundary storage: in/out for gamma, in/out for
 * gammaTilde (BoundaryStorage.h:440-490). */
int sc_boundary_sizes(const sc_ctx *ctx, int *sizes);

/* How the angles are swept: the number of angle chunks (the sweep scratch and
 * frame buffers of all angles are held within a device-memory budget, 35% of
 * the free memory at creation or SCB_SCRATCH_MB; one chunk unless a grain is
 * too large) and whether mixed mode pairs each angle with its mirror angle
 * theta + pi (one sweep serves both).  Either pointer may be NULL. */
int sc_sweep_plan(const sc_ctx *ctx, int *n_chunks, int *paired);

/* Boundary coherence values, interleaved (re, im), count*Ne complex values.
 * which: 0 in-gamma, 1 out-gamma, 2 in-gammaTilde, 3 out-gammaTilde. */
int sc_get_boundary(sc_ctx *ctx, int which, double *values);
int sc_set_boundary(sc_ctx *ctx, int which, const double *values);

/* Sets the boundary initial condition (homogeneous solutions at the exit
 * nodes followed by the boundary condition),
 * IntegrationIteratorOzaki::setBoundaryInitialCondition
 * (IntegrationIteratorOzaki.h:244-300). */
int sc_boundary_initial(sc_ctx *ctx);

/* Frame Green sums of one angle for the current state and boundary values
 * (before the boundary extension): F = sum_n r_n (f + f~*) [2][N1][N1],
 * Re G [N1][N1], Re I [N1][N1] (GreensFunctionStatic.h:125-157,
 * ComputeFreeEnergy.h:106-160).  Updates the out-going boundary values of that
 * angle as the sweep does. */
int sc_angle_greens(sc_ctx *ctx, int angle, double *f, double *g_re, double *i_re);

/* Vector potential of a current density [2][N0][N0] through the separable
 * Poisson filters (ComputeVectorPotential::solve, ComputeVectorPotential.h:727-745),
 * internal units. */
int sc_poisson(sc_ctx *ctx, const double *j, double *a_out);

/* Allocation-free Poisson solve, for callers that cannot call cudaMalloc: a
 * plugin inside a framework that has reserved the device memory for its own
 * pool and passes it only the buffers it owns, or a service whose device
 * footprint is fixed at start-up.  No counterpart in the reference: it
 * computes what sc_poisson computes (ComputeVectorPotential::solve), with every
 * buffer owned by the caller and the intermediates in a fixed 24 MiB device
 * array of the library instead of allocated memory.
 *   d_filters  [n_filters][2*n0-1] device, the separable filters (sc_setup_filters)
 *   positive   [n_filters] host, their signs (sc_setup_filters)
 *   factor     -h^2 * scale (scale from sc_setup_filters, h the lattice spacing)
 *   n_grain    lattice sites of the grain (the current's mean is sum / n_grain)
 *   d_j        [2][n0][n0] device current density; d_a [2][n0][n0] device result
 *   stream     cudaStream_t the work is issued on (asynchronous)
 * Limit: n0 <= 724 (6 n0^2 + 128 doubles of scratch); larger n0 returns SC_ERR_SIZE
 * before any work.  It allocates nothing (no cudaMalloc, no allocating
 * library call).  The first call on a device (and the first after that
 * device's context was re-created, e.g. by cudaDeviceReset) looks up the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture.  Each kernel launch is checked as it is issued; a launch
 * error returns SC_ERR_CUDA.  All calls share the array: calls whose work
 * overlaps on the GPU race on it and must be ordered by the caller. */
int sc_poisson_noalloc(int n0, int n_filters, const double *d_filters, const int *positive,
                       double factor, int n_grain, const double *d_j, double *d_a, void *stream);

/* ---- LDOS postprocess (Keldysh path) ------------------------------------- */

/* Context of an LDOS postprocess: replaces the Context that src/postprocess.cu
 * :60-400 builds (IntegrationIteratorKeldysh, ComputeLDOS,
 * RiccatiSolverConfined with BoundaryConditionSpecular).  simulation_json is
 * the simulation_config.json of the loaded run; postprocess_json holds the
 * "spectroscopy" (energy_min, energy_max, num_energies, energy_broadening) and
 * "numerics" (num_fermi_momenta, convergence_criterion, norm,
 * num_energies_per_block, num_iterations_*) sections.  The real energies
 * E_k + i delta are swept one block at a time.  Load Delta and A with
 * sc_set_state (A in internal units: the file's A times lambda^2).  On such a
 * context sc_compute returns SC_ERR_STATE; sc_burn_in converges the boundary
 * of the current block; in sc_get_scalars slot 7 holds the LDOS residual. */
int sc_ldos_create(const char *simulation_json, const char *postprocess_json, int mode,
                   sc_ctx **out);
int sc_ldos_dims(const sc_ctx *ctx, int *n_energies, int *per_block, int *n_blocks);
/* The real energies E_k (IntegrationIteratorKeldysh.h:91-124) and delta. */
int sc_ldos_energies(const sc_ctx *ctx, double *energies, double *broadening);
/* Switches the sweep to energy block b and re-initialises the boundary with
 * homogeneous values (IntegrationIteratorKeldysh.h:250-268). */
int sc_ldos_begin_block(sc_ctx *ctx, int block);
/* n LDOS iterations of the current block (IntegrationIteratorKeldysh::compute,
 * IntegrationIteratorKeldysh.h:300-389; ComputeLDOS.h:123-193): sweeps, Im g
 * per energy rotated back, boundary condition, residual of the block's LDOS.
 * *converged: max(LDOS, boundary) residual below the criterion. */
int sc_ldos_iterate(sc_ctx *ctx, int n, double *residual, int *converged);
/* The whole postprocess loop (runPostprocess, run_simulation.h:44-104):
 * per block burn-in (burnin < 0: until the boundary converges), then
 * iterations until converged and at least it_min (at most it_max, < 0 = no
 * limit); stops at the first block that does not converge.  Loops without a
 * limit stop after 100000 iterations. */
int sc_ldos_run(sc_ctx *ctx, int burnin, int it_min, int it_max, int *converged,
                int *iterations);
/* The LDOS of every energy [n_energies][N0][N0] (ComputeLDOS::getResult). */
int sc_ldos_get(sc_ctx *ctx, double *ldos);
int sc_ldos_get_device(sc_ctx *ctx, double *d_ldos);

/* ---- batched grains -------------------------------------------------------- */

/* Many independent grains advanced together: one context per configuration
 * (each its own Context in the reference, src/simulation.cu:95-537, run one by
 * one there), with a shared pool for the sweep work buffers.  Every call of
 * sc_batch_compute runs one self-consistency iteration of each grain that has
 * not finished (converged and at least num_iterations_min, or
 * num_iterations_max reached, each grain by its own configuration); a grain
 * that finishes leaves the batch.  The Riccati sweep of all grains of a wave
 * (the grains whose work buffers fit the pool together) is one persistent
 * launch; from the second iteration on, the iteration is a CUDA graph. */
typedef struct sc_batch sc_batch;
int sc_batch_create(const char *const *configs, int n, int mode, sc_batch **out);
int sc_batch_destroy(sc_batch *b);
const char *sc_batch_last_error(const sc_batch *b);
int sc_batch_size(const sc_batch *b, int *n);
/* The context of grain i (owned by the batch: set its state, read its
 * results and scalars through the sc_* calls above; do not destroy it). */
int sc_batch_grain(sc_batch *b, int i, sc_ctx **ctx);
/* Up to n iterations of the active grains; *n_active: grains still running. */
int sc_batch_compute(sc_batch *b, int n, int *n_active);
/* Per grain: still active, iterations done, last residual (arrays of size n). */
int sc_batch_status(const sc_batch *b, int *active, int *iterations, double *residual);
/* Per grain (array of size n) how it stands: still running, finished
 * converged, finished at its num_iterations_max without converging (the
 * reference's "FAILURE! Simulation did not converge", run_simulation.h:174-181),
 * or diverged.  No counterpart in the reference: a grain whose iteration gives
 * a non-finite residual or free energy (a NaN or infinity anywhere in its
 * order parameter, current or vector potential reaches both) is frozen with
 * its last state, leaves the batch and is reported here; the other grains
 * continue unchanged. */
#define SC_GRAIN_RUNNING 0
#define SC_GRAIN_CONVERGED 1
#define SC_GRAIN_AT_CAP 2
#define SC_GRAIN_DIVERGED 3
int sc_batch_grain_state(const sc_batch *b, int *state);
/* CUDA-graph replay of the iteration on (default) or off. */
int sc_batch_set_graph(sc_batch *b, int enable);
/* Mapping of the persistent sweep: each grain takes the fewest threads per
 * trajectory column (1, 2, 4 or 8) that keep at most energies_per_thread
 * energies on a thread, and minb selects the resident-block variant (1: up
 * to 255 registers per thread, 3: at most 168, 4: at most 128, 6: at most 80;
 * 3 with at most four energies per thread, 6 with at most two; the default is four energies per thread and
 * minb 4).  In mixed precision a cap of two or four runs the packed FP32 sweep (each grain's energies per thread
 * rounded up to even).  sc_batch_autotune times the feasible choices on the current state (after at least one
 * iteration) and keeps the fastest. */
int sc_batch_config(sc_batch *b, int energies_per_thread, int minb);
int sc_batch_get_config(const sc_batch *b, int *energies_per_thread, int *minb, int *n_waves);
int sc_batch_autotune(sc_batch *b, int *energies_per_thread, int *minb, double *best_ms);
/* Device time of the sweeps of all waves (average of `repeats`), state unchanged. */
int sc_batch_time_sweeps(sc_batch *b, int repeats, double *ms);
int sc_batch_launch_count(const sc_batch *b, long long *count);

/* Measures the FP64 (precision 64) or FP32 (precision 32) FMA throughput of
 * the current device in FLOP/s: the CUDA-core denominator of the sweep's
 * compute roofline (the reference has no counterpart; a measurement aid). */
int sc_measure_fma_peak(int precision, double *flops_per_second);

/* Per-kernel CUDA-event timing on the context's stream.  kernel: 0 Riccati
 * sweep, 1 rotation back to the reference grid, 2 Poisson filters, 3 boundary
 * condition, 4 frame fields (the rotated order parameter, Doppler shift and
 * labels of each chunk's trajectory sites).  sc_profile_read returns the summed device time and number of
 * timed launches since the last read, and resets them. */
int sc_profile(sc_ctx *ctx, int enable);
int sc_profile_read(sc_ctx *ctx, int kernel, double *total_ms, long long *launches);

/* Number of this library's kernel launches issued by ctx so far. */
int sc_launch_count(const sc_ctx *ctx, long long *count);

/* ---- host-only setup probes (no GPU needed) ------------------------------ */

/* The static tables of a configuration, built without touching CUDA: lattice
 * sizes, Ozaki energies, frame labels, boundary-storage sizes and Poisson
 * filters (the set-up part of Context::initialize, Context.h:285-375). */
typedef struct sc_setup sc_setup;
int sc_setup_create(const char *config_json, sc_setup **out);
const char *sc_setup_last_error(void);
int sc_setup_destroy(sc_setup *s);
int sc_setup_dims(const sc_setup *s, int *n0, int *n1, int *n_angles, int *n_energies,
                  int *n_comp);
/* Imaginary parts of the Ozaki energies and their residues
 * (IntegrationIteratorOzaki.h:108-200). */
int sc_setup_energies(const sc_setup *s, double *e_im, double *residues);
int sc_setup_frame(const sc_setup *s, int angle, signed char *labels, int *box);
int sc_setup_domain(const sc_setup *s, signed char *domain);
int sc_setup_boundary_sizes(const sc_setup *s, int *sizes);
/* Separable Poisson filters [n][2*N0-1], their signs and the common scale
 * (ComputeVectorPotential.h:212-416).  Call with NULL arrays to get n first. */
int sc_setup_filters(const sc_setup *s, int *n_filters, double *filters, int *positive,
                     double *scale);
int sc_setup_site_updates(const sc_setup *s, long long *per_iteration);
/* Fermi-surface tables of the configuration (FermiSurfaceCircle.h:84-164, or
 * FermiSurfaceTightBinding.h:384-470 with physics.fermi_surface.type =
 * "tight_binding"): table [8][n_angles] = polar angle phi, system angle,
 * Fermi momentum x, y, Fermi velocity x, y (divided by the mean speed),
 * integrand factor, Riccati step h/|v_F|; info [4] = mean |p_F|, mean |v_F|
 * (the tight-binding averages before normalisation, FermiSurfaceTightBinding
 * .h:79-80; 1 on the circle), momentum origin x, y.  Either may be NULL. */
int sc_setup_fermi_surface(const sc_setup *s, double *table, double *info);

/* Bulk s-wave thermodynamics (host only).
 * sc_bulk_order_parameter_s_wave: computeOrderParameterBulkSWave
 * (OrderParameterBulk.h:88-221), the bulk gap at temperature T/Tc in units of
 * 2 pi k_B Tc; the reference's defaults are criterion 10 eps, 10 iterations,
 * cutoff 100.  A d-wave (or g-wave) component's bulk amplitude is this value
 * times D_WAVE_BULK / S_WAVE_BULK (OrderParameterComponent.h:210-235).
 * sc_bulk_free_energy_s_wave: computeFreeEnergyBulkSWave
 * (OrderParameterBulk.h:224-246), the bulk free energy density at that gap
 * (reference default cutoff 100).
 * sc_bulk_yoshida_s_wave: computeYoshidaBulkSWave (OrderParameterBulk.h:256-277),
 * the Yoshida function that sets the London response j = -Y A of the bulk. */
int sc_bulk_order_parameter_s_wave(double temperature, double convergence_criterion,
                                   int max_iterations, double energy_cutoff, double *out);
int sc_bulk_free_energy_s_wave(double temperature, double order_parameter, double energy_cutoff,
                               double *out);
int sc_bulk_yoshida_s_wave(double temperature, double order_parameter, double energy_cutoff,
                           double *out);

/* Load-path helpers for runs saved on another lattice (host only).
 * sc_grid_extend: extendValuesAtBoundary (domain_ops.h:11-69) of n_fields
 * planes [n_fields][n][n] in place, with the domain labels of that lattice.
 * sc_grid_resample: GridFunctions::resample (GridFunctions_GPU.h:547-600,
 * 1056-1091), bilinear onto an n_new lattice keeping the 3-site safety
 * margin; sites that would read past the old lattice (only inside the margin
 * when shrinking) take the nearest edge value.  Used by the drivers as the
 * reference's CSV reader does (csv.h:180-205, 297-395). */
int sc_grid_extend(int n, const signed char *domain, int n_fields, double *values);
int sc_grid_resample(int n_old, int n_new, int n_fields, const double *src, double *dst);

#ifdef __cplusplus
}
#endif

#endif /* SCB200_H_ */
