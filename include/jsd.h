/*
 * jsd.h -- C ABI of the B200 velocity-vorticity channel-flow step.
 *
 * The reference (dakling/jax-spectral-dns) is pure Python/JAX and has no FFI;
 * this ABI is the boundary under its equation classes. Each entry point names
 * the reference call it replaces (paths inside the reference package).
 *
 * Conventions
 *  - All arrays passed to the step functions are DEVICE pointers owned by the
 *    caller. A state is 3 spectral fields (u, v, w), each Ny x Mx x Mz complex
 *    doubles stored as interleaved (re, im), plane by plane:
 *        element (c, y, ix, iz) at ((c * Ny + y) * Mx + ix) * Mz + iz
 *    kx, kz in FFT order [0..K, -K..-1]; y index 0 is y = +1. Coefficients use
 *    the reference normalisation: ortho FFT on the reference's physical grid
 *    (Px_ref x Pz_ref) divided by s = Lx Lz / (4 pi^2).
 *  - Host pointers in jsd_desc are copied at plan creation.
 *  - Every function returns 0 on success or a negative JSD_ERR_* code; the
 *    message of the last error on the calling thread is jsd_last_error().
 *  - A plan owns its device workspace and launches on the stream passed to
 *    each call. Plans are not thread-safe; distinct plans may run concurrently.
 */
#ifndef JSD_H
#define JSD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JSD_ABI_VERSION 5  /* 2: jsd_desc gained n_batch, re_tau_batch; 3: JSD_ERR_NONFINITE, wait limit;
                               4: jsd_set_source; 5: jsd_split_eig_in */

enum jsd_status {
  JSD_OK = 0,
  JSD_ERR_ARG = -1,      /* invalid argument or unsupported configuration */
  JSD_ERR_CUDA = -2,     /* CUDA runtime error (message has the detail) */
  JSD_ERR_NOMEM = -3,    /* device allocation failed */
  JSD_ERR_STATE = -4,    /* call out of order (e.g. dual step without history) */
  JSD_ERR_NONFINITE = -5 /* the state became NaN or infinite (reported by jsd_device_error) */
};

enum jsd_kind {
  JSD_KIND_NS = 0,            /* NavierStokesVelVort            (navier_stokes.py:310) */
  JSD_KIND_PERTURBATION = 1,  /* NavierStokesVelVortPerturbation (navier_stokes_perturbation.py:341) */
  JSD_KIND_DUAL = 2           /* NavierStokesVelVortPerturbationDual (navier_stokes_perturbation_dual.py:376) */
};

/* Discretisation and operator tables. The tables are the FP64 quantities the
 * host builds once per box (Chebyshev matrix D, the eigen-decomposition
 * D2_int = V diag(lam) V^-1 of the interior second-derivative matrix, and the
 * reference's (0,0) mean-flow matrices); see jax_spectral_dns/_ops.py. */
typedef struct jsd_desc {
  int mx, ny, mz;          /* Fourier modes in x and z (odd), Chebyshev points */
  int px_ref, pz_ref;      /* reference physical grid (normalisation, Domain.create, domain.py:201-317) */
  int px_fft, pz_fft;      /* device FFT lengths, >= 3*(m/2)+1 with factors 2,3,5,7 */
  double lx, lz;           /* box lengths */
  int kind;                /* enum jsd_kind */
  int linearise;           /* drop the quadratic term (perturbation / dual) */
  int constant_mass_flux;  /* navier_stokes.py:1205-1214 */
  double re_tau;           /* Reynolds number of the implicit operators */
  double dt;               /* time step of the implicit operators */
  double dt_explicit;      /* time step multiplying the explicit terms (-dt for the dual) */
  double flow_rate_target; /* Q0 for the constant-mass-flux correction */
  const double* base_u;    /* [ny] base profile U(y) (perturbation / dual) or NULL */
  const double* base_du;   /* [ny] dU/dy or NULL */
  const double* D;         /* [ny*ny] Chebyshev first-derivative matrix, row-major */
  const double* V;         /* [(ny-2)^2] eigenvectors of D2[1:-1,1:-1] (columns) */
  const double* Vinv;      /* [(ny-2)^2] */
  const double* lam;       /* [ny-2] eigenvalues */
  const double* sgn;       /* [ny-2] parity of each eigenvector under y -> -y (+1/-1) */
  const double* c0;        /* [ny-2] Vinv @ D2[1:-1, 0] */
  const double* cN;        /* [ny-2] Vinv @ D2[1:-1, -1] */
  const double* w0;        /* [ny-2] D[0, 1:-1] @ V */
  const double* wN;        /* [ny-2] D[-1, 1:-1] @ V */
  const double* y_weights; /* [ny] Chebyshev integration weights (field.py:2618-2650) */
  const double* rhs_ns;    /* [3*(2ny)^2] (0,0) explicit matrices per RK stage (navier_stokes.py:1000-1022) */
  const double* lhs_inv_ns;/* [3*(2ny)^2] (0,0) implicit inverses per RK stage */
  int precision;           /* JSD_PRECISION_FP64, or JSD_PRECISION_MIXED: FP32 transforms and products,
                              split-TF32 tensor-core y-derivatives; solves stay FP64 */
  /* Batch of independent runs on the same box (no counterpart in the
   * reference, which steps one field at a time). n_batch <= 1: one run.
   * n_batch > 1: every field holds the runs side by side, plane by plane,
   *     element (c, y, run, ix, iz) at (((c * Ny + y) * n_batch + run) * Mx + ix) * Mz + iz,
   * so each y-operator is one product over all runs; re_tau_batch[n_batch]
   * gives each run's Reynolds number and rhs_ns / lhs_inv_ns hold n_batch
   * consecutive sets of 3 matrices. NS and perturbation equations without
   * mass-flux control. */
  int n_batch;
  const double* re_tau_batch;
} jsd_desc;

enum jsd_precision { JSD_PRECISION_FP64 = 0, JSD_PRECISION_MIXED = 1 };

typedef struct jsd_plan jsd_plan;

/* Builds the device operators, FFT tables and workspace.
 * Replaces NavierStokesVelVort.assemble_matrices / prepare_assemble_rk_matrices
 * (navier_stokes.py:437-502, 920-1022) and FourierDomain.assemble_poisson_matrix
 * (domain.py:857-889). */
int jsd_plan_create(const jsd_desc* desc, jsd_plan** plan);

int jsd_plan_destroy(jsd_plan* plan);

/* Advances `state` in place by n_steps RK3/Crank-Nicolson steps on `stream`.
 * dpdx is a device double (mean pressure gradient), read and, with constant
 * mass flux, updated. first_step is the global index of the first step (used
 * by the dual to select the forward state).
 * Replaces NavierStokesVelVort.perform_time_step / perform_runge_kutta_step
 * (navier_stokes.py:1778-1813, 1219-1775). */
int jsd_step(jsd_plan* plan, void* state, double* dpdx, int first_step, int n_steps, void* stream);

/* jsd_step that also records the trajectory: states (device, n_steps + 1
 * consecutive states) receives the initial state and the state after each
 * step. Replaces solve_scan with write_entire_output (navier_stokes.py:1960-1990),
 * the forward run the dual needs (navier_stokes_perturbation_dual.py:850-939). */
int jsd_step_trajectory(jsd_plan* plan, void* state, double* dpdx, int first_step, int n_steps, void* states,
                        void* stream);

/* Source terms of the following steps (device arrays owned by the caller,
 * read in every stage until replaced): hv and hg (state layout of one field,
 * Ny x Mx x Mz complex) are added to the nonlinear terms h_v and h_g, s00
 * (2 Ny complex: x then z component) to the (0,0) mean-flow forcing. All
 * three NULL switches them off. Single-run plans. Replaces the source_hat
 * hooks of perform_runge_kutta_step (navier_stokes.py:1461-1491, 1697-1703)
 * that the dual's dissipation objective fills
 * (navier_stokes_perturbation_dual.py:962-990). */
int jsd_set_source(jsd_plan* plan, const void* hv, const void* hg, const void* s00);

/* Dual equations: register the forward trajectory u_0 .. u_{n_states-1}
 * (device, n_states consecutive states). Dual step t uses u_{n_states-1-t}
 * for all three stages (navier_stokes_perturbation_dual.py:591-602). */
int jsd_set_history(jsd_plan* plan, const void* states, int n_states);

/* Constant-mass-flux correction of the streamwise field: Q is the flow rate of
 * state's u, u <- hat(no_hat(u) - (Q - Q0)/2) (walls included) and, when dpdx
 * is not NULL, dpdx += (Q - Q0)/dt_explicit.
 * Replaces update_pressure_gradient + update_velocity_field_data
 * (navier_stokes.py:724-805; perturbation variant navier_stokes_perturbation.py:420-466). */
int jsd_correct_mass_flux(jsd_plan* plan, void* state, double* dpdx, void* stream);

/* Kinetic energy E = 1/(2V) int |u|^2 / 2 of a state, written to the device
 * double `out`. Replaces VectorField.no_hat().energy() (field.py:607-611,
 * 1468-1474). */
int jsd_energy(jsd_plan* plan, const void* state, double* out, void* stream);

/* Kinetic energy of every active run of a batch plan: out[run], run <
 * jsd_batch_active (device pointer). The single-run entry points (jsd_energy,
 * jsd_flow_rate, jsd_correct_mass_flux, jsd_nonlinear_terms) reject batch
 * plans. No counterpart in the reference. */
int jsd_energy_runs(jsd_plan* plan, const void* state, double* out, void* stream);

/* Step only the first n_runs runs of a batch plan from now on (1 <= n_runs <=
 * n_batch): the caller keeps its state packed for n_runs runs, i.e. drops
 * finished runs from the end of the run order. Runs keep their Reynolds
 * numbers. No counterpart in the reference. */
int jsd_set_batch_active(jsd_plan* plan, int n_runs);

/* Discrete adjoint of the linearised perturbation step: replaces `cotangent`
 * (device, state layout), the gradient of an objective with respect to the
 * state after n_steps steps of this plan, by its gradient with respect to the
 * state before them, i.e. applies the exact transpose of n_steps steps (for
 * the real inner product of the real and imaginary parts) in reverse. The
 * linearised step is linear and the same every step, so no forward states are
 * needed. Linearised perturbation plans of one run, coupling term on, no
 * mass-flux control. Stands in for jax.grad through the reference's forward
 * solve (optimiser.py:120, with navier_stokes.py:1219-1813); unlike the
 * reference's dual solver (navier_stokes_perturbation_dual.py:850-1120), which
 * it does not replace, it is the exact derivative of the discrete step. */
int jsd_step_adjoint(jsd_plan* plan, void* cotangent, int n_steps, void* stream);

/* Gradient of jsd_energy's value with respect to the real and imaginary parts
 * of every coefficient of `state`, written to `out` (device, state layout):
 * the derivative of VectorField.no_hat().energy() (field.py:607-611,
 * 1468-1474). */
int jsd_energy_grad(jsd_plan* plan, const void* state, void* out, void* stream);

/* coupling_term of the perturbation and dual equations
 * (navier_stokes_perturbation.py:401-415; the extra terms of
 * navier_stokes_perturbation.py:217-237 and ..._dual.py:270-292 when off).
 * Default on. */
int jsd_set_coupling_term(jsd_plan* plan, int on);

/* Replace the base profile U(y) and dU/dy (device arrays of Ny doubles,
 * copied on `stream`) for the following steps: the time-dependent base of
 * NavierStokesVelVortPerturbationInstationary.vel_base_fn
 * (navier_stokes_perturbation_instationary.py:37-83) is set once per step. */
int jsd_set_base_flow(jsd_plan* plan, const double* base_u, const double* base_du, void* stream);
int jsd_batch_active(const jsd_plan* plan);

/* Kinetic energy of a state without a plan and without allocating anything.
 * No counterpart in the reference. For callers that cannot allocate device
 * memory: code that runs under a host framework which has already reserved
 * the GPU's memory for its own pool, or in-situ monitoring hooks inside a
 * time loop that must not allocate or free (cudaMalloc/cudaFree can
 * synchronise the device and fragment a long-running job's memory).
 * The caller passes the state (layout as above), the grid, the reference
 * physical grid sizes, the box lengths, the Ny Chebyshev integration weights
 * (device array, field.py:2618-2650) and a device double for the result.
 * Limit: ny <= 4096. The per-plane scratch is a fixed 32 KiB device array
 * inside the library, held by every GPU that loads it until the process exits.
 * The first call on a device looks up that array's address (with that device
 * current) and keeps it for the life of the process, so it assumes the
 * device's primary context is not reset or recreated in between (after
 * cudaDeviceReset the kept address is stale); make that first call before
 * any stream capture. All calls share
 * the array, so calls that overlap on the GPU (e.g. on two streams) race;
 * each call overwrites the entries it reads, so sequential calls need no
 * clearing. Calls no cudaMalloc/cudaFree. */
int jsd_energy_noalloc(const void* state, int mx, int ny, int mz, int px_ref, int pz_ref, double lx, double lz,
                       const double* y_weights, double* out, void* stream);

/* Flow rate Q = int u(x=0, y, z=0) dy of the streamwise component, written to
 * the device double `out`. Replaces NavierStokesVelVort.get_flow_rate
 * (navier_stokes.py:709-722). */
int jsd_flow_rate(jsd_plan* plan, const void* u_field, double* out, void* stream);

/* Nonlinear-term hook: h_v, h_g (spectral, Ny x Mx x Mz each) of `state` at
 * forward step t. Replaces nonlinear_update_fn's (h_v, h_g) outputs
 * (navier_stokes.py:324-332, 48-73). */
int jsd_nonlinear_terms(jsd_plan* plan, const void* state, int time_step, void* h_v, void* h_g, void* stream);

/* Bytes of device workspace the plan holds. */
size_t jsd_workspace_bytes(const jsd_plan* plan);

/* Autotuner (no counterpart in the reference, where XLA picks its own
 * kernels): times every FP64 tensor-core tile configuration of the library on
 * the plan's three GEMM call sites (y-derivatives, eigenbasis transforms in,
 * back-transforms out) with the plan's own sizes and workspace, and keeps the
 * fastest per site, and likewise chooses among the x-pass kernel variants of
 * the nonlinear terms. Overwrites workspace only (no state); synchronises the
 * stream, so it must not be called during stream capture. */
int jsd_autotune(jsd_plan* plan, void* stream);

/* Tile configuration in use at GEMM call site `site` (0 y-derivatives,
 * 1 eigenbasis in, 2 eigenbasis out), or -1 for a bad argument; if times_ms is
 * not null it receives the autotuner's per-configuration times (7 floats, 0
 * for configurations not timed). */
int jsd_gemm_config(const jsd_plan* plan, int site, float* times_ms);

/* Use tile configuration `config` (0..6) at GEMM call site `site`. Every
 * configuration sums over K in the same order, so results do not depend on
 * the choice. No counterpart in the reference. */
int jsd_set_gemm_config(jsd_plan* plan, int site, int config);

/* x-pass kernel of the nonlinear terms in use: 0 register FFT with S lanes per
 * x line, 1 register FFT with 2 S lanes per line, 2 shared-memory FFT; if
 * times_ms is not null it receives the autotuner's times of the three (0 for
 * variants not timed or not available). No counterpart in the reference. */
int jsd_xmid_variant(const jsd_plan* plan, float* times_ms);

/* Force x-pass variant 0, 1 or 2 (JSD_ERR_ARG when it does not apply to the
 * plan's FFT length, precision or equation). No counterpart in the reference. */
int jsd_set_xmid_variant(jsd_plan* plan, int variant);

/* Split-TF32 product kernel of a mixed-precision plan (y-derivatives, and
 * the eigenbasis-in products of the nonlinear terms when those are split):
 * 0 mma.sync (k_sgemm3), 1 tcgen05 with the accumulator in tensor memory
 * (k_tc05_split, Ny <= 129, the default); -1 for FP64 plans. times_ms (2 floats, may be
 * null) receives the autotuner's timings. No counterpart in the reference. */
int jsd_split_kernel(const jsd_plan* plan, float* times_ms);
int jsd_set_split_kernel(jsd_plan* plan, int kernel);

/* Eigenbasis-in products of the nonlinear terms (V^-1 D q, V^-1 H1,
 * V^-1 h_g) of a mixed-precision plan: 1 in split TF32 on the split kernel
 * (the default for the Navier-Stokes equations: the terms themselves come
 * out of FP32 transforms and products), 0 FP64-accurate (DMMA or int8
 * Ozaki, as jsd_eig_kernel says; the default with a base flow, whose
 * coupling terms are part of these products);
 * -1 for FP64 plans. The state's own eigenbasis products (V^-1 v, V^-1
 * omega_y, V and D V back) stay FP64-accurate either way, and so do the
 * products of linearised terms (formed in FP64, not by FP32 transforms).
 * No counterpart in the reference. */
int jsd_split_eig_in(const jsd_plan* plan);
int jsd_set_split_eig_in(jsd_plan* plan, int on);

/* Eigenbasis product kernel of a plan at GEMM site 1 (eigenbasis in) or 2
 * (eigenbasis out): 0 FP64 DMMA (the default of FP64 plans), 1
 * FP64-accurate Ozaki products on the int8 tensor cores (k_oz8_gemm,
 * Ny <= 129; the default of mixed-precision plans, whose autotuning keeps the
 * faster kernel per site); -1 for a bad site.
 * times_ms (2 floats, may be null) receives the autotuner's timings (best
 * DMMA tile, Ozaki). No counterpart in the reference. */
int jsd_eig_kernel(const jsd_plan* plan, int site, float* times_ms);
int jsd_set_eig_kernel(jsd_plan* plan, int site, int kernel);

/* Device-side failure detection; synchronises the stream and clears the
 * plan's error flag. Returns JSD_ERR_CUDA when a kernel of the plan gave up a
 * bounded wait since the last check (its results are then invalid), else
 * JSD_ERR_NONFINITE when a stage produced a NaN or an infinity (every stage
 * checks the new state as it reconstructs it), else 0. The reference's only
 * check is a host assert on the objective (gradient_descent_solver.py:125). */
int jsd_device_error(jsd_plan* plan, void* stream);

/* Polls of an mbarrier before a pipeline wait of the plan's tcgen05 kernels
 * gives up and raises the wait bit of the error flag (0 restores the
 * default, 4194304). The kernel then stops, waits for its own copies and MMAs
 * in flight, frees its tensor memory and returns. No counterpart in the
 * reference. */
int jsd_set_wait_limit(jsd_plan* plan, int polls);
int jsd_wait_limit(const jsd_plan* plan);

/* Number of kernel launches one call of jsd_step issues per time step after
 * its first; the first step of each call issues jsd_launches_first_step_extra
 * more (it derives omega_y, and dv/dy for linearised plans, from the caller's
 * state; later stages carry both from the previous stage's solve). */
int jsd_launches_per_step(const jsd_plan* plan);
int jsd_launches_first_step_extra(const jsd_plan* plan);

/* Optional timing of kernel classes with CUDA events (no effect unless
 * enabled). jsd_profile_read returns and clears, for one class, the summed
 * device time (ms), the number of launches and the summed algorithmic work
 * (FLOPs for JSD_PROF_GEMM, bytes for the others). No reference counterpart. */
enum jsd_prof_class {
  JSD_PROF_GEMM = 0,    /* FP64 y-contractions (DMMA) */
  JSD_PROF_ZINV = 1,    /* inverse z transforms */
  JSD_PROF_XMID = 2,    /* x transforms + products */
  JSD_PROF_ZFWD = 3,    /* forward z transforms + truncation */
  JSD_PROF_EIGEN = 4,   /* eigenbasis update + influence correction */
  JSD_PROF_LINEAR = 5,  /* linearised terms */
  JSD_PROF_SGEMM = 6    /* split-TF32 y-derivatives (mixed precision) */
};
int jsd_profile_enable(jsd_plan* plan, int enable);
int jsd_profile_read(jsd_plan* plan, int kernel_class, double* total_ms, long long* launches, double* work);

const char* jsd_last_error(void);
int jsd_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* JSD_H */
