/*
 * shhd_b200.h — C ABI of the B200 step engine for the 2-D spectral
 * Hohenberg–Halperin / fluctuating-hydrodynamics solver.
 *
 * The engine replaces, for one process on one GPU, the reference solver's
 * per-step hot path: FluidSolver::step (src/fluid_solver.h:97-99) driving a
 * TimeIntegrator (src/time_integrator.h:141) over the FCalculator RHS
 * operators (src/fcalculator.h:64-69) on heFFTe transforms
 * (src/fourier_transform.h:39-51).  State stays in device memory between
 * calls; host arrays cross the boundary only in set/get calls.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative SHHD_E* code; the
 *     message of the last failure on the calling thread is shhd_last_error().
 *   - Host arrays are caller-owned and only read or written during the call.
 *   - A state array is the reference's State layout (src/state.cc:22-38,
 *     src/domain.cc:21-30): nfields blocks (rho, psi_0..psi_{N-1}, jx, jy) of
 *     (nx/2+1)*ny complex values, gx fastest, as interleaved doubles.
 *   - An engine may hold `batch` independent members (noise realisations or
 *     jobs of one shape); member m's noise stream is keyed by
 *     member_offset + m.
 *   - One host thread at a time per engine; every engine owns a CUDA stream.
 */
#ifndef SHHD_B200_H
#define SHHD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct shhd_engine shhd_engine;

#define SHHD_MAX_ORDER_PARAMETERS 8
#define SHHD_MAX_FORCES 8
#define SHHD_MAX_FE_PARAMS 4      /* parameters of a free-energy plugin style */

/* error codes */
#define SHHD_OK 0
#define SHHD_EINVAL (-1)      /* bad argument or configuration */
#define SHHD_ECUDA (-2)       /* CUDA runtime failure */
#define SHHD_ENOMEM (-3)      /* device allocation failed */
#define SHHD_ENUMERIC (-4)    /* zero density met by v = j / rho (fcalculator_workspace.cc:122-133) */
#define SHHD_EUNSUPPORTED (-5)/* configuration outside what the engine implements */

enum shhd_mode { SHHD_COMPRESSIBLE = 0, SHHD_INCOMPRESSIBLE = 1, SHHD_QUIESCENT = 2 };
enum shhd_integrator { SHHD_EULER = 0, SHHD_SRK3 = 1 };
enum shhd_precision { SHHD_FP64 = 0, SHHD_FP32 = 1 };
enum shhd_noise_source { SHHD_NOISE_PHILOX = 0, SHHD_NOISE_EXTERNAL = 1 };
enum shhd_free_energy { SHHD_FE_NONE = 0, SHHD_FE_PHI4 = 1, SHHD_FE_QUADRATIC = 2, SHHD_FE_PLUGIN = 3 };

typedef struct shhd_sine_force {
    int target;      /* 0 momentum, 1 order parameter */
    int component;   /* momentum: 0 = x, 1 = y; order parameter: index */
    int axis;        /* 0 = x, 1 = y */
    int nk;
    double amplitude;
} shhd_sine_force;

typedef struct shhd_gradient_force {
    int component;   /* order parameter index */
    int direction;   /* 0 = x, 1 = y */
    double amplitude;
} shhd_gradient_force;

/* Solver configuration: the reference's Params fields that shape the step
 * (src/simulationinfo.h:35-175), with the model plugins given as data. */
typedef struct shhd_config {
    int active_nx, active_ny;   /* `grid` (active modes) */
    int nx, ny;                 /* compute grid after `dealias` */
    double lx, ly;              /* `length` */
    double dt;                  /* `timestep` */
    int mode;                   /* enum shhd_mode   (`time_evolution` */
    int integrator;             /* enum shhd_integrator  .../...) */
    int num_order_parameters;   /* `order_parameters` */
    /* `model free_energy`: mu_a = (k0 + k2 k^2 + k4 k^4) psi_a (spectral) + u3 psi_a^3 (physical;
     * a plugin style's mu_a instead, fe_plugin below) */
    int free_energy;            /* enum shhd_free_energy */
    double mu_k0[SHHD_MAX_ORDER_PARAMETERS];
    double mu_k2[SHHD_MAX_ORDER_PARAMETERS];
    double mu_k4[SHHD_MAX_ORDER_PARAMETERS];
    double mu_u3[SHHD_MAX_ORDER_PARAMETERS];
    /* `model thermo linear_eos`: p = cT^2 rho (spectral only) */
    double cT;
    /* `model transport constant` */
    double eta, zeta;
    double mobility[SHHD_MAX_ORDER_PARAMETERS];
    /* `fix ... nonlinear` */
    int momentum_advection, order_parameter_advection;
    /* `fix ... noise` */
    int noise_momentum, noise_order_parameter;
    int64_t noise_seed;
    double kBT, chi;
    /* `fix ... force/sine`, `fix ... force/gradient` */
    int n_sine_forces;
    shhd_sine_force sine_forces[SHHD_MAX_FORCES];
    int n_gradient_forces;
    shhd_gradient_force gradient_forces[SHHD_MAX_FORCES];
    /* engine options (no reference counterpart) */
    int precision;              /* enum shhd_precision */
    int noise_source;           /* enum shhd_noise_source */
    int batch;                  /* members advanced together (1 ... 65535) */
    int member_offset;          /* first member id for the noise key */
    /* free_energy == SHHD_FE_PLUGIN: the compiled-in style (1 ... shhd_free_energy_plugin_count(),
     * include/shhd_b200_free_energy.cuh) and its parameters [parameter][order parameter]; the
     * linear part is mu_k0, mu_k2 (keys a[], b[]) */
    int fe_plugin;
    double fe_param[SHHD_MAX_FE_PARAMS][SHHD_MAX_ORDER_PARAMETERS];
} shhd_config;

typedef struct shhd_info {
    int nfields;                /* num_order_parameters + 3 */
    size_t state_doubles;       /* doubles in one member's state array (reference layout) */
    size_t active_modes;        /* active modes per field: (active_nx/2) * (active_ny - 1) */
    int n_inverse, n_forward;   /* transforms per stage: C2R fields, R2C product fields */
    int n_evolved;              /* fields the integrator updates */
    size_t device_bytes;        /* device memory the engine holds */
    double bytes_per_stage;     /* HBM bytes the fused kernels must move per stage (all members) */
    double fft_flops_per_stage; /* 5 n log2 n per complex line equivalent */
    int64_t step_index;         /* steps taken since creation */
    double time;                /* simulation time */
} shhd_info;

/* Thread-local message of the last failure. */
const char* shhd_last_error(void);

/* Free-energy plugin styles compiled into this library (no reference counterpart as a call; it
 * lists what FreeEnergyRegistry::register_free_energy_style registered,
 * src/model_free_energy_registry.h:65-85): their number, and the name of style id (1-based;
 * NULL when out of range).  Host only; needs no GPU. */
int shhd_free_energy_plugin_count(void);
const char* shhd_free_energy_plugin_name(int id);
/* Script key of parameter k of style id ("u[]": one value per order parameter, written u[0],
 * u[1], ...; "g": one value), or NULL when out of range. */
const char* shhd_free_energy_plugin_key(int id, int k);

/* Fill *cfg with the reference defaults (src/simulationinfo.h:35-98):
 * grid 128^2, L = 2 pi, no dealiasing, dt 0.005, srk3/compressible, N = 0,
 * noise off with seed 12345, kBT 1, chi 1; plus FP64, Philox noise, batch 1. */
int shhd_config_default(shhd_config* cfg);

/* Parse a reference input script (the hot-path commands of
 * src/param_parser.cc:42-163,165-339,551-805) into *cfg, applying the same
 * validation and error messages.  `set`, `measure`, `thermo`, `restart` and
 * `run` lines are accepted and ignored.  Host only; needs no GPU. */
int shhd_config_from_script(const char* script_text, shhd_config* cfg);

/* Replaces constructing FluidSolver (src/fluid_solver.h:52-95): allocates
 * the device state, workspaces and plans for cfg->batch members on the
 * current CUDA device. */
int shhd_engine_create(const shhd_config* cfg, shhd_engine** out);

/* Releases all device memory and the stream. */
void shhd_engine_destroy(shhd_engine* engine);

int shhd_engine_info(const shhd_engine* engine, shhd_info* info);

/* Upload one member's state (reference State layout, n_doubles =
 * info.state_doubles).  Entries outside the active modes
 * (src/spectral_mask.cc:45-52) must be zero, as every reference State is
 * after its mask is applied; anything else is rejected. */
int shhd_engine_set_state(shhd_engine* engine, int member, const double* state, size_t n_doubles);

/* Download one member's state into the reference layout (inactive entries zero). */
int shhd_engine_get_state(shhd_engine* engine, int member, double* state, size_t n_doubles);

/* Replaces FluidSolver::step / TimeIntegrator::step (time_integrator.h:141)
 * called nsteps times (project.h:134-139): enqueues nsteps steps of all
 * members on the engine's stream and waits for them. */
int shhd_engine_step(shhd_engine* engine, int nsteps);

/* Same as shhd_engine_step without waiting; errors raised on the device are
 * reported by the next shhd_engine_synchronize. */
int shhd_engine_step_async(shhd_engine* engine, int nsteps);
int shhd_engine_synchronize(shhd_engine* engine);

/* For noise_source == SHHD_NOISE_EXTERNAL: the stochastic right-hand sides
 * the next step uses, as the reference integrators hold them
 * (stochastic_rhs_a_ / stochastic_rhs_b_, srk3_compressible.h:23-24; Euler uses
 * sto_a only).  Reference layout; sto_b may be NULL for Euler. */
int shhd_engine_set_external_noise(shhd_engine* engine, int member, const double* sto_a, const double* sto_b, size_t n_doubles);

/* Deterministic right-hand side of the current state (rho_det, psi_det,
 * j_det of src/fcalculator.cc:60-150) in the reference layout. */
int shhd_engine_rhs(shhd_engine* engine, int member, double* det, size_t n_doubles);

/* Per-member controls of a batched engine (no reference counterpart; used by
 * the serving loop).  Member m draws its noise with key (seed, key) at step
 * (engine step index - step_origin), scaled by noise_scale (the factor
 * sqrt(kBT_m / kBT) for a member whose temperature differs from the
 * configuration's); inactive members are skipped by every kernel.  Defaults:
 * key = member_offset + m, step_origin 0, noise_scale 1, active.  Resets the
 * member's cached reference density (a new trajectory). */
int shhd_engine_set_member(shhd_engine* engine, int member, uint32_t key, int64_t step_origin, double noise_scale, int active);

/* Replay of captured CUDA graphs (no reference counterpart).  With chunk > 0,
 * a step call is split into replays of captured graphs, each holding one call
 * of a fixed number of steps (its launches and the advance of the device-side
 * step counter that keys the noise): as many of `chunk` as fit, then of each
 * power of two below `chunk`, largest first, so any call costs at most about
 * log2(chunk) + n / chunk graph launches; the result equals the same sequence
 * of calls made directly.  Graphs are captured on first use of each size.
 * Euler uses even sizes only (its two state buffers swap every step; the
 * chunk is rounded up to even) and steps a leftover single step directly.
 * 0 (the default) launches every kernel directly.  Per-kernel profiling uses
 * direct launches. */
int shhd_engine_set_graph_chunk(shhd_engine* engine, int chunk);

/* Structure factor of one field (no reference counterpart; the reference's
 * closest data are `snapshot space spectral` dumps, measure_snapshot.cc).
 * shhd_engine_sk_accumulate enqueues, on the engine stream, the addition of
 * S(k) = V |u_k|^2 / Np^4 averaged over the active members to an FP64
 * accumulator on the device (one sample; u_k the unnormalised padded-grid
 * coefficient, so S(k) -> kBT / (k0 + k2 k^2) for a quadratic free energy in
 * equilibrium).  shhd_engine_sk_read copies the sum of the samples in the
 * engine's mode order [gx < active_nx/2][j < active_ny - 1] (j = ky for
 * ky >= 0, else ky + active_ny - 1), sets *count to the number of samples and,
 * with reset != 0, clears the accumulator.  One field at a time. */
int shhd_engine_sk_accumulate(shhd_engine* engine, int field);
int shhd_engine_sk_read(shhd_engine* engine, double* out, size_t n_modes, int64_t* count, int reset);

/* Autotuner (no reference counterpart).  Times trial_steps steps of every
 * kernel family valid for the configuration (FP32 compute sizes 96-1536: the
 * pair-line kernels and the single-line kernels; otherwise the one family)
 * with direct launches and as one replayed graph, on the engine's current
 * state, then restores the state, step counter and time (and the accumulators
 * of enabled per-step measures: Green-Kubo sums, flux taps) and keeps the fastest
 * combination.  *family: 4 two-pair row pass, 3 split row pass, 2 register
 * row pass, 1 pair-line, 0 other; *graph_chunk: the chosen chunk (0 = direct
 * launches); ms_per_step (optional, room for 10): the measured ms per step of
 * each valid candidate in order (family 0 direct, family 0 graph, family 1
 * direct, family 1 graph, ... family 4 graph).  Family 2 is the pair-line
 * family with the register-resident row pass, valid for FP32 engines whose
 * compute rows have 1536 points; family 3 the pair-line family with the row
 * pass split into an inverse and a forward kernel over a physical-row buffer
 * (allocated while the family is selected); family 4 the pair-line family
 * whose row pass transforms two output pairs at a time, valid for compressible
 * dynamics whose last two input pair-lines are (rho, jx), (jy, -).  The
 * families are timed at the rule's launch shapes; then, with the chosen family
 * and chunk, the launch shapes of its pair-line kernels where shared memory
 * leaves a choice (shhd_engine_set_launch_shape: row pass at 2 or 3 blocks per
 * SM, column forward at 3 or 4), and the fastest is kept (read it back with
 * shhd_engine_launch_shape).  Allocates a temporary copy of the state. */
int shhd_engine_autotune(shhd_engine* engine, int trial_steps, int* family, int* graph_chunk, double* ms_per_step);

/* Select the kernel family (no reference counterpart): -1 the default choice
 * (1 where valid, else 0), 0 never the pair-line kernels,
 * 1 pair-line where valid, 2 pair-line with the
 * register-resident row pass where valid, 3 pair-line with the split row pass
 * where valid, 4 pair-line with the two-pair row pass where valid (2, 3 and 4
 * otherwise as 1).  Results agree across families within the precision's
 * tolerance; families 1 and 4 agree bit for bit.  Drops captured graphs. */
int shhd_engine_set_family(shhd_engine* engine, int family);

/* The family the engine launches: 4, 3, 2, 1 or 0 as above. */
int shhd_engine_family(const shhd_engine* engine);

/* Launch shapes of the pair-line stage kernels (no reference counterpart): the
 * row pass compiled with registers for row_blocks blocks per SM (2 or 3), the
 * column forward on columns of 384 points and more for col_blocks (3 or 4);
 * 0 keeps the rule (row pass: 3 where shared memory holds three blocks;
 * column forward: 4 where it holds four, on 1536-point columns and for plans
 * without a momentum group).  Where shared memory holds fewer blocks than the
 * registers are budgeted for, fewer run per SM; results do not depend on the
 * shape.  Kept across shhd_engine_set_family; the autotuner sets its choice.
 * Drops captured graphs. */
int shhd_engine_set_launch_shape(shhd_engine* engine, int row_blocks, int col_blocks);

/* The launch shapes the engine uses: *row_blocks 2 or 3 (0 when the row kernel
 * is not the pair-line row pass), *col_blocks 2, 3 or 4 (0 without pair-line
 * kernels); either pointer may be NULL. */
int shhd_engine_launch_shape(const shhd_engine* engine, int* row_blocks, int* col_blocks);

/* Initial conditions generated on the device: the reference's `set` styles
 * (initial_condition_*.cc), one field of one member per call, every active
 * mode evaluated in FP64 (FP32 engines round once and keep the (0, 0) value
 * in their FP64 copy).  Wave numbers are 2 pi g / L; Ng = nx * ny (padded).
 *
 *   GAUSSIAN_MODES      sigma(k) xi_k at k != 0, sigma(k)^2 = s0 / (c0 + c2 k^2
 *                       + c4 k^4), xi_k the equilibrium styles' complex unit
 *                       Gaussian for (seed, channel, kx, ky); `mean` at (0, 0).
 *                       uniform (s0 = 0), equilibrium/gaussian density and
 *                       order parameter, equilibrium/gaussian/compressible
 *                       momentum (channel = direction).
 *   TRANSVERSE_GAUSSIAN equilibrium/gaussian/incompressible momentum, direction
 *                       `channel`: (-ky/k or kx/k) sqrt(s0) xi_k (key channel 0).
 *   RANDOM_VORTICITY    random_vorticity, direction `channel`: the shell
 *                       exp(-((|n| - n0)/sigma)^2 / 2) with one random phase per
 *                       mode (seed, gx, ky), as velocity, normalised so the rms
 *                       velocity is `amplitude` (urms), times `rho0`.
 *   BUMP                gaussian: amplitude Ng 2 pi sx sy / (Lx Ly)
 *                       exp(-(sx^2 kx^2 + sy^2 ky^2)/2) e^{-i(kx x0 + ky y0)},
 *                       plus `mean` (base * Ng) at (0, 0).
 *   SINE                sine: -i amplitude Ng / 2 at (nkx, nky) (and its
 *                       conjugate on the kx = 0 line), `mean` at (0, 0).
 *
 * Errors are the reference's (e.g. a nonpositive chemical-potential
 * coefficient, a zero random-vorticity norm or reference density). */
enum shhd_ic_style {
    SHHD_IC_GAUSSIAN_MODES = 0,
    SHHD_IC_TRANSVERSE_GAUSSIAN = 1,
    SHHD_IC_RANDOM_VORTICITY = 2,
    SHHD_IC_BUMP = 3,
    SHHD_IC_SINE = 4
};

typedef struct shhd_initial_field {
    int style;                 /* enum shhd_ic_style */
    int channel;               /* key channel (GAUSSIAN_MODES) or direction 0 = x, 1 = y */
    uint64_t seed;             /* counter-based key (low 32 bits used) */
    double mean;               /* (0, 0) coefficient */
    double s0, c0, c2, c4;     /* variance law of GAUSSIAN_MODES / TRANSVERSE_GAUSSIAN (c0 = 1 for density, momentum) */
    double amplitude;          /* BUMP, SINE: amplitude; RANDOM_VORTICITY: urms */
    double rho0;               /* RANDOM_VORTICITY: reference density */
    double n0, sigma;          /* RANDOM_VORTICITY: shell radius and width in mode numbers */
    double x0, y0;             /* BUMP: centre */
    double sigma_x, sigma_y;   /* BUMP: widths */
    int nkx, nky;              /* SINE: mode numbers */
} shhd_initial_field;

int shhd_engine_set_initial_field(shhd_engine* engine, int member, int field, const shhd_initial_field* spec);

/* The incompressible check on the initial momentum (initial_condition.cc:7-40),
 * evaluated in FP64 on the two momentum specs: SHHD_EINVAL with the
 * reference's message when |k . j| > 1e-10 + 1e-10 |k| |j| at an active
 * k != 0. */
int shhd_engine_check_transverse(shhd_engine* engine, const shhd_initial_field* jx, const shhd_initial_field* jy);

/* GAUSSIAN_MODES with the given arguments (shorthand of shhd_engine_set_initial_field). */
int shhd_engine_set_gaussian_field(shhd_engine* engine, int member, int field, uint64_t seed, int channel, double mean, double s0,
                                   double c0, double c2, double c4);

/* Energy columns of the time-series measure (measure_time_series.cc:152-188,
 * 305-470) for one member, FP64 sums: out[0..3] = E_T, E_K, E_psi, E_C.
 * E_K: compressible, the sum over the padded grid of (jx^2 + jy^2) / (2 rho) dA
 * from the inverse-transformed fields; incompressible, cell / (2 Ng rho0) times
 * the weighted spectral sum of |j|^2; quiescent, 0.  E_C: compressible,
 * cT^2 cell / (2 Ng rho0) times the weighted sum of |rho|^2 over k != 0.  E_psi:
 * the quadratic chemical-potential terms spectrally, plus u psi^4 / 4 dA over
 * the padded grid for phi4.  The physical-space sums use their own transforms
 * (allocated on first use). */
int shhd_engine_energies(shhd_engine* engine, int member, double* out, size_t n);

/* k = 0 flux columns of the time-series measure (measure_time_series.cc:190-229):
 * after enabling, every step records, per member, the stage-weighted (0, 0)
 * coefficients of the momentum and order-parameter fluxes (pressure and
 * advective terms; gradient terms and noise vanish at k = 0).  read gives the
 * last step's values divided by nx * ny: out[0..2] = pi_xx, pi_xy, pi_yy, then
 * Jpsi[a]_x, Jpsi[a]_y per order parameter (n >= 3 + 2 * num_order_parameters).
 * Enabling drops captured graphs. */
int shhd_engine_flux0_enable(shhd_engine* engine);
int shhd_engine_flux0_read(shhd_engine* engine, int member, double* out, size_t n);

/* One sample of the ave/profile measure (measure_ave_profile.cc:180-374) for
 * one member.  axis 0 bins over x (averaging over y), axis 1 bins over y.
 * profile_line: the spectral line of `field` the profile needs, FP64 complex
 * as interleaved doubles: axis 0 the ky = 0 row over the active kx
 * (active_nx / 2 entries), axis 1 the kx = 0 column in the engine's ky order (ky = 0 .. Na/2 - 1, then
 * -(Na/2 - 1) .. -1).  The transverse sum of the field is the 1-D inverse
 * transform of that line.  profile_velocity: the compressible velocity
 * component j_c / rho summed over the transverse axis on the padded grid
 * (nx or ny doubles), FP64 sums on the device; SHHD_EINVAL with the
 * reference's message on a zero density. */
int shhd_engine_profile_line(shhd_engine* engine, int member, int field, int axis, double* out, size_t n);
int shhd_engine_profile_velocity(shhd_engine* engine, int member, int component, int axis, double* out, size_t n);

/* The step's flux buffer along one spectral line, for the ave/profile flux
 * targets (measure_ave_profile.cc:216-238): after enabling an axis (0: the
 * ky = 0 row, 1: the kx = 0 column), every step records per member the
 * stage-weighted fluxes the deterministic RHS records at the line's modes,
 * the first noise draw's flux / sqrt(dt) and, incompressible, the projection
 * pressure.  read gives the last step's values as interleaved complex doubles
 * [comp][line], comp = pi_xx, pi_xy, pi_yy, then Jpsi[a]_x, Jpsi[a]_y; the line
 * in the order of shhd_engine_profile_line.  Refused with replayed (external)
 * noise when the noise is on.  Enabling drops captured graphs. */
int shhd_engine_flux_line_enable(shhd_engine* engine, int axis);

/* Which steps an enabled flux tap records (tap 0: the k = 0 fluxes, 1: the
 * ky = 0 line, 2: the kx = 0 line): the steps whose engine step index after
 * the step is phase modulo period (default every step).  A measure that
 * samples every nevery steps needs no other; the others cost one early-exit
 * launch per stage.  Changing it drops captured graphs. */
int shhd_engine_flux_tap_schedule(shhd_engine* engine, int tap, int64_t period, int64_t phase);
int shhd_engine_flux_line_read(shhd_engine* engine, int axis, int member, double* out, size_t n);

/* Spectral L2 columns of the time-series measure (measure_time_series.cc:
 * |rho|^2, |d_rho|^2, |j|^2, |d_j|^2, |psi[a]|^2, |d_psi[a]|^2) for one member
 * of the current state, in FP64 on the device: out[2 f] = (V / Np^2) / Np^2
 * * sum w |u_f|^2 and out[2 f + 1] the same with a factor k^2, over the active
 * modes but (0, 0), w = 2 off the kx = 0 line (n = 2 * nfields).  The
 * momentum columns are the sums of the jx and jy entries. */
int shhd_engine_l2_sums(shhd_engine* engine, int member, double* out, size_t n);

/* Yokota-Green-Kubo stress measure (measure_yokota_green_kubo.cc:16-225),
 * accumulated on the device in FP64.  shhd_engine_gk_enable selects the wave
 * vectors as the reference does (selection 0 "diagonal": (n, n), 1 "all"),
 * and from then on every step adds, per member and mode, the step's momentum
 * flux pi_xy (stage-weighted deterministic flux plus the first noise draw's
 * flux / sqrt(dt)) to the block integral I and, every `nevery` steps of a
 * block of `nblock`, |I|^2 / (2 tau kBT V) to the sum for that tau.  A
 * member's blocks count from its own first step (serving: step_origin).
 * shhd_engine_gk_read copies one member's sums in [tau][mode] order
 * (ntau = nblock / nevery; the reference's S_mean = sum / *nsample) and the
 * number of completed blocks since the last reset.  Needs kBT > 0, momentum
 * dynamics and the engine's own (Philox) noise. */
int shhd_engine_gk_enable(shhd_engine* engine, int nevery, int nblock, int selection);
int shhd_engine_gk_read(shhd_engine* engine, int member, double* sums, size_t n, int64_t* nsample, int reset);

/* Step counter and time (project.h:136-137). */
int shhd_engine_set_time(shhd_engine* engine, int64_t step_index, double time);

/* Kernel statistics (no reference counterpart).  Kinds: 0 column inverse,
 * 1 row pass, 2 column forward + epilogue, 3 other.  Launch counts and
 * algorithmic HBM bytes accumulate always; per-kernel device time (CUDA
 * events around each launch on the engine stream) only while profiling is on. */
int shhd_engine_set_profiling(shhd_engine* engine, int on);
int shhd_engine_kernel_stats(shhd_engine* engine, double* total_ms, int64_t* launches, double* bytes);
int shhd_engine_reset_stats(shhd_engine* engine);

/* CUDA stream the engine launches on (cudaStream_t as void*). */
void* shhd_engine_stream(shhd_engine* engine);

/* Device pointers of the current state of all members, in the engine's own
 * active-mode layout [member][field][gx < active_nx/2][j < active_ny-1]
 * (j = ky for 0 <= ky < active_ny/2, else ky + active_ny - 1), complex
 * float or double per `precision`.  Valid until the next step call. */
const void* shhd_engine_state_device(const shhd_engine* engine);

/* Deterministic right-hand side of one state without any device allocation.
 * No counterpart in the reference: it exists for hosts that must not call
 * cudaMalloc, such as a solver running inside a framework whose caching
 * allocator already owns the GPU's memory, or a plugin loaded into a process
 * that reserved its device memory up front.  Such a caller passes device
 * buffers it owns: state_dev (the input State, reference layout, FP64) and
 * rhs_dev (same layout; receives what shhd_engine_rhs would return for that
 * state), n_doubles = info.state_doubles, cfg->batch = 1.  The work is
 * enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream) and
 * the call returns once it has finished.
 *
 * Every intermediate lives in one array of SHHD_NOALLOC_SCRATCH_BYTES compiled
 * into the library, which each GPU that loads the library holds until the
 * process exits.  A configuration that needs more is rejected with SHHD_EINVAL
 * and a message giving the size it needs (32 MiB covers, for example, a 256^2
 * grid with 3/2 padding, two order parameters and advection in FP64).  Each
 * call looks up the current device's address of the array.  The call is
 * synchronous: it waits on `stream` for its input checks and again for its
 * result before returning, so it cannot be recorded into a CUDA graph; on a
 * stream that is being captured it returns SHHD_EINVAL and enqueues nothing.
 * All calls share the one array, which keeps the
 * last call's contents, so calls whose work overlaps on the GPU (other
 * streams or host threads) race: serialise them. */
#define SHHD_NOALLOC_SCRATCH_BYTES (32u << 20)
int shhd_rhs_noalloc(const shhd_config* cfg, const double* state_dev, double* rhs_dev, size_t n_doubles, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SHHD_B200_H */
