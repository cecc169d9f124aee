/*
 * uph.h -- C ABI of the B200 SPH hot path.
 *
 * The library advances the reference solver's per-timestep hot path on one
 * GPU: neighbour search (cell list in place of the kd-tree), the smoothing
 * kernel, the continuity and Tait-EOS update, pressure / viscous / wall forces
 * and the leapfrog kick-drift.  Every entry point takes plain pointers and
 * sizes, returns a uph_status and never exits the process.
 *
 * Particle order and layout follow the reference's System struct
 * (src/lib/System.h:13-153): index ranges
 *     [0, n_fluid)                          fluid
 *     [n_fluid, +n_solid)                   solid
 *     [.., +n_fixed)                        fixed boundary
 *     [.., +n_moving)                       moving boundary
 * and vectors are row-major [n][2] doubles, exactly the memory behind the
 * reference's double** matrices (System.c:10-18, CreateMatrix), so a caller
 * can pass sys->Position[0] and friends directly.
 *
 * Reference interfaces each group replaces:
 *   uph_search_neighbors  <- SearchNeighbors       src/lib/Search.cc:5
 *   uph_sim_derivatives   <- derivatives           src/lib/derivatives.h:12 (derivatives.c:3137)
 *   uph_sim_step          <- the time loop         src/bin/sph.cc:90-168
 *   uph_params_from_deck  <- CreateSystem params   src/lib/System.c:38-345
 *   uph_deck_read         <- input + inputbp read  src/lib/input.c:22-164, src/lib/inputbp.c:12-191
 * The layout-compatible System drop-in (derivatives / SearchNeighbors with
 * the reference's own signatures) is declared in uph_system.h.
 */
#ifndef UPH_H
#define UPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UPH_ABI_VERSION 1

typedef enum uph_status {
  UPH_OK = 0,
  UPH_BAD_ARG = 1,           /* a pointer, size or parameter is invalid */
  UPH_OUT_OF_DOMAIN = 2,     /* a particle left the cell grid's domain */
  UPH_NEIGHBOR_OVERFLOW = 3, /* a pair or cell capacity was exceeded */
  UPH_NAN = 4,               /* a non-finite value appeared in the state */
  UPH_TIMEOUT = 5,           /* a bounded device-side wait gave up */
  UPH_CUDA_ERROR = 6,        /* a CUDA runtime call failed */
  UPH_NO_DEVICE = 7,         /* no CUDA device is visible */
  UPH_UNSUPPORTED = 8,       /* a reference mode this library does not implement */
  UPH_OUT_OF_MEMORY = 9,
  UPH_IO_ERROR = 10          /* a deck file is missing or malformed, or an output file cannot be written */
} uph_status;

/* Physics profiles.
 *   REF   : the reference's active formulation, derivatives.c:4196-4326 with
 *           flagInitSimul == 1 -- poly-7 convolution / deconvolution kernel
 *           pair, predictor rates, local fluctuations, rate-form Tait with
 *           pressure / density diffusion, single-step deviatoric viscosity,
 *           gravity, sponge layer and the selected wall force.
 *   WCSPH : textbook weakly-compressible SPH on the same particles: the
 *           reference's cubic spline Kernel() (derivatives.c:44-66),
 *           continuity, algebraic Tait EOS (derivatives.c:1674-1682) feeding
 *           the pressure force, Monaghan artificial viscosity (Monaghan 1992,
 *           ARA&A 30:543, beta = 0) and the reference's wall forces, advanced
 *           with the same leapfrog structure as sph.cc:90-168. */
enum { UPH_PROFILE_REF = 0, UPH_PROFILE_WCSPH = 1 };

/* Pair arithmetic: FP64 everywhere, or (WCSPH only) FP32 pair forces and
 * density rates with FP64 positions, velocities and integration. */
enum { UPH_PREC_FP64 = 0, UPH_PREC_FP32_PAIR = 1 };

typedef struct uph_params {
  int32_t profile;   /* UPH_PROFILE_* */
  int32_t precision; /* UPH_PREC_* */
  int32_t n_fluid, n_solid, n_fixed, n_moving;

  /* parameters.dat fields, in file order (System.c:60-94) */
  double stroke, wave_period, local_depth, flat_bottom_length;
  double density0, adiabatic_constant, gravity, dx, dy;
  int32_t dim;
  double viscosity0, mach_number, peclet_number, epsilon, alpha;
  int32_t virtual_type, print_step, screen_step;
  double time_step, lid_velocity;
  int32_t near_neighbor, select_boundary_force;
  double lennard_select, spring_constant0, damping_constant0;
  int32_t flag_init_simul, gravity_flag;
  double thermal_diffusivity0;
  int32_t moving_boundary, number_of_initialization_steps;
  double pressure_probe_x, pressure_probe_y;
  int32_t stress_type, dissipation_control_volume;

  /* derived values (System.c:292-335, input.c:107) */
  double speed_of_sound;     /* c0 */
  double compression_factor; /* B = rho0 c0^2 / gamma */
  double omega;              /* 2 pi / wave_period */
  double eta;                /* h = eta * dx */
  double h;                  /* smoothing length of every particle */
  double lennard_coefficient;
  double sponge_factor0, sponge_position0;
  int32_t wave_absorption;

  /* WCSPH only: Monaghan viscosity coefficient (beta = 0) */
  double av_alpha;

  /* Neighbour search.  knn_cap = 0 keeps every pair inside the radius.  The
   * reference keeps only each fluid query's 40 nearest points
   * (derivatives.c:1085, Search.cc:27-33): knn_cap = 40 does the same --
   * query i keeps its knn_cap nearest in-radius points, ties ordered by
   * reference index, and a pair (i, j) exists iff j is kept by i.  Both
   * settings agree whenever no query has more than knn_cap in-radius
   * neighbours (uph_sim_stats reports the largest count).  REF profile
   * only; at most 64. */
  int32_t knn_cap;

  /* Cell-grid domain: every interacting particle must stay inside
   * [lo, hi] or the step fails with UPH_OUT_OF_DOMAIN. */
  double domain_lo[2], domain_hi[2];
} uph_params;

/* Host particle arrays in the reference's layout.  "all" arrays hold
 * n = n_fluid + n_solid + n_fixed + n_moving entries, "fluid" arrays n_fluid.
 * Field names are the reference's System names.  A NULL pointer is allowed
 * where noted. */
typedef struct uph_state {
  double *Position;            /* all  [n][2] */
  double *Velocity;            /* all  [n][2] */
  double *localVelocity;       /* all  [n][2] */
  double *density;             /* all */
  double *localDensity;        /* all */
  double *DynamicPressure;     /* all */
  double *localPressure;       /* all */
  double *mass;                /* all */
  int32_t *itype;              /* all */
  double *Velocity_min;        /* fluid [n_fluid][2] */
  double *density_min;         /* fluid */
  double *DynamicPressure_min; /* fluid */
  double *spongeFactor;        /* fluid, may be NULL (zero) */
  /* rates of the last derivatives() evaluation (fluid) */
  double *ddensitydt, *dpdt, *dvdt;                      /* dvdt [n_fluid][2] */
  double *ddensitydt_approx, *dpdt_approx, *dvdt_approx; /* dvdt_approx [n_fluid][2] */
  double *densityFluctuation, *pressureFluctuation;      /* fluid */
  double *velocityFluctuation;                           /* fluid [n_fluid][2] */
  double *Pressure;                                      /* all, algebraic Tait (diagnostic) */
} uph_state;

typedef struct uph_stats {
  int64_t niac;            /* interaction pairs (i < j) of the last evaluation */
  int32_t max_neighbors;   /* largest in-radius neighbour count of a fluid particle */
  int32_t itime;           /* completed leapfrog steps */
  double kinetic_energy;   /* sum 0.5 m |v|^2 over fluid (derivatives.c:2254-2264) */
  double potential_energy; /* sum m g y over fluid */
  double total_mass;       /* sum m over fluid */
  double max_abs_density_error; /* max |rho - rho0| / rho0 over fluid */
  int64_t list_builds;     /* cell-list builds that re-binned the particles since the simulation was made
                              (a step rebuilds when a particle moved more than the skin; uploads and storage
                              re-sorts sort too) */
} uph_stats;

typedef struct uph_sim uph_sim;

/* ---- set-up -------------------------------------------------------------- */

/* Fills `out` from the 34-field parameters.dat (System.c:60-94) and applies the
 * derivations of System.c:292-335.  Counts are left to the caller (or
 * uph_deck_read).  eta_override > 0 replaces eta = sqrt(nearNeighbor / 4 pi). */
uph_status uph_params_from_file(const char *parameters_dat, double eta_override, uph_params *out);

/* Recomputes the derived fields of `p` from its parameters.dat fields. */
uph_status uph_params_derive(uph_params *p, double eta_override);

/* Reads a deck directory (parameters.dat + the particle files of
 * input.c:57-72 / inputbp.c:88-150) into caller-owned arrays.  Call once with
 * st == NULL to get the counts in *p, allocate, then again to fill. */
uph_status uph_deck_read(const char *deck_dir, double eta_override, uph_params *p, uph_state *st);

/* ---- resident simulation -------------------------------------------------- */

/* Allocates device state for p's particle counts on the current CUDA device. */
uph_status uph_sim_create(const uph_params *p, uph_sim **out);
uph_status uph_sim_destroy(uph_sim *sim);

/* Issues all later work of `sim` on this cudaStream_t (NULL: the sim's own). */
uph_status uph_sim_set_stream(uph_sim *sim, void *cuda_stream);

/* Host -> device.  `itime` is the number of leapfrog steps already taken by
 * this state (0 for a fresh deck: the next step is the reference's itime==1
 * branch).  Rates are read too: the next step's predictor needs them. */
uph_status uph_sim_upload(uph_sim *sim, const uph_state *st, int32_t itime);

/* Device -> host, reference order.  NULL fields are skipped. */
uph_status uph_sim_download(uph_sim *sim, uph_state *st);

/* Advances `nsteps` leapfrog steps (sph.cc:90-168) on the device. */
uph_status uph_sim_step(uph_sim *sim, int32_t nsteps);

/* Records the kernel sequence of a `steps_per_graph`-step call into a CUDA
 * graph on the first such call (after the simulation's first step) and
 * replays it on later calls of the same length: one host launch per call
 * instead of ~10 per step.  0 turns graphs off.  (The reference has no
 * counterpart; its loop is sph.cc:90-168.) */
uph_status uph_sim_set_graph(uph_sim *sim, int32_t steps_per_graph);

/* Whether the rate pass applies the leapfrog step in its epilogue
 * (default 1): the pass then writes each fluid particle's corrected state
 * and the next step's predictor into the simulation's second state buffer,
 * which becomes the current one, and no separate corrector launch runs.
 * The state is bit-identical either way (0 runs the pass and the corrector
 * as two launches).  Applies to the WCSPH profile, and to the REF profile
 * with flagInitSimul 1 and stressType 1, while diagnostics are off;
 * elsewhere the corrector always runs separately.  (The reference's
 * corrector is sph.cc:137-168.) */
uph_status uph_sim_set_fused_step(uph_sim *sim, int32_t enable);

/* Whether the rate passes keep a candidate list per fluid particle between
 * cell-list builds (default 1): at a build's first pass each particle lists
 * the records of its tile's block within the search radius plus twice the
 * largest displacement before the next build (up to 24 of them), and the
 * passes until the next build test only those instead of walking the cell
 * stencil.  The pairs, their order and so the results are bit-identical
 * either way.  (The reference rebuilds its kd-tree search every call,
 * Search.cc:5-44.) */
uph_status uph_sim_set_candidate_lists(uph_sim *sim, int32_t enable);

/* Execution tuning (no counterpart in the reference): cell width = search
 * radius / reach (reach 1-3), particle-storage tile edge in cells (power of
 * two <= 32) and the storage re-sort interval in steps.  Defaults 2, 8, 16. */
uph_status uph_sim_set_tuning(uph_sim *sim, int32_t reach, int32_t tile, int32_t reorder_interval);

/* Picks the tuning by timing `trial_steps` steps per candidate on this
 * simulation (a coordinate search over reach, tile and interval; it advances
 * the simulation by about 9 (trial_steps + 2) steps) and applies the fastest.
 * Results are cached per size class, so later sims of the same class are
 * tuned without trials.  choice[3] receives (reach, tile, interval);
 * *ms_per_step the best trial's time (0 when taken from the cache). */
uph_status uph_sim_autotune(uph_sim *sim, int32_t trial_steps, int32_t choice[3], double *ms_per_step);

/* Shakes the moving-boundary block horizontally, one entry per moving
 * particle (reference order): x = x0 + half_stroke (1 - cos(omega t)),
 * u = half_stroke omega sin(omega t).  This generalises the reference's
 * piston and sloshing walls (inputbp.c:194-207, 244-276) to tanks that move
 * rigidly with their own amplitude and period.  NULL pointers switch back to
 * the movingBoundary mode of the parameters. */
uph_status uph_sim_set_wall_motion(uph_sim *sim, const double *x0, const double *half_stroke,
                                   const double *omega);

/* Base coordinates of the lid (movingBoundary 3: x = base + lidVelocity t)
 * or the gate (movingBoundary 2: y = base + lidVelocity min(t, t_stop)),
 * one per moving boundary particle in reference order: the reference's
 * tempPosition / tempPositionGate deck columns (inputbp.c:209-243).  An
 * upload sets them from the uploaded positions (at itime 0: the positions
 * themselves); this call replaces them. */
uph_status uph_sim_set_wall_base(uph_sim *sim, const double *base);

/* One rate evaluation at time t on the uploaded state, no integration: what
 * the reference's derivatives() computes for the hot path. */
uph_status uph_sim_derivatives(uph_sim *sim, double t);

/* Pairs (i < j, reference indices) of the last evaluation, ordered by i then
 * j, with rij2, the convolution kernel w and the gradient dwcdx [niac][2]
 * (derivatives.c:1088-1105).  *niac gets the pair count even when it is
 * larger than `cap` (then UPH_NEIGHBOR_OVERFLOW and nothing is written).
 * Any output pointer may be NULL. */
uph_status uph_sim_pairs(uph_sim *sim, int64_t cap, int32_t *i_pair, int32_t *j_pair, double *rij2,
                         double *w, double *dwcdx, int64_t *niac);

/* The virtual mirror particles of the last evaluation (virtualType 1, 3, 4,
 * 5, 7, 8; derivatives.c:3194-4192), in the reference's order: the reference
 * index of virtual particle k is n_fluid + n_solid + n_fixed + n_moving + k.
 * position [count][2]; src: the reference index of the fluid particle it
 * copies; rule: the mirror that made it (each appears once per type):
 * 0 left wall (u flipped), 1 right wall (u), 2 bottom (v), 3 top (v),
 * 4 bottom-left corner (u, v), 5 bottom-right corner (u, v), 6 the slope of
 * virtualType 1 (velocities reflected in it).  *count is set even when it exceeds `cap` (then
 * UPH_BAD_ARG and nothing is written when an array is given); all arrays may
 * be NULL.  They are never in a pair (j < Nf + Ns + Nb - 1,
 * derivatives.c:1081-1083): they are points of the knn-capped search only. */
uph_status uph_sim_virtual(uph_sim *sim, int64_t cap, double *position, int32_t *src, int32_t *rule,
                           int64_t *count);

/* The reference's approxVorticity of every fluid particle ([n_fluid], by
 * reference index) on the current state and pair set: each pair adds
 * V_partner (dv_y dx - dv_x dy) w / (r^2 + 0.01 h^2) to both of its
 * particles (ApproximateVortcity, derivatives.c:2840-2885).  A diagnostic
 * printed in out<k>.dat; REF profile. */
uph_status uph_sim_approx_vorticity(uph_sim *sim, double *vorticity);

uph_status uph_sim_stats(uph_sim *sim, uph_stats *out);

/* The reference's per-evaluation diagnostics, computed on the device at the
 * state each derivatives() call sees (before the step's corrector), as
 * sph.cc's output() later prints them:
 *   kinetic/potential energy: TotalKineticEnergy (derivatives.c:2254-2264),
 *           sums of 0.5 m |v|^2 and m g y over the fluid;
 *   point:  NeighborsToPressurePoint (derivatives.c:2290-2338) -- Gaussian-
 *           weighted DynamicPressure over fluid within 3h of the probe with
 *           p > 0: w = (exp(-r^2/h^2) - e^-9) m / (2 pi h^2 (0.5 - 5 e^-9) rho),
 *           point_pressure = sum p w / sum w, pressure_norm = sum w (1 when
 *           nothing is in range, and point_pressure then keeps its previous
 *           value, 0 at creation), point_neighbors = count;
 *   two:    NeighborsToPressurePointTwo + EnsembleAveragedPointPressureTwo
 *           (derivatives.c:2340-2393) -- mean p over fluid within 2h of the
 *           second probe with p > 0.
 * Sums run in a fixed order (not the reference's serial one).  itime is the
 * step whose evaluation the values belong to (0: none yet). */
typedef struct uph_diagnostics {
  double kinetic_energy, potential_energy;
  double point_pressure, pressure_norm, point_pressure_two;
  int32_t point_neighbors, point_neighbors_two;
  int32_t itime;
} uph_diagnostics;

/* Turns the diagnostics on (one extra kernel per step) or off.  The first
 * probe is parameters.dat's pressureProbeX/Y (System.c:91-92); the reference
 * never sets the second one, so its (0, 0) is what reproduces its files. */
uph_status uph_sim_set_diagnostics(uph_sim *sim, int32_t enable, double probe_x, double probe_y, double probe_x2,
                                   double probe_y2);
/* The values of the last evaluation (UPH_BAD_ARG while diagnostics are off). */
uph_status uph_sim_diagnostics(uph_sim *sim, uph_diagnostics *out);

/* The reference's output() (output.c:19-140) for a downloaded state, in
 * `directory`: writes out<itime>.dat (one line per particle: index, x, y, u,
 * v, density, mass, hsml, DynamicPressure, damGateFlag, approxVorticity,
 * itype, specificDissipationRate, localDensity in the reference's formats;
 * hsml is p->h, dam_gate_flag may be NULL (written as 0), and the vorticity
 * and dissipation rate, which feed nothing on this path, are written as 0)
 * and appends a line to TotalKineticEnergy.dat, PointPressure.dat and
 * PointPressureTwo.dat from `diag`; at itime == number_of_initialization_steps
 * it appends the fluid to FluidParticleInit.dat (its tempPosition and
 * tempPositionGate columns, deck inputs nothing on this path reads, as 0).
 * The dissipation and control-volume files (PowerCalc.dat, ControlVol*.dat)
 * are not written.  The appended files are the caller's to truncate at the
 * start of a run, as sph.cc does before its time loop. */
uph_status uph_write_output(const char *directory, int32_t itime, const uph_params *p, const uph_state *st,
                            const int32_t *dam_gate_flag, const uph_diagnostics *diag);

/* Device time per kernel family since the last reset, measured with CUDA
 * events when profiling is on.  names: comma-separated list written to
 * `names` (size `names_len`); ms / launches: arrays of `n` entries. */
uph_status uph_sim_profile(uph_sim *sim, int32_t enable);
uph_status uph_sim_kernel_times(uph_sim *sim, int32_t n, double *ms, int64_t *launches, char *names,
                                size_t names_len, int32_t *n_written);
/* Kernels this sim has launched since creation. */
int64_t uph_sim_launch_count(const uph_sim *sim);

/* ---- one-shot neighbour search -------------------------------------------- */

/* SearchNeighbors semantics (Search.cc:5-44): pairs (s, j) with s <
 * n_fluid, j > s, rij2 < dist, j < particle_boundary, DBL_EPSILON < rij2
 * (no self matches), ordered by s then j.  knn (the reference passes 40;
 * at most 64, 0 = no cap) keeps each query's knn nearest in-radius points,
 * ties by index, as uph_params.knn_cap.  Host arrays in, host arrays out. */
uph_status uph_search_neighbors(const double *position, int32_t n_fluid, int32_t n_all,
                                int32_t particle_boundary, int32_t knn, double dist, int64_t cap,
                                int32_t *i_pair, int32_t *j_pair, double *rij2, int64_t *niac);

/* The same search for callers that must not allocate GPU memory: code that
 * runs inside a host application's own memory pool, a real-time loop where
 * an allocation could stall, or a plugin host that forbids cudaMalloc after
 * start-up.  No counterpart in the reference.
 * position, i_pair, j_pair and rij2 are DEVICE buffers owned by the caller;
 * the grid box [lo, hi] must contain every position.  Scratch lives in one
 * statically sized __device__ array of the library (about 11 MiB, held by
 * every GPU that loads the library until exit); no call allocates.
 * Limits: n_all <= 262,144 particles and at most 524,288 search cells of width
 * sqrt(dist) over [lo, hi]; larger inputs return UPH_BAD_ARG.  A cell holding
 * more than 4,096 particles returns UPH_NEIGHBOR_OVERFLOW with *niac = 0.
 * Unlike uph_search_neighbors (and the reference's 40-NN search) there is no
 * knn cap: every in-radius pair is returned.  Pair offsets and *niac are
 * 64-bit; *niac is the full count even when it exceeds cap (then
 * UPH_NEIGHBOR_OVERFLOW, and only the first cap pairs are written).
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  Calls share the array, so calls that
 * overlap on the GPU race.  The call synchronises `stream` (a cudaStream_t,
 * NULL for the default stream) to return *niac and the status. */
uph_status uph_search_neighbors_noalloc(const double *position, int32_t n_fluid, int32_t n_all,
                                        int32_t particle_boundary, double dist, const double lo[2],
                                        const double hi[2], int64_t cap, int32_t *i_pair, int32_t *j_pair,
                                        double *rij2, int64_t *niac, void *stream);

/* ---- self-tests ------------------------------------------------------------ */

/* y[k] = the reciprocal the rate passes use in place of 1.0 / x[k] (a
 * Newton-Raphson refinement of the hardware's approximate FP64 reciprocal),
 * for n DEVICE values on `stream`; for testing its error against IEEE
 * division.  No counterpart in the reference (which divides). */
uph_status uph_rcp_selftest(const double *x, double *y, int64_t n, void *stream);

/* ---- errors ---------------------------------------------------------------- */

const char *uph_status_string(uph_status s);
/* Last error message of the calling thread ("" when none). */
const char *uph_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* UPH_H */
