/*
 * uph_surrogate.h -- C ABI of the learned surrogate.
 *
 * The reference has no learned part; everything declared here is a project
 * addition that sits beside the plain solver of uph.h.  A message-passing
 * network over the solver's own radius-2h neighbour graph predicts how the
 * fluid state changes over `macro_steps` SPH steps; it is trained on the GPU
 * from trajectories the plain solver generates, and when it advances a
 * simulation the plain solver re-runs every `judge_every`-th macro step as
 * the judge of its density and free-surface error, taking over whenever a
 * threshold is exceeded.
 *
 * Network (latent width 128, `rounds` rounds, BF16 weights and activations
 * on the tcgen05 tensor cores, FP32 accumulation):
 *   h    = Enc2 relu(Enc1 f + b) + b                 f: node features
 *   per round:  [P | Q] = W_pq h + b
 *               s_i = sum_j relu(P_i + Q_j + W_e e_ij)
 *                 e_ij = ((dx, dy, r) / R, (rho_j - rho_i) / (rho0 s_e))  (FP32)
 *               m_i = W_2 s_i
 *               h  <- h + N2 relu(N1 [h ; m] + b) + b
 *   out  = Dec2 relu(Dec1 h + b) + b                 5 normalised increments
 * Node features: u/U, v/U, (rho/rho0 - 1)/s_rho and the node's kind
 * (fluid itype 1, moving wall itype 3, any other fixed).  Fluid increments
 * over one macro step of length T = macro_steps * dt:
 *   x += T u + s0 o0,  y += T v + s1 o1,  u += s2 o2,  v += s3 o3,
 *   rho += s4 o4,  p = Tait(rho).
 *
 * All pointers are device pointers unless marked host; calls are
 * asynchronous on the handle's stream except where they return host values.
 * Device-side failures (neighbour capacity, non-finite values, a bounded
 * wait that gave up) surface as uph_status codes at the next synchronising
 * call.
 */
#ifndef UPH_SURROGATE_H
#define UPH_SURROGATE_H

#include <stdint.h>

#include "uph.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] = A[M x K] . B[N x K]^T on the tcgen05 tensor cores: BF16
 * inputs (row-major, K contiguous), FP32 accumulation in TMEM.  K must be a
 * multiple of 64, N of 128, leading dimensions of 8.
 *   splits == 1: optional bias[N] and ReLU, then FP32 and/or BF16 output;
 *   splits  > 1: K is split across CTAs, FP32 partials (splits * M * N
 *                floats in `partials`) are summed in a fixed order into
 *                c_f32 (dense, ldc == N), added to its contents when
 *                accumulate != 0. */
uph_status uph_tc_gemm_bf16(const void *A, int32_t lda, const void *B, int32_t ldb, int32_t M, int32_t N,
                            int32_t K, const float *bias, int32_t relu, float *c_f32, void *c_bf16, int32_t ldc,
                            int32_t splits, float *partials, int32_t accumulate, unsigned *err, void *stream);

/* Failure-detection self test of the tensor-core kernels' bounded waits: one
 * 128 x 128 x 64 tile (A, B device BF16 [128 x 64], c_f32 device [128 x 128])
 * whose CTA first waits on an mbarrier that nothing arrives at.  The wait
 * gives up after about a second, the kernel sets ERR_TIMEOUT in the device
 * word *err, frees its TMEM and returns.  Returns UPH_TIMEOUT when that
 * happened; the CUDA context stays usable. */
uph_status uph_tc_wait_selftest(const void *A, const void *B, float *c_f32, unsigned *err, void *stream);

typedef struct uph_surrogate uph_surrogate;

#define UPH_SUR_LATENT 128
#define UPH_SUR_OUTPUTS 5
#define UPH_SUR_MAX_DEGREE 32
#define UPH_SUR_MAX_ROUNDS 4

typedef struct {
  int32_t rounds;        /* message-passing rounds, 1..UPH_SUR_MAX_ROUNDS (3) */
  int32_t macro_steps;   /* SPH steps one network step covers */
  double radius;         /* graph radius R (the SPH interaction radius 2h) */
  double dt;             /* SPH time step */
  double rho0;           /* reference density */
  double vel_scale;      /* U */
  double rho_scale;      /* s_rho */
  double edge_rho_scale; /* s_e: unit of the edge density difference, relative to rho0 */
  double out_scale[UPH_SUR_OUTPUTS]; /* s0..s4 */
} uph_sur_config;

/* One graph's nodes: fluid nodes first ([0, n_fluid)), then walls.  Every
 * node lies inside [lo, hi]; at most UPH_SUR_MAX_DEGREE partners each. */
typedef struct {
  int32_t n, n_fluid;
  const double *x, *y, *u, *v, *rho;
  const int32_t *itype;
  double lo_x, lo_y, hi_x, hi_y;
} uph_sur_nodes;

uph_status uph_sur_create(const uph_sur_config *cfg, int32_t node_capacity, uph_surrogate **out);
uph_status uph_sur_destroy(uph_surrogate *s);
uph_status uph_sur_set_stream(uph_surrogate *s, void *stream);
/* number of FP32 parameters for `rounds` rounds (storage layout: the
 * blocks enc1.w enc1.b enc2.w enc2.b, per round pq.w pq.b we[128 x 4 edge
 * features] w2 n1.w
 * n1.b n2.w n2.b, then dec1.w dec1.b dec2.w dec2.b; matrices [out x in]) */
int64_t uph_sur_param_count(int32_t rounds);
uph_status uph_sur_set_params(uph_surrogate *s, const float *host, int64_t count);
uph_status uph_sur_get_params(uph_surrogate *s, float *host, int64_t count);
/* on != 0 (the default): uph_sur_forward and uph_sur_advance run the
 * network through the fused node-chain kernels (one per round, every layer
 * of a round on chip); 0: one GEMM per layer, as the training path does.
 * Both compute the same network. */
uph_status uph_sur_set_fused(uph_surrogate *s, int32_t on);
/* resets the Adam moments and step count */
uph_status uph_sur_reset_optimizer(uph_surrogate *s);

/* network outputs [n x 5] (normalised increments) for every node */
uph_status uph_sur_forward(uph_surrogate *s, const uph_sur_nodes *nodes, float *out);
/* forward + mean-squared-error loss against target [n_fluid x 5] + backward:
 * writes dL/dparams into grad (count floats; NULL keeps them internal) and
 * the loss into *loss (host; NULL skips the synchronisation) */
uph_status uph_sur_gradients(uph_surrogate *s, const uph_sur_nodes *nodes, const float *target, float *grad,
                             double *loss);
/* one Adam step on the gradients of the last uph_sur_gradients call, with
 * the gradient scaled down to global norm <= clip when clip > 0 */
uph_status uph_sur_adam(uph_surrogate *s, double lr, double beta1, double beta2, double eps, double clip);

typedef struct {
  int32_t judge_every;     /* every judge_every-th macro step is re-run by the plain solver (10) */
  int32_t fallback_macro;  /* after a failed check the plain solver runs this many macro steps */
  double max_rho_err;      /* RMS relative density error allowed (0.01) */
  double max_surface_err;  /* free-surface height error allowed, fraction of depth (0.02) */
  double depth;            /* still-water depth */
  double surface_x0, surface_x1;  /* free-surface bins span [x0, x1) ... */
  int32_t surface_bins;            /* ... in this many equal bins (<= 4096) */
} uph_sur_judge;

typedef struct {
  int64_t macro_steps;      /* macro steps advanced */
  int64_t network_steps;    /* macro steps the network advanced */
  int64_t judged_steps;     /* macro steps checked against the plain solver */
  int64_t failed_checks;    /* checks over a threshold (each starts a fallback) */
  int64_t plain_steps;      /* SPH steps the plain solver ran */
  int64_t graph_overflows;  /* macro steps handed to the plain solver because a
                               node had more than UPH_SUR_MAX_DEGREE partners
                               (each also starts a fallback) */
  int64_t rejected_steps;   /* predictions the sanity guard rejected (a value
                               not finite, a density beyond rho0 (1 +- 0.05), a
                               particle moved further than the graph radius or
                               out of the simulation's domain);
                               the plain solver took the macro step and the
                               fallback after it */
  double last_rho_err, last_surface_err;
  double max_rho_err, max_surface_err;
} uph_sur_report;

/* Advances a WCSPH simulation by `macro_steps` macro steps (each
 * cfg.macro_steps SPH steps).  A predicted fluid position closer than
 * 0.25 R to a wall particle (advanced by its velocity) is moved back out to
 * 0.25 R and its velocity into the wall removed; every prediction then
 * passes a sanity guard; a network step replaces the fluid state and
 * restarts the simulation's leapfrog.  A judged step also runs the plain solver over
 * the same macro step from the same state and compares the prediction with
 * its result (RMS relative density error, largest free-surface height
 * difference): a passing prediction is kept, a failing one leaves the plain
 * state and hands the next fallback_macro macro steps to the plain solver.  Counts accumulate into *report (host).  The judge
 * schedule (macro steps since the last check, fallback steps left) carries
 * over between calls on the same simulation and restarts for another one. */
uph_status uph_sur_advance(uph_surrogate *s, uph_sim *sim, int32_t macro_steps, const uph_sur_judge *judge,
                           uph_sur_report *report);

#ifdef __cplusplus
}
#endif

#endif /* UPH_SURROGATE_H */
