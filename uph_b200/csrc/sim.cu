// uph_sim: resident device state and the step loop behind the C ABI.
//
// Device layout (all SoA doubles unless noted), "slot" order:
//   slots [0, nf)  fluid particles, spatially sorted by cell,
//   slots [nf, n)  solid / fixed / moving boundary particles, sorted by cell.
// S.orig[slot] is the particle's reference index; uploads and downloads
// permute through it, so callers only ever see reference order.  Every
// `reorder_interval` steps the fluid slots are re-sorted by their current
// cell so that a warp's particles keep sharing neighbour cells.
#include <float.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tile_pass.cuh"
#include "sim_access.cuh"

using namespace uph;

namespace uph {
}

namespace {

// Storage re-sorts keep a tile's particles in nearby slots; the tiled
// passes find particles through the cell list, so a stale order only costs
// coalescing.
constexpr int kReorderInterval = 64;
constexpr int kErrorCheckInterval = 64;
constexpr int kCellReach = 2;

enum KernelFamily { KF_PREDICT, KF_WALLS, KF_REFRESH, KF_CELLS, KF_PASS, KF_CORRECT, KF_REORDER, KF_COUNT };
const char *kFamilyNames[KF_COUNT] = {"predict", "wall_motion", "refresh", "cell_list", "rate_pass", "correct",
                                      "reorder"};

// staging buffers in reference order (the caller's layout)
struct Staging {
  double *pos, *vel, *lvel;  // [n][2]
  double *rho, *lrho, *p, *lp, *mass, *pressure;
  int32_t *itype;
  double *vmin;  // [nf][2]
  double *rhomin, *pmin, *sponge, *drho, *dp, *drho_a, *dp_a, *frho, *fp;
  double *acc, *acc_a, *fvel;  // [nf][2]
  double *tmp_x, *tmp_y;       // positions split for the key kernel
};

// the pressure-probe points of the per-evaluation diagnostics
struct DiagProbes {
  double x1, y1, x2, y2;
};

// the diagnostics of the last evaluation, as the reference's System holds them
struct DevDiag {
  double kinetic_energy, potential_energy;
  double point_pressure, pressure_norm, point_pressure_two;
  int point_neighbors, point_neighbors_two;
  int itime;
};

constexpr int kDiagRows = 7;

}  // namespace

struct uph_sim {
  uph_params hp;
  DevParams P;
  SlotArrays S, S2;
  CellGrid G;
  Staging T;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  unsigned *d_err = nullptr;
  // the rate pass's statistics, zeroed by the cell-list launch before it
  unsigned long long *d_niac = nullptr;
  int *d_max_nb = nullptr;
  int *d_perm = nullptr;  // scratch for uploads
  int itime = 0;
  int steps_since_reorder = 0;
  bool have_rates = false;
  int64_t launches = 0;
  bool profiling = false;
  // profiling: event pairs recorded around every kernel family without
  // synchronising; read back after the call's own final synchronisation
  static constexpr int kEventPool = 2048;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_family;
  int ev_used = 0;
  double fam_ms[KF_COUNT] = {0};
  int64_t fam_launch[KF_COUNT] = {0};
  std::vector<void *> allocations;
  double *d_partials = nullptr;
  int n_partials = 0;
  // device step counter (steps completed) and moving-wall table
  int *d_itime = nullptr;
  double *d_wall_tab = nullptr;
  WallTable W = {nullptr, nullptr, nullptr, 0};
  // CUDA graph of `graph_steps` steps, recorded on the first eligible call
  int graph_steps = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  const double *graph_buffer = nullptr;  // S.x when recorded: the buffer parity it needs
  int graph_since_after = 0;
  int64_t graph_launches = 0;
  int64_t graph_replays = 0;
  // tuning: storage re-sort interval and the grid arrays' capacity in cells
  int reorder_interval = kReorderInterval;
  long long grid_capacity = 0;
  long long tile_gen_capacity = 0;
  // the fluid state was replaced from outside (the learned surrogate): the
  // next step starts the leapfrog afresh with the first-step half kick
  bool restart = false;
  int64_t serial = 0;  // distinct for every simulation this process creates
  // the REF pass applies the leapfrog step (uph_sim_set_fused_step)
  bool fused_step = true;
  // the tiled passes keep per-particle candidate lists between cell-list
  // builds (uph_sim_set_candidate_lists)
  bool cand_lists = true;
  // per-evaluation diagnostics (off by default)
  bool diag_enabled = false;
  DiagProbes diag_probes = {0, 0, 0, 0};
  int diag_blocks = 0;
  double *d_diag_part = nullptr;  // [kDiagRows][diag_blocks]
  unsigned *d_diag_done = nullptr;
  DevDiag *d_diag = nullptr;
  // virtual mirror particles (virtual.cu): generated every evaluation when
  // the virtualType has rules; their own cell list feeds the knn cut
  VirtualBuf vb = {};
  CellGrid gv = {};
  double deriv_t = 0.0;  // the time of a uph_sim_derivatives call
  // pair export (uph_sim_pairs): counts and offsets by reference index, and
  // the pair arrays, grown as needed and kept
  int *pe_cnt = nullptr, *pe_off = nullptr, *pe_bsum = nullptr;
  int32_t *pe_ip = nullptr, *pe_jp = nullptr;
  double *pe_r2 = nullptr, *pe_w = nullptr, *pe_dw = nullptr;
  int64_t pe_cap = 0;
  bool kcut_fresh = false;  // the knn cut matches the current positions and cell list
};

namespace {

template <typename T>
cudaError_t dalloc(uph_sim *s, T **p, size_t count)
{
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
  if (e == cudaSuccess) s->allocations.push_back((void *)*p);
  return e;
}

cudaError_t alloc_slots(uph_sim *s, SlotArrays &A, int n, int nf)
{
  cudaError_t e = cudaSuccess;
  double **all[] = {&A.x, &A.y, &A.u, &A.v, &A.ut, &A.vt, &A.rho, &A.rhot, &A.p, &A.pt, &A.m, &A.inv_rho,
                    &A.inv_rhot, &A.pressure};
  for (double **p : all)
    if ((e = dalloc(s, p, (size_t)n)) != cudaSuccess) return e;
  if ((e = dalloc(s, &A.itype, (size_t)n)) != cudaSuccess) return e;
  if ((e = dalloc(s, &A.orig, (size_t)n)) != cudaSuccess) return e;
  double **fl[] = {&A.rho_min, &A.p_min, &A.u_min, &A.v_min, &A.sponge, &A.drho, &A.dp, &A.ax, &A.ay,
                   &A.drho_a, &A.dp_a, &A.ax_a, &A.ay_a, &A.frho, &A.fp, &A.fu, &A.fv};
  for (double **p : fl)
    if ((e = dalloc(s, p, (size_t)nf)) != cudaSuccess) return e;
  return cudaSuccess;
}

// adds the recorded event pairs to the per-family totals; the caller has
// synchronised the stream (or this waits for the last event)
void flush_profile(uph_sim *s)
{
  for (int k = 0; k < s->ev_used; k++) {
    cudaEvent_t a = s->ev_pool[2 * k], b = s->ev_pool[2 * k + 1];
    cudaEventSynchronize(b);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess) {
      s->fam_ms[s->ev_family[k]] += ms;
      s->fam_launch[s->ev_family[k]]++;
    }
  }
  s->ev_used = 0;
}

struct Timer {
  uph_sim *s;
  int fam;
  int slot = -1;
  Timer(uph_sim *s_, int f) : s(s_), fam(f)
  {
    if (!s->profiling || s->ev_pool.empty()) return;
    if (s->ev_used == uph_sim::kEventPool) flush_profile(s);
    slot = s->ev_used++;
    s->ev_family[slot] = fam;
    cudaEventRecord(s->ev_pool[2 * slot], s->stream);
  }
  ~Timer()
  {
    if (slot >= 0) cudaEventRecord(s->ev_pool[2 * slot + 1], s->stream);
  }
};

// ---- permutation kernels ------------------------------------------------------

__global__ void k_split_xy(const double *__restrict__ pos, double *__restrict__ x, double *__restrict__ y, int n)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    x[k] = pos[2 * k];
    y[k] = pos[2 * k + 1];
  }
}

// slots <- staging (reference order) through perm[slot] = reference index
__global__ void k_gather_upload(SlotArrays S, Staging T, const int *__restrict__ perm, int n, int nf, double rho0)
{
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = perm[s];
  S.orig[s] = o;
  S.x[s] = T.pos[2 * o];
  S.y[s] = T.pos[2 * o + 1];
  S.u[s] = T.vel[2 * o];
  S.v[s] = T.vel[2 * o + 1];
  S.ut[s] = T.lvel[2 * o];
  S.vt[s] = T.lvel[2 * o + 1];
  S.rho[s] = T.rho[o];
  S.p[s] = T.p[o];
  // walls and solids: localDensity = rho0 and localPressure = 0, as inputbp
  // sets them before every derivatives() (inputbp.c:289-290)
  S.rhot[s] = s < nf ? T.lrho[o] : rho0;
  S.pt[s] = s < nf ? T.lp[o] : 0.0;
  S.m[s] = T.mass[o];
  S.itype[s] = T.itype[o];
  S.pressure[s] = T.pressure[o];
  if (s < nf) {
    S.rho_min[s] = T.rhomin[o];
    S.p_min[s] = T.pmin[o];
    S.u_min[s] = T.vmin[2 * o];
    S.v_min[s] = T.vmin[2 * o + 1];
    S.sponge[s] = T.sponge[o];
    S.drho[s] = T.drho[o];
    S.dp[s] = T.dp[o];
    S.ax[s] = T.acc[2 * o];
    S.ay[s] = T.acc[2 * o + 1];
    S.drho_a[s] = T.drho_a[o];
    S.dp_a[s] = T.dp_a[o];
    S.ax_a[s] = T.acc_a[2 * o];
    S.ay_a[s] = T.acc_a[2 * o + 1];
    S.frho[s] = T.frho[o];
    S.fp[s] = T.fp[o];
    S.fu[s] = T.fvel[2 * o];
    S.fv[s] = T.fvel[2 * o + 1];
  }
}

// staging (reference order) <- slots
__global__ void k_scatter_download(SlotArrays S, Staging T, int n, int nf)
{
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = S.orig[s];
  T.pos[2 * o] = S.x[s];
  T.pos[2 * o + 1] = S.y[s];
  T.vel[2 * o] = S.u[s];
  T.vel[2 * o + 1] = S.v[s];
  T.lvel[2 * o] = S.ut[s];
  T.lvel[2 * o + 1] = S.vt[s];
  T.rho[o] = S.rho[s];
  T.lrho[o] = S.rhot[s];
  T.p[o] = S.p[s];
  T.lp[o] = S.pt[s];
  T.mass[o] = S.m[s];
  T.itype[o] = S.itype[s];
  T.pressure[o] = S.pressure[s];
  if (s < nf) {
    T.rhomin[o] = S.rho_min[s];
    T.pmin[o] = S.p_min[s];
    T.vmin[2 * o] = S.u_min[s];
    T.vmin[2 * o + 1] = S.v_min[s];
    T.sponge[o] = S.sponge[s];
    T.drho[o] = S.drho[s];
    T.dp[o] = S.dp[s];
    T.acc[2 * o] = S.ax[s];
    T.acc[2 * o + 1] = S.ay[s];
    T.drho_a[o] = S.drho_a[s];
    T.dp_a[o] = S.dp_a[s];
    T.acc_a[2 * o] = S.ax_a[s];
    T.acc_a[2 * o + 1] = S.ay_a[s];
    T.frho[o] = S.frho[s];
    T.fp[o] = S.fp[s];
    T.fvel[2 * o] = S.fu[s];
    T.fvel[2 * o + 1] = S.fv[s];
  }
}

// D <- S through perm[new slot] = old slot, for slots [0, count)
// D's slot s takes S's slot perm[s] for the fluid (s < nf) and slot s for
// the rest (walls keep their order)
__global__ void k_reorder(SlotArrays D, SlotArrays S, const int *__restrict__ perm, int count, int nf)
{
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  const int o = s < nf ? perm[s] : s;
  D.x[s] = S.x[o]; D.y[s] = S.y[o]; D.u[s] = S.u[o]; D.v[s] = S.v[o];
  D.ut[s] = S.ut[o]; D.vt[s] = S.vt[o]; D.rho[s] = S.rho[o]; D.rhot[s] = S.rhot[o];
  D.p[s] = S.p[o]; D.pt[s] = S.pt[o]; D.m[s] = S.m[o]; D.inv_rho[s] = S.inv_rho[o];
  D.inv_rhot[s] = S.inv_rhot[o]; D.pressure[s] = S.pressure[o]; D.itype[s] = S.itype[o]; D.orig[s] = S.orig[o];
  if (s < nf) {
    D.rho_min[s] = S.rho_min[o]; D.p_min[s] = S.p_min[o]; D.u_min[s] = S.u_min[o]; D.v_min[s] = S.v_min[o];
    D.sponge[s] = S.sponge[o]; D.drho[s] = S.drho[o]; D.dp[s] = S.dp[o]; D.ax[s] = S.ax[o]; D.ay[s] = S.ay[o];
    D.drho_a[s] = S.drho_a[o]; D.dp_a[s] = S.dp_a[o]; D.ax_a[s] = S.ax_a[o]; D.ay_a[s] = S.ay_a[o];
    D.frho[s] = S.frho[o]; D.fp[s] = S.fp[o]; D.fu[s] = S.fu[o]; D.fv[s] = S.fv[o];
  }
}

// The wall slots of S copied into D, the other buffer, so that a pass that
// writes its post-step state into D (StepOut) finds the walls' fields there.
__global__ void k_copy_walls(SlotArrays D, SlotArrays S, int nf, int n)
{
  const int s = nf + blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  D.x[s] = S.x[s]; D.y[s] = S.y[s]; D.u[s] = S.u[s]; D.v[s] = S.v[s];
  D.ut[s] = S.ut[s]; D.vt[s] = S.vt[s]; D.rho[s] = S.rho[s]; D.rhot[s] = S.rhot[s];
  D.p[s] = S.p[s]; D.pt[s] = S.pt[s]; D.m[s] = S.m[s]; D.inv_rho[s] = S.inv_rho[s];
  D.inv_rhot[s] = S.inv_rhot[s]; D.pressure[s] = S.pressure[s]; D.itype[s] = S.itype[s]; D.orig[s] = S.orig[s];
}

bool p_lid_or_gate(const DevParams &P)
{
  return (P.moving_boundary == 2 || P.moving_boundary == 3) && P.flag_init_simul == 1;
}

// The base coordinate of the lid (x, movingBoundary 3) or gate (y,
// movingBoundary 2) particles, per reference index - m0, such that the wall
// law at the upload's time t0 reproduces the uploaded position; at t0 = 0 (a
// fresh deck) the base is the position itself, as the reference's
// tempPosition / tempPositionGate columns are for its decks.
__global__ void k_wall_base(DevParams P, SlotArrays S, double *base, double t0)
{
  const int s = P.nf + blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  const int o = S.orig[s];
  if (o < P.m0 || o >= P.b1) return;
  const double U = P.lid_velocity;
  double b;
  if (P.moving_boundary == 3)
    b = S.x[s] - U * t0;
  else
    b = S.y[s] - (t0 <= 0.0 ? 0.0 : U * fmin(t0, P.gate_stop));
  base[o - P.m0] = b;
}

// counting sort of ids [first, first+count) by cell, result: G.list[0, count)
// = ids in key order, ties by id.  storage_order selects the tile-major
// storage key instead of the row-major cell-list id.
uph_status sort_range(uph_sim *s, const double *x, const double *y, int first, int count, bool storage_order)
{
  uph_status r = launch_cell_build(s->P, x, y, first, count, s->G, s->d_err, storage_order, nullptr, s->stream);
  s->launches += 1;
  return r;
}

// the cell list of all interacting particles, when the skin test asks for
// it; zeroes the pass statistics given and advances the step counter given
uph_status build_cell_list(uph_sim *s, const PassStats *stats = nullptr, int *step_counter = nullptr)
{
  Timer t(s, KF_CELLS);
  uph_status r = launch_cell_build(s->P, s->S.x, s->S.y, 0, s->P.n, s->G, s->d_err, false, stats, s->stream, true,
                                   step_counter);
  s->launches += 1;
  return r;
}

// the next cell-list build must bin every particle afresh (positions or
// slots changed outside the leapfrog)
uph_status force_rebuild(uph_sim *s)
{
  s->kcut_fresh = false;
  UPH_CUDA(cudaMemsetAsync(s->P.rebuild, 1, sizeof(unsigned), s->stream));
  return UPH_OK;
}

// The particle constants (mass, type, reference index, sponge factor) of S
// copied into S2: a pass that applies the step (StepOut) writes its
// post-step state into S2 without them.
uph_status sync_constants(uph_sim *s)
{
  const size_t n = s->P.n, nf = s->P.nf;
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  UPH_CUDA(cudaMemcpyAsync(s->S2.m, s->S.m, sizeof(double) * n, k, s->stream));
  UPH_CUDA(cudaMemcpyAsync(s->S2.itype, s->S.itype, sizeof(int32_t) * n, k, s->stream));
  UPH_CUDA(cudaMemcpyAsync(s->S2.orig, s->S.orig, sizeof(int32_t) * n, k, s->stream));
  if (nf > 0) UPH_CUDA(cudaMemcpyAsync(s->S2.sponge, s->S.sponge, sizeof(double) * nf, k, s->stream));
  return UPH_OK;
}

uph_status reorder_fluid(uph_sim *s)
{
  Timer t(s, KF_REORDER);
  const int nf = s->P.nf, n = s->P.n;
  uph_status r = sort_range(s, s->S.x, s->S.y, 0, nf, true);
  if (r != UPH_OK) return r;
  // the fluid's new order is the list the sort left in G.list[0, nf)
  k_reorder<<<(n + 255) / 256, 256, 0, s->stream>>>(s->S2, s->S, s->G.list, n, nf);
  s->launches += 1;
  SlotArrays tmp = s->S;
  s->S = s->S2;
  s->S2 = tmp;
  s->steps_since_reorder = 0;
  uph_status r2 = sync_constants(s);
  if (r2 != UPH_OK) return r2;
  return force_rebuild(s);
}

uph_status check_error_word(uph_sim *s)
{
  unsigned err = 0;
  UPH_CUDA(cudaMemcpyAsync(&err, s->d_err, sizeof err, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  UPH_CUDA(cudaGetLastError());
  if (err & ERR_NAN) return fail(UPH_NAN, "a non-finite value appeared in the particle state");
  if (err & ERR_OUT_OF_DOMAIN) return fail(UPH_OUT_OF_DOMAIN, "a particle left the cell-grid domain");
  if (err & ERR_NEIGHBOR_OVERFLOW) return fail(UPH_NEIGHBOR_OVERFLOW, "neighbour capacity exceeded");
  if (err & ERR_TIMEOUT) {
    // a cell-list build that gave up at a grid barrier leaves its histogram
    // and barrier words part-way: clear them for the next build
    cudaMemsetAsync(s->G.count, 0, sizeof(int) * s->G.ncell, s->stream);
    cudaMemsetAsync(s->G.bar, 0, kGridWords * sizeof(unsigned), s->stream);
    cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), s->stream);
    return fail(UPH_TIMEOUT, "a device-side wait timed out");
  }
  return UPH_OK;
}

// refresh: recompute 1/rho, 1/rhot (and the WCSPH pressure) first; a
// predictor that ran since the last state change has done it already
// step: a leapfrog step of uph_sim_step starts (the device step counter
// advances)
// F: the rate pass applies the step too (StepOut), writing the post-step
// state into F->D; null: the pass writes the rates into s->S
uph_status rate_pass(uph_sim *s, bool refresh, bool step = false, const StepOut *F = nullptr)
{
  if (refresh) {
    Timer t(s, KF_REFRESH);
    launch_refresh_inverse(s->P, s->S, 0, s->P.nf, s->stream);
    s->launches++;
  }
  const PassStats st{s->d_niac, s->d_max_nb};
  uph_status r = build_cell_list(s, &st, step ? s->d_itime : nullptr);
  if (r != UPH_OK) return r;
  VirtualPoints vp = {nullptr, nullptr, CellGrid{}};
  if (s->P.nvrules > 0) {
    Timer t(s, KF_CELLS);
    launch_virtual(s->P, s->S, s->vb, s->deriv_t, step ? s->d_itime : nullptr, s->stream);
    s->launches += 3;
    if (s->P.knn > 0) {
      r = launch_cell_build(s->P, s->vb.x, s->vb.y, 0, s->vb.cap, s->gv, s->d_err, false, nullptr, s->stream,
                            false, nullptr, s->vb.count);
      if (r != UPH_OK) return r;
      s->launches++;
      vp = VirtualPoints{s->vb.x, s->vb.y, s->gv};
    }
  }
  if (s->P.knn > 0) {
    launch_knn_cut(s->P, s->S, s->G, vp, s->stream);
    s->launches++;
    s->kcut_fresh = true;
  }
  Timer t(s, KF_PASS);
  // the tiled passes' candidate lists (uph_sim_set_candidate_lists), for
  // the steps of uph_sim_step: a lone evaluation (uph_sim_derivatives, after
  // an upload that rebuilt the list) would only write lists nobody reads
  CellGrid gp = s->G;
  if (!s->cand_lists || !step) {
    gp.vl = nullptr;
    gp.vl_n = nullptr;
  }
  if (s->P.profile != UPH_PROFILE_REF)
    r = launch_wcsph_pass(s->P, s->S, gp, st, F ? *F : StepOut{}, s->stream);
  else if (s->P.flag_init_simul == 0)
    r = launch_packing_pass(s->P, s->S, s->G, st, s->stream);
  else
    r = launch_ref_pass(s->P, s->S, gp, st, F ? *F : StepOut{}, s->stream);
  if (r != UPH_OK) return r;
  s->launches++;
  if (s->P.stress_type == 2 && s->P.profile == UPH_PROFILE_REF && s->P.flag_init_simul == 1) {
    launch_viscous_two_step(s->P, s->S, s->G, s->stream);
    s->launches += 2;
  }
  s->have_rates = true;
  return UPH_OK;
}

uph_status validate(const uph_params *p)
{
  if (p->n_fluid < 0 || p->n_solid < 0 || p->n_fixed < 0 || p->n_moving < 0)
    return fail(UPH_BAD_ARG, "negative particle count");
  const long long n = (long long)p->n_fluid + p->n_solid + p->n_fixed + p->n_moving;
  if (n <= 0 || n > (1LL << 30)) return fail(UPH_BAD_ARG, "particle count out of range");
  if (p->profile != UPH_PROFILE_REF && p->profile != UPH_PROFILE_WCSPH) return fail(UPH_BAD_ARG, "unknown profile");
  if (p->precision != UPH_PREC_FP64 && p->precision != UPH_PREC_FP32_PAIR)
    return fail(UPH_BAD_ARG, "unknown precision");
  if (p->precision == UPH_PREC_FP32_PAIR && p->profile != UPH_PROFILE_WCSPH)
    return fail(UPH_UNSUPPORTED, "FP32 pair arithmetic is implemented for the WCSPH profile only");
  if (!(p->h > 0) || !(p->dx > 0)) return fail(UPH_BAD_ARG, "smoothing length and dx must be positive");
  if (p->dim != 2) return fail(UPH_UNSUPPORTED, "only dim = 2 exists in the reference");
  if (p->flag_init_simul != 1 && p->flag_init_simul != 0)
    return fail(UPH_UNSUPPORTED, "flagInitSimul must be 0 (particle packing) or 1");
  if (p->flag_init_simul == 0 && p->profile != UPH_PROFILE_REF)
    return fail(UPH_UNSUPPORTED, "particle packing (flagInitSimul 0) belongs to the REF profile");
  if (p->stress_type == 2 && p->profile != UPH_PROFILE_REF)
    return fail(UPH_UNSUPPORTED, "stressType 2 belongs to the REF profile");
  if (p->knn_cap < 0) return fail(UPH_BAD_ARG, "negative knn_cap");
  if (p->knn_cap > kKnnMax)
    return fail(UPH_UNSUPPORTED, "knn_cap above " + std::to_string(kKnnMax) + " is not implemented");
  if (p->knn_cap > 0 && p->profile != UPH_PROFILE_REF)
    return fail(UPH_UNSUPPORTED, "the k-NN cap is implemented for the REF profile only");
  if (!(p->domain_hi[0] > p->domain_lo[0]) || !(p->domain_hi[1] > p->domain_lo[1]))
    return fail(UPH_BAD_ARG, "empty cell-grid domain");
  for (int d = 0; d < 2; d++)
    if (!isfinite(p->domain_lo[d]) || !isfinite(p->domain_hi[d]))
      return fail(UPH_BAD_ARG, "non-finite cell-grid domain");
  return UPH_OK;
}

// (Re)allocates the per-cell arrays for the current grid geometry; they grow
// only, so a smaller grid after re-tuning keeps the old allocation.
cudaError_t alloc_grid(uph_sim *s)
{
  CellGrid &G = s->G;
  const long long ncell = (long long)s->P.ncx * s->P.ncy;
  if (ncell > (1LL << 28)) return cudaErrorInvalidValue;
  G.ncell = (int)ncell;
  G.nblock_sums = scan_block_sums_needed((int)ncell);
  s->gv.ncell = (int)ncell;
  // the tiles' candidate-list generations: none matches any build's
  const long long ntiles = (long long)s->P.ntx * (s->P.ncy / s->P.tile);
  if (ntiles > s->tile_gen_capacity) {
    if (G.tile_gen) cudaFree(G.tile_gen);
    G.tile_gen = nullptr;
    cudaError_t e = cudaMalloc((void **)&G.tile_gen, sizeof(unsigned) * ntiles);
    if (e != cudaSuccess) return e;
    s->tile_gen_capacity = ntiles;
  }
  if (ntiles > 0) {
    cudaError_t e = cudaMemset(G.tile_gen, 0xff, sizeof(unsigned) * ntiles);
    if (e != cudaSuccess) return e;
  }
  // cudaMemset runs on the legacy default stream, which the simulation's
  // non-blocking stream does not wait for: the memsets here must have
  // completed before the caller's next launch (a list build that started on
  // stale counts would scatter out of range)
  if (ncell <= s->grid_capacity) return cudaDeviceSynchronize();
  for (int **p : {&G.count, &G.start, &G.fill, &G.block_sums, &s->gv.count, &s->gv.start, &s->gv.fill}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  cudaError_t e;
  if ((e = cudaMalloc((void **)&G.count, sizeof(int) * ncell)) != cudaSuccess) return e;
  if ((e = cudaMalloc((void **)&G.start, sizeof(int) * (ncell + 1))) != cudaSuccess) return e;
  if ((e = cudaMalloc((void **)&G.fill, sizeof(int) * ncell)) != cudaSuccess) return e;
  if ((e = cudaMalloc((void **)&G.block_sums, sizeof(int) * (G.nblock_sums + 1))) != cudaSuccess) return e;
  // the one-launch build keeps count all zero between builds
  if ((e = cudaMemset(G.count, 0, sizeof(int) * ncell)) != cudaSuccess) return e;
  if (s->P.nvrules > 0) {
    CellGrid &V = s->gv;
    if ((e = cudaMalloc((void **)&V.count, sizeof(int) * ncell)) != cudaSuccess) return e;
    if ((e = cudaMalloc((void **)&V.start, sizeof(int) * (ncell + 1))) != cudaSuccess) return e;
    if ((e = cudaMalloc((void **)&V.fill, sizeof(int) * ncell)) != cudaSuccess) return e;
    if ((e = cudaMemset(V.count, 0, sizeof(int) * ncell)) != cudaSuccess) return e;
  }
  s->grid_capacity = ncell;
  return cudaDeviceSynchronize();
}

// Cell width radius / reach; cells per axis rounded up to whole tiles.  A
// sparse domain (few particles spread far apart, as SearchNeighbors may be
// given) gets wider cells so the grid stays within kMaxGridCells: the
// stencil of `reach` cells then reaches further than the radius, which only
// adds candidates -- the pair test is the exact distance predicate.
constexpr double kMaxGridCells = double(1 << 26);

void set_grid_geometry(DevParams &P, int reach, int tile)
{
  P.reach = reach;
  P.tile = tile;
  double cell = sqrt(P.r2cut) / P.reach * (1.0 + kCellSkin) * (1.0 + 1e-9);
  double tiles_x, tiles_y;
  for (int grow = 0; grow < 200; grow++) {  // finite domains (validate) end in a few rounds
    const double nx = ceil((P.hi_x - P.lo_x) / cell);
    const double ny = ceil((P.hi_y - P.lo_y) / cell);
    tiles_x = ceil(fmax(nx, 1.0) / tile);
    tiles_y = ceil(fmax(ny, 1.0) / tile);
    if (tiles_x * tiles_y * tile * tile <= kMaxGridCells) break;
    cell *= 1.5;
  }
  P.cell = cell;
  P.inv_cell = 1.0 / cell;
  // a pair within the radius stays within `reach` cells of where both were
  // binned while each moved at most (reach cell - radius) / 2 per axis
  P.skin = 0.5 * (P.reach * cell * (1.0 - 1e-9) - sqrt(P.r2cut));
  P.ntx = (int)tiles_x;
  P.ncx = P.ntx * tile;
  P.ncy = (int)tiles_y * tile;
}

// The mirror rules of each virtualType, in the reference's loop order
// (derivatives.c:3195-4189).  Type 2's loops are commented out in the
// reference; other types have none.
void set_virtual_rules(DevParams &P, const uph_params *p)
{
  const double L = p->flat_bottom_length, D = p->local_depth;
  auto rule = [&](int kind, int pos, double a, double b) {
    P.vrule[P.nvrules++] = VirtualRule{kind, pos, a, b};
  };
  P.nvrules = 0;
  P.flat_bottom_length = L;
  P.local_depth = D;
  switch (p->virtual_type) {
    case 1:  // waves on a slope (:3195-3320); slope 1/15 (System.c:309)
      rule(VK_LEFT, VP_LEFT, 0.0, 0.0);
      rule(VK_BOTTOM, VP_CONST, L, 0.0);
      rule(VK_CORNER_L, VP_LEFT, 0.0, 0.0);
      rule(VK_SLOPE, VP_CONST, L, 1.0 / 15.0);
      break;
    case 3:  // vortex spin-down (:3471-3625)
      rule(VK_LEFT, VP_CONST, 0.0, 0.0);
      rule(VK_BOTTOM, VP_CONST, L, 0.0);
      rule(VK_TOP, VP_CONST, D, p->dx);
      rule(VK_CORNER_L, VP_LEFT, 0.0, 0.0);
      rule(VK_RIGHT, VP_CONST, L, 0.0);
      break;
    case 4:  // dam break with a gate (:3783-3906)
    case 8:  // dam break (:3907-4031)
      rule(VK_LEFT, VP_CONST, 0.0, 0.0);
      rule(VK_BOTTOM, VP_CONST, L, 0.0);
      rule(VK_CORNER_L, VP_LEFT, 0.0, 0.0);
      rule(VK_RIGHT, VP_CONST, L, 0.0);
      break;
    case 5:  // sloshing tank (:3626-3782)
      rule(VK_LEFT, VP_LEFT, 0.0, 0.0);
      rule(VK_CORNER_L, VP_LEFT, 0.0, 0.0);
      rule(VK_CORNER_R, VP_RIGHT, 0.0, 0.0);
      rule(VK_RIGHT, VP_RIGHT, 0.0, 0.0);
      break;
    case 7:  // hydrostatic tank (:4032-4189)
      rule(VK_LEFT, VP_CONST, 0.0, 0.0);
      rule(VK_BOTTOM, VP_CONST, L, 0.0);
      rule(VK_TOP, VP_CONST, D, 0.0);
      rule(VK_CORNER_L, VP_LEFT, 0.0, 0.0);
      rule(VK_RIGHT, VP_CONST, L, 0.0);
      break;
    default:
      break;
  }
  // inputbp.c's if-else chain: the piston law moves the left boundary for
  // movingBoundary 1 and, failing 1, 2 and 3, for the sloshing walls; the
  // lid and gate leave it where it was (0: nothing else sets it); the
  // remaining case sets 0
  const int mb = p->moving_boundary;
  const bool piston = mb == 1 && p->flag_init_simul == 1;
  const bool lid_or_gate = (mb == 3 || mb == 2) && p->flag_init_simul == 1;
  P.vleft_moves = piston || (!lid_or_gate && !piston && p->virtual_type == 5);
}

DevParams make_dev_params(const uph_params *p)
{
  DevParams P;
  memset(&P, 0, sizeof P);
  P.nf = p->n_fluid;
  P.n = p->n_fluid + p->n_solid + p->n_fixed + p->n_moving;
  P.pb = P.n - 1;
  P.b0 = p->n_fluid + p->n_solid;
  P.b1 = P.n;
  P.m0 = p->n_fluid + p->n_solid + p->n_fixed;
  P.profile = p->profile;
  P.precision = p->precision;
  const double h = p->h;
  P.h = h;
  P.inv_h = 1.0 / h;
  P.inv_h2 = 1.0 / (h * h);
  P.r2cut = h * h * 4;                                  // derivatives.c:1086
  P.eta2 = 0.01 * h * h;
  P.w_alpha = 2145.0 / (1347584.0 * M_PI * h * h);      // derivatives.c:769
  P.dw_alpha = -1.0 * (2145.0 / (192512.0 * M_PI * h * h));  // derivatives.c:788, 817
  P.dw_alpha_h2 = P.dw_alpha * P.inv_h2;
  P.cs_alpha = 10.0 / (7. * M_PI * h * h);              // derivatives.c:46
  P.rho0 = p->density0;
  P.gamma = p->adiabatic_constant;
  P.c0 = p->speed_of_sound;
  P.B = p->compression_factor;
  P.rho0c2 = p->density0 * p->speed_of_sound * p->speed_of_sound;
  P.g = p->gravity;
  P.gravity_flag = p->gravity_flag;
  P.mu0 = p->viscosity0;
  P.two_mu0 = 2.0 * p->viscosity0;
  P.kappa = p->thermal_diffusivity0;
  P.eps = p->epsilon;
  P.stress_type = p->stress_type;
  P.boundary_force = p->select_boundary_force;
  P.k_spring = p->spring_constant0;
  P.c_damp = p->damping_constant0;
  P.dx = p->dx;
  P.dy = p->dy;
  P.lj_coeff = p->lennard_coefficient;
  P.mach_c = p->mach_number * p->speed_of_sound;
  P.moving_boundary = p->moving_boundary;
  P.flag_init_simul = p->flag_init_simul;
  P.wave_absorption = p->wave_absorption;
  P.stroke = p->stroke;
  P.omega = p->omega;
  P.lid_velocity = p->lid_velocity;
  // inputbp.c:226 (a zero speed never starts the gate: stop at t = 0)
  P.gate_stop = p->lid_velocity != 0.0 ? 1.5 * (p->local_depth - 15.0 * p->dx) / p->lid_velocity : 0.0;
  P.av_alpha_c0 = p->av_alpha * p->speed_of_sound;
  P.dt = p->time_step;
  P.lo_x = p->domain_lo[0];
  P.lo_y = p->domain_lo[1];
  P.hi_x = p->domain_hi[0];
  P.hi_y = p->domain_hi[1];
  set_virtual_rules(P, p);
  if (P.nvrules > 0) {
    // mirror images lie up to 4h beyond the fluid (the top rule's
    // D + 2 |y - D|): the grid covers them too
    const double pad = 8.0 * p->h;
    P.lo_x -= pad;
    P.lo_y -= pad;
    P.hi_x += pad;
    P.hi_y += pad;
  }
  // cells of half the search radius: a 5 x 5 block holds 25 h^2 of candidates
  // against 36 h^2 for a 3 x 3 block of radius-wide cells.  A cell then holds
  // about ((1 + skin) h / dx)^2 particles of a lattice; the default tile (11
  // cells at h = 1.3 dx) shrinks for wider kernels so that a tile's
  // particles fit one round of a CTA and its block the tiled passes'
  // shared-memory records.
  int tile = kCellTile;
  const double hdx = p->dx > 0 ? h / p->dx : 1.0;
  if (hdx > 1.4) tile = std::max(2, (int)floor(kCellTile * 1.3 / hdx));
  set_grid_geometry(P, kCellReach, tile);
  P.knn = p->knn_cap;
  P.kcut_d2 = nullptr;
  P.kcut_j = nullptr;
  P.str_xx = P.str_xy = P.str_yy = nullptr;
  P.xbin = P.ybin = nullptr;
  P.rebuild = nullptr;
  return P;
}

}  // namespace

// ---- C ABI ---------------------------------------------------------------------

extern "C" uph_status uph_sim_create(const uph_params *p, uph_sim **out)
{
  if (!p || !out) return fail(UPH_BAD_ARG, "uph_sim_create: NULL argument");
  *out = nullptr;
  uph_status v = validate(p);
  if (v != UPH_OK) return v;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(UPH_NO_DEVICE, "no CUDA device is visible");
  uph_sim *s = new uph_sim();
  s->hp = *p;
  s->P = make_dev_params(p);
  const long long ncell = (long long)s->P.ncx * s->P.ncy;
  if (ncell > (1LL << 28)) {
    delete s;
    return fail(UPH_BAD_ARG, "cell grid larger than 2^28 cells; shrink the domain");
  }
  const int n = s->P.n, nf = s->P.nf;
#define TRY(x)                       \
  do {                               \
    cudaError_t e_ = (x);            \
    if (e_ != cudaSuccess) {         \
      uph_sim_destroy(s);            \
      return cuda_fail(e_, #x);      \
    }                                \
  } while (0)
  TRY(alloc_slots(s, s->S, n, nf));
  TRY(alloc_slots(s, s->S2, n, nf));
  CellGrid &G = s->G;
  TRY(dalloc(s, &G.list, (size_t)n));
  TRY(dalloc(s, &G.cell_of, (size_t)n));
  if (s->P.knn > 0) {
    TRY(dalloc(s, &s->P.kcut_d2, (size_t)nf));
    TRY(dalloc(s, &s->P.kcut_j, (size_t)nf));
  }
  if (s->P.stress_type == 2 && s->P.profile == UPH_PROFILE_REF) {
    TRY(dalloc(s, &s->P.str_xx, (size_t)n));
    TRY(dalloc(s, &s->P.str_xy, (size_t)n));
    TRY(dalloc(s, &s->P.str_yy, (size_t)n));
  }
  {
    double *m0 = nullptr;
    TRY(dalloc(s, &m0, 1));
    TRY(cudaMemset(m0, 0, sizeof(double)));
    s->P.pack_mass0 = m0;
  }
  TRY(dalloc(s, &s->P.xbin, (size_t)n));
  TRY(dalloc(s, &s->P.ybin, (size_t)n));
  TRY(dalloc(s, &s->P.rebuild, 1));
  TRY(cudaMemset(s->P.rebuild, 1, sizeof(unsigned)));
  TRY(dalloc(s, &G.gen, 1));
  TRY(cudaMemset(G.gen, 0, sizeof(unsigned)));
  TRY(dalloc(s, &G.vl, (size_t)nf * kVlMax));
  TRY(dalloc(s, &G.vl_n, (size_t)nf));
  TRY(dalloc(s, &G.rank, (size_t)n));
  TRY(dalloc(s, &G.totals, (size_t)kCellBuildMaxBlocks + 1));
  TRY(dalloc(s, &G.bar, kGridWords));
  TRY(cudaMemset(G.bar, 0, kGridWords * sizeof(unsigned)));
  if (s->P.nvrules > 0) {
    VirtualBuf &V = s->vb;
    V.cap = s->P.nvrules * nf;
    TRY(dalloc(s, &V.flags, (size_t)V.cap));
    TRY(dalloc(s, &V.offs, (size_t)V.cap));
    TRY(dalloc(s, &V.block_sums, (size_t)scan_block_sums_needed(V.cap) + 1));
    TRY(dalloc(s, &V.count, 1));
    TRY(cudaMemset(V.count, 0, sizeof(int)));
    TRY(dalloc(s, &V.x, (size_t)V.cap));
    TRY(dalloc(s, &V.y, (size_t)V.cap));
    TRY(dalloc(s, &V.src, (size_t)V.cap));
    TRY(dalloc(s, &V.rule, (size_t)V.cap));
    CellGrid &Gv = s->gv;
    TRY(dalloc(s, &Gv.list, (size_t)V.cap));
    TRY(dalloc(s, &Gv.cell_of, (size_t)V.cap));
    TRY(dalloc(s, &Gv.rank, (size_t)V.cap));
    TRY(dalloc(s, &Gv.totals, (size_t)kCellBuildMaxBlocks + 1));
    TRY(dalloc(s, &Gv.bar, kGridWords));
    TRY(cudaMemset(Gv.bar, 0, kGridWords * sizeof(unsigned)));
  }
  TRY(alloc_grid(s));
  Staging &T = s->T;
  double **tall[] = {&T.rho, &T.lrho, &T.p, &T.lp, &T.mass, &T.pressure, &T.tmp_x, &T.tmp_y};
  for (double **q : tall) TRY(dalloc(s, q, (size_t)n));
  double **tall2[] = {&T.pos, &T.vel, &T.lvel};
  for (double **q : tall2) TRY(dalloc(s, q, 2 * (size_t)n));
  TRY(dalloc(s, &T.itype, (size_t)n));
  double **tfl[] = {&T.rhomin, &T.pmin, &T.sponge, &T.drho, &T.dp, &T.drho_a, &T.dp_a, &T.frho, &T.fp};
  for (double **q : tfl) TRY(dalloc(s, q, (size_t)nf));
  double **tfl2[] = {&T.vmin, &T.acc, &T.acc_a, &T.fvel};
  for (double **q : tfl2) TRY(dalloc(s, q, 2 * (size_t)nf));
  TRY(dalloc(s, &s->d_err, 1));
  TRY(dalloc(s, &s->d_niac, 1));
  TRY(dalloc(s, &s->d_max_nb, 1));
  TRY(dalloc(s, &s->d_perm, (size_t)n));
  TRY(dalloc(s, &s->d_itime, 1));
  TRY(dalloc(s, &s->d_wall_tab, 4 * (size_t)(p->n_moving > 0 ? p->n_moving : 1)));
  s->W.base = s->d_wall_tab + 3 * (size_t)(p->n_moving > 0 ? p->n_moving : 1);
  s->n_partials = 1024;
  TRY(dalloc(s, &s->d_partials, (size_t)s->n_partials * 4));
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int want = (p->n_fluid + 255) / 256;
    s->diag_blocks = want < 2 * sms ? (want > 0 ? want : 1) : 2 * sms;
  }
  TRY(dalloc(s, &s->d_diag_part, (size_t)s->diag_blocks * kDiagRows));
  TRY(dalloc(s, &s->d_diag_done, 1));
  TRY(dalloc(s, &s->d_diag, 1));
  TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  s->own_stream = true;
  {
    static std::atomic<int64_t> created{0};
    s->serial = ++created;
  }
  // the memsets above ran on the legacy default stream, which the
  // non-blocking stream does not wait for
  TRY(cudaDeviceSynchronize());
  TRY(cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), s->stream));
  TRY(cudaMemsetAsync(s->d_diag_done, 0, sizeof(unsigned), s->stream));
  TRY(cudaMemsetAsync(s->d_diag, 0, sizeof(DevDiag), s->stream));
#undef TRY
  *out = s;
  return UPH_OK;
}

namespace {
void drop_graph(uph_sim *s);
}

extern "C" uph_status uph_sim_destroy(uph_sim *s)
{
  if (!s) return UPH_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  for (void *p : s->allocations) cudaFree(p);
  for (void *p : {(void *)s->G.count, (void *)s->G.start, (void *)s->G.fill, (void *)s->G.block_sums,
                  (void *)s->G.tile_gen,
                  (void *)s->gv.count, (void *)s->gv.start, (void *)s->gv.fill, (void *)s->pe_ip, (void *)s->pe_jp,
                  (void *)s->pe_r2, (void *)s->pe_w, (void *)s->pe_dw})
    if (p) cudaFree(p);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  for (cudaEvent_t e : s->ev_pool)
    if (e) cudaEventDestroy(e);
  delete s;
  return UPH_OK;
}

extern "C" uph_status uph_sim_set_stream(uph_sim *s, void *stream)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  if (s->own_stream) cudaStreamDestroy(s->stream);
  if (stream) {
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
  } else {
    UPH_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return UPH_OK;
}

namespace {

template <typename T>
cudaError_t h2d(T *dst, const T *src, size_t count, cudaStream_t st)
{
  if (!src) return cudaMemsetAsync(dst, 0, sizeof(T) * count, st);
  return cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, st);
}

template <typename T>
cudaError_t d2h(T *dst, const T *src, size_t count, cudaStream_t st)
{
  if (!dst) return cudaSuccess;
  return cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToHost, st);
}

}  // namespace

extern "C" uph_status uph_sim_upload(uph_sim *s, const uph_state *st, int32_t itime)
{
  if (!s || !st) return fail(UPH_BAD_ARG, "uph_sim_upload: NULL argument");
  if (!st->Position || !st->Velocity || !st->density || !st->DynamicPressure || !st->mass || !st->itype)
    return fail(UPH_BAD_ARG, "uph_sim_upload: Position, Velocity, density, DynamicPressure, mass and itype are required");
  if (itime < 0) return fail(UPH_BAD_ARG, "uph_sim_upload: negative itime");
  const int n = s->P.n, nf = s->P.nf;
  cudaStream_t q = s->stream;
  Staging &T = s->T;
  UPH_CUDA(h2d(T.pos, st->Position, 2 * (size_t)n, q));
  UPH_CUDA(h2d(T.vel, st->Velocity, 2 * (size_t)n, q));
  UPH_CUDA(h2d(T.lvel, st->localVelocity ? st->localVelocity : st->Velocity, 2 * (size_t)n, q));
  UPH_CUDA(h2d(T.rho, st->density, (size_t)n, q));
  UPH_CUDA(h2d(T.lrho, st->localDensity ? st->localDensity : st->density, (size_t)n, q));
  UPH_CUDA(h2d(T.p, st->DynamicPressure, (size_t)n, q));
  UPH_CUDA(h2d(T.lp, st->localPressure, (size_t)n, q));
  UPH_CUDA(h2d(T.mass, st->mass, (size_t)n, q));
  // the packing pass's volume scale is the mass of reference particle 0
  UPH_CUDA(cudaMemcpyAsync(const_cast<double *>(s->P.pack_mass0), st->mass, sizeof(double), cudaMemcpyHostToDevice,
                           q));
  UPH_CUDA(h2d(T.itype, st->itype, (size_t)n, q));
  UPH_CUDA(h2d(T.pressure, st->Pressure, (size_t)n, q));
  UPH_CUDA(h2d(T.vmin, st->Velocity_min, 2 * (size_t)nf, q));
  UPH_CUDA(h2d(T.rhomin, st->density_min, (size_t)nf, q));
  UPH_CUDA(h2d(T.pmin, st->DynamicPressure_min, (size_t)nf, q));
  UPH_CUDA(h2d(T.sponge, st->spongeFactor, (size_t)nf, q));
  UPH_CUDA(h2d(T.drho, st->ddensitydt, (size_t)nf, q));
  UPH_CUDA(h2d(T.dp, st->dpdt, (size_t)nf, q));
  UPH_CUDA(h2d(T.acc, st->dvdt, 2 * (size_t)nf, q));
  UPH_CUDA(h2d(T.drho_a, st->ddensitydt_approx, (size_t)nf, q));
  UPH_CUDA(h2d(T.dp_a, st->dpdt_approx, (size_t)nf, q));
  UPH_CUDA(h2d(T.acc_a, st->dvdt_approx, 2 * (size_t)nf, q));
  UPH_CUDA(h2d(T.frho, st->densityFluctuation, (size_t)nf, q));
  UPH_CUDA(h2d(T.fp, st->pressureFluctuation, (size_t)nf, q));
  UPH_CUDA(h2d(T.fvel, st->velocityFluctuation, 2 * (size_t)nf, q));
  UPH_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), q));
  // spatial order: fluid and walls sorted by cell separately
  k_split_xy<<<(n + 255) / 256, 256, 0, q>>>(T.pos, T.tmp_x, T.tmp_y, n);
  s->launches++;
  uph_status r = sort_range(s, T.tmp_x, T.tmp_y, 0, nf, true);
  if (r != UPH_OK) return r;
  UPH_CUDA(cudaMemcpyAsync(s->d_perm, s->G.list, sizeof(int) * nf, cudaMemcpyDeviceToDevice, q));
  if (n > nf) {
    r = sort_range(s, T.tmp_x, T.tmp_y, nf, n - nf, true);
    if (r != UPH_OK) return r;
    UPH_CUDA(cudaMemcpyAsync(s->d_perm + nf, s->G.list, sizeof(int) * (n - nf), cudaMemcpyDeviceToDevice, q));
  }
  k_gather_upload<<<(n + 255) / 256, 256, 0, q>>>(s->S, T, s->d_perm, n, nf, s->P.rho0);
  launch_refresh_inverse(s->P, s->S, 0, n, q);
  launch_wall_pressure(s->P, s->S, q);
  if (p_lid_or_gate(s->P) && s->hp.n_moving > 0) {
    // the lid's / gate's base coordinates from the uploaded positions
    const int nw = n - nf;
    k_wall_base<<<(nw + 255) / 256, 256, 0, q>>>(s->P, s->S, const_cast<double *>(s->W.base), itime * s->P.dt);
    s->launches++;
  }
  if (n > nf) {
    k_copy_walls<<<(n - nf + 255) / 256, 256, 0, q>>>(s->S2, s->S, nf, n);
    s->launches++;
  }
  r = sync_constants(s);
  if (r != UPH_OK) return r;
  s->launches += 3;
  s->itime = itime;
  UPH_CUDA(cudaMemcpyAsync(s->d_itime, &s->itime, sizeof(int), cudaMemcpyHostToDevice, q));
  s->steps_since_reorder = 0;
  r = force_rebuild(s);
  if (r != UPH_OK) return r;
  s->have_rates = false;
  s->restart = false;
  return check_error_word(s);
}

extern "C" uph_status uph_sim_download(uph_sim *s, uph_state *st)
{
  if (!s || !st) return fail(UPH_BAD_ARG, "uph_sim_download: NULL argument");
  const int n = s->P.n, nf = s->P.nf;
  cudaStream_t q = s->stream;
  Staging &T = s->T;
  k_scatter_download<<<(n + 255) / 256, 256, 0, q>>>(s->S, T, n, nf);
  s->launches++;
  UPH_CUDA(d2h(st->Position, T.pos, 2 * (size_t)n, q));
  UPH_CUDA(d2h(st->Velocity, T.vel, 2 * (size_t)n, q));
  UPH_CUDA(d2h(st->localVelocity, T.lvel, 2 * (size_t)n, q));
  UPH_CUDA(d2h(st->density, T.rho, (size_t)n, q));
  UPH_CUDA(d2h(st->localDensity, T.lrho, (size_t)n, q));
  UPH_CUDA(d2h(st->DynamicPressure, T.p, (size_t)n, q));
  UPH_CUDA(d2h(st->localPressure, T.lp, (size_t)n, q));
  UPH_CUDA(d2h(st->mass, T.mass, (size_t)n, q));
  UPH_CUDA(d2h(st->itype, T.itype, (size_t)n, q));
  UPH_CUDA(d2h(st->Pressure, T.pressure, (size_t)n, q));
  UPH_CUDA(d2h(st->Velocity_min, T.vmin, 2 * (size_t)nf, q));
  UPH_CUDA(d2h(st->density_min, T.rhomin, (size_t)nf, q));
  UPH_CUDA(d2h(st->DynamicPressure_min, T.pmin, (size_t)nf, q));
  UPH_CUDA(d2h(st->spongeFactor, T.sponge, (size_t)nf, q));
  UPH_CUDA(d2h(st->ddensitydt, T.drho, (size_t)nf, q));
  UPH_CUDA(d2h(st->dpdt, T.dp, (size_t)nf, q));
  UPH_CUDA(d2h(st->dvdt, T.acc, 2 * (size_t)nf, q));
  UPH_CUDA(d2h(st->ddensitydt_approx, T.drho_a, (size_t)nf, q));
  UPH_CUDA(d2h(st->dpdt_approx, T.dp_a, (size_t)nf, q));
  UPH_CUDA(d2h(st->dvdt_approx, T.acc_a, 2 * (size_t)nf, q));
  UPH_CUDA(d2h(st->densityFluctuation, T.frho, (size_t)nf, q));
  UPH_CUDA(d2h(st->pressureFluctuation, T.fp, (size_t)nf, q));
  UPH_CUDA(d2h(st->velocityFluctuation, T.fvel, 2 * (size_t)nf, q));
  UPH_CUDA(cudaStreamSynchronize(q));
  return UPH_OK;
}

namespace {

bool walls_move(const uph_sim *s)
{
  const int mb = s->P.moving_boundary;
  return s->hp.n_moving > 0 && (s->W.enabled || ((mb == 1 || mb == 2 || mb == 3) && s->P.flag_init_simul == 1));
}

// Enqueues `nsteps` leapfrog steps on the sim's stream.  Where the rate pass
// applies the step (StepOut) each step is the list launch and the pass, and
// the two state buffers swap; else the pass and the corrector.  With
// `capturing` the sequence is being recorded into a CUDA graph: no host
// synchronisation, no profiling events, and an even number of buffer swaps
// (one more storage re-sort where needed) so the graph ends on the buffer it
// started on.
void launch_diagnostics(uph_sim *s);

uph_status enqueue_steps(uph_sim *s, int nsteps, bool capturing)
{
  const bool moving = walls_move(s);
  const bool fuse = s->fused_step && !s->diag_enabled &&
                    (s->P.profile == UPH_PROFILE_WCSPH ||
                     (s->P.flag_init_simul == 1 && s->P.stress_type != 2 && s->P.precision == UPH_PREC_FP64));
  int swaps = 0;  // buffer swaps: fused steps and storage re-sorts
  for (int k = 0; k < nsteps; k++) {
    const int itime = ++s->itime;
    const bool first = itime == 1 || (k == 0 && s->restart);
    // the predictor of steps after the first of this call ran inside the
    // previous step's corrector
    if (!first && k == 0) {
      Timer tm(s, KF_PREDICT);
      launch_predict(s->P, s->S, s->stream);
      s->launches++;
    }
    // the walls of steps after the first of this call moved inside the
    // previous step's corrector
    if (moving && k == 0) {
      Timer tm(s, KF_WALLS);
      launch_wall_motion(s->P, s->S, s->W, 0.0, s->d_itime, s->d_err, s->stream);
      s->launches++;
    }
    const bool more = k + 1 < nsteps;
    uph_status r;
    if (fuse) {
      // the pass writes the post-step state into the other buffer
      const StepOut F{s->S2, s->W, s->d_err, s->d_itime, 1, first ? 1 : 0, more ? 1 : 0, moving ? (more ? 2 : 1) : 0};
      r = rate_pass(s, first, true, &F);
      if (r != UPH_OK) return r;
      const SlotArrays tmp = s->S;
      s->S = s->S2;
      s->S2 = tmp;
      swaps++;
      if (k == 0) s->restart = false;
    } else {
      r = rate_pass(s, first, true);
      if (r != UPH_OK) return r;
      if (k == 0) s->restart = false;
      if (s->diag_enabled) launch_diagnostics(s);
      Timer tm(s, KF_CORRECT);
      launch_correct(s->P, s->S, s->W, first, more, more && moving, s->d_err, s->d_itime, s->stream);
      s->launches++;
    }
    if (++s->steps_since_reorder >= s->reorder_interval) {
      r = reorder_fluid(s);
      if (r != UPH_OK) return r;
      swaps++;
    }
    // a particle that left the grid is clamped into a border cell, which can
    // make that cell arbitrarily crowded: stop early rather than run on
    if (!capturing && (k + 1) % kErrorCheckInterval == 0 && k + 1 < nsteps) {
      r = check_error_word(s);
      if (r != UPH_OK) return r;
    }
  }
  if (capturing && (swaps & 1)) {
    uph_status r = reorder_fluid(s);
    if (r != UPH_OK) return r;
  }
  s->kcut_fresh = false;  // the correctors moved the particles
  return UPH_OK;
}

void drop_graph(uph_sim *s)
{
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->graph_exec = nullptr;
  s->graph = nullptr;
}

}  // namespace

extern "C" uph_status uph_sim_step(uph_sim *s, int32_t nsteps)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  if (nsteps < 0) return fail(UPH_BAD_ARG, "negative step count");
  // graph replay: a call of exactly graph_steps steps that is not the
  // simulation's first step and starts on the buffer the graph was recorded on
  if (s->graph_steps > 0 && nsteps == s->graph_steps && s->itime >= 1 && !s->profiling && !s->restart) {
    if (s->graph_exec && s->graph_buffer != s->S.x) drop_graph(s);
    if (!s->graph_exec) {
      const int itime0 = s->itime, since0 = s->steps_since_reorder;
      const int64_t launches0 = s->launches;
      const double *buffer0 = s->S.x;
      s->steps_since_reorder = 0;
      UPH_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      uph_status r = enqueue_steps(s, nsteps, true);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(s->stream, &g);
      // replaying leaves the re-sort counter where the recording left it
      const int since_after = s->steps_since_reorder;
      // the recording ran nothing: restore the host-side counters
      s->itime = itime0;
      s->steps_since_reorder = since0;
      s->graph_launches = s->launches - launches0;
      s->launches = launches0;
      if (r != UPH_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
      }
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
      s->graph = g;
      UPH_CUDA(cudaGraphInstantiate(&s->graph_exec, g, 0));
      s->graph_buffer = buffer0;
      s->graph_since_after = since_after;
    }
    UPH_CUDA(cudaGraphLaunch(s->graph_exec, s->stream));
    s->itime += nsteps;
    s->steps_since_reorder = s->graph_since_after;
    s->launches += s->graph_launches;
    s->graph_replays++;
    UPH_CUDA(cudaGetLastError());
    return check_error_word(s);
  }
  uph_status r = enqueue_steps(s, nsteps, false);
  if (r != UPH_OK) return r;
  UPH_CUDA(cudaGetLastError());
  return check_error_word(s);
}

extern "C" uph_status uph_sim_set_graph(uph_sim *s, int32_t steps_per_graph)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  if (steps_per_graph < 0) return fail(UPH_BAD_ARG, "negative graph length");
  drop_graph(s);
  s->graph_steps = steps_per_graph;
  return UPH_OK;
}

extern "C" uph_status uph_sim_set_fused_step(uph_sim *s, int32_t enable)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  drop_graph(s);
  s->fused_step = enable != 0;
  return UPH_OK;
}

extern "C" uph_status uph_sim_set_candidate_lists(uph_sim *s, int32_t enable)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  drop_graph(s);
  s->cand_lists = enable != 0;
  // lists written before a switch off are not trusted after a switch back on
  return force_rebuild(s);
}

extern "C" uph_status uph_sim_set_wall_motion(uph_sim *s, const double *x0, const double *half_stroke,
                                              const double *omega)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  const int nm = s->hp.n_moving;
  if (!x0 || !half_stroke || !omega) {
    s->W.enabled = 0;
    drop_graph(s);
    return UPH_OK;
  }
  if (nm <= 0) return fail(UPH_BAD_ARG, "uph_sim_set_wall_motion: the sim has no moving boundary particles");
  UPH_CUDA(cudaMemcpyAsync(s->d_wall_tab, x0, sizeof(double) * nm, cudaMemcpyHostToDevice, s->stream));
  UPH_CUDA(cudaMemcpyAsync(s->d_wall_tab + nm, half_stroke, sizeof(double) * nm, cudaMemcpyHostToDevice, s->stream));
  UPH_CUDA(cudaMemcpyAsync(s->d_wall_tab + 2 * nm, omega, sizeof(double) * nm, cudaMemcpyHostToDevice, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  s->W.x0 = s->d_wall_tab;
  s->W.hs = s->d_wall_tab + nm;
  s->W.om = s->d_wall_tab + 2 * nm;
  s->W.enabled = 1;
  drop_graph(s);
  return UPH_OK;
}

extern "C" uph_status uph_sim_set_wall_base(uph_sim *s, const double *base)
{
  if (!s || !base) return fail(UPH_BAD_ARG, "uph_sim_set_wall_base: NULL argument");
  const int nm = s->hp.n_moving;
  if (nm <= 0) return fail(UPH_BAD_ARG, "uph_sim_set_wall_base: the sim has no moving boundary particles");
  UPH_CUDA(cudaMemcpyAsync(const_cast<double *>(s->W.base), base, sizeof(double) * nm, cudaMemcpyHostToDevice,
                           s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  drop_graph(s);
  return UPH_OK;
}

extern "C" uph_status uph_sim_derivatives(uph_sim *s, double t)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  // the piston position is a closed form of t, so applying it again after the
  // caller's own inputbp() changes nothing
  if (walls_move(s)) {
    launch_wall_motion(s->P, s->S, s->W, t, nullptr, s->d_err, s->stream);
    s->launches++;
  }
  s->deriv_t = t;
  uph_status r = rate_pass(s, true);
  if (r != UPH_OK) return r;
  UPH_CUDA(cudaGetLastError());
  return check_error_word(s);
}

extern "C" uph_status uph_sim_virtual(uph_sim *s, int64_t cap, double *position, int32_t *src, int32_t *rule,
                                      int64_t *count)
{
  if (!s || !count) return fail(UPH_BAD_ARG, "uph_sim_virtual: NULL argument");
  *count = 0;
  if (s->P.nvrules <= 0 || !s->have_rates) return UPH_OK;
  int nv = 0;
  UPH_CUDA(cudaMemcpyAsync(&nv, s->vb.count, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  *count = nv;
  if (!position && !src && !rule) return UPH_OK;
  if (cap < nv) return fail(UPH_BAD_ARG, "uph_sim_virtual: " + std::to_string(nv) + " virtual particles, capacity " +
                                             std::to_string(cap));
  if (nv > 0) {
    if (position) {
      std::vector<double> x(nv), y(nv);
      UPH_CUDA(cudaMemcpyAsync(x.data(), s->vb.x, sizeof(double) * nv, cudaMemcpyDeviceToHost, s->stream));
      UPH_CUDA(cudaMemcpyAsync(y.data(), s->vb.y, sizeof(double) * nv, cudaMemcpyDeviceToHost, s->stream));
      UPH_CUDA(cudaStreamSynchronize(s->stream));
      for (int k = 0; k < nv; k++) {
        position[2 * k] = x[k];
        position[2 * k + 1] = y[k];
      }
    }
    if (src) UPH_CUDA(cudaMemcpyAsync(src, s->vb.src, sizeof(int) * nv, cudaMemcpyDeviceToHost, s->stream));
    if (rule) UPH_CUDA(cudaMemcpyAsync(rule, s->vb.rule, sizeof(int) * nv, cudaMemcpyDeviceToHost, s->stream));
    UPH_CUDA(cudaStreamSynchronize(s->stream));
  }
  return UPH_OK;
}

// ---- pair export ---------------------------------------------------------------

namespace {

__device__ __forceinline__ double pr2(double dx, double dy) { return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)); }

// count pairs whose i (smaller reference index) is the fluid particle in slot a
__global__ void k_pair_count(DevParams P, SlotArrays S, CellGrid G, int *__restrict__ cnt_by_orig)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double xa = S.x[a], ya = S.y[a];
  const int oa = S.orig[a];
  const double cd = P.knn > 0 ? P.kcut_d2[a] : 0.0;
  const int cj = P.knn > 0 ? P.kcut_j[a] : 0;
  NeighbourCursor cur;
  cur.init(P, G, G.cell_of[a]);
  int cnt = 0, k;
  while (cur.next(k)) {
    const int b = G.list[k];
    const int ob = S.orig[b];
    if (ob <= oa || ob >= P.pb) continue;
    const double r2 = pr2(xa - S.x[b], ya - S.y[b]);
    if (r2 < P.r2cut && r2 > DBL_EPSILON && (P.knn <= 0 || knn_key_le(r2, ob, cd, cj))) cnt++;
  }
  cnt_by_orig[oa] = cnt;
}

// the kernel values of a listed pair, as CalculateKernel exports them
__device__ __forceinline__ void pair_kernel(const DevParams &P, double r2, double &W, double &F)
{
  const double r = sqrt(r2), q = r * P.inv_h;
  if (P.profile == UPH_PROFILE_REF) {
    const double q2 = q * q, t = 1.0 - 0.25 * q2, t2 = t * t, t4 = t2 * t2;
    const double pp = (((((305.0 * q2 - 628.0) * q2 + 1184.0) * q2 - 1984.0) * q2 + 2816.0) * q2 - 3072.0) * q2 + 2048.0;
    const double pp7 = (((((305.0 * q2 - 1106.0) * q2 + 1912.0) * q2 - 2912.0) * q2 + 3712.0) * q2 - 3584.0) * q2 + 2048.0;
    W = P.w_alpha * (t4 * t4) * pp;
    F = P.dw_alpha * (t4 * t2 * t) * pp7 * P.inv_h2;
  } else if (q < 1.0) {
    W = P.cs_alpha * (1 - 1.5 * q * q + 0.75 * q * q * q);
    F = P.cs_alpha * (-3 + 2.25 * q) * P.inv_h2;
  } else {
    const double t = 2 - q;
    W = P.cs_alpha * 0.25 * t * t * t;
    F = -P.cs_alpha * 0.75 * t * t / (P.h * r);
  }
}

constexpr int kPairSortLocal = 128;  // partners a query orders in thread-local memory

// The pairs whose i is the fluid particle in slot a, ordered by j, written
// from off[i]: the partners are gathered as (j, slot) keys, ordered by j in
// thread-local memory (more than kPairSortLocal: in place in the outputs),
// then each pair's values written once.
__global__ void k_pair_write(DevParams P, SlotArrays S, CellGrid G, const int *__restrict__ off, int32_t *ip,
                             int32_t *jp, double *rij2, double *w, double *dw)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double xa = S.x[a], ya = S.y[a];
  const int oa = S.orig[a];
  const int base = off[oa], total = off[oa + 1] - base;
  const double cd = P.knn > 0 ? P.kcut_d2[a] : 0.0;
  const int cj = P.knn > 0 ? P.kcut_j[a] : 0;
  const bool local = total <= kPairSortLocal;
  int kj[kPairSortLocal], kb[kPairSortLocal];
  int cnt = 0, k;
  NeighbourCursor cur;
  cur.init(P, G, G.cell_of[a]);
  while (cur.next(k)) {
    const int b = G.list[k];
    const int ob = S.orig[b];
    if (ob <= oa || ob >= P.pb) continue;
    const double dx = xa - S.x[b], dy = ya - S.y[b];
    const double r2 = pr2(dx, dy);
    if (!(r2 < P.r2cut && r2 > DBL_EPSILON)) continue;
    if (P.knn > 0 && !knn_key_le(r2, ob, cd, cj)) continue;
    if (local) {
      // insertion by j
      int i = cnt++;
      while (i > 0 && kj[i - 1] > ob) {
        kj[i] = kj[i - 1];
        kb[i] = kb[i - 1];
        i--;
      }
      kj[i] = ob;
      kb[i] = b;
      continue;
    }
    double W, F;
    pair_kernel(P, r2, W, F);
    const int o = base + cnt++;
    if (ip) ip[o] = oa;
    if (jp) jp[o] = ob;
    if (rij2) rij2[o] = r2;
    if (w) w[o] = W;
    if (dw) {
      dw[2 * o] = F * dx;
      dw[2 * o + 1] = F * dy;
    }
  }
  if (local) {
    for (int e = 0; e < cnt; e++) {
      const int b = kb[e], o = base + e;
      const double dx = xa - S.x[b], dy = ya - S.y[b];
      const double r2 = pr2(dx, dy);
      double W, F;
      pair_kernel(P, r2, W, F);
      if (ip) ip[o] = oa;
      if (jp) jp[o] = kj[e];
      if (rij2) rij2[o] = r2;
      if (w) w[o] = W;
      if (dw) {
        dw[2 * o] = F * dx;
        dw[2 * o + 1] = F * dy;
      }
    }
    return;
  }
  // order the segment by j (insertion sort in place)
  if (jp) {
    for (int i = base + 1; i < base + cnt; i++) {
      const int vj = jp[i];
      const double vr = rij2 ? rij2[i] : 0, vw = w ? w[i] : 0, vx = dw ? dw[2 * i] : 0, vy = dw ? dw[2 * i + 1] : 0;
      int j = i - 1;
      while (j >= base && jp[j] > vj) {
        jp[j + 1] = jp[j];
        if (rij2) rij2[j + 1] = rij2[j];
        if (w) w[j + 1] = w[j];
        if (dw) { dw[2 * (j + 1)] = dw[2 * j]; dw[2 * (j + 1) + 1] = dw[2 * j + 1]; }
        j--;
      }
      jp[j + 1] = vj;
      if (rij2) rij2[j + 1] = vr;
      if (w) w[j + 1] = vw;
      if (dw) { dw[2 * (j + 1)] = vx; dw[2 * (j + 1) + 1] = vy; }
    }
  }
}

// ApproximateVortcity (derivatives.c:2840-2885) for the fluid particle in
// slot a: every pair adds V_partner (dv_y dx - dv_x dy) w / (r^2 + 0.01 h^2)
// to both of its particles (the expression is the same from either side),
// dx = x_i - x_j, dv = v_i - v_j, V = m / rho.  Written by reference index.
__global__ void k_approx_vorticity(DevParams P, SlotArrays S, CellGrid G, double *__restrict__ out)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double xa = S.x[a], ya = S.y[a], ua = S.u[a], va = S.v[a];
  const int oa = S.orig[a];
  const double cd = P.knn > 0 ? P.kcut_d2[a] : 0.0;
  const int cj = P.knn > 0 ? P.kcut_j[a] : 0;
  double acc = 0.0;
  int k;
  NeighbourCursor cur;
  cur.init(P, G, G.cell_of[a]);
  while (cur.next(k)) {
    const int b = G.list[k];
    const int ob = S.orig[b];
    if (b == a || max(oa, ob) >= P.pb) continue;
    const double dx = xa - S.x[b], dy = ya - S.y[b];
    const double r2 = pr2(dx, dy);
    if (!(r2 < P.r2cut && r2 > DBL_EPSILON)) continue;
    if (P.knn > 0 && !(ob > oa ? knn_key_le(r2, ob, cd, cj) : knn_key_le(r2, oa, P.kcut_d2[b], P.kcut_j[b])))
      continue;
    double W, F;
    pair_kernel(P, r2, W, F);
    const double aij = ((va - S.v[b]) * dx - (ua - S.u[b]) * dy) * W * (1.0 / (r2 + P.eta2));
    acc += S.m[b] / S.rho[b] * aij;
  }
  out[oa] = acc;
}

}  // namespace

extern "C" uph_status uph_sim_approx_vorticity(uph_sim *s, double *vorticity)
{
  if (!s || !vorticity) return fail(UPH_BAD_ARG, "uph_sim_approx_vorticity: NULL argument");
  const int nf = s->P.nf;
  if (nf <= 0) return UPH_OK;
  if (s->P.profile != UPH_PROFILE_REF) return fail(UPH_UNSUPPORTED, "approxVorticity is a REF-profile diagnostic");
  cudaStream_t q = s->stream;
  uph_status r = build_cell_list(s);
  if (r != UPH_OK) return r;
  if (s->P.knn > 0 && !s->kcut_fresh) {
    VirtualPoints vp = {nullptr, nullptr, CellGrid{}};
    if (s->P.nvrules > 0 && s->have_rates) vp = VirtualPoints{s->vb.x, s->vb.y, s->gv};
    launch_knn_cut(s->P, s->S, s->G, vp, q);
    s->launches++;
    s->kcut_fresh = true;
  }
  double *d = s->T.rho;  // staging, nf entries free until the next upload or download
  k_approx_vorticity<<<(nf + 127) / 128, 128, 0, q>>>(s->P, s->S, s->G, d);
  s->launches++;
  UPH_CUDA(cudaMemcpyAsync(vorticity, d, sizeof(double) * nf, cudaMemcpyDeviceToHost, q));
  UPH_CUDA(cudaStreamSynchronize(q));
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

extern "C" uph_status uph_sim_pairs(uph_sim *s, int64_t cap, int32_t *i_pair, int32_t *j_pair, double *rij2,
                                    double *w, double *dwcdx, int64_t *niac)
{
  if (!s || !niac) return fail(UPH_BAD_ARG, "uph_sim_pairs: NULL argument");
  const int nf = s->P.nf;
  cudaStream_t q = s->stream;
  // the cell list of the last evaluation is still valid unless a reorder moved slots since
  uph_status r = build_cell_list(s);
  if (r != UPH_OK) return r;
  if (s->P.knn > 0 && !s->kcut_fresh) {
    // the virtual particles of the last evaluation, when the virtualType has them
    VirtualPoints vp = {nullptr, nullptr, CellGrid{}};
    if (s->P.nvrules > 0 && s->have_rates) vp = VirtualPoints{s->vb.x, s->vb.y, s->gv};
    launch_knn_cut(s->P, s->S, s->G, vp, q);
    s->launches++;
    s->kcut_fresh = true;
  }
  if (!s->pe_cnt) {
    const int nb = scan_block_sums_needed(nf > 0 ? nf : 1);
    UPH_CUDA(dalloc(s, &s->pe_cnt, (size_t)nf + 1));
    UPH_CUDA(dalloc(s, &s->pe_off, (size_t)nf + 1));
    UPH_CUDA(dalloc(s, &s->pe_bsum, (size_t)nb));
  }
  int *cnt = s->pe_cnt, *off = s->pe_off, *bsum = s->pe_bsum;
  uph_status result = UPH_OK;
  int total = 0;
  if (nf > 0) {
    k_pair_count<<<(nf + 127) / 128, 128, 0, q>>>(s->P, s->S, s->G, cnt);
    launch_exclusive_scan(cnt, off, nf, bsum, q);
    s->launches += 4;
    cudaMemcpyAsync(&total, off + nf, sizeof(int), cudaMemcpyDeviceToHost, q);
    cudaStreamSynchronize(q);
  }
  *niac = total;
  if (total > cap) {
    result = fail(UPH_NEIGHBOR_OVERFLOW, "pair buffer too small: " + std::to_string(total) + " pairs");
  } else if (total > 0) {
    if (total > s->pe_cap) {
      // grow by a quarter beyond what is needed, so small growth reallocates rarely
      UPH_CUDA(cudaStreamSynchronize(q));
      for (void *p : {(void *)s->pe_ip, (void *)s->pe_jp, (void *)s->pe_r2, (void *)s->pe_w, (void *)s->pe_dw})
        if (p) cudaFree(p);
      s->pe_ip = s->pe_jp = nullptr;
      s->pe_r2 = s->pe_w = s->pe_dw = nullptr;
      s->pe_cap = 0;
      const int64_t cap2 = (int64_t)total + total / 4 + 1024;
      UPH_CUDA(cudaMalloc((void **)&s->pe_ip, sizeof(int32_t) * cap2));
      UPH_CUDA(cudaMalloc((void **)&s->pe_jp, sizeof(int32_t) * cap2));
      UPH_CUDA(cudaMalloc((void **)&s->pe_r2, sizeof(double) * cap2));
      UPH_CUDA(cudaMalloc((void **)&s->pe_w, sizeof(double) * cap2));
      UPH_CUDA(cudaMalloc((void **)&s->pe_dw, sizeof(double) * 2 * cap2));
      s->pe_cap = cap2;
    }
    int32_t *dip = s->pe_ip, *djp = s->pe_jp;
    double *dr = s->pe_r2, *dww = s->pe_w, *ddw = s->pe_dw;
    k_pair_write<<<(nf + 127) / 128, 128, 0, q>>>(s->P, s->S, s->G, off, dip, djp, dr, dww, ddw);
    s->launches++;
    if (i_pair) cudaMemcpyAsync(i_pair, dip, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, q);
    if (j_pair) cudaMemcpyAsync(j_pair, djp, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, q);
    if (rij2) cudaMemcpyAsync(rij2, dr, sizeof(double) * total, cudaMemcpyDeviceToHost, q);
    if (w) cudaMemcpyAsync(w, dww, sizeof(double) * total, cudaMemcpyDeviceToHost, q);
    if (dwcdx) cudaMemcpyAsync(dwcdx, ddw, sizeof(double) * 2 * total, cudaMemcpyDeviceToHost, q);
  }
  UPH_CUDA(cudaStreamSynchronize(q));
  UPH_CUDA(cudaGetLastError());
  return result;
}

// ---- statistics -----------------------------------------------------------------

namespace {

// per-block partial sums (KE, PE, mass) and max |rho - rho0| / rho0; the host
// adds the partials in block order, so the result is deterministic
__global__ void k_stats(DevParams P, SlotArrays S, double *partials, int nblocks_total)
{
  __shared__ double sh[4][256];
  double ke = 0, pe = 0, m = 0, de = 0;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P.nf; a += gridDim.x * blockDim.x) {
    const double ma = S.m[a], u = S.u[a], v = S.v[a];
    ke += 0.5 * ma * (u * u + v * v);
    pe += ma * P.g * S.y[a];
    m += ma;
    de = fmax(de, fabs(S.rho[a] - P.rho0) / P.rho0);
  }
  sh[0][threadIdx.x] = ke;
  sh[1][threadIdx.x] = pe;
  sh[2][threadIdx.x] = m;
  sh[3][threadIdx.x] = de;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
      sh[2][threadIdx.x] += sh[2][threadIdx.x + o];
      sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) partials[k * nblocks_total + blockIdx.x] = sh[k][0];
}

// Per-evaluation diagnostics (TotalKineticEnergy, derivatives.c:2254-2264;
// NeighborsToPressurePoint / ...Two, derivatives.c:2290-2393) over the fluid
// at the state the rate pass just read.  Each block writes its partials
// [KE, PE, sum p w, sum w, n1, sum p, n2]; the last block to finish (counted
// with an atomic after a fence) adds them in block order and updates the
// persistent values, so the result is deterministic and needs no host step.
__global__ void k_diagnostics(DevParams P, SlotArrays S, DiagProbes q, double *partials, int nblocks_total,
                              unsigned *done, DevDiag *out, const int *d_itime)
{
  __shared__ double sh[kDiagRows][256];
  __shared__ bool last;
  const double e9 = exp(-9.0);
  const double coeff1 = 0.5 - 5.0 * e9;
  const double h = P.h;
  double acc[kDiagRows] = {0, 0, 0, 0, 0, 0, 0};
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P.nf; a += gridDim.x * blockDim.x) {
    const double ma = S.m[a], u = S.u[a], v = S.v[a], xa = S.x[a], ya = S.y[a];
    acc[0] += 0.5 * ma * (u * u + v * v);
    acc[1] += ma * P.g * ya;
    const double pa = S.p[a];
    if (!(pa > 0.0)) continue;
    double dx = xa - q.x1, dy = ya - q.y1;
    double r = sqrt(dx * dx + dy * dy);
    if (r <= 3.0 * h) {
      const double w = (exp(-r * r / (h * h)) - e9) * ma / (2.0 * M_PI * h * h * coeff1 * S.rho[a]);
      acc[2] += pa * w;
      acc[3] += w;
      acc[4] += 1.0;
    }
    dx = xa - q.x2;
    dy = ya - q.y2;
    r = sqrt(dx * dx + dy * dy);
    if (r < 2.0 * h) {
      acc[5] += pa;
      acc[6] += 1.0;
    }
  }
  for (int k = 0; k < kDiagRows; k++) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int k = 0; k < kDiagRows; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < kDiagRows; k++) partials[k * nblocks_total + blockIdx.x] = sh[k][0];
    __threadfence();
    last = atomicAdd(done, 1u) == (unsigned)nblocks_total - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if ((int)threadIdx.x < kDiagRows) {
    const volatile double *row = partials + threadIdx.x * nblocks_total;
    double t = 0.0;
    for (int b = 0; b < nblocks_total; b++) t += row[b];
    sh[threadIdx.x][0] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int n1 = (int)sh[4][0], n2 = (int)sh[6][0];
    out->kinetic_energy = sh[0][0];
    out->potential_energy = sh[1][0];
    out->point_neighbors = n1;
    out->pressure_norm = n1 ? sh[3][0] : 1.0;
    if (n1) out->point_pressure = sh[2][0] / sh[3][0];
    out->point_neighbors_two = n2;
    out->point_pressure_two = n2 ? sh[5][0] / n2 : 0.0;
    out->itime = d_itime ? *d_itime : 0;  // the steps started, this one included
    *done = 0u;
  }
}

void launch_diagnostics(uph_sim *s)
{
  k_diagnostics<<<s->diag_blocks, 256, 0, s->stream>>>(s->P, s->S, s->diag_probes, s->d_diag_part, s->diag_blocks,
                                                       s->d_diag_done, s->d_diag, s->d_itime);
  s->launches++;
}

}  // namespace

extern "C" uph_status uph_sim_set_diagnostics(uph_sim *s, int32_t enable, double x, double y, double x2, double y2)
{
  if (!s) return fail(UPH_BAD_ARG, "uph_sim_set_diagnostics: NULL sim");
  drop_graph(s);  // the recorded steps carry the old setting
  s->diag_enabled = enable != 0;
  s->diag_probes = DiagProbes{x, y, x2, y2};
  return UPH_OK;
}

extern "C" uph_status uph_sim_diagnostics(uph_sim *s, uph_diagnostics *out)
{
  if (!s || !out) return fail(UPH_BAD_ARG, "uph_sim_diagnostics: NULL argument");
  memset(out, 0, sizeof *out);
  if (!s->diag_enabled) return fail(UPH_BAD_ARG, "uph_sim_diagnostics: diagnostics are off (uph_sim_set_diagnostics)");
  DevDiag d;
  UPH_CUDA(cudaMemcpyAsync(&d, s->d_diag, sizeof d, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  out->kinetic_energy = d.kinetic_energy;
  out->potential_energy = d.potential_energy;
  out->point_pressure = d.point_pressure;
  out->pressure_norm = d.pressure_norm;
  out->point_pressure_two = d.point_pressure_two;
  out->point_neighbors = d.point_neighbors;
  out->point_neighbors_two = d.point_neighbors_two;
  out->itime = d.itime;
  return UPH_OK;
}

extern "C" uph_status uph_sim_stats(uph_sim *s, uph_stats *out)
{
  if (!s || !out) return fail(UPH_BAD_ARG, "uph_sim_stats: NULL argument");
  memset(out, 0, sizeof *out);
  const int nb = s->n_partials;
  k_stats<<<nb, 256, 0, s->stream>>>(s->P, s->S, s->d_partials, nb);
  s->launches++;
  std::vector<double> part(4 * (size_t)nb);
  unsigned long long niac = 0;
  int mx = 0;
  UPH_CUDA(cudaMemcpyAsync(part.data(), s->d_partials, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaMemcpyAsync(&niac, s->d_niac, sizeof niac, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaMemcpyAsync(&mx, s->d_max_nb, sizeof mx, cudaMemcpyDeviceToHost, s->stream));
  unsigned builds = 0;
  UPH_CUDA(cudaMemcpyAsync(&builds, s->G.gen, sizeof builds, cudaMemcpyDeviceToHost, s->stream));
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  for (int b = 0; b < nb; b++) {
    out->kinetic_energy += part[b];
    out->potential_energy += part[nb + b];
    out->total_mass += part[2 * nb + b];
    out->max_abs_density_error = fmax(out->max_abs_density_error, part[3 * nb + b]);
  }
  out->niac = s->have_rates ? (int64_t)niac : 0;
  out->max_neighbors = s->have_rates ? mx : 0;
  out->itime = s->itime;
  out->list_builds = builds;
  return UPH_OK;
}

// ---- tuning -----------------------------------------------------------------------

extern "C" uph_status uph_sim_set_tuning(uph_sim *s, int32_t reach, int32_t tile, int32_t reorder_interval)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  if (reach < 1 || reach > 3) return fail(UPH_BAD_ARG, "cell reach must be 1, 2 or 3");
  // the tiled pass stages a tile plus `reach` cells on each side: at most 32 cells per axis
  if (tile < 1 || tile + 2 * reach > kTileRowsMax)
    return fail(UPH_BAD_ARG, "tile must be positive and tile + 2 reach at most 32");
  if (reorder_interval < 1 || reorder_interval > 4096) return fail(UPH_BAD_ARG, "reorder interval out of range");
  DevParams P2 = s->P;
  set_grid_geometry(P2, reach, tile);
  if ((long long)P2.ncx * P2.ncy > (1LL << 28)) return fail(UPH_BAD_ARG, "tuned cell grid larger than 2^28 cells");
  UPH_CUDA(cudaStreamSynchronize(s->stream));
  s->P = P2;
  UPH_CUDA(alloc_grid(s));
  s->reorder_interval = reorder_interval;
  drop_graph(s);
  // storage order follows the new tile from now on
  return reorder_fluid(s);
}

namespace {

struct TuneKey {
  int profile, precision, nf_class, cell_class;
  bool operator<(const TuneKey &o) const
  {
    if (profile != o.profile) return profile < o.profile;
    if (precision != o.precision) return precision < o.precision;
    if (nf_class != o.nf_class) return nf_class < o.nf_class;
    return cell_class < o.cell_class;
  }
};

std::mutex g_tune_mutex;
std::map<TuneKey, std::array<int, 3>> g_tune_cache;

int log2_class(double v) { return v < 1.0 ? 0 : (int)floor(log2(v)); }

// ms per step of `steps` steps (after two warm-up steps) with the current tuning
uph_status time_steps(uph_sim *s, int steps, double *ms)
{
  uph_status r = enqueue_steps(s, 2, false);
  if (r != UPH_OK) return r;
  cudaEvent_t a, b;
  UPH_CUDA(cudaEventCreate(&a));
  UPH_CUDA(cudaEventCreate(&b));
  cudaEventRecord(a, s->stream);
  r = enqueue_steps(s, steps, false);
  cudaEventRecord(b, s->stream);
  cudaEventSynchronize(b);
  float f = 0.f;
  cudaEventElapsedTime(&f, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (r != UPH_OK) return r;
  *ms = f / steps;
  return check_error_word(s);
}

}  // namespace

// Coordinate search over (cell reach, storage tile, re-sort interval): the
// reach first with tile 11 and interval 64, then the tile at the best reach,
// then the interval.  Each trial times `trial_steps` steps of this very
// simulation, so tuning advances it by about 9 (trial_steps + 2) steps.
// Results are cached per size class (profile, precision, log2 of the fluid
// count, log2 of the radius-wide cell count); a sim of a cached class is set
// without trials.
extern "C" uph_status uph_sim_autotune(uph_sim *s, int32_t trial_steps, int32_t choice[3], double *ms_per_step)
{
  if (!s || !choice) return fail(UPH_BAD_ARG, "uph_sim_autotune: NULL argument");
  if (trial_steps < 1) return fail(UPH_BAD_ARG, "uph_sim_autotune: trial_steps must be positive");
  DevParams P1 = s->P;
  set_grid_geometry(P1, 1, 1);
  const TuneKey key{s->P.profile, s->P.precision, log2_class(s->P.nf), log2_class((double)P1.ncx * P1.ncy)};
  std::array<int, 3> best{kCellReach, kCellTile, kReorderInterval};
  bool cached = false;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      best = it->second;
      cached = true;
    }
  }
  double best_ms = 0.0;
  if (!cached) {
    auto trial = [&](std::array<int, 3> c, double *ms) -> uph_status {
      uph_status r = uph_sim_set_tuning(s, c[0], c[1], c[2]);
      if (r != UPH_OK) return r;
      return time_steps(s, trial_steps, ms);
    };
    best_ms = 1e300;
    for (int axis = 0; axis < 3; axis++) {
      static const int options[3][3] = {{1, 2, 3}, {9, 11, 13}, {16, 64, 256}};
      std::array<int, 3> axis_best = best;
      for (int v : options[axis]) {
        std::array<int, 3> c = best;
        c[axis] = v;
        double ms = 0.0;
        uph_status r = trial(c, &ms);
        if (r == UPH_BAD_ARG) continue;  // e.g. a grid too large for this reach
        if (r != UPH_OK) return r;
        if (ms < best_ms) {
          best_ms = ms;
          axis_best = c;
        }
      }
      best = axis_best;
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best;
  }
  uph_status r = uph_sim_set_tuning(s, best[0], best[1], best[2]);
  if (r != UPH_OK) return r;
  for (int k = 0; k < 3; k++) choice[k] = best[k];
  if (ms_per_step) *ms_per_step = best_ms;
  return UPH_OK;
}

// ---- profiling --------------------------------------------------------------------

extern "C" uph_status uph_sim_profile(uph_sim *s, int32_t enable)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  if (enable && s->ev_pool.empty()) {
    s->ev_pool.resize(2 * uph_sim::kEventPool, nullptr);
    s->ev_family.resize(uph_sim::kEventPool, 0);
    for (cudaEvent_t &e : s->ev_pool) UPH_CUDA(cudaEventCreate(&e));
  }
  flush_profile(s);
  s->profiling = enable != 0;
  for (int k = 0; k < KF_COUNT; k++) {
    s->fam_ms[k] = 0;
    s->fam_launch[k] = 0;
  }
  return UPH_OK;
}

extern "C" uph_status uph_sim_kernel_times(uph_sim *s, int32_t n, double *ms, int64_t *launches, char *names,
                                           size_t names_len, int32_t *n_written)
{
  if (!s) return fail(UPH_BAD_ARG, "NULL sim");
  flush_profile(s);
  const int m = n < KF_COUNT ? n : KF_COUNT;
  std::string all;
  for (int k = 0; k < m; k++) {
    if (ms) ms[k] = s->fam_ms[k];
    if (launches) launches[k] = s->fam_launch[k];
    if (k) all += ",";
    all += kFamilyNames[k];
  }
  if (names && names_len) {
    strncpy(names, all.c_str(), names_len - 1);
    names[names_len - 1] = 0;
  }
  if (n_written) *n_written = m;
  return UPH_OK;
}

extern "C" int64_t uph_sim_launch_count(const uph_sim *s) { return s ? s->launches : 0; }

// ---- one-shot neighbour search ------------------------------------------------------

namespace {

__global__ void k_load_positions(SlotArrays S, const double *__restrict__ pos, int n)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  S.x[k] = pos[2 * k];
  S.y[k] = pos[2 * k + 1];
  S.orig[k] = k;
}


}  // namespace

extern "C" uph_status uph_search_neighbors(const double *position, int32_t n_fluid, int32_t n_all,
                                           int32_t particle_boundary, int32_t knn, double dist, int64_t cap,
                                           int32_t *i_pair, int32_t *j_pair, double *rij2, int64_t *niac)
{
  if (!position || !niac || n_fluid < 0 || n_all < n_fluid || n_all <= 0)
    return fail(UPH_BAD_ARG, "uph_search_neighbors: bad arguments");
  *niac = 0;
  if (n_fluid == 0 || !(dist > 0.0)) return UPH_OK;
  double lo[2] = {position[0], position[1]}, hi[2] = {position[0], position[1]};
  for (int k = 0; k < n_all; k++)
    for (int d = 0; d < 2; d++) {
      const double v = position[2 * k + d];
      if (!isfinite(v)) return fail(UPH_NAN, "uph_search_neighbors: non-finite position");
      lo[d] = fmin(lo[d], v);
      hi[d] = fmax(hi[d], v);
    }
  uph_params p;
  memset(&p, 0, sizeof p);
  p.n_fluid = n_fluid;
  p.n_fixed = n_all - n_fluid;
  p.dim = 2;
  p.flag_init_simul = 1;
  p.dx = 1.0;
  p.h = 0.5 * sqrt(dist);
  p.density0 = 1.0;
  if (knn > kKnnMax) return fail(UPH_UNSUPPORTED, "knn above " + std::to_string(kKnnMax) + " is not implemented");
  p.knn_cap = knn > 0 ? knn : 0;
  const double pad = sqrt(dist);
  p.domain_lo[0] = lo[0] - pad;
  p.domain_lo[1] = lo[1] - pad;
  p.domain_hi[0] = hi[0] + pad;
  p.domain_hi[1] = hi[1] + pad;
  uph_sim *s = nullptr;
  uph_status r = uph_sim_create(&p, &s);
  if (r != UPH_OK) return r;
  // the reference's own threshold and boundary index, not ones derived from h
  s->P.r2cut = dist;
  s->P.pb = particle_boundary;
  cudaStream_t q = s->stream;
  double *dpos = s->T.pos;
  r = UPH_OK;
  if (cudaMemcpyAsync(dpos, position, sizeof(double) * 2 * n_all, cudaMemcpyHostToDevice, q) != cudaSuccess) {
    uph_sim_destroy(s);
    return fail(UPH_CUDA_ERROR, "uph_search_neighbors: upload failed");
  }
  k_load_positions<<<(n_all + 255) / 256, 256, 0, q>>>(s->S, dpos, n_all);
  r = force_rebuild(s);
  if (r == UPH_OK) r = build_cell_list(s);
  // an overcrowded cell (or a position outside the grid) stops here, before
  // any kernel walks the candidates
  if (r == UPH_OK) r = check_error_word(s);
  if (r == UPH_OK) r = check_error_word(s);
  if (r == UPH_OK) {
    s->have_rates = true;
    // uph_sim_pairs without the cell-list rebuild side effects on positions
    r = uph_sim_pairs(s, cap, i_pair, j_pair, rij2, nullptr, nullptr, niac);
  }
  uph_sim_destroy(s);
  return r;
}

// ---- access for the learned surrogate (sim_access.cuh) ----------------------
namespace uph {

SimView sim_view(uph_sim *s)
{
  SimView v;
  v.P = s->P;
  v.S = s->S;
  v.W = s->W;
  v.stream = s->stream;
  v.err = s->d_err;
  v.itime = s->itime;
  v.walls_move = walls_move(s);
  v.serial = s->serial;
  return v;
}

uph_status sim_jump(uph_sim *s, int nsteps)
{
  s->itime += nsteps;
  UPH_CUDA(cudaMemcpyAsync(s->d_itime, &s->itime, sizeof(int), cudaMemcpyHostToDevice, s->stream));
  // the moving walls at the new time, as after a step that ended there
  if (walls_move(s)) {
    launch_wall_motion(s->P, s->S, s->W, s->itime * s->P.dt, nullptr, s->d_err, s->stream);
    s->launches++;
  }
  s->restart = true;
  {
    uph_status r = force_rebuild(s);
    if (r != UPH_OK) return r;
  }
  // the storage re-sort waits for the next plain step (the state moves
  // about 0.1 dx per jump, so the slot order stays spatially coherent)
  s->steps_since_reorder += nsteps;
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}

uph_status sim_check(uph_sim *s) { return check_error_word(s); }

void sim_count_launches(uph_sim *s, int n) { s->launches += n; }

}  // namespace uph
