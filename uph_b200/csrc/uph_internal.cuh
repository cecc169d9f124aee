// Internal definitions shared by the CUDA translation units of libuph.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "uph.h"

namespace uph {

// ---- device error word bits (set by kernels, read by the host) -------------
enum : unsigned {
  ERR_OUT_OF_DOMAIN = 1u,
  ERR_NAN = 2u,
  ERR_NEIGHBOR_OVERFLOW = 4u,
  ERR_TIMEOUT = 8u,
};

// Bounded device-side waits give up after this long on the GPU's global
// timer (and after an iteration cap), set ERR_TIMEOUT and clean up.
constexpr unsigned long long kWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Particle data in storage ("slot") order.  Fluid particles occupy slots
// [0, nf), the other interacting particles [nf, n).  Storage order is
// spatially sorted (cell order) so that a warp's particles share neighbours.
struct SlotArrays {
  double *x, *y, *u, *v;  // Position, Velocity
  double *ut, *vt;        // localVelocity
  double *rho, *rhot;     // density, localDensity
  double *p, *pt;         // DynamicPressure, localPressure
  double *m;              // mass
  double *inv_rho;        // 1 / density (refreshed before every rate evaluation)
  double *inv_rhot;       // 1 / localDensity
  int32_t *itype;
  int32_t *orig;          // reference index of the particle in this slot
  // fluid-only (first nf slots)
  double *rho_min, *p_min, *u_min, *v_min;
  double *sponge;
  double *drho, *dp, *ax, *ay;              // ddensitydt, dpdt, dvdt
  double *drho_a, *dp_a, *ax_a, *ay_a;      // *_approx
  double *frho, *fp, *fu, *fv;              // density/pressure/velocity fluctuation
  double *pressure;                         // algebraic Tait (all slots)
};

// One mirror rule of the reference's virtual particles: which fluid
// particles it copies (within 2h of a wall line, 3h of the slope) and where
// it puts the copy.  Line positions given as a source: a constant, or the
// left/right boundary position of the step's time.
enum VirtualKind {
  VK_LEFT,      // |x - X| < 2h: x' = X - |x - X|, u' = -u
  VK_RIGHT,     // |x - X| < 2h: x' = X + |x - X|, u' = -u
  VK_BOTTOM,    // y < 2h and x <= L: y' = -y, v' = -v
  VK_TOP,       // |(y - D) - e| < 2h: y' = D + 2 |(y - D) - e|, v' = -v
  VK_CORNER_L,  // |x - X| < 2h and y < 2h: x' = X - |x - X|, y' = -y, both flipped
  VK_CORNER_R,  // |x - X| < 2h and y < 2h: x' = X + |x - X|, y' = -y, both flipped
  VK_SLOPE      // distance to y = s (x - L) below 3h and x > L: reflected in that line
};
enum VirtualPos { VP_CONST, VP_LEFT, VP_RIGHT };
struct VirtualRule {
  int kind;
  int pos;   // VirtualPos of X (VK_LEFT / RIGHT / CORNER_*)
  double a;  // X for VP_CONST; L (BOTTOM, SLOPE); D (TOP)
  double b;  // e (TOP); slope s (SLOPE)
};
constexpr int kMaxVirtualRules = 5;

// Constants of one simulation as the kernels see them.
struct DevParams {
  int nf, n;        // fluid slots, all slots
  int pb;           // ParticleBoundary = Nf + Ns + Nb - 1 (reference indices)
  int b0, b1;       // boundary reference index range [Nf+Ns, Nf+Ns+Nb)
  int m0;           // first moving-boundary reference index
  int profile, precision;
  double h, inv_h, inv_h2;
  double r2cut;     // (h*h)*4, the reference's search radius squared
  double eta2;      // 0.01 h^2
  double w_alpha;   // poly-7 convolution normalisation (derivatives.c:769)
  double dw_alpha;  // -alpha_0 of the poly-7 deconvolution (derivatives.c:788)
  double dw_alpha_h2;  // dw_alpha / h^2
  double cs_alpha;  // cubic spline sigma = 10 / (7 pi h^2) (derivatives.c:46)
  double rho0, gamma, c0, B, rho0c2, g;
  int gravity_flag;
  double mu0, kappa, eps;
  double two_mu0;  // 2 mu0
  int stress_type;
  int boundary_force;
  double k_spring, c_damp, dx, dy;
  double lj_coeff, mach_c;  // LennardCoefficient, machNumber * SpeedOfSound
  int moving_boundary, flag_init_simul, wave_absorption;
  double stroke, omega;
  double lid_velocity;  // lidVelocity: the lid (movingBoundary 3) and gate (2) speed
  double gate_stop;     // the gate stops at 1.5 (LocalDepth - 15 dx) / lidVelocity (inputbp.c:226)
  double av_alpha_c0;       // WCSPH: alpha * c0
  double dt;
  // cell grid
  double lo_x, lo_y, cell, inv_cell;
  double hi_x, hi_y;  // declared domain; the grid itself is rounded up to whole tiles
  int ncx, ncy;  // cells per axis, multiples of `tile`
  int tile;      // storage-order tile edge in cells
  int ntx;       // tiles per row
  int reach;     // cells are >= radius / reach wide; partners lie within `reach` cells
  // k-nearest cap of the reference's search (derivatives.c:1085 passes 40):
  // 0 = every in-radius pair; else each fluid query s keeps its knn nearest
  // in-radius points, ordered by (r^2, reference index), and a pair (i, j)
  // exists iff j is among query i's kept points.  kcut_* [nf], by slot: the
  // largest kept key of the query, (+inf, INT_MAX) when nothing is cut.
  int knn;
  double *kcut_d2;
  int *kcut_j;
  // stressType 2: each particle's shear stress over its density squared,
  // sigma / rho^2 (xx, xy = yx, yy), indexed by slot
  double *str_xx, *str_xy, *str_yy;
  // virtual mirror particles (derivatives.c:3194-4192; virtual.cu): the
  // virtualType's mirror rules in the reference's order
  int nvrules;
  VirtualRule vrule[kMaxVirtualRules];
  int vleft_moves;  // LeftBoundaryPosition follows the piston law (inputbp.c:194-207, 244-250)
  double flat_bottom_length, local_depth;
  // particle packing (flag_init_simul == 0): mass of reference particle 0,
  // the reference's volume scale mass[0] / rho0 (derivatives.c:2967)
  const double *pack_mass0;
  // Skin of the cell list: cells are (1 + kCellSkin) radius / reach wide, so
  // the list stays complete while no particle has moved more than `skin`
  // (per axis) from where the last build binned it (xbin, ybin by slot).
  // The corrector and the wall motion raise *rebuild when one has; the
  // build kernel skips its work while *rebuild is 0.
  double skin;
  double *xbin, *ybin;
  unsigned *rebuild;
};

constexpr double kCellSkin = 0.05;

constexpr int kKnnMax = 64;  // largest knn cap the kernels keep per query

// (r2, j) <= (cd, cj) in the cap's order
__host__ __device__ __forceinline__ bool knn_key_le(double r2, int j, double cd, int cj)
{
  return r2 < cd || (r2 == cd && j <= cj);
}

// The cell list numbers cells row-major (cy * ncx + cx), so the cells of one
// stencil row are one contiguous range of the list.  Particle *storage* is
// sorted by a tile-major key instead: kCellTile x kCellTile cells form a
// tile, tiles row-major, cells inside a tile row-major.  The REF rate pass
// runs one CTA per tile (tile_pass.cuh), so a tile's fluid particles are
// nearly contiguous slots.  The tile edge is a tuning parameter
// (DevParams::tile, default 11: 121 cells of (1 + skin) h hold about 225
// particles of a lattice at h = 1.3 dx, one per thread of a 256-thread CTA,
// with room for compression before a second round of the CTA is needed).
constexpr int kCellTile = 11;

__host__ __device__ __forceinline__ int storage_key(int cx, int cy, int ntx, int tile)
{
  const int tx = cx / tile, lx = cx % tile, ty = cy / tile, ly = cy % tile;
  return ((ty * ntx + tx) * tile + ly) * tile + lx;
}

// Per-particle horizontal shaking of the moving boundary block (reference
// indices [m0, b1)): x = x0 + hs (1 - cos w t), u = ut = hs w sin w t.
// Indexed by reference index - m0, so it does not move with re-sorts.
struct WallTable {
  const double *x0, *hs, *om;
  int enabled;
  // the lid's and the gate's per-particle base coordinate (the reference's
  // tempPosition / tempPositionGate), indexed by reference index - m0
  const double *base;
};

constexpr int kGridWords = 2;

struct CellGrid {
  int ncell;
  int *count;    // [ncell]
  int *start;    // [ncell + 1]
  int *fill;     // [ncell]
  int *list;     // [n] slots in cell order
  int *cell_of;  // [n]
  int *block_sums;
  int nblock_sums;
  // one-launch build (launch_cell_build): rank of each slot in its cell,
  // per-block totals and the grid barrier's two words; count and bar are all
  // zero between builds
  int *rank;       // [n]
  int *totals;     // [kCellBuildMaxBlocks + 1]
  unsigned *bar;   // [kGridWords]
  // The tiled passes' candidate lists (the simulation's main grid only; null
  // on other grids).  gen counts the builds that rebuilt the list.  A tile
  // whose tile_gen equals gen has, for each of its fluid particles (by
  // slot), vl_n candidates in vl[slot * kVlMax ...]: the records of its
  // block within the list radius (the search radius plus twice the largest
  // displacement a rebuild allows), in the stencil walk's order, or vl_n ==
  // kVlOverflow when there were more than kVlMax.
  unsigned *gen;           // [1]
  unsigned *tile_gen;      // [number of tiles]
  unsigned short *vl;      // [nf * kVlMax]
  unsigned char *vl_n;     // [nf]
};
constexpr int kVlMax = 24;
constexpr unsigned char kVlOverflow = 255;

// Statistics of a rate pass, zeroed by the cell-list launch before it: pairs
// (i < j) counted from the i side, and the largest in-radius neighbour count
// of a fluid particle.
struct PassStats {
  unsigned long long *niac;
  int *max_nb;
};

std::string &last_error();
uph_status fail(uph_status s, const std::string &msg);
uph_status cuda_fail(cudaError_t e, const char *what);

#define UPH_CUDA(call)                                  \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::uph::cuda_fail(e_, #call); \
  } while (0)

// ---- launches implemented in the .cu files ---------------------------------
// cell list
void launch_cell_keys(const DevParams &P, const double *x, const double *y, int first, int count,
                      CellGrid &G, unsigned *err, bool storage_order, cudaStream_t s);
void launch_exclusive_scan(const int *in, int *out, int n, int *block_sums, cudaStream_t s);
int scan_block_sums_needed(int n);  // size of launch_exclusive_scan's block_sums
// the same scan with 64-bit offsets and totals (pair counts); out has n + 1 entries
void launch_exclusive_scan64(const int *in, long long *out, int n, long long *block_sums, cudaStream_t s);
void launch_cell_scatter(const CellGrid &G, int first, int count, cudaStream_t s);
// a cell with more ids than this is left unsorted and flags ERR_NEIGHBOR_OVERFLOW
constexpr int kMaxCellOccupancy = 4096;
void launch_cell_sort_segments(const CellGrid &G, unsigned *err, cudaStream_t s);
// The whole build (keys and histogram, scan, scatter, per-cell sort) as one
// cooperative launch with three bounded grid barriers.  count must be all
// zero on entry and is again on return.
constexpr int kCellBuildThreads = 512;
constexpr int kCellBuildMaxBlocks = 1024;
// check_rebuild: build only when *P.rebuild is set (and then clear it and
// record the binned positions); otherwise always build.  stats, when given,
// are zeroed for the rate pass that follows, whether or not the list is
// rebuilt.
// step_counter, when given, is advanced by one (a leapfrog step starts);
// dyn_count, when given, lowers count to the device value it points to.
uph_status launch_cell_build(const DevParams &P, const double *x, const double *y, int first, int count,
                             CellGrid &G, unsigned *err, bool storage_order, const PassStats *stats,
                             cudaStream_t s, bool check_rebuild = false, int *step_counter = nullptr,
                             const int *dyn_count = nullptr);

// A leapfrog step applied by the rate pass itself.  The pass reads the state
// of S (staged in shared memory, so other tiles' particles must not change
// under it) and writes each fluid particle's post-step state -- corrected,
// with the next step's predictor when predict_next, and with the rates and
// the algebraic pressure when not -- into D, the simulation's other buffer;
// the caller then swaps the two.  D must hold the same particle constants
// (mass, type, reference index, sponge factor) as S, and the walls' fields;
// where walls move the pass also moves D's walls: walls == 1
// to this step's time, *d_itime dt (where S's walls are), walls == 2 to the
// next step's, (*d_itime + 1) dt.  enabled == 0: the pass writes only the
// rates, into S.
struct StepOut {
  SlotArrays D;
  WallTable W;
  unsigned *err;
  const int *d_itime;
  int enabled, first_step, predict_next, walls;
};

// REF / WCSPH rate pass over the fluid slots: one CTA per storage tile
// (tile_pass.cuh); the cell list must be current.
uph_status launch_ref_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st,
                           const StepOut &F, cudaStream_t s);
// the REF profile's particle-packing pass (flag_init_simul == 0) in its place
uph_status launch_packing_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st,
                               cudaStream_t s);
// The virtual mirror particles of one evaluation (virtual.cu), and their own
// cell list on the simulation's grid; grid.list == nullptr: none.
struct VirtualPoints {
  const double *x, *y;  // [count], in the reference's order
  CellGrid grid;
};
// the knn cap's cut of every fluid query (P.kcut_*), from the cell list and
// the virtual points
void launch_knn_cut(const DevParams &P, const SlotArrays &S, const CellGrid &G, const VirtualPoints &V,
                    cudaStream_t s);
// Scratch and results of the virtual particles: flags and offsets by
// (rule, reference fluid index), positions, source fluid index and rule of
// each virtual particle, and their count.
struct VirtualBuf {
  int cap;  // P.nvrules * nf
  int *flags, *offs, *block_sums;
  int *count;
  double *x, *y;
  int *src, *rule;  // reference fluid index copied; the VirtualKind of the rule
};
// Generates the virtual particles of the time (*d_itime) dt, or t_host when
// d_itime is null (derivatives.c:3194-4192).
void launch_virtual(const DevParams &P, const SlotArrays &S, const VirtualBuf &V, double t_host, const int *d_itime,
                    cudaStream_t s);
// stressType 2, after the rate pass: the shear stress of every listed
// particle (P.str_*), then its divergence added to the corrector's dv/dt
void launch_viscous_two_step(const DevParams &P, const SlotArrays &S, const CellGrid &G, cudaStream_t s);
uph_status launch_wcsph_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st,
                             const StepOut &F, cudaStream_t s);

// leapfrog
void launch_predict(const DevParams &P, const SlotArrays &S, cudaStream_t s);
// predict_next: the next step's predictor too; walls_next: the next step's
// wall motion too (threads past the fluid)
void launch_correct(const DevParams &P, const SlotArrays &S, const WallTable &W, int first_step, int predict_next,
                    int walls_next, unsigned *err, const int *d_itime, cudaStream_t s);
void launch_refresh_inverse(const DevParams &P, const SlotArrays &S, int first, int count, cudaStream_t s);
// t = (*d_itime + 1) dt when d_itime is given: the counter holds the steps
// started (the cell-list launch of each step of uph_sim_step advances it)
// and lives on the device so CUDA-graph replays see the right time;
// else t = t_host
void launch_wall_motion(const DevParams &P, const SlotArrays &S, const WallTable &W, double t_host,
                        const int *d_itime, unsigned *err, cudaStream_t s);
void launch_wall_pressure(const DevParams &P, const SlotArrays &S, cudaStream_t s);

// BF16 tcgen05 GEMM, C[M x N] = A . B^T with FP32 accumulation.  An operand
// is K-major ([rows x K], ld >= K) unless its *_trans flag says it is stored
// [K x rows] (ld >= rows).  Epilogue, in order: + bias[N], + a BF16
// residual, + old c_f32 (accumulate), ReLU, zero where mask <= 0; then FP32
// and/or BF16 stores.
// splits > 1 splits K over CTAs into `partials` (splits * M * N floats) and
// sums them in split order into a dense c_f32 (ldc == N).
struct GemmCall {
  const void *A = nullptr;
  int lda = 0, a_trans = 0;
  const void *B = nullptr;
  int ldb = 0, b_trans = 0;
  int M = 0, N = 0, K = 0;
  int k_valid = 0;  // transposed operands: K rows >= k_valid read as zero (0: K)
  const float *bias = nullptr;
  int relu = 0;
  const void *mask = nullptr;
  int ldm = 0;
  int accumulate = 0;
  const void *residual = nullptr;  // BF16 [M x ldr]
  int ldr = 0;
  float *c_f32 = nullptr;
  void *c_bf16 = nullptr;
  int ldc = 0;
  int ldc16 = 0;  // leading dimension of c_bf16 (0: ldc)
  int splits = 1;
  float *partials = nullptr;
  unsigned *err = nullptr;
  int stall = 0;  // self-test: each CTA first waits on a barrier nothing arrives at
};
uph_status launch_tc_gemm(const GemmCall &c, cudaStream_t s);

}  // namespace uph
