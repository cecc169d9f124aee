// The fused rate pass of the WCSPH profile on the same cell list and pair
// set as the REF pass:
//   drho_a = sum_b m_b (v_a - v_b) . grad_a W_ab
//   dv_a   = -sum_b m_b (p_a/rho_a^2 + p_b/rho_b^2 + Pi_ab) grad_a W_ab + g + walls
//   Pi_ab  = -alpha c0 h (v_ab . x_ab) / (r^2 + 0.01 h^2) / rhobar_ab   if v_ab . x_ab < 0
// with the reference's cubic spline Kernel() (derivatives.c:44-66) and the
// algebraic Tait pressure (derivatives.c:1674-1682) evaluated before the pass.
// Monaghan's viscosity (Monaghan 1992, Annu. Rev. Astron. Astrophys. 30:543,
// beta = 0) has no counterpart in the reference.  Wall forces are the
// reference's (derivatives.c:2396-2449 and the other selectBoundaryForce
// modes), in FP64.
//
// Real = double: everything in FP64.  Real = float: the pair arithmetic and
// the per-particle sums run in FP32 on the staged records' FP32 operands --
// positions relative to the CTA's block origin (so small separations keep
// their precision), velocities, m, p / rho^2 and rho, each rounded once from
// FP64 when the record is staged; the pair test itself stays the exact FP64
// predicate so both precisions see the same pairs.
//
// Execution as in the REF pass: a cheap listing phase (distance test only)
// per thread into shared memory, then the pair arithmetic over the lists.
#include "leapfrog.cuh"
#include "tile_pass.cuh"

namespace uph {

// selectBoundaryForce modes that act on listed pairs (i side = this fluid particle)
__device__ __forceinline__ void wcsph_wall_pair(const DevParams &P, int itb, double r2d, double dxd, double dyd,
                                                double dud, double dvd, double ma, double &wx, double &wy)
{
  const double rr = sqrt(r2d);
  if (P.boundary_force == 3 && (itb == 2 || itb == 3 || itb == 5)) {
    const double r0 = 3.0 * P.dx;
    if (rr < r0) {
      const double rv = dxd * dud + dyd * dvd;
      const double c1 = P.k_spring * (r0 - rr) / (rr * ma);
      const double c2 = P.c_damp * rv / (rr * rr * ma);
      wx -= c1 * dxd + c2 * dxd;
      wy -= c1 * dyd + c2 * dyd;
    }
  } else if (P.boundary_force == 4 && (itb == 2 || itb == 3) && rr < P.dx) {
    const double norm = 7.0 / (64.0 * 3.142 * P.h * P.h);
    const double qq = rr / P.h;
    double phi = 0.0;
    if (qq < 2.0) {
      const double t = 2.0 - qq;
      phi = norm * (1.0 + 2.0 * qq) * (t * t) * (t * t);
    }
    const double c = P.mach_c * P.mach_c / 5.0 * phi / ((rr - P.dx / 5.0) * rr);
    wx += c * dxd;
    wy += c * dyd;
  } else if (P.boundary_force == 5 && itb == 2 && rr < P.dx) {
    wx -= (P.k_spring * dxd + P.c_damp * dud) / ma;
    wy -= (P.k_spring * dyd + P.c_damp * dvd) / ma;
  }
}

// One staged particle.  FP64 position, velocity and mass always (the exact
// pair test and the FP64 wall forces need them); the pair arithmetic's
// operands in Real: for FP32, the position relative to the CTA's block
// origin and the velocity, and m, p / rho^2 and rho rounded once from FP64,
// so the pair loop runs in FP32 without a per-pair FP64 difference.
template <typename Real>
struct WcRec;
template <>
struct __align__(16) WcRec<double> {
  double x, y, u, v, m, A1, rho;
  int orig, itype;
};
template <>
struct __align__(16) WcRec<float> {
  double x, y, u, v, m;
  float xr, yr, ur, vr, mr, A1, rho;
  int orig, itype;
};
static_assert(sizeof(WcRec<double>) == 64 && sizeof(WcRec<float>) == 80, "record sizes");

// (ox, oy): the origin FP32 positions are taken relative to
template <typename Real>
__device__ __forceinline__ WcRec<Real> load_wc_rec(const SlotArrays &S, int s, double ox, double oy)
{
  WcRec<Real> r;
  r.x = S.x[s];
  r.y = S.y[s];
  r.u = S.u[s];
  r.v = S.v[s];
  r.m = S.m[s];
  const double ir = S.inv_rho[s];
  r.A1 = (Real)(S.p[s] * ir * ir);
  r.rho = (Real)S.rho[s];
  if constexpr (sizeof(Real) == sizeof(float)) {
    r.xr = (float)(r.x - ox);
    r.yr = (float)(r.y - oy);
    r.ur = (float)r.u;
    r.vr = (float)r.v;
    r.mr = (float)r.m;
  }
  r.orig = S.orig[s];
  r.itype = S.itype[s];
  return r;
}

template <typename Real>
struct WcStagedSrc {
  const WcRec<Real> *rec;
  const float2 *posf;  // block-relative FP32 positions for the listing
  __device__ __forceinline__ double2 xy(int k) const { return *reinterpret_cast<const double2 *>(&rec[k].x); }
  __device__ __forceinline__ float2 xyf(int k) const { return posf[k]; }
  __device__ __forceinline__ int orig(int k) const { return rec[k].orig; }
  __device__ __forceinline__ double mass(int k) const { return rec[k].m; }
  __device__ __forceinline__ WcRec<Real> get(int k) const { return rec[k]; }
};
template <typename Real>
struct WcGlobalSrc {
  SlotArrays S;
  double ox, oy;
  __device__ __forceinline__ double2 xy(int s) const { return make_double2(S.x[s], S.y[s]); }
  __device__ __forceinline__ float2 xyf(int) const { return make_float2(0.f, 0.f); }  // not used: no pre-test
  __device__ __forceinline__ int orig(int s) const { return S.orig[s]; }
  __device__ __forceinline__ double mass(int s) const { return S.m[s]; }
  __device__ __forceinline__ WcRec<Real> get(int s) const { return load_wc_rec<Real>(S, s, ox, oy); }
};

struct WcAcc {
  double wx, wy;  // wall forces, FP64 like the reference
};

// the sums of one pair (a, b), a = the own particle
template <typename Real>
__device__ __forceinline__ void wc_pair(const DevParams &P, const WcRec<Real> &a, const WcRec<Real> &b, bool isI,
                                        Real &drho, Real &ax, Real &ay, WcAcc &W)
{
  const Real h = (Real)P.h, inv_h = (Real)P.inv_h, inv_h2 = (Real)P.inv_h2;
  const Real sigma = (Real)P.cs_alpha;
  const Real eta2 = (Real)P.eta2, ac = (Real)P.av_alpha_c0;
  Real dx, dy, du, dv, mb, r, inv_r;
  if constexpr (sizeof(Real) == sizeof(float)) {
    // FP32 throughout: block-relative positions, approximate square root
    // and reciprocals (MUFU), errors far below the FP32 sums'
    dx = a.xr - b.xr;
    dy = a.yr - b.yr;
    du = a.ur - b.ur;
    dv = a.vr - b.vr;
    mb = b.mr;
  } else {
    dx = a.x - b.x;
    dy = a.y - b.y;
    du = a.u - b.u;
    dv = a.v - b.v;
    mb = b.m;
  }
  const Real r2 = dx * dx + dy * dy;
  if constexpr (sizeof(Real) == sizeof(float)) {
    inv_r = r2 > 0.0f ? rsqrtf(r2) : 0.0f;
    r = r2 * inv_r;
  } else {
    r = sqrt(r2);
  }
  const Real q = r * inv_h;
  Real F;
  if (q < (Real)1) {
    F = sigma * ((Real)-3 + (Real)2.25 * q) * inv_h2;
  } else {
    const Real t = (Real)2 - q;
    if constexpr (sizeof(Real) == sizeof(float))
      F = -sigma * 0.75f * t * t * inv_h * inv_r;
    else
      F = -sigma * 0.75 * t * t * inv_h * rcp_nr(r);
  }
  const Real gx = F * dx, gy = F * dy;
  drho += mb * (du * gx + dv * gy);
  const Real vr = du * dx + dv * dy;
  Real pi_ab = 0;
  if (vr < (Real)0) {
    if constexpr (sizeof(Real) == sizeof(float)) {
      const float mu = h * vr * __fdividef(1.0f, r2 + eta2);
      pi_ab = -ac * mu * __fdividef(2.0f, a.rho + b.rho);
    } else {
      const double mu = h * vr * rcp_nr(r2 + eta2);
      pi_ab = -ac * mu * rcp_nr(0.5 * (a.rho + b.rho));
    }
  }
  const Real pij = a.A1 + b.A1 + pi_ab;
  ax -= mb * pij * gx;
  ay -= mb * pij * gy;
  if (isI && a.itype == 1 && b.itype >= 2) {
    const double dxd = a.x - b.x, dyd = a.y - b.y;
    wcsph_wall_pair(P, b.itype, exact_r2(dxd, dyd), dxd, dyd, a.u - b.u, a.v - b.v, a.m, W.wx, W.wy);
  }
}

// nshort, vl_out, vl_cnt: the candidate lists, as in the REF pass's
// ref_particle
template <bool kBrute, bool kF32, typename Real, typename Src, typename Cursor, typename Entry>
__device__ __forceinline__ void wc_particle(const DevParams &P, const Src &src, Cursor &cur, bool active, int self,
                                            const WcRec<Real> &o, const F32Test &ft, Entry *s_nb, Real &drho,
                                            Real &ax, Real &ay, WcAcc &W, unsigned &my_pairs, int &my_nb, int nshort,
                                            unsigned short *vl_out, int &vl_cnt)
{
  constexpr Entry kRole = sizeof(Entry) == 2 ? (Entry)kRoleI16 : (Entry)kRoleI;
  const int col = threadIdx.x;
  bool more = active;
  while (__any_sync(0xffffffffu, more)) {
    int cnt = 0;
    if (kF32 && nshort >= 0) {
      if constexpr (kF32) {
        if (more)
          cnt = tile_list_short<kBrute, false>(P, src, nshort, self, o.orig, o.x, o.y, ft, s_nb, col, my_pairs, my_nb,
                                               W.wx, W.wy, 0.0, 0);
      }
      more = false;
    } else {
      cnt = tile_list<kBrute, kTileChunk, false, kF32>(P, src, cur, more, self, o.orig, o.x, o.y, ft, s_nb, col,
                                                       my_pairs, my_nb, W.wx, W.wy, 0.0, 0, vl_out, vl_cnt);
    }
    __syncwarp();
    for (int e = 0; e < cnt; e++) {
      const Entry ent = s_nb[e * kTileThreads + col];
      const WcRec<Real> b = src.get((int)(ent & (Entry)~kRole));
      wc_pair<Real>(P, o, b, (ent & kRole) != 0, drho, ax, ay, W);
    }
    __syncwarp();
  }
}

// dv/dt with the wall forces, gravity and the sponge layer
template <typename Real>
__device__ __forceinline__ void wc_accel(const DevParams &P, const SlotArrays &S, int a, const WcRec<Real> &o, Real ax,
                                         Real ay, const WcAcc &W, double &axd, double &ayd)
{
  axd = (double)ax + W.wx;
  ayd = (double)ay + W.wy;
  if (P.gravity_flag == 1) ayd -= P.g;
  if (P.moving_boundary == 1 && P.wave_absorption == 1) axd -= S.sponge[a] * o.u;
}

template <typename Real>
__device__ __forceinline__ void wc_epilogue(const DevParams &P, const SlotArrays &S, int a, const WcRec<Real> &o,
                                            Real drho, Real ax, Real ay, const WcAcc &W)
{
  double axd, ayd;
  wc_accel(P, S, a, o, ax, ay, W, axd, ayd);
  S.drho[a] = (double)drho;
  S.dp[a] = 0.0;
  S.ax[a] = axd;
  S.ay[a] = ayd;
  S.drho_a[a] = (double)drho;
  S.dp_a[a] = 0.0;
  S.ax_a[a] = axd;
  S.ay_a[a] = ayd;
  S.frho[a] = 0.0;
  S.fp[a] = 0.0;
  S.fu[a] = 0.0;
  S.fv[a] = 0.0;
}

// The epilogue of a pass that applies the step (StepOut), as the stand-alone
// corrector does it for WCSPH (integrate.cu): the corrector with the rates
// just summed (no predictor rates or fluctuations of their own: the same
// rates, zeros), the Tait pressure of the corrected density, the drift and,
// with predict_next, the next step's predictor, written to slot a of the
// other buffer.  Rates and the algebraic pressure are stored only by the
// last step of a call, and the particle's constants not at all (see the REF
// pass's ref_step_epilogue).
template <typename Real>
__device__ __forceinline__ void wc_step_epilogue(const DevParams &P, const SlotArrays &S, const StepOut &F, int a,
                                                 const WcRec<Real> &o, Real drho, Real ax, Real ay, const WcAcc &W)
{
  const SlotArrays &D = F.D;
  double axd, ayd;
  wc_accel(P, S, a, o, ax, ay, W, axd, ayd);
  const double drhod = (double)drho;
  if (!F.predict_next) {
    D.drho[a] = drhod;
    D.dp[a] = 0.0;
    D.ax[a] = axd;
    D.ay[a] = ayd;
    D.drho_a[a] = drhod;
    D.dp_a[a] = 0.0;
    D.ax_a[a] = axd;
    D.ay_a[a] = ayd;
    D.frho[a] = 0.0;
    D.fp[a] = 0.0;
    D.fu[a] = 0.0;
    D.fv[a] = 0.0;
  }
  const LeapRates R = {drhod, 0.0, axd, ayd, 0.0, 0.0, 0.0, 0.0};
  double rmin = 0.0, pmin = 0.0, umin = 0.0, vmin = 0.0;
  if (!F.first_step || !F.predict_next) {
    rmin = S.rho_min[a];
    pmin = S.p_min[a];
    umin = S.u_min[a];
    vmin = S.v_min[a];
  }
  const LeapState c = F.first_step ? leap_correct(P.dt, P.eps, true, S.rho[a], S.p[a], o.u, o.v, R)
                                   : leap_correct(P.dt, P.eps, false, rmin, pmin, umin, vmin, R);
  const double p = tait(P, c.rho);
  const double x = leap_drift(P.dt, o.x, c.u), y = leap_drift(P.dt, o.y, c.v);
  D.x[a] = x;
  D.y[a] = y;
  if (!isfinite(c.rho) || !isfinite(p) || !isfinite(x) || !isfinite(y) || !isfinite(c.u) || !isfinite(c.v))
    atomicOr(F.err, ERR_NAN);
  note_moved(P, a, x, y, F.err);
  if (F.predict_next) {
    const LeapPred q = leap_predict(P.dt, P.eps, c.rho, p, c.u, c.v, drhod, 0.0, axd, ayd, 0.0, 0.0, 0.0, 0.0);
    D.rho_min[a] = c.rho;
    D.p_min[a] = p;
    D.u_min[a] = c.u;
    D.v_min[a] = c.v;
    D.u[a] = q.u;
    D.v[a] = q.v;
    D.ut[a] = q.ut;
    D.vt[a] = q.vt;
    D.pt[a] = q.pt;
    D.rho[a] = q.rho;
    D.rhot[a] = q.rt;
    D.p[a] = tait(P, q.rho);
    D.inv_rho[a] = q.ir;
    D.inv_rhot[a] = q.irt;
  } else {
    D.rho_min[a] = rmin;
    D.p_min[a] = pmin;
    D.u_min[a] = umin;
    D.v_min[a] = vmin;
    D.u[a] = c.u;
    D.v[a] = c.v;
    D.ut[a] = c.ut;
    D.vt[a] = c.vt;
    D.pt[a] = c.pt;
    D.rho[a] = c.rho;
    D.rhot[a] = c.rt;
    D.p[a] = p;
    D.pressure[a] = p;
    D.inv_rho[a] = __ddiv_rn(1.0, c.rho);
    D.inv_rhot[a] = __ddiv_rn(1.0, c.rt);
  }
}

constexpr int kWcRecCap = 640;
constexpr size_t kWcListBytes = sizeof(unsigned short) * kTileChunk * kTileThreads;
template <typename Real>
constexpr size_t wc_smem()
{
  return sizeof(TileBlock) + kWcListBytes + (sizeof(WcRec<Real>) + sizeof(float2)) * kWcRecCap;
}
static_assert(sizeof(WcRec<float>) * kWcRecCap >= sizeof(unsigned) * kTileChunk * kTileThreads,
              "the fallback's 32-bit lists live in the record area");

// One tile of the WCSPH pass, as the REF pass's (tile_pass.cuh).
template <bool kBrute, typename Real>
__device__ __forceinline__ void wc_tile(const DevParams &P, const SlotArrays &S, const CellGrid &G, const StepOut &F,
                                        int tile, unsigned char *smem, unsigned &my_pairs, int &my_nb)
{
  TileBlock &B = *reinterpret_cast<TileBlock *>(smem);
  unsigned short *s_nb16 = reinterpret_cast<unsigned short *>(smem + sizeof(TileBlock));
  WcRec<Real> *rec = reinterpret_cast<WcRec<Real> *>(smem + sizeof(TileBlock) + kWcListBytes);
  float2 *s_posf = reinterpret_cast<float2 *>(rec + kWcRecCap);
  tile_setup(P, G, tile, B);
  const int ncore = B.ncore;
  if (ncore == 0) return;
  const bool staged = B.nrec <= kWcRecCap;
  // the origin of the block: FP32 positions are taken relative to it
  const double ox = P.lo_x + B.bx0 * P.cell, oy = P.lo_y + B.by0 * P.cell;
  if (staged) {
    // this tile's candidate lists are current if written since the last
    // build (G.vl null: the lists are off, every particle walks the stencil)
    const unsigned gen = G.vl ? *G.gen : 0u;
    const bool vl_use = G.vl && G.tile_gen[tile] == gen;
    // two records per thread at a time, every load issued before the first
    // store (two rounds of loads: the slots, then their fields)
    for (int k0 = threadIdx.x; k0 < B.nrec; k0 += 2 * kTileThreads) {
      const int k1 = k0 + kTileThreads;
      const bool two = k1 < B.nrec;
      const int s0 = G.list[tile_record_pos(B, k0)];
      const int s1 = two ? G.list[tile_record_pos(B, k1)] : s0;
      // the candidate lists the core's fluid particles will read after the
      // staging: fetched into L2 meanwhile (the halo's too, for their tiles)
      if (vl_use) {
        if (s0 < P.nf) {
          prefetch_l2(G.vl + (size_t)s0 * kVlMax);
          prefetch_l2(G.vl_n + s0);
        }
        if (two && s1 < P.nf) {
          prefetch_l2(G.vl + (size_t)s1 * kVlMax);
          prefetch_l2(G.vl_n + s1);
        }
      }
      const WcRec<Real> r0 = load_wc_rec<Real>(S, s0, ox, oy);
      const WcRec<Real> r1 = load_wc_rec<Real>(S, s1, ox, oy);
      rec[k0] = r0;
      s_posf[k0] = make_float2((float)(r0.x - ox), (float)(r0.y - oy));
      if (two) {
        rec[k1] = r1;
        s_posf[k1] = make_float2((float)(r1.x - ox), (float)(r1.y - oy));
      }
    }
    __syncthreads();
    const WcStagedSrc<Real> src{rec, s_posf};
    for (int base = 0; base < ncore; base += kTileThreads) {
      const int k = base + threadIdx.x;
      int kr = 0, pos = 0, a = 0, cx = B.bx0, cy = B.by0;
      if (k < ncore) {
        tile_core_cell(B, k, kr, pos, cx, cy);
        a = G.list[pos];
      }
      const bool active = k < ncore && a < P.nf;
      // the epilogue's reads of the particle's own *_min state: fetched into
      // L2 now, while the pair loop runs
      if (F.enabled && active && (!F.first_step || !F.predict_next)) {
        prefetch_l2(S.rho_min + a);
        prefetch_l2(S.p_min + a);
        prefetch_l2(S.u_min + a);
        prefetch_l2(S.v_min + a);
      }
      const WcRec<Real> o = rec[active ? kr : 0];
      StagedCursor cur;
      cur.c.init(B, P.reach, active ? cx : B.bx0, active ? cy : B.by0);
      const float2 of = s_posf[active ? kr : 0];
      const F32Test ft = make_f32_test(P, B, of.x, of.y);
      Real drho = 0, ax = 0, ay = 0;
      WcAcc W = {0.0, 0.0};
      int nb = 0;
      int nshort = -1, vl_cnt = 0;
      unsigned short *vl_out = nullptr;
      if (active && G.vl) nshort = load_candidates(G, a, vl_use, s_nb16, threadIdx.x, vl_out);
      wc_particle<kBrute, true, Real>(P, src, cur, active, kr, o, ft, s_nb16, drho, ax, ay, W, my_pairs, nb, nshort,
                                      vl_out, vl_cnt);
      if (vl_out) G.vl_n[a] = vl_cnt <= kVlMax ? (unsigned char)vl_cnt : kVlOverflow;
      my_nb = max(my_nb, nb);
      if (active) {
        if (F.enabled)
          wc_step_epilogue<Real>(P, S, F, a, o, drho, ax, ay, W);
        else
          wc_epilogue<Real>(P, S, a, o, drho, ax, ay, W);
      }
    }
    if (G.vl && !vl_use && threadIdx.x == 0) G.tile_gen[tile] = gen;
  } else {
    unsigned *s_nb32 = reinterpret_cast<unsigned *>(rec);
    const WcGlobalSrc<Real> src{S, ox, oy};
    for (int base = 0; base < ncore; base += kTileThreads) {
      const int k = base + threadIdx.x;
      int kr = 0, pos = 0, a = 0;
      if (k < ncore) {
        tile_core(B, k, kr, pos);
        a = G.list[pos];
      }
      const bool active = k < ncore && a < P.nf;
      const int as = active ? a : 0;
      const WcRec<Real> o = load_wc_rec<Real>(S, as, ox, oy);
      GlobalCursor cur;
      cur.list = G.list;
      cur.c.init(P, G, G.cell_of[as]);
      const F32Test ft = {};
      Real drho = 0, ax = 0, ay = 0;
      WcAcc W = {0.0, 0.0};
      int nb = 0;
      int vl_none = 0;
      wc_particle<kBrute, false, Real>(P, src, cur, active, as, o, ft, s_nb32, drho, ax, ay, W, my_pairs, nb, -1,
                                       nullptr, vl_none);
      my_nb = max(my_nb, nb);
      if (active) {
        if (F.enabled)
          wc_step_epilogue<Real>(P, S, F, a, o, drho, ax, ay, W);
        else
          wc_epilogue<Real>(P, S, a, o, drho, ax, ay, W);
      }
    }
  }
}

// The WCSPH rate pass: one CTA per storage tile (tile_pass.cuh).
// With F.enabled the pass also applies the step (StepOut), wall motion first
// as in the REF pass.
template <bool kBrute, typename Real>
__global__ void __launch_bounds__(kTileThreads, 3) k_wcsph_pass(const DevParams P, const SlotArrays S, const CellGrid G,
                                                             PassStats st, const StepOut F)
{
  extern __shared__ __align__(16) unsigned char smem[];
  if (F.enabled && F.walls) {
    const double t = (*F.d_itime + (F.walls == 2 ? 1 : 0)) * P.dt;
    for (int w = P.nf + blockIdx.x * kTileThreads + threadIdx.x; w < P.n; w += gridDim.x * kTileThreads)
      wall_move_one(P, F.D, F.W, w, t, F.err);
  }
  unsigned my_pairs = 0;
  int my_nb = 0;  // largest in-radius count of this thread's particles
  wc_tile<kBrute, Real>(P, S, G, F, blockIdx.x, smem, my_pairs, my_nb);
  pass_stats(st, my_pairs, my_nb);
}

template <bool kBrute, typename Real>
uph_status launch_wc(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st, const StepOut &F,
                     cudaStream_t s)
{
  static bool attr_set[64] = {};  // once per device
  int dev = 0;
  UPH_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    UPH_CUDA(cudaFuncSetAttribute(k_wcsph_pass<kBrute, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)wc_smem<Real>()));
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  const int ntiles = P.ntx * (P.ncy / P.tile);
  k_wcsph_pass<kBrute, Real><<<ntiles, kTileThreads, wc_smem<Real>(), s>>>(P, S, G, st, F);
  return UPH_OK;
}

uph_status launch_wcsph_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st,
                             const StepOut &F, cudaStream_t s)
{
  if (P.nf <= 0) return UPH_OK;
  const bool brute = P.boundary_force != 3 && P.boundary_force != 4 && P.boundary_force != 5;
  if (P.precision == UPH_PREC_FP32_PAIR)
    return brute ? launch_wc<true, float>(P, S, G, st, F, s) : launch_wc<false, float>(P, S, G, st, F, s);
  return brute ? launch_wc<true, double>(P, S, G, st, F, s) : launch_wc<false, double>(P, S, G, st, F, s);
}

}  // namespace uph
