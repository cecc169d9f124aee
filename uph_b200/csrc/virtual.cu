// Virtual mirror particles of the reference's derivatives()
// (derivatives.c:3194-4192, virtualType 1, 3, 4, 5, 7, 8).
//
// Every call the reference copies the fluid particles within 2h of each of
// the virtualType's wall lines (3h of the slope of type 1) to their mirror
// images, loop after loop, appending them after the boundary particles
// (reference indices from Nf + Ns + Nb on, itype 4).  The pair filter keeps
// j < Nf + Ns + Nb - 1 (derivatives.c:1081-1083), so a virtual particle is
// never in a pair: it is a point of the 40-nearest search, where it can take
// one of a query's 40 places, and a row of the System (and of out<k>.dat).
//
// Here the copies are generated on the device in the reference's order: one
// flag per (rule, reference fluid index), an exclusive scan over the flags
// in that order, then each flagged copy written at its scanned index.  The
// positions are computed with the reference's expressions in its operation
// order, without multiply-add contraction (this file is compiled with
// --fmad=false), so they are bit-identical to the reference's.
#include "uph_internal.cuh"

namespace uph {

namespace {

// LeftBoundaryPosition of inputbp at time t: the piston law for
// movingBoundary 1 and for the sloshing walls (inputbp.c:196, 246), else 0
// (inputbp.c:280).  RightBoundaryPosition: FlatBottomLength + left
// (inputbp.c:248), set only with the sloshing walls.
__device__ __forceinline__ double left_position(const DevParams &P, double t)
{
  return P.vleft_moves ? 0.5 * P.stroke * (1.0 - cos(P.omega * t)) : 0.0;
}

__device__ __forceinline__ double rule_line(const DevParams &P, const VirtualRule &r, double left)
{
  if (r.pos == VP_LEFT) return left;
  if (r.pos == VP_RIGHT) return P.flat_bottom_length + left;
  return r.a;
}

// Whether fluid particle (x, y) has a copy under rule r, and where.
__device__ __forceinline__ bool mirror(const DevParams &P, const VirtualRule &r, double left, double x, double y,
                                       double &xv, double &yv)
{
  const double h2 = 2.0 * P.h;
  switch (r.kind) {
    case VK_LEFT:
    case VK_RIGHT: {
      const double X = rule_line(P, r, left);
      const double d = fabs(x - X);
      if (!(d < h2)) return false;
      xv = r.kind == VK_LEFT ? X - d : X + d;
      yv = y;
      return true;
    }
    case VK_BOTTOM:
      if (!((y < h2) && (x <= r.a))) return false;
      xv = x;
      yv = -y;
      return true;
    case VK_TOP: {
      const double d = fabs(y - r.a - r.b);
      if (!(d < h2)) return false;
      xv = x;
      yv = r.a + 2 * d;
      return true;
    }
    case VK_CORNER_L:
    case VK_CORNER_R: {
      const double X = rule_line(P, r, left);
      const double d = fabs(x - X);
      const double dy = y;
      if (!((d < h2) && (dy < h2))) return false;
      xv = r.kind == VK_CORNER_L ? X - d : X + d;
      yv = -y;
      return true;
    }
    case VK_SLOPE: {
      const double s = r.b;
      const double denoms = 1 + s * s;
      const double nums = 1 - s * s;
      const double yi = s * r.a;
      const double d = (1.0 / sqrt(denoms)) * fabs(s * x - y - yi);
      if (!((d < 3.0 * P.h) && (x > r.a))) return false;
      xv = (nums * x + 2.0 * s * y + 2.0 * s * yi) / denoms;
      yv = (2.0 * s * x - nums * y - 2.0 * yi) / denoms;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ double eval_time(const DevParams &P, double t_host, const int *d_itime)
{
  return d_itime ? *d_itime * P.dt : t_host;
}

__global__ void k_virtual_flags(const DevParams P, const SlotArrays S, VirtualBuf V, double t_host,
                                const int *d_itime)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double left = left_position(P, eval_time(P, t_host, d_itime));
  const double x = S.x[a], y = S.y[a];
  const int o = S.orig[a];
  for (int r = 0; r < P.nvrules; r++) {
    double xv, yv;
    V.flags[r * P.nf + o] = mirror(P, P.vrule[r], left, x, y, xv, yv) ? 1 : 0;
  }
}

__global__ void k_virtual_emit(const DevParams P, const SlotArrays S, VirtualBuf V, double t_host,
                               const int *d_itime)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double left = left_position(P, eval_time(P, t_host, d_itime));
  const double x = S.x[a], y = S.y[a];
  const int o = S.orig[a];
  for (int r = 0; r < P.nvrules; r++) {
    const int f = r * P.nf + o;
    if (f == V.cap - 1) *V.count = V.offs[f] + V.flags[f];
    if (!V.flags[f]) continue;
    double xv = 0.0, yv = 0.0;
    mirror(P, P.vrule[r], left, x, y, xv, yv);
    const int k = V.offs[f];
    V.x[k] = xv;
    V.y[k] = yv;
    V.src[k] = o;
    V.rule[k] = P.vrule[r].kind;
  }
}

}  // namespace

void launch_virtual(const DevParams &P, const SlotArrays &S, const VirtualBuf &V, double t_host, const int *d_itime,
                    cudaStream_t s)
{
  if (P.nf <= 0 || P.nvrules <= 0) return;
  const int blocks = (P.nf + 255) / 256;
  k_virtual_flags<<<blocks, 256, 0, s>>>(P, S, V, t_host, d_itime);
  launch_exclusive_scan(V.flags, V.offs, V.cap, V.block_sums, s);
  k_virtual_emit<<<blocks, 256, 0, s>>>(P, S, V, t_host, d_itime);
}

}  // namespace uph
