/*
 * Test infrastructure (oracle only).  CPU restatement, in plain C, of the
 * reference's per-timestep hot path, kept in the reference's own form: an
 * explicit pair list (i < j) and one scatter loop per physical term, each
 * adding to i and j exactly as the reference's loops do.  The CUDA library
 * uses a different formulation (owner-computes gather over a cell list), so
 * agreement between the two is a real check.
 *
 * Pinned against the reference compiled from its own sources
 * (oracle/_ref/libuph_ref.so, built by oracle/Makefile) by
 * tests/test_oracle_pin.py and by the committed golden vectors in
 * tests/golden/.
 *
 * Single threaded and FP64 throughout; compiled with -ffp-contract=off so no
 * multiply-add is fused.  Not part of the product.
 */
#include "uph_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct uph_oracle {
  uph_params p;
  int nf, n, pb; /* fluid count, all particles, ParticleBoundary */
  int itime;
  /* state, reference layout */
  double *pos, *vel, *lvel, *rho, *lrho, *pr, *lpr, *mass, *pressure;
  int *itype;
  double *vmin, *rhomin, *prmin, *sponge;
  double *drho, *dp, *acc, *drho_a, *dp_a, *acc_a, *frho, *fp, *fvel;
  /* moving-wall file positions (inputbp.c re-reads them every step) */
  double *wall_x0;
  /* pairs */
  int64_t niac, pcap;
  int32_t *ip, *jp;
  double *rij2, *w, *dw;
  int max_nb;
  double *tmp; /* 2n scratch, the reference's per-thread tmp row */
  double *wall_tab; /* optional shaking table of the moving block: x0, hs, om */
};

static void *xcalloc(size_t n, size_t s)
{
  void *p = calloc(n ? n : 1, s);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    exit(1);
  }
  return p;
}

uph_oracle *uph_oracle_create(const uph_params *p)
{
  uph_oracle *o = (uph_oracle *)xcalloc(1, sizeof *o);
  o->p = *p;
  o->nf = p->n_fluid;
  o->n = p->n_fluid + p->n_solid + p->n_fixed + p->n_moving;
  o->pb = o->n - 1; /* Nf + Ns + Nb - 1, derivatives.c:1082-1084 */
  const size_t n = (size_t)o->n, nf = (size_t)o->nf;
  o->pos = xcalloc(2 * n, 8); o->vel = xcalloc(2 * n, 8); o->lvel = xcalloc(2 * n, 8);
  o->rho = xcalloc(n, 8); o->lrho = xcalloc(n, 8); o->pr = xcalloc(n, 8); o->lpr = xcalloc(n, 8);
  o->mass = xcalloc(n, 8); o->pressure = xcalloc(n, 8); o->itype = xcalloc(n, 4);
  o->vmin = xcalloc(2 * nf, 8); o->rhomin = xcalloc(nf, 8); o->prmin = xcalloc(nf, 8); o->sponge = xcalloc(nf, 8);
  o->drho = xcalloc(nf, 8); o->dp = xcalloc(nf, 8); o->acc = xcalloc(2 * nf, 8);
  o->drho_a = xcalloc(nf, 8); o->dp_a = xcalloc(nf, 8); o->acc_a = xcalloc(2 * nf, 8);
  o->frho = xcalloc(nf, 8); o->fp = xcalloc(nf, 8); o->fvel = xcalloc(2 * nf, 8);
  o->wall_x0 = xcalloc(n, 8);
  o->tmp = xcalloc(2 * n, 8);
  o->pcap = 16 * (int64_t)n + 1024;
  o->ip = xcalloc((size_t)o->pcap, 4); o->jp = xcalloc((size_t)o->pcap, 4);
  o->rij2 = xcalloc((size_t)o->pcap, 8); o->w = xcalloc((size_t)o->pcap, 8); o->dw = xcalloc(2 * (size_t)o->pcap, 8);
  return o;
}

void uph_oracle_destroy(uph_oracle *o)
{
  if (!o) return;
  void *ptrs[] = {o->pos, o->vel, o->lvel, o->rho, o->lrho, o->pr, o->lpr, o->mass, o->pressure, o->itype,
                  o->vmin, o->rhomin, o->prmin, o->sponge, o->drho, o->dp, o->acc, o->drho_a, o->dp_a, o->acc_a,
                  o->frho, o->fp, o->fvel, o->wall_x0, o->tmp, o->ip, o->jp, o->rij2, o->w, o->dw, o->wall_tab};
  for (size_t k = 0; k < sizeof ptrs / sizeof ptrs[0]; k++) free(ptrs[k]);
  free(o);
}

#define CP_IN(dst, src, cnt)                                   \
  do {                                                         \
    if (src) memcpy((dst), (src), sizeof(*(dst)) * (size_t)(cnt)); \
  } while (0)
#define CP_OUT(dst, src, cnt)                                  \
  do {                                                         \
    if (dst) memcpy((dst), (src), sizeof(*(src)) * (size_t)(cnt)); \
  } while (0)

int uph_oracle_set_state(uph_oracle *o, const uph_state *s, int itime)
{
  const int n = o->n, nf = o->nf;
  CP_IN(o->pos, s->Position, 2 * n); CP_IN(o->vel, s->Velocity, 2 * n); CP_IN(o->lvel, s->localVelocity, 2 * n);
  CP_IN(o->rho, s->density, n); CP_IN(o->lrho, s->localDensity, n); CP_IN(o->pr, s->DynamicPressure, n);
  CP_IN(o->lpr, s->localPressure, n); CP_IN(o->mass, s->mass, n); CP_IN(o->itype, s->itype, n);
  CP_IN(o->vmin, s->Velocity_min, 2 * nf); CP_IN(o->rhomin, s->density_min, nf);
  CP_IN(o->prmin, s->DynamicPressure_min, nf);
  if (s->spongeFactor) memcpy(o->sponge, s->spongeFactor, 8 * (size_t)nf); else memset(o->sponge, 0, 8 * (size_t)nf);
  CP_IN(o->drho, s->ddensitydt, nf); CP_IN(o->dp, s->dpdt, nf); CP_IN(o->acc, s->dvdt, 2 * nf);
  CP_IN(o->drho_a, s->ddensitydt_approx, nf); CP_IN(o->dp_a, s->dpdt_approx, nf);
  CP_IN(o->acc_a, s->dvdt_approx, 2 * nf);
  CP_IN(o->frho, s->densityFluctuation, nf); CP_IN(o->fp, s->pressureFluctuation, nf);
  CP_IN(o->fvel, s->velocityFluctuation, 2 * nf); CP_IN(o->pressure, s->Pressure, n);
  for (int k = 0; k < n; k++) o->wall_x0[k] = o->pos[2 * k];
  o->itime = itime;
  return 0;
}

int uph_oracle_get_state(const uph_oracle *o, uph_state *s)
{
  const int n = o->n, nf = o->nf;
  CP_OUT(s->Position, o->pos, 2 * n); CP_OUT(s->Velocity, o->vel, 2 * n); CP_OUT(s->localVelocity, o->lvel, 2 * n);
  CP_OUT(s->density, o->rho, n); CP_OUT(s->localDensity, o->lrho, n); CP_OUT(s->DynamicPressure, o->pr, n);
  CP_OUT(s->localPressure, o->lpr, n); CP_OUT(s->mass, o->mass, n); CP_OUT(s->itype, o->itype, n);
  CP_OUT(s->Velocity_min, o->vmin, 2 * nf); CP_OUT(s->density_min, o->rhomin, nf);
  CP_OUT(s->DynamicPressure_min, o->prmin, nf); CP_OUT(s->spongeFactor, o->sponge, nf);
  CP_OUT(s->ddensitydt, o->drho, nf); CP_OUT(s->dpdt, o->dp, nf); CP_OUT(s->dvdt, o->acc, 2 * nf);
  CP_OUT(s->ddensitydt_approx, o->drho_a, nf); CP_OUT(s->dpdt_approx, o->dp_a, nf);
  CP_OUT(s->dvdt_approx, o->acc_a, 2 * nf);
  CP_OUT(s->densityFluctuation, o->frho, nf); CP_OUT(s->pressureFluctuation, o->fp, nf);
  CP_OUT(s->velocityFluctuation, o->fvel, 2 * nf); CP_OUT(s->Pressure, o->pressure, n);
  return 0;
}

/* ---------------------------------------------------------------- search -- */

/* Radius search with SearchNeighbors' filter (Search.cc:31-40): (s, j) with
 * s < n_fluid, j > s, DBL_EPSILON < d2 < dist (libnabo excludes self matches
 * by default), j < particle_boundary; ordered by s then j.  d2 is
 * dx*dx + dy*dy with dx = x_s - x_j. */
int64_t uph_oracle_search(const double *pos, int n_fluid, int n_all, int particle_boundary, double dist, int64_t cap,
                          int32_t *i_pair, int32_t *j_pair, double *rij2, int *max_inradius)
{
  if (n_all <= 0 || n_fluid <= 0 || !(dist > 0)) return 0;
  double xmin = pos[0], xmax = pos[0], ymin = pos[1], ymax = pos[1];
  for (int k = 1; k < n_all; k++) {
    xmin = fmin(xmin, pos[2 * k]); xmax = fmax(xmax, pos[2 * k]);
    ymin = fmin(ymin, pos[2 * k + 1]); ymax = fmax(ymax, pos[2 * k + 1]);
  }
  const double cs = sqrt(dist) * (1.0 + 1e-9);
  const long ncx = (long)((xmax - xmin) / cs) + 1, ncy = (long)((ymax - ymin) / cs) + 1;
  int *cell = xcalloc((size_t)n_all, 4), *start = xcalloc((size_t)(ncx * ncy + 1), 4),
      *order = xcalloc((size_t)n_all, 4), *fill = xcalloc((size_t)(ncx * ncy), 4);
  for (int k = 0; k < n_all; k++) {
    long cx = (long)((pos[2 * k] - xmin) / cs), cy = (long)((pos[2 * k + 1] - ymin) / cs);
    if (cx >= ncx) cx = ncx - 1;
    if (cy >= ncy) cy = ncy - 1;
    cell[k] = (int)(cy * ncx + cx);
    start[cell[k] + 1]++;
  }
  for (long c = 0; c < ncx * ncy; c++) start[c + 1] += start[c];
  memcpy(fill, start, sizeof(int) * (size_t)(ncx * ncy));
  for (int k = 0; k < n_all; k++) order[fill[cell[k]]++] = k;
  int64_t niac = 0;
  int mx = 0;
  int *nb = xcalloc(1024, 4);
  int nbcap = 1024;
  for (int s = 0; s < n_fluid; s++) {
    const long cx = cell[s] % ncx, cy = cell[s] / ncx;
    int cnt = 0, inr = 0;
    for (long by = cy - 1; by <= cy + 1; by++) {
      if (by < 0 || by >= ncy) continue;
      for (long bx = cx - 1; bx <= cx + 1; bx++) {
        if (bx < 0 || bx >= ncx) continue;
        for (int q = start[by * ncx + bx]; q < start[by * ncx + bx + 1]; q++) {
          const int j = order[q];
          const double dx = pos[2 * s] - pos[2 * j], dy = pos[2 * s + 1] - pos[2 * j + 1];
          const double d2 = dx * dx + dy * dy;
          if (d2 <= DBL_EPSILON || !(d2 < dist)) continue;
          inr++;
          if (j > s && j < particle_boundary) {
            if (cnt == nbcap) { nbcap *= 2; nb = realloc(nb, sizeof(int) * (size_t)nbcap); }
            nb[cnt++] = j;
          }
        }
      }
    }
    if (inr > mx) mx = inr;
    /* ascending j */
    for (int a = 1; a < cnt; a++) {
      int v = nb[a], b = a - 1;
      while (b >= 0 && nb[b] > v) { nb[b + 1] = nb[b]; b--; }
      nb[b + 1] = v;
    }
    for (int a = 0; a < cnt; a++) {
      if (niac < cap) {
        const int j = nb[a];
        const double dx = pos[2 * s] - pos[2 * j], dy = pos[2 * s + 1] - pos[2 * j + 1];
        i_pair[niac] = s;
        j_pair[niac] = j;
        rij2[niac] = dx * dx + dy * dy;
      }
      niac++;
    }
  }
  free(nb); free(cell); free(start); free(order); free(fill);
  if (max_inradius) *max_inradius = mx;
  return niac;
}

/* ----------------------------------------------------------- REF kernels -- */

/* PolyOrderSevenConvolutionKernel, derivatives.c:767-784 */
static double ref_w(double r, double h)
{
  const double alpha_d = 2145.0 / (1347584.0 * M_PI * h * h);
  const double q = r / h;
  if (q >= 0.0 && q <= 2.0) {
    const double q2 = q * q, q4 = q2 * q2, q6 = q2 * q4, q8 = q2 * q6, q10 = q2 * q8, q12 = q2 * q10;
    const double t = 1 - 0.25 * q2;
    const double qq = t * t * t * t * t * t * t * t;
    const double pp = (2048 - 3072 * q2 + 2816 * q4 - 1984 * q6 + 1184 * q8 - 628 * q10 + 305 * q12);
    return alpha_d * qq * pp;
  }
  return 0.0;
}

/* PolyOrderSevenDeconvolutionKernel, derivatives.c:786-823.  The two
 * correction coefficients are C integer divisions (-131/329 and
 * 150882/1840097, lines 792-793) and evaluate to 0, so only the alpha_0 term
 * contributes. */
static double ref_dw_factor(double r, double h)
{
  const double alpha_0 = 2145.0 / (192512.0 * M_PI * h * h);
  const double deconvCoeff0 = 1.0;
  const double q = r / h;
  if (q >= 0.0 && q <= 2.0) {
    const double q2 = q * q, q4 = q2 * q2, q6 = q2 * q4, q8 = q2 * q6, q10 = q2 * q8, q12 = q2 * q10;
    const double t = 1 - 0.25 * q2;
    const double qq7 = t * t * t * t * t * t * t;
    const double pp7 = (2048 - 3584 * q2 + 3712 * q4 - 2912 * q6 + 1912 * q8 - 1106 * q10 + 305 * q12);
    return -deconvCoeff0 * alpha_0 * qq7 * pp7; /* "sums"; dwcdx[d] = sums*dx[d]/(h*h) */
  }
  return 0.0;
}

/* Kernel() (cubic spline), derivatives.c:44-66; returns W, writes dW */
static double cubic_w_dw(const double dx[2], double r, double h, double dw[2])
{
  const double alpha = 10.0 / (7. * M_PI * h * h);
  const double q = r / h;
  dw[0] = dw[1] = 0.0;
  if (q >= 0.0 && q < 1.0) {
    const double q2 = q * q, q3 = q * q * q;
    for (int d = 0; d < 2; d++) dw[d] = alpha * (-3 + 2.25 * q) * dx[d] / (h * h);
    return alpha * (1 - 1.5 * q2 + 0.75 * q3);
  } else if (q >= 1.0 && q < 2.0) {
    const double qp2 = (2 - q) * (2 - q), qp3 = qp2 * (2 - q);
    for (int d = 0; d < 2; d++) dw[d] = -alpha * 0.75 * qp2 * dx[d] / (h * r);
    return alpha * 0.25 * qp3;
  }
  return 0.0;
}

/* pairs + kernel values, CalculateKernel derivatives.c:1063-1106 */
static void build_pairs(uph_oracle *o)
{
  const double h0 = o->p.h;
  const double dist = h0 * h0 * 4; /* sys->hsml[0] * sys->hsml[0] * 4, derivatives.c:1086 */
  int mx = 0;
  int64_t niac = uph_oracle_search(o->pos, o->nf, o->n, o->pb, dist, o->pcap, o->ip, o->jp, o->rij2, &mx);
  if (niac > o->pcap) {
    o->pcap = niac + 1024;
    o->ip = realloc(o->ip, 4 * (size_t)o->pcap); o->jp = realloc(o->jp, 4 * (size_t)o->pcap);
    o->rij2 = realloc(o->rij2, 8 * (size_t)o->pcap); o->w = realloc(o->w, 8 * (size_t)o->pcap);
    o->dw = realloc(o->dw, 16 * (size_t)o->pcap);
    niac = uph_oracle_search(o->pos, o->nf, o->n, o->pb, dist, o->pcap, o->ip, o->jp, o->rij2, &mx);
  }
  o->niac = niac;
  o->max_nb = mx;
  for (int64_t k = 0; k < niac; k++) {
    const int i = o->ip[k], j = o->jp[k];
    const double h = 0.5 * (h0 + h0);
    double dx[2];
    for (int d = 0; d < 2; d++) dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
    const double r = sqrt(o->rij2[k]);
    if (o->p.profile == UPH_PROFILE_REF) {
      o->w[k] = ref_w(r, h);
      const double sums = ref_dw_factor(r, h);
      for (int d = 0; d < 2; d++) o->dw[2 * k + d] = sums * dx[d] / (h * h);
    } else {
      o->w[k] = cubic_w_dw(dx, r, h, &o->dw[2 * k]);
    }
  }
}

#define PAIR_LOOP for (int64_t k = 0; k < o->niac; k++)
#define I_ (o->ip[k])
#define J_ (o->jp[k])

static void zero_tmp(uph_oracle *o) { memset(o->tmp, 0, sizeof(double) * 2 * (size_t)o->n); }
static void add_scalar(uph_oracle *o, double *out) { for (int i = 0; i < o->nf; i++) out[i] = o->tmp[i] + out[i]; }
static void add_vector(uph_oracle *o, double *out)
{
  for (int i = 0; i < 2 * o->nf; i++) out[i] = o->tmp[i] + out[i];
}

/* PredictingDensityEquation, derivatives.c:1217-1252 (mass[j] on both sides) */
static void pred_density(uph_oracle *o)
{
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    double dv[2];
    for (int d = 0; d < 2; d++) dv[d] = o->vel[2 * i + d] - o->lvel[2 * j + d];
    for (int d = 0; d < 2; d++) {
      const double vdw = dv[d] * o->dw[2 * k + d];
      o->tmp[i] += o->mass[j] * vdw;
      o->tmp[j] += o->mass[j] * vdw;
    }
  }
  add_scalar(o, o->drho_a);
}

/* PredictingDynamicPressureEquation, derivatives.c:1254-1331 */
static void pred_pressure(uph_oracle *o)
{
  const uph_params *P = &o->p;
  const double c2 = P->density0 * P->speed_of_sound * P->speed_of_sound;
  const double gam = P->adiabatic_constant, kap = P->thermal_diffusivity0;
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    double dx[2], dv[2];
    for (int d = 0; d < 2; d++) {
      dv[d] = o->vel[2 * i + d] - o->vel[2 * j + d];
      dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
    }
    double vdw = 0.0, rdwij = 0.0;
    for (int d = 0; d < 2; d++) {
      vdw += dv[d] * o->dw[2 * k + d];
      rdwij += dx[d] * o->dw[2 * k + d];
    }
    const double pi = (c2 + gam * o->pr[i]), pj = (c2 + gam * o->pr[j]);
    const double volumej = o->mass[j] / o->rho[j];
    const double volumei = o->mass[j] / o->rho[i];
    const double vj = o->mass[j] / o->rho[i], vi = o->mass[i] / o->rho[j];
    o->tmp[i] += vj * pi * vdw;
    o->tmp[j] += vi * pj * vdw;
    const double h = P->h;
    const double eta2 = 0.01 * h * h;
    const double nu = rdwij / (o->rij2[k] + eta2);
    const double epj = 4.0 * pi / (pi + pj), epi = 4.0 * pj / (pi + pj);
    o->tmp[i] += gam * kap * volumej * (o->pr[i] - o->pr[j]) * nu * epj;
    o->tmp[j] += gam * kap * volumei * (o->pr[j] - o->pr[i]) * nu * epi;
    const double rho = (o->rho[i] + o->rho[j]) / (o->rho[i] * o->rho[j]);
    const double rhoi = (o->rho[i] - o->rho[j]) * rho, rhoj = (o->rho[j] - o->rho[i]) * rho;
    o->tmp[i] -= kap * volumej * pi * rhoi * nu;
    o->tmp[j] -= kap * pj * volumei * rhoj * nu;
  }
  add_scalar(o, o->dp_a);
}

/* PredictingPressureGradientForce, derivatives.c:1333-1377 */
static void pred_pgf(uph_oracle *o)
{
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    const double rhoi = 1.0 / (o->rho[i] * o->rho[i]), rhoj = 1.0 / (o->rho[j] * o->rho[j]);
    const double pij = o->pr[i] * rhoi + o->pr[j] * rhoj;
    for (int d = 0; d < 2; d++) {
      o->tmp[2 * i + d] -= o->mass[j] * pij * o->dw[2 * k + d];
      o->tmp[2 * j + d] += o->mass[i] * pij * o->dw[2 * k + d];
    }
  }
  add_vector(o, o->acc_a);
}

/* LocalDensityFluctuation / LocalPressureFluctuation, derivatives.c:2100-2172 */
static void fluct_scalar(uph_oracle *o, const double *f, double *out)
{
  memset(out, 0, sizeof(double) * (size_t)o->nf);
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    const double volumei = o->mass[i] / o->rho[i], volumej = o->mass[j] / o->rho[j];
    const double avgpart = (f[i] - f[j]) * o->w[k];
    o->tmp[i] -= volumej * avgpart;
    o->tmp[j] += volumei * avgpart;
  }
  add_scalar(o, out);
}

/* LocalVelocityFluctuation, derivatives.c:2060-2097 (both terms go to i) */
static void fluct_velocity(uph_oracle *o)
{
  memset(o->fvel, 0, sizeof(double) * 2 * (size_t)o->nf);
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    for (int d = 0; d < 2; d++) {
      const double avgpart = (o->vel[2 * i + d] - o->vel[2 * j + d]) * o->w[k];
      o->tmp[2 * i + d] -= o->mass[j] * avgpart / o->lrho[i];
      o->tmp[2 * i + d] += o->mass[i] * avgpart / o->lrho[j];
    }
  }
  add_vector(o, o->fvel);
}

/* DensityEquation, derivatives.c:1520-1567 */
static void density_eq(uph_oracle *o)
{
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    double dvij[2], dvji[2];
    for (int d = 0; d < 2; d++) {
      dvij[d] = o->vel[2 * i + d] - o->lvel[2 * j + d];
      dvji[d] = o->vel[2 * j + d] - o->lvel[2 * i + d];
    }
    for (int d = 0; d < 2; d++) {
      const double vdwij = dvij[d] * o->dw[2 * k + d], vdwji = dvji[d] * o->dw[2 * k + d];
      const double volumei = o->mass[i] / o->rho[i], volumej = o->mass[j] / o->rho[j];
      const double mj = volumej * o->lrho[j], mi = volumei * o->lrho[i];
      o->tmp[i] += mj * vdwij;
      o->tmp[j] -= mi * vdwji;
    }
  }
  add_scalar(o, o->drho);
}

/* EquationOfState, derivatives.c:1674-1682 (fluid + solid + boundary) */
static void eos(uph_oracle *o)
{
  for (int i = 0; i < o->n; i++) {
    const double density = o->rho[i] / o->p.density0;
    o->pressure[i] = o->p.compression_factor * (pow(density, o->p.adiabatic_constant) - 1.0);
  }
}

/* DynamicPressureEquation, derivatives.c:1569-1672 */
static void dyn_pressure(uph_oracle *o)
{
  const uph_params *P = &o->p;
  const double c2 = P->density0 * P->speed_of_sound * P->speed_of_sound;
  const double gam = P->adiabatic_constant, kap = P->thermal_diffusivity0;
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    double dx[2], dvij[2], dvji[2];
    for (int d = 0; d < 2; d++) {
      dvij[d] = o->vel[2 * i + d] - o->lvel[2 * j + d];
      dvji[d] = o->vel[2 * j + d] - o->lvel[2 * i + d];
      dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
    }
    double vdwij = 0.0, vdwji = 0.0, rdwij = 0.0;
    for (int d = 0; d < 2; d++) {
      vdwij += dvij[d] * o->dw[2 * k + d];
      vdwji += dvji[d] * o->dw[2 * k + d];
      rdwij += dx[d] * o->dw[2 * k + d];
    }
    const double pi = (c2 + gam * o->pr[i]), pj = (c2 + gam * o->pr[j]);
    const double volumei = o->mass[i] / o->rho[i], volumej = o->mass[j] / o->rho[j];
    const double reducedVolumei = volumei * o->lrho[i] / o->rho[j];
    const double reducedVolumej = volumej * o->lrho[j] / o->rho[i];
    o->tmp[i] += reducedVolumej * pi * vdwij;
    o->tmp[j] -= reducedVolumei * pj * vdwji;
    const double h = P->h;
    const double eta2 = 0.01 * h * h;
    const double nu = rdwij / (o->rij2[k] + eta2);
    const double epj = 4.0 * pi / (pi + pj), epi = 4.0 * pj / (pi + pj);
    o->tmp[i] += gam * kap * volumej * (o->pr[i] - o->lpr[j]) * nu * epj;
    o->tmp[j] += gam * kap * volumei * (o->pr[j] - o->lpr[i]) * nu * epi;
    const double rho = (o->rho[i] + o->rho[j]) / (o->rho[i] * o->rho[j]);
    const double rhoi = (o->rho[i] - o->lrho[j]) * rho, rhoj = (o->rho[j] - o->lrho[i]) * rho;
    o->tmp[i] -= kap * volumej * pi * rhoi * nu;
    o->tmp[j] -= kap * pj * volumei * rhoj * nu;
  }
  add_scalar(o, o->dp);
}

/* PressureGradientForce, derivatives.c:1109-1163 */
static void pgf(uph_oracle *o)
{
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    const double rhoi = o->lrho[j] / (o->rho[i] * o->rho[i] * o->rho[j]);
    const double rhoj = o->lrho[i] / (o->rho[j] * o->rho[j] * o->rho[i]);
    const double pij = o->pr[i] * rhoi + o->pr[j] * rhoj;
    for (int d = 0; d < 2; d++) {
      o->tmp[2 * i + d] -= o->mass[j] * pij * o->dw[2 * k + d];
      o->tmp[2 * j + d] += o->mass[i] * pij * o->dw[2 * k + d];
    }
  }
  add_vector(o, o->acc);
}

/* ViscousForcesSingleStep (predicting = 0), derivatives.c:1770-1839, and
 * PredictingViscousForcesSingleStep (predicting = 1), derivatives.c:1448-1515 */
static void viscous(uph_oracle *o, int predicting)
{
  const double mu0 = o->p.viscosity0, h = o->p.h;
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    double dx[2], dvij[2], dvji[2];
    for (int d = 0; d < 2; d++) {
      dvij[d] = o->vel[2 * i + d] - o->vel[2 * j + d];
      dvji[d] = predicting ? dvij[d] : o->vel[2 * j + d] - o->vel[2 * i + d];
      dx[d] = o->pos[2 * j + d] - o->pos[2 * i + d];
    }
    const double eta2 = 0.01 * h * h;
    const double invR2 = 1.0 / (o->rij2[k] + eta2);
    double rhoi, rhoj;
    if (predicting) {
      rhoi = 1.0 / (o->rho[i] * o->rho[i]);
      rhoj = 1.0 / (o->rho[j] * o->rho[j]);
    } else {
      rhoi = o->lrho[j] / (o->rho[i] * o->rho[i] * o->rho[j]);
      rhoj = o->lrho[i] / (o->rho[j] * o->rho[j] * o->rho[i]);
    }
    const double eff = 2.0 * (o->rho[i] * mu0) * (o->rho[j] * mu0) / (o->rho[i] * mu0 + o->rho[j] * mu0);
    const double iS00 = eff * (dx[0] * dvij[0] - dx[1] * dvij[1]) * invR2;
    const double iS01 = eff * (dx[0] * dvij[1] + dx[1] * dvij[0]) * invR2;
    const double iS10 = eff * (dx[1] * dvij[0] + dx[0] * dvij[1]) * invR2;
    const double iS11 = eff * (dx[1] * dvij[1] - dx[0] * dvij[0]) * invR2;
    const double jS00 = eff * (dx[0] * dvji[0] - dx[1] * dvji[1]) * invR2;
    const double jS01 = eff * (dx[0] * dvji[1] + dx[1] * dvji[0]) * invR2;
    const double jS10 = eff * (dx[1] * dvji[0] + dx[0] * dvji[1]) * invR2;
    const double jS11 = eff * (dx[1] * dvji[1] - dx[0] * dvji[0]) * invR2;
    double ax = (iS00 * rhoi + jS00 * rhoj) * o->dw[2 * k];
    ax += (iS01 * rhoi + jS01 * rhoj) * o->dw[2 * k + 1];
    double ay = (iS10 * rhoi + jS10 * rhoj) * o->dw[2 * k];
    ay += (iS11 * rhoi + jS11 * rhoj) * o->dw[2 * k + 1];
    o->tmp[2 * i] += o->mass[j] * ax;
    o->tmp[2 * i + 1] += o->mass[j] * ay;
    o->tmp[2 * j] -= o->mass[i] * ax;
    o->tmp[2 * j + 1] -= o->mass[i] * ay;
  }
  add_vector(o, predicting ? o->acc_a : o->acc);
}

/* BodyForce / PredictingBodyForce, derivatives.c:1167-1178, 1379-1390 */
static void body(uph_oracle *o, double *acc)
{
  if (o->p.gravity_flag == 1)
    for (int i = 0; i < o->nf; i++) {
      acc[2 * i] -= 0.0;
      acc[2 * i + 1] -= o->p.gravity;
    }
}

/* SpongeLayerWaveReflectionAbsorption, derivatives.c:2827-2838 */
static void sponge(uph_oracle *o)
{
  if (o->p.moving_boundary == 1 && o->p.wave_absorption == 1)
    for (int i = 0; i < o->nf; i++) {
      o->acc[2 * i] -= o->sponge[i] * o->vel[2 * i];
      o->acc[2 * i + 1] -= 0.0;
    }
}

static int wall_type_spring(int t) { return t == 2 || t == 3 || t == 5; }

/* SpringBoundaryForces / PredictingSpringBoundaryForces,
 * derivatives.c:2396-2449 and 1392-1446 (identical arithmetic) */
static void spring(uph_oracle *o, double *acc)
{
  const double r0 = 3.0 * o->p.dx;
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    if (o->itype[i] == 1 && wall_type_spring(o->itype[j])) {
      double dx[2], dv[2], rr = 0.0, rvij = 0.0;
      for (int d = 0; d < 2; d++) {
        dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
        dv[d] = o->vel[2 * i + d] - o->vel[2 * j + d];
        rr += dx[d] * dx[d];
        rvij += dx[d] * dv[d];
      }
      rr = sqrt(rr);
      if (rr < r0)
        for (int d = 0; d < 2; d++) {
          o->tmp[2 * i + d] -= o->p.spring_constant0 * (r0 - rr) * dx[d] / (rr * o->mass[i]);
          o->tmp[2 * i + d] -= o->p.damping_constant0 * rvij * dx[d] / (rr * rr * o->mass[i]);
        }
    }
  }
  add_vector(o, acc);
}

/* SerialSpringBoundaryForces, derivatives.c:2452-2479 */
static void serial_spring(uph_oracle *o)
{
  const double r0 = o->p.dx;
  PAIR_LOOP {
    const int i = I_, j = J_;
    if (o->itype[i] == 1 && o->itype[j] == 2) {
      double dx[2], dv[2], rr = 0.0;
      for (int d = 0; d < 2; d++) {
        dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
        dv[d] = o->vel[2 * i + d] - o->vel[2 * j + d];
        rr += dx[d] * dx[d];
      }
      rr = sqrt(rr);
      if (rr < r0)
        for (int d = 0; d < 2; d++)
          o->acc[2 * i + d] -= (o->p.spring_constant0 * dx[d] + o->p.damping_constant0 * dv[d]) / o->mass[i];
    }
  }
}

/* ImprovedMonaghan, derivatives.c:1955-2012 */
static void improved_monaghan(uph_oracle *o)
{
  const double r0 = o->p.dx;
  const double cM = o->p.mach_number * o->p.speed_of_sound;
  zero_tmp(o);
  PAIR_LOOP {
    const int i = I_, j = J_;
    if (o->itype[i] == 1 && (o->itype[j] == 2 || o->itype[j] == 3)) {
      double dx[2], rr = 0.0;
      for (int d = 0; d < 2; d++) {
        dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
        rr += dx[d] * dx[d];
      }
      rr = sqrt(rr);
      if (rr < r0) {
        const double h = 0.5 * (o->p.h + o->p.h);
        const double normFactor = 7.0 / (64.0 * 3.142 * h * h);
        const double q = rr / h;
        double phi = 0.0;
        if (q >= 0.0 && q < 2.0) {
          const double q4 = (2.0 - q) * (2.0 - q) * (2.0 - q) * (2.0 - q);
          phi = normFactor * (1.0 + 2.0 * q) * q4;
        }
        const double boundarySpacing = 5.0;
        const double rd = (rr - o->p.dx / boundarySpacing);
        const double maxSpeed = cM * cM / boundarySpacing;
        for (int d = 0; d < 2; d++) o->tmp[2 * i + d] += maxSpeed * phi * dx[d] / (rd * rr);
      }
    }
  }
  add_vector(o, o->acc);
}

/* LeonnardJonesBoundaryForces, derivatives.c:1184-1211: every fluid particle
 * against every boundary particle (the last one included) */
static void lennard_jones(uph_oracle *o)
{
  const double r0 = o->p.dx;
  const int b0 = o->nf + o->p.n_solid, b1 = b0 + o->p.n_fixed + o->p.n_moving;
  for (int j = b0; j < b1; j++)
    for (int i = 0; i < o->nf; i++) {
      double dx[2];
      for (int d = 0; d < 2; d++) dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
      const double r2 = dx[0] * dx[0] + dx[1] * dx[1];
      if (r2 < r0 * r0) {
        double r = r0 / sqrt(r2);
        r *= r;
        r *= r;
        const double pb = o->p.lennard_coefficient * r * (r * r - 1.) / r2;
        for (int d = 0; d < 2; d++) o->acc[2 * i + d] += pb * dx[d];
      }
    }
}

/* MonaghanBoundaryForce, derivatives.c:1919-1953 (the default mode) */
static void monaghan_boundary(uph_oracle *o)
{
  const int b0 = o->nf + o->p.n_solid, b1 = b0 + o->p.n_fixed + o->p.n_moving;
  const double cM = o->p.mach_number * o->p.speed_of_sound;
  for (int j = b0; j < b1; j++)
    for (int i = 0; i < o->nf; i++) {
      double dx[2];
      for (int d = 0; d < 2; d++) dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
      const double r2 = dx[0] * dx[0] + dx[1] * dx[1];
      const double r = sqrt(r2);
      const double h = o->p.h;
      const double q = r / h;
      double phi = 0.0;
      if (q >= 0.0 && q < 2.0) {
        const double q3 = (2.0 - q) * (2.0 - q) * (2.0 - q);
        phi = 0.125 * (1.0 + 1.5 * q) * q3;
      }
      for (int d = 0; d < 2; d++) {
        const double gama = cM * cM / (o->p.density0 * o->p.dx * o->p.dy);
        o->acc[2 * i + d] += gama * phi * o->mass[j] * dx[d] / r2;
      }
    }
}

/* per-particle shaking of the moving block: x = x0 + hs (1 - cos(om t)) */
void uph_oracle_set_wall_motion(uph_oracle *o, const double *x0, const double *hs, const double *om)
{
  const int nm = o->p.n_moving;
  free(o->wall_tab);
  o->wall_tab = NULL;
  if (!x0 || nm <= 0) return;
  o->wall_tab = (double *)xcalloc(3 * (size_t)nm, 8);
  memcpy(o->wall_tab, x0, 8 * (size_t)nm);
  memcpy(o->wall_tab + nm, hs, 8 * (size_t)nm);
  memcpy(o->wall_tab + 2 * nm, om, 8 * (size_t)nm);
}

/* inputbp.c:194-207: piston wavemaker (movingBoundary 1), or the table above */
static void wall_motion(uph_oracle *o, double t)
{
  const int m0 = o->nf + o->p.n_solid + o->p.n_fixed, nm = o->p.n_moving;
  if (o->wall_tab) {
    for (int k = 0; k < nm; k++) {
      const double hs = o->wall_tab[nm + k], om = o->wall_tab[2 * nm + k];
      o->pos[2 * (m0 + k)] = o->wall_tab[k] + hs * (1.0 - cos(om * t));
      o->vel[2 * (m0 + k)] = hs * om * sin(om * t);
      o->lvel[2 * (m0 + k)] = o->vel[2 * (m0 + k)];
    }
    return;
  }
  if (o->p.moving_boundary == 1 && o->p.flag_init_simul == 1) {
    const double lbp = 0.5 * o->p.stroke * (1.0 - cos(o->p.omega * t));
    const double lbv = 0.5 * o->p.stroke * o->p.omega * sin(o->p.omega * t);
    const int m0 = o->nf + o->p.n_solid + o->p.n_fixed;
    for (int k = 0; k < o->p.n_moving; k++) {
      o->pos[2 * (m0 + k)] = lbp;
      o->vel[2 * (m0 + k)] = lbv;
      o->lvel[2 * (m0 + k)] = lbv;
    }
  }
}

/* ------------------------------------------------------------ WCSPH rates -- */

/* Textbook weakly-compressible SPH on the same pair list:
 *   p_a      = B ((rho_a/rho0)^gamma - 1)                  (derivatives.c:1674-1682)
 *   drho_a   = sum_b m_b (v_a - v_b) . grad_a W_ab
 *   dv_a     = -sum_b m_b (p_a/rho_a^2 + p_b/rho_b^2 + Pi_ab) grad_a W_ab + g + walls
 *   Pi_ab    = -alpha c0 mu_ab / rhobar_ab if v_ab . x_ab < 0 else 0,
 *   mu_ab    = h v_ab . x_ab / (r^2 + 0.01 h^2)            (Monaghan 1992, beta = 0)
 * The predictor rates equal the corrector rates and the fluctuation fields
 * are zero, so the sph.cc leapfrog becomes a plain kick-drift-kick. */
static void wcsph_rates(uph_oracle *o)
{
  const uph_params *P = &o->p;
  for (int i = 0; i < o->n; i++) {
    const double density = o->rho[i] / P->density0;
    o->pr[i] = P->compression_factor * (pow(density, P->adiabatic_constant) - 1.0);
    o->pressure[i] = o->pr[i];
  }
  memset(o->drho, 0, 8 * (size_t)o->nf);
  memset(o->dp, 0, 8 * (size_t)o->nf);
  memset(o->acc, 0, 16 * (size_t)o->nf);
  const double h = P->h, eta2 = 0.01 * h * h, ac = P->av_alpha * P->speed_of_sound;
  zero_tmp(o);
  double *trho = (double *)xcalloc((size_t)o->n, 8);
  PAIR_LOOP {
    const int i = I_, j = J_;
    double dx[2], dv[2];
    for (int d = 0; d < 2; d++) {
      dx[d] = o->pos[2 * i + d] - o->pos[2 * j + d];
      dv[d] = o->vel[2 * i + d] - o->vel[2 * j + d];
    }
    const double vdw = dv[0] * o->dw[2 * k] + dv[1] * o->dw[2 * k + 1];
    trho[i] += o->mass[j] * vdw;
    trho[j] += o->mass[i] * vdw;
    const double vr = dv[0] * dx[0] + dv[1] * dx[1];
    double pi_ab = 0.0;
    if (vr < 0.0) {
      const double mu = h * vr / (o->rij2[k] + eta2);
      pi_ab = -ac * mu / (0.5 * (o->rho[i] + o->rho[j]));
    }
    const double pij = o->pr[i] / (o->rho[i] * o->rho[i]) + o->pr[j] / (o->rho[j] * o->rho[j]) + pi_ab;
    for (int d = 0; d < 2; d++) {
      o->tmp[2 * i + d] -= o->mass[j] * pij * o->dw[2 * k + d];
      o->tmp[2 * j + d] += o->mass[i] * pij * o->dw[2 * k + d];
    }
  }
  for (int i = 0; i < o->nf; i++) o->drho[i] = trho[i];
  free(trho);
  add_vector(o, o->acc);
  body(o, o->acc);
  sponge(o);
}

/* --------------------------------------------------------- derivatives() -- */

/* derivatives.c:4291-4315: the selected wall force on dvdt */
static void boundary_force(uph_oracle *o)
{
  switch (o->p.select_boundary_force) {
  case 1: lennard_jones(o); break;
  case 3: spring(o, o->acc); break;
  case 4: improved_monaghan(o); break;
  case 5: serial_spring(o); break;
  default: monaghan_boundary(o); break;
  }
}

int uph_oracle_derivatives(uph_oracle *o, double t)
{
  const uph_params *P = &o->p;
  const int nf = o->nf;
  /* derivatives.c:3147-3157 */
  memset(o->drho, 0, 8 * (size_t)nf); memset(o->dp, 0, 8 * (size_t)nf); memset(o->acc, 0, 16 * (size_t)nf);
  memset(o->drho_a, 0, 8 * (size_t)nf); memset(o->dp_a, 0, 8 * (size_t)nf); memset(o->acc_a, 0, 16 * (size_t)nf);
  wall_motion(o, t); /* inputbp(sys, t), derivatives.c:3168 */
  build_pairs(o);    /* CalculateKernel, derivatives.c:4196 */
  if (P->profile == UPH_PROFILE_WCSPH) {
    wcsph_rates(o);
    boundary_force(o);
    memcpy(o->drho_a, o->drho, 8 * (size_t)nf);
    memcpy(o->acc_a, o->acc, 16 * (size_t)nf);
    memset(o->frho, 0, 8 * (size_t)nf); memset(o->fp, 0, 8 * (size_t)nf); memset(o->fvel, 0, 16 * (size_t)nf);
    return 0;
  }
  /* derivatives.c:4197-4276, flagInitSimul == 1 */
  pred_density(o);
  pred_pressure(o);
  pred_pgf(o);
  fluct_scalar(o, o->rho, o->frho);
  fluct_scalar(o, o->pr, o->fp);
  fluct_velocity(o);
  density_eq(o);
  eos(o);
  dyn_pressure(o);
  pgf(o);
  if (P->stress_type == 1) {
    viscous(o, 0);
    viscous(o, 1);
  }
  body(o, o->acc);
  body(o, o->acc_a);
  sponge(o);
  boundary_force(o);
  spring(o, o->acc_a); /* every mode pairs with PredictingSpringBoundaryForces */
  return 0;
}

/* --------------------------------------------------------------- leapfrog -- */

/* src/bin/sph.cc:90-168, statement by statement */
int uph_oracle_step(uph_oracle *o, int nsteps)
{
  const double dt = o->p.time_step;
  const int nf = o->nf;
  const double eps = o->p.epsilon;
  for (int s = 0; s < nsteps; s++) {
    const int itime = ++o->itime;
    const double t = itime * dt;
    if (itime != 1) {
      memcpy(o->rhomin, o->rho, 8 * (size_t)nf);
      memcpy(o->prmin, o->pr, 8 * (size_t)nf);
      memcpy(o->lrho, o->rho, 8 * (size_t)nf);
      memcpy(o->lpr, o->pr, 8 * (size_t)nf);
      memcpy(o->lvel, o->vel, 16 * (size_t)nf); /* walls keep their deck values */
      for (int i = 0; i < nf; i++) {
        o->rho[i] += 0.5 * dt * o->drho_a[i];
        o->lrho[i] = o->lrho[i] + 0.5 * dt * o->drho_a[i] + o->frho[i];
        o->pr[i] += 0.5 * dt * o->dp_a[i];
        o->lpr[i] = o->lpr[i] + 0.5 * dt * o->dp_a[i] + o->fp[i];
      }
      for (int i = 0; i < nf; i++)
        for (int d = 0; d < 2; d++) {
          o->vmin[2 * i + d] = o->vel[2 * i + d];
          o->vel[2 * i + d] += 0.5 * dt * o->acc_a[2 * i + d];
          o->lvel[2 * i + d] = o->vel[2 * i + d] + 0.5 * dt * o->acc_a[2 * i + d] + eps * o->fvel[2 * i + d];
        }
    }
    uph_oracle_derivatives(o, t);
    if (itime == 1) {
      for (int i = 0; i < nf; i++) {
        o->lrho[i] = o->rho[i] + 0.5 * dt * o->drho[i] + o->frho[i];
        o->rho[i] += 0.5 * dt * o->drho[i];
        o->lpr[i] = o->pr[i] + 0.5 * dt * o->dp[i] + o->fp[i];
        o->pr[i] += 0.5 * dt * o->dp[i];
      }
      for (int i = 0; i < nf; i++)
        for (int d = 0; d < 2; d++) {
          o->lvel[2 * i + d] = o->vel[2 * i + d] + 0.5 * dt * o->acc[2 * i + d] + eps * o->fvel[2 * i + d];
          o->vel[2 * i + d] += 0.5 * dt * o->acc[2 * i + d];
          o->pos[2 * i + d] += dt * o->vel[2 * i + d];
        }
    } else {
      for (int i = 0; i < nf; i++) {
        o->lrho[i] = o->rhomin[i] + dt * o->drho[i] + o->frho[i];
        o->rho[i] = o->rhomin[i] + dt * o->drho[i];
        o->lpr[i] = o->prmin[i] + dt * o->dp[i] + o->fp[i];
        o->pr[i] = o->prmin[i] + dt * o->dp[i];
      }
      for (int i = 0; i < nf; i++)
        for (int d = 0; d < 2; d++) {
          o->lvel[2 * i + d] = o->vmin[2 * i + d] + dt * o->acc[2 * i + d] + eps * o->fvel[2 * i + d];
          o->vel[2 * i + d] = o->vmin[2 * i + d] + dt * o->acc[2 * i + d];
          o->pos[2 * i + d] += dt * o->vel[2 * i + d];
        }
    }
    if (o->p.profile == UPH_PROFILE_WCSPH)
      for (int i = 0; i < nf; i++) { /* the WCSPH pressure is Tait's law of the new density */
        const double density = o->rho[i] / o->p.density0;
        o->pr[i] = o->p.compression_factor * (pow(density, o->p.adiabatic_constant) - 1.0);
        o->pressure[i] = o->pr[i];
      }
  }
  return 0;
}

int64_t uph_oracle_pairs(const uph_oracle *o, int64_t cap, int32_t *i_pair, int32_t *j_pair, double *rij2, double *w,
                         double *dwcdx)
{
  if (o->niac <= cap) {
    if (i_pair) memcpy(i_pair, o->ip, 4 * (size_t)o->niac);
    if (j_pair) memcpy(j_pair, o->jp, 4 * (size_t)o->niac);
    if (rij2) memcpy(rij2, o->rij2, 8 * (size_t)o->niac);
    if (w) memcpy(w, o->w, 8 * (size_t)o->niac);
    if (dwcdx) memcpy(dwcdx, o->dw, 16 * (size_t)o->niac);
  }
  return o->niac;
}

int uph_oracle_max_neighbors(const uph_oracle *o) { return o->max_nb; }

void uph_oracle_energies(const uph_oracle *o, double out[3])
{
  double ke = 0.0, pe = 0.0, m = 0.0;
  for (int i = 0; i < o->nf; i++) {
    ke += 0.5 * o->mass[i] * (o->vel[2 * i] * o->vel[2 * i] + o->vel[2 * i + 1] * o->vel[2 * i + 1]);
    pe += o->mass[i] * o->p.gravity * o->pos[2 * i + 1];
    m += o->mass[i];
  }
  out[0] = ke;
  out[1] = pe;
  out[2] = m;
}
