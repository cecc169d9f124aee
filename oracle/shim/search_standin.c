/*
 * Test infrastructure (oracle only).  A stand-in for the reference's
 * neighbour search `SearchNeighbors` (src/lib/Search.cc:5-44), which needs
 * libnabo and Eigen -- neither is vendored by the reference, neither has a
 * pinned version, and neither is installed here.
 *
 * What the reference does (Search.cc:12-40, called from
 * src/lib/derivatives.c:1076-1086):
 *   - builds a libnabo kd-tree (createKDTreeTreeHeap) over all
 *     `NumberOfParticles` positions and runs an exact k-nearest-neighbour
 *     query (k = NumberOfNeighbors = 40) for every fluid particle s;
 *   - libnabo's default option flags forbid self matches: a data point whose
 *     squared distance to the query is <= DBL_EPSILON is never returned
 *     (libnabo's published documentation of ALLOW_SELF_MATCH), and results
 *     are left unsorted (SORT_RESULTS unset);
 *   - keeps the pair (s, j) iff j > s, dists(k,s) < dist and
 *     j < ParticleBoundary, with dists the squared distances
 *     (x_s - x_j)^2 + (y_s - y_j)^2;
 *   - emits pairs ordered by s, then by libnabo's internal heap order.
 *
 * This stand-in computes the same set with a uniform cell grid:
 *   - candidates are all points with DBL_EPSILON < d^2 < dist (points outside
 *     the radius are filtered by the reference anyway, so the k-NN set
 *     restricted to the radius is exactly the in-radius set whenever a query
 *     has at most k in-radius candidates);
 *   - if a query has more than k in-radius candidates, the k nearest are kept
 *     with ties broken by ascending index.  libnabo's tie order is unknown, so
 *     such queries are counted (uph_standin_truncated_queries) and parity
 *     cases assert that the count is zero;
 *   - pairs are emitted ordered by s, then by ascending j.  Only the
 *     summation order of the reference's pair loops depends on this order.
 * d^2 is evaluated as dx*dx + dy*dy in that order; this file is compiled with
 * -ffp-contract=off so no fused multiply-add changes the rounding.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static long g_truncated = 0;     /* queries where the k-NN cap removed in-radius points */
static int g_max_inradius = 0;   /* largest in-radius candidate count seen (all queries) */
static long g_capacity = -1;     /* pair-array capacity; <0 means unchecked */
static long g_overflow = 0;      /* calls whose pair count exceeded the capacity */

void uph_standin_reset_stats(void) { g_truncated = 0; g_max_inradius = 0; g_overflow = 0; }
long uph_standin_truncated_queries(void) { return g_truncated; }
int uph_standin_max_inradius(void) { return g_max_inradius; }
long uph_standin_overflows(void) { return g_overflow; }
void uph_standin_set_capacity(long cap) { g_capacity = cap; }

typedef struct { double d2; int j; } cand_t;

static int cand_cmp(const void *a, const void *b)
{
  const cand_t *x = (const cand_t *)a, *y = (const cand_t *)b;
  if (x->d2 < y->d2) return -1;
  if (x->d2 > y->d2) return 1;
  return (x->j > y->j) - (x->j < y->j);
}

static int int_cmp(const void *a, const void *b)
{
  int x = ((const cand_t *)a)->j, y = ((const cand_t *)b)->j;
  return (x > y) - (x < y);
}

int SearchNeighbors(const double **Position, int *i_pair, int *j_pair, double *rij2,
                    const int NumberOfFluidParticles, const int NumberOfParticles,
                    int ParticleBoundary, const int NumberOfNeighbors, const double dist)
{
  const int n = NumberOfParticles;
  if (n <= 0 || NumberOfFluidParticles <= 0 || !(dist > 0.0))
    return 0;
  double xmin = Position[0][0], xmax = xmin, ymin = Position[0][1], ymax = ymin;
  for (int p = 1; p < n; p++) {
    const double x = Position[p][0], y = Position[p][1];
    if (x < xmin) xmin = x;
    if (x > xmax) xmax = x;
    if (y < ymin) ymin = y;
    if (y > ymax) ymax = y;
  }
  /* cells a hair wider than the radius so a 3x3 block always covers it */
  const double cs = sqrt(dist) * (1.0 + 1e-9);
  long ncx = (long)((xmax - xmin) / cs) + 1, ncy = (long)((ymax - ymin) / cs) + 1;
  if (ncx * ncy > 64L * 1024 * 1024) {
    fprintf(stderr, "search stand-in: grid of %ld x %ld cells is too large\n", ncx, ncy);
    exit(1);
  }
  int *cell = (int *)malloc(sizeof(int) * n);
  int *start = (int *)calloc((size_t)(ncx * ncy + 1), sizeof(int));
  int *order = (int *)malloc(sizeof(int) * n);
  for (int p = 0; p < n; p++) {
    long cx = (long)((Position[p][0] - xmin) / cs), cy = (long)((Position[p][1] - ymin) / cs);
    if (cx >= ncx) cx = ncx - 1;
    if (cy >= ncy) cy = ncy - 1;
    cell[p] = (int)(cy * ncx + cx);
    start[cell[p] + 1]++;
  }
  for (long c = 0; c < ncx * ncy; c++)
    start[c + 1] += start[c];
  {
    int *fill = (int *)malloc(sizeof(int) * (size_t)(ncx * ncy));
    memcpy(fill, start, sizeof(int) * (size_t)(ncx * ncy));
    for (int p = 0; p < n; p++) /* ascending index inside every cell */
      order[fill[cell[p]]++] = p;
    free(fill);
  }

  int cap = 256;
  cand_t *cand = (cand_t *)malloc(sizeof(cand_t) * cap);
  long niac = 0;
  for (int s = 0; s < NumberOfFluidParticles; s++) {
    const double xs = Position[s][0], ys = Position[s][1];
    const long cx = cell[s] % ncx, cy = cell[s] / ncx;
    int nc = 0;
    for (long by = cy - 1; by <= cy + 1; by++) {
      if (by < 0 || by >= ncy) continue;
      for (long bx = cx - 1; bx <= cx + 1; bx++) {
        if (bx < 0 || bx >= ncx) continue;
        const long c = by * ncx + bx;
        for (int q = start[c]; q < start[c + 1]; q++) {
          const int j = order[q];
          const double dx = xs - Position[j][0];
          const double dy = ys - Position[j][1];
          const double d2 = dx * dx + dy * dy;
          if (d2 <= DBL_EPSILON || !(d2 < dist))
            continue;
          if (nc == cap) {
            cap *= 2;
            cand = (cand_t *)realloc(cand, sizeof(cand_t) * cap);
          }
          cand[nc].d2 = d2;
          cand[nc].j = j;
          nc++;
        }
      }
    }
    if (nc > g_max_inradius)
      g_max_inradius = nc;
    if (nc > NumberOfNeighbors) {
      g_truncated++;
      qsort(cand, nc, sizeof(cand_t), cand_cmp);
      nc = NumberOfNeighbors;
    }
    qsort(cand, nc, sizeof(cand_t), int_cmp);
    for (int k = 0; k < nc; k++) {
      const int j = cand[k].j;
      if (j > s && j < ParticleBoundary) {
        if (g_capacity >= 0 && niac >= g_capacity) {
          g_overflow++;
          fprintf(stderr, "search stand-in: more than %ld pairs; raise the pair capacity\n", g_capacity);
          exit(1);
        }
        i_pair[niac] = s;
        j_pair[niac] = j;
        rij2[niac] = cand[k].d2;
        niac++;
      }
    }
  }
  free(cand);
  free(order);
  free(start);
  free(cell);
  return (int)niac;
}
