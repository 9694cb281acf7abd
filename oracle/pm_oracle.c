/* CPU oracle: C restatement of ProtoMol's periodic cutoff nonbonded system
 * force (LJ with C2 switching + Coulomb with C1 switching) and of the
 * real-space term of its Ewald sum.
 *
 * TEST INFRASTRUCTURE ONLY (see pm_oracle.h).  Every function cites the
 * reference code it restates; paths are relative to protomol/src/protomol/.
 * The operation order inside each function follows the reference so that the
 * FP64 results match it bit for bit on orthogonal periodic boxes.
 */
#include "pm_oracle.h"

#include <math.h>
#include <stdlib.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <string.h>

#define PMO_EPSILON 1.0e-14                 /* base/PMConstants.cpp:47 */
#define PMO_INV_TIMEFACTOR 0.02045482828087295 /* base/PMConstants.cpp:51 */
#define PMO_MAX_INT_2 (2147483647 / 2)       /* base/PMConstants.cpp:44 */

/* ---------------------------------------------------------------------- */
/* PeriodicBoundaryConditions (topology/PeriodicBoundaryConditions.cpp:32-77,
 * orthogonal branch only).                                                */
typedef struct {
  double e[3];       /* e1.x, e2.y, e3.z */
  double er[3];      /* reciprocal basis components myE1r.x, ... */
  double origin[3];
  double min[3], max[3];
  double h[3], h2[3]; /* myH, myH2 */
  double d;           /* myD: squared half of the smallest box length */
} pbc_t;

static void pbc_set(pbc_t *b, const double box[3], const double origin[3]) {
  /* e1 = (Lx,0,0), e2 = (0,Ly,0), e3 = (0,0,Lz).
   * a1 = e2 x e3, myE1r = a1 / e1.a1 (PeriodicBoundaryConditions.cpp:56-61) */
  const double lx = box[0], ly = box[1], lz = box[2];
  double a1x = ly * lz - 0.0 * 0.0;
  double a2y = lz * lx - 0.0 * 0.0;
  double a3z = lx * ly - 0.0 * 0.0;
  double d1 = lx * a1x + 0.0 * 0.0 + 0.0 * 0.0;
  double d2 = 0.0 * 0.0 + ly * a2y + 0.0 * 0.0;
  double d3 = 0.0 * 0.0 + 0.0 * 0.0 + lz * a3z;
  int k;
  b->e[0] = lx; b->e[1] = ly; b->e[2] = lz;
  b->er[0] = a1x / d1; b->er[1] = a2y / d2; b->er[2] = a3z / d3;
  for (k = 0; k < 3; k++) {
    /* a = origin - (e1+e2+e3)*0.5, b = origin + (e1+e2+e3)*0.5 (:63-71) */
    double s = (k == 0 ? lx + 0.0 + 0.0 : k == 1 ? 0.0 + ly + 0.0 : 0.0 + 0.0 + lz);
    double a = origin[k] - s * 0.5;
    double c = origin[k] + s * 0.5;
    b->origin[k] = origin[k];
    b->min[k] = a < c ? a : c;
    b->max[k] = a < c ? c : a;
  }
  {
    double dx = (lx * 0.5) * (lx * 0.5);
    double dy = (ly * 0.5) * (ly * 0.5);
    double dz = (lz * 0.5) * (lz * 0.5);
    double m = dy < dz ? dy : dz;
    b->d = dx < m ? dx : m; /* myD = min(myDX, min(myDY, myDZ)) (:73-76) */
  }
  for (k = 0; k < 3; k++) {
    b->h[k] = b->max[k] - b->min[k];
    b->h2[k] = b->h[k] * 0.5;
  }
}

static double norm2(const double v[3]) {
  return v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
}

/* minimalDifference(c1, c2, distSquared)
 * (topology/PeriodicBoundaryConditions.h:72-110, orthogonal branch). */
static void pbc_min_diff(const pbc_t *b, const double *c1, const double *c2,
                         double diff[3], double *dist2) {
  int k;
  for (k = 0; k < 3; k++) diff[k] = c2[k] - c1[k];
  *dist2 = norm2(diff);
  if (*dist2 > b->d) {
    for (k = 0; k < 3; k++) {
      if (diff[k] < -b->h2[k])
        diff[k] += b->h[k];
      else if (diff[k] > b->h2[k])
        diff[k] -= b->h[k];
    }
    *dist2 = norm2(diff);
    if (*dist2 > b->d) {
      for (k = 0; k < 3; k++) diff[k] -= b->e[k] * rint(b->er[k] * diff[k]);
      *dist2 = norm2(diff);
    }
  }
}

/* minimalPosition(c) (topology/PeriodicBoundaryConditions.h:113-147). */
static void pbc_min_pos(const pbc_t *b, const double *c, double out[3]) {
  int k;
  for (k = 0; k < 3; k++) out[k] = c[k] - b->origin[k];
  if (norm2(out) <= b->d) return;
  for (k = 0; k < 3; k++) {
    if (out[k] < -b->h2[k])
      out[k] += b->h[k];
    else if (out[k] > b->h2[k])
      out[k] -= b->h[k];
  }
  if (norm2(out) <= b->d) return;
  for (k = 0; k < 3; k++) out[k] = out[k] - b->e[k] * rint(b->er[k] * out[k]);
}

/* ---------------------------------------------------------------------- */
/* ExclusionTable::add / check (topology/ExclusionTable.cpp:103-120,
 * topology/ExclusionTable.h:116-131): pair keyed by (min, max) atom index,
 * later additions overwrite earlier ones.                                 */
typedef struct {
  long long key;
  int kind;
  int order;
} excl_t;

static int excl_cmp(const void *pa, const void *pb) {
  const excl_t *a = (const excl_t *)pa, *b = (const excl_t *)pb;
  if (a->key != b->key) return a->key < b->key ? -1 : 1;
  return a->order < b->order ? -1 : (a->order > b->order);
}

static int excl_check(const excl_t *t, int m, int i, int j) {
  long long key;
  int lo = 0, hi = m - 1, found = 0;
  if (j < i) { int tmp = i; i = j; j = tmp; }
  key = ((long long)i << 32) | (unsigned)j;
  /* last entry with this key wins */
  while (lo <= hi) {
    int mid = (lo + hi) / 2;
    if (t[mid].key <= key) {
      if (t[mid].key == key) found = t[mid].kind;
      lo = mid + 1;
    } else
      hi = mid - 1;
  }
  return found;
}

/* ---------------------------------------------------------------------- */
/* Switching functions and potentials.                                      */
typedef struct {
  double ron2, rc2, s1, s2, s3; /* C2 (switch/C2SwitchingFunction.cpp:12-18) */
  double c_rc2, c15_1, c05_3, c15_3; /* C1 (switch/C1SwitchingFunction.cpp:12-16) */
  double cut2;                  /* OneAtomPairTwo mySquaredCutoff (OneAtomPairTwo.h:38-40) */
} sw_t;

static void sw_set(sw_t *w, double ron, double rc_lj, double rc_coul) {
  double t = rc_lj * rc_lj - ron * ron;
  w->ron2 = ron * ron;
  w->rc2 = rc_lj * rc_lj;
  w->s1 = 1.0 / ((t * t) * t);                  /* power<3> = (x*x)*x */
  w->s2 = rc_lj * rc_lj - 3.0 * ron * ron;
  w->s3 = 4.0 / ((t * t) * t);
  w->c_rc2 = rc_coul * rc_coul;
  w->c15_1 = 1.5 / rc_coul;
  w->c05_3 = 0.5 / (rc_coul * rc_coul * rc_coul);
  w->c15_3 = 1.5 / (rc_coul * rc_coul * rc_coul);
  w->cut2 = w->rc2 > w->c_rc2 ? w->rc2 : w->c_rc2;
}

/* C2SwitchingFunction::operator() (switch/C2SwitchingFunction.h:42-53). */
static void c2_switch(const sw_t *w, double d2, double *value, double *deriv) {
  *deriv = 0.0;
  if (d2 > w->rc2)
    *value = 0.0;
  else if (d2 >= w->ron2) {
    double c2 = w->rc2 - d2;
    double c4 = c2 * (w->s2 + 2.0 * d2);
    *value = w->s1 * (c2 * c4);
    *deriv = w->s3 * (c2 * c2 - c4);
  } else
    *value = 1.0;
}

/* C1SwitchingFunction::operator() (switch/C1SwitchingFunction.h:41-50). */
static void c1_switch(const sw_t *w, double d2, double *value, double *deriv) {
  double dist;
  if (d2 > w->c_rc2) {
    *value = 0.0;
    *deriv = 0.0;
    return;
  }
  dist = sqrt(d2);
  *value = 1.0 - dist * (w->c15_1 - d2 * w->c05_3);
  *deriv = -w->c15_1 / dist + dist * w->c15_3;
}

/* ---------------------------------------------------------------------- */
typedef struct {
  const pmo_system *s;
  const double *pos;
  double *forces;
  double e_coul, e_lj;
  double vir[9], mvir[9];
  int virial_mode;
  pbc_t pbc;
  sw_t sw;
  excl_t *excl;
  int nexcl;
  double *molpos; /* [nmol*3] when virial_mode == 2 */
  long long pairs;
  int count_only;
  /* Ewald real-space term (form 1 = A&S poly5 erfc, the reference's default
   * build; form 2 = libm erfc, its -DUSE_EWALD_EXACT_ERF build) */
  int form;
  double ew_alpha, ew_alpha2, ew_2api, ew_rc2;
  double walk_cut;   /* cutoff of the cell enumerator */
} ctx_t;

/* ScalarStructure::addVirial(force12, diff) (type/ScalarStructure.cpp:36-54) */
static void add_virial(double *t, const double f[3], const double d[3]) {
  double xy = f[0] * d[1];
  double xz = f[0] * d[2];
  double yz = f[1] * d[2];
  t[0] += f[0] * d[0];
  t[1] += xy;
  t[2] += xz;
  t[3] += xy;
  t[4] += f[1] * d[1];
  t[5] += yz;
  t[6] += xz;
  t[7] += yz;
  t[8] += f[2] * d[2];
}

/* OneAtomPairTwo::doOneAtomPair (force/OneAtomPairTwo.h:57-125) with
 * LennardJonesForce (force/LennardJonesForce.h:29-61) first and
 * CoulombForce (force/CoulombForce.h:27-38) second. */
static void one_pair(ctx_t *c, int i, int j) {
  const pmo_system *s = c->s;
  double diff[3], d2, r2, e1, f1, e2, f2, sv, sd, fij[3], fs;
  int mi, mj, same, excl = 0, k;
  pbc_min_diff(&c->pbc, c->pos + 3 * i, c->pos + 3 * j, diff, &d2);
  if (d2 > c->sw.cut2) return;
  mi = s->mol[i];
  mj = s->mol[j];
  same = (mi == mj);
  if (same) excl = excl_check(c->excl, c->nexcl, i, j);
  if (excl == 2) return;
  if (c->count_only) {
    c->pairs++;
    return;
  }
  r2 = 1.0 / d2;
  { /* Lennard-Jones */
    const double *p = s->lj + 4 * (s->type[i] * s->ntypes + s->type[j]);
    double A = excl != 1 ? p[0] : p[2];
    double B = excl != 1 ? p[1] : p[3];
    double r6 = r2 * r2 * r2;
    double r12 = r6 * r6;
    double r6B = B * r6;
    double r12A = A * r12;
    e1 = r12A - r6B;
    f1 = 12.0 * r12A * r2 - 6.0 * r6B * r2;
  }
  { /* Coulomb on pre-scaled charges */
    e2 = s->qscaled[i] * s->qscaled[j] * sqrt(r2);
    if (excl == 1) e2 *= s->coulomb_scaling;
    f2 = e2 * r2;
  }
  c2_switch(&c->sw, d2, &sv, &sd);
  f1 = f1 * sv - e1 * sd;
  e1 = e1 * sv;
  c1_switch(&c->sw, d2, &sv, &sd);
  f2 = f2 * sv - e2 * sd;
  e2 = e2 * sv;
  c->e_lj += e1;
  c->e_coul += e2;
  fs = f1 + f2;
  for (k = 0; k < 3; k++) fij[k] = diff[k] * fs;
  for (k = 0; k < 3; k++) {
    c->forces[3 * i + k] -= fij[k];
    c->forces[3 * j + k] += fij[k];
  }
  if (!same && c->virial_mode >= 2) {
    double cd[3], cd2;
    pbc_min_diff(&c->pbc, c->molpos + 3 * mi, c->molpos + 3 * mj, cd, &cd2);
    add_virial(c->vir, fij, diff);
    add_virial(c->mvir, fij, cd);
  } else if (c->virial_mode >= 1)
    add_virial(c->vir, fij, diff);
}

/* Abramowitz & Stegun 7.1.26 polynomial for erfc(x) e^{x^2}
 * (base/MathUtilities.cpp:39-49): t = 1 / (1 + p x), t (a1 + t (a2 + ...)). */
static double ew_poly5(double ar) {
  const double a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741,
               a4 = -1.453152027, a5 = 1.061405429, p = 0.3275911;
  double t = 1.0 / (1.0 + p * ar);
  return (t) * (a1 + (t) * (a2 + (t) * (a3 + (t) * (a4 + (t) * a5))));
}

/* One (i, j) visit of NonbondedFullEwaldSystemForce::realTerm
 * (force/nonbonded/NonbondedFullEwaldSystemForce.h:776-851) with the
 * CutoffSwitchingFunction (switch/CutoffSwitchingFunction.h:41-44) and only
 * the zero lattice vector (every box edge >= 2 rc, so buildLatticeVectors,
 * topology/PeriodicBoundaryConditions.cpp:80-104, adds no image within rc).
 * The force on i is summed into fi; the caller adds fi to forces[i] after
 * its j loop, as the reference does. */
static void ewald_pair(ctx_t *c, int i, int j, double fi[3]) {
  const pmo_system *s = c->s;
  double rij[3], r2, r, qq, energy, force, fij[3];
  int mi = s->mol[i], mj = s->mol[j], same = (mi == mj), excl = 0, k;
  pbc_min_diff(&c->pbc, c->pos + 3 * i, c->pos + 3 * j, rij, &r2);
  if (same) excl = excl_check(c->excl, c->nexcl, i, j);
  if (i == j) excl = 2;
  if (excl == 2) return;
  r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
  if (r2 > c->ew_rc2) return;
  if (c->count_only) {
    c->pairs++;
    return;
  }
  r = sqrt(r2);
  qq = s->qscaled[i] * s->qscaled[j];
  if (excl == 1) qq *= s->coulomb_scaling;
  if (c->form == 1) {
    double rr = 1.0 / r;
    double ar = c->ew_alpha * r;
    double e = qq * exp(-ar * ar);
    energy = ew_poly5(ar) * e * rr;
    force = ((energy + c->ew_2api * e) * rr * rr);
  } else {
    double a = erfc(c->ew_alpha * r) / r;
    energy = qq * a;
    force = qq * (a + c->ew_2api * exp(-c->ew_alpha2 * r2)) / r2;
  }
  /* switching value 1, derivative 0 inside the cutoff */
  force = force * 1.0 - energy * 0.0;
  energy = energy * 1.0;
  c->e_coul += energy;
  for (k = 0; k < 3; k++) fij[k] = rij[k] * force;
  for (k = 0; k < 3; k++) {
    fi[k] -= fij[k];
    c->forces[3 * j + k] += fij[k];
  }
  if (!same && c->virial_mode >= 2) {
    double cd[3], cd2;
    pbc_min_diff(&c->pbc, c->molpos + 3 * mi, c->molpos + 3 * mj, cd, &cd2);
    add_virial(c->vir, fij, rij);
    add_virial(c->mvir, fij, cd);
  } else if (c->virial_mode >= 1)
    add_virial(c->vir, fij, rij);
}

/* All j of one i for the Ewald walk: j over cell B, or from i itself in a
 * self cell (NonbondedFullEwaldSystemForce.h:776-853).  next == NULL walks
 * j = bfirst .. n-1 (the all-pairs cross-check). */
static void ewald_atom(ctx_t *c, int a, int bfirst, const int *next) {
  double fi[3] = {0.0, 0.0, 0.0};
  int bb, k;
  for (bb = bfirst; bb != -1; bb = next ? next[bb] : (bb + 1 < c->s->n ? bb + 1 : -1))
    ewald_pair(c, a, bb, fi);
  if (!c->count_only)
    for (k = 0; k < 3; k++) c->forces[3 * a + k] += fi[k];
}

/* molecularCenterOfMass with Kahan summation over the molecule's atoms in
 * ascending index order (topology/TopologyUtilities.cpp:645-683). */
static int build_molpos(ctx_t *c) {
  const pmo_system *s = c->s;
  int nmol = 0, i, k;
  double *sum, *comp, *mass;
  int *seen;
  for (i = 0; i < s->n; i++)
    if (s->mol[i] + 1 > nmol) nmol = s->mol[i] + 1;
  c->molpos = (double *)calloc((size_t)nmol * 3 + 1, sizeof(double));
  sum = (double *)calloc((size_t)nmol * 3 + 1, sizeof(double));
  comp = (double *)calloc((size_t)nmol * 3 + 1, sizeof(double));
  mass = (double *)calloc((size_t)nmol + 1, sizeof(double));
  seen = (int *)calloc((size_t)nmol + 1, sizeof(int));
  if (!c->molpos || !sum || !comp || !mass || !seen) {
    free(sum); free(comp); free(mass); free(seen);
    return PMO_ENOMEM;
  }
  for (i = 0; i < s->n; i++) {
    int m = s->mol[i];
    double w = s->mass ? s->mass[i] : 1.0;
    if (!seen[m]) {
      seen[m] = 1;
      mass[m] = w;
      for (k = 0; k < 3; k++) sum[3 * m + k] = c->pos[3 * i + k] * w;
    } else {
      mass[m] += w;
      for (k = 0; k < 3; k++) {
        double x = c->pos[3 * i + k] * w;
        double y = x - comp[3 * m + k];
        double t = sum[3 * m + k] + y;
        comp[3 * m + k] = (t - sum[3 * m + k]) - y;
        sum[3 * m + k] = t;
      }
    }
  }
  for (i = 0; i < nmol; i++)
    for (k = 0; k < 3; k++)
      c->molpos[3 * i + k] = seen[i] ? sum[3 * i + k] / mass[i] : 0.0;
  free(sum); free(comp); free(mass); free(seen);
  return PMO_OK;
}

/* ---------------------------------------------------------------------- */
/* Cell list + cell-pair walk.
 *  - CubicCellManager::initialize (topology/CubicCellManager.cpp:46-65):
 *    cell edge = box / max(1, floor(box / cellsize)) per axis.
 *  - ArrayCellListStructure::initialize (topology/ArrayCellListStructure.cpp:
 *    22-128): n = max(1, floor(box / edge + EPSILON)); cells stored x-major,
 *    z fastest.
 *  - Topology::updateCellLists (topology/Topology.h:44-86): atoms inserted
 *    from N-1 down to 0 at the head of their cell's list, cell =
 *    floor((origin - min + minimalPosition(p)) / edge).
 *  - CellListEnumerator<Periodic, Cubic>::initialize/next
 *    (topology/CellListEnumeratorPeriodicBoundaries.h:25-134): neighbour
 *    deltas with sum(((|k|-1)+ * edge)^2) < cutoff^2, reduced to basis cells,
 *    de-duplicated, sorted (x, y, z); each cell pair visited from the lower
 *    array index, self pair first.
 *  - NonbondedCutoffForce::doEvaluate (force/nonbonded/NonbondedCutoffForce.h:
 *    37-54): i over cell A, j over cell B (or i's successors in a self cell).
 */
typedef struct { int x, y, z; } cell3;

static int cell3_cmp(const void *pa, const void *pb) {
  const cell3 *a = (const cell3 *)pa, *b = (const cell3 *)pb;
  if (a->x != b->x) return a->x < b->x ? -1 : 1;
  if (a->y != b->y) return a->y < b->y ? -1 : 1;
  if (a->z != b->z) return a->z < b->z ? -1 : 1;
  return 0;
}

static int imod(int a, int maxn, int n) { return (a + maxn) % n; }

static int walk_cells(ctx_t *c) {
  const pmo_system *s = c->s;
  const pbc_t *b = &c->pbc;
  double vdiff[3], edge[3], inv[3];
  int nd[3], maxn[3], n1[3], maxn1[3], k, i;
  int *head, *next;
  int ncell, begin, end, ndelta = 0;
  cell3 *deltas;
  double cut2 = c->walk_cut * c->walk_cut;
  for (k = 0; k < 3; k++) {
    double m = floor((b->max[k] - b->min[k]) / s->cellsize);
    vdiff[k] = b->max[k] - b->min[k];
    edge[k] = vdiff[k] / (1.0 > m ? 1.0 : m);
  }
  for (k = 0; k < 3; k++) inv[k] = 1.0 / edge[k];
  for (k = 0; k < 3; k++) {
    int v = (int)floor(vdiff[k] / edge[k] + PMO_EPSILON);
    nd[k] = v > 1 ? v : 1;
    maxn[k] = PMO_MAX_INT_2 - PMO_MAX_INT_2 % nd[k];
    n1[k] = -nd[k] / 2;
    maxn1[k] = maxn[k] - n1[k];
  }
  ncell = nd[0] * nd[1] * nd[2];
  head = (int *)malloc(sizeof(int) * (size_t)ncell);
  next = (int *)malloc(sizeof(int) * (size_t)(s->n > 0 ? s->n : 1));
  if (!head || !next) { free(head); free(next); return PMO_ENOMEM; }
  for (i = 0; i < ncell; i++) head[i] = -1;
  for (i = s->n - 1; i >= 0; i--) {
    double mp[3];
    int cc[3], idx;
    pbc_min_pos(b, c->pos + 3 * i, mp);
    for (k = 0; k < 3; k++) {
      double p = (b->origin[k] - b->min[k]) + mp[k];
      cc[k] = (int)floor(p * inv[k]);
      /* The reference writes outside its cell array when rounding puts a
       * coordinate exactly on the upper box face; clamp instead. */
      if (cc[k] < 0) cc[k] = 0;
      if (cc[k] >= nd[k]) cc[k] = nd[k] - 1;
    }
    idx = (cc[0] * nd[1] + cc[1]) * nd[2] + cc[2];
    next[i] = head[idx];
    head[idx] = i;
  }
  /* neighbour deltas */
  {
    int lim[3];
    for (k = 0; k < 3; k++) {
      int v = (int)(c->walk_cut / edge[k] + 1.0 + PMO_EPSILON);
      lim[k] = v < nd[k] ? v : nd[k];
    }
    deltas = (cell3 *)malloc(sizeof(cell3) *
                             (size_t)((2 * lim[0] + 1) * (2 * lim[1] + 1) * (2 * lim[2] + 1)));
    if (!deltas) { free(head); free(next); return PMO_ENOMEM; }
    {
      double xx = edge[0] * edge[0], yy = edge[1] * edge[1], zz = edge[2] * edge[2];
      int kx, ly, mz;
      for (kx = -lim[0]; kx <= lim[0]; kx++) {
        int x = abs(kx) - 1;
        double d0;
        if (x < 0) x = 0;
        d0 = x * x * xx;
        for (ly = -lim[1]; ly <= lim[1]; ly++) {
          int y = abs(ly) - 1;
          double d1;
          if (y < 0) y = 0;
          d1 = d0 + y * y * yy;
          for (mz = -lim[2]; mz <= lim[2]; mz++) {
            int z = abs(mz) - 1;
            if (z < 0) z = 0;
            if (d1 + z * z * zz < cut2) {
              cell3 md;
              int q, dup = 0;
              md.x = (kx + maxn1[0]) % nd[0] + n1[0];
              md.y = (ly + maxn1[1]) % nd[1] + n1[1];
              md.z = (mz + maxn1[2]) % nd[2] + n1[2];
              if (md.x == 0 && md.y == 0 && md.z == 0) dup = 1;
              for (q = 0; q < ndelta && !dup; q++)
                if (deltas[q].x == md.x && deltas[q].y == md.y && deltas[q].z == md.z) dup = 1;
              if (!dup) deltas[ndelta++] = md;
            }
          }
        }
      }
    }
    qsort(deltas, (size_t)ndelta, sizeof(cell3), cell3_cmp);
  }
  /* cell-pair walk */
  begin = ncell;
  end = 0;
  for (i = 0; i < ncell; i++)
    if (head[i] >= 0) {
      if (begin == ncell) begin = i;
      end = i + 1;
    }
  if (begin == ncell) begin = end = 0;
  {
    int ci = begin, cj = begin, counter = 0;
    while (ci != end) {
      int a, bb;
      if (c->form)
        for (a = head[ci]; a != -1; a = next[a])
          ewald_atom(c, a, (ci != cj) ? head[cj] : a, next);
      else
        for (a = head[ci]; a != -1; a = next[a])
          for (bb = (ci != cj) ? head[cj] : next[a]; bb != -1; bb = next[bb])
            one_pair(c, a, bb);
      /* next() */
      do {
        if (ci != end) {
          cj = end;
          while (counter != ndelta) {
            int x = ci / (nd[1] * nd[2]);
            int y = (ci / nd[2]) % nd[1];
            int z = ci % nd[2];
            const cell3 *d = &deltas[counter++];
            int jx = imod(x + d->x, maxn[0], nd[0]);
            int jy = imod(y + d->y, maxn[1], nd[1]);
            int jz = imod(z + d->z, maxn[2], nd[2]);
            int jdx = (jx * nd[1] + jy) * nd[2] + jz;
            if (head[jdx] >= 0) { cj = jdx; break; }
          }
          if (cj == end) {
            ++ci;
            while (ci != end && head[ci] < 0) ++ci;
            cj = ci;
            counter = 0;
          }
        }
      } while (ci > cj);
    }
  }
  free(deltas);
  free(head);
  free(next);
  return PMO_OK;
}

static int ctx_init(ctx_t *c, const pmo_system *s, const double *pos,
                    double *forces, int virial_mode) {
  int e;
  memset(c, 0, sizeof(*c));
  if (!s || s->n < 0 || !pos || s->ntypes <= 0 || s->cellsize <= 0.0 ||
      s->rc_lj <= 0.0 || s->rc_coul <= 0.0 || s->rc_alg <= 0.0 ||
      s->ron < 0.0 || s->ron >= s->rc_lj || s->box[0] <= 0.0 ||
      s->box[1] <= 0.0 || s->box[2] <= 0.0)
    return PMO_EBADARG;
  c->s = s;
  c->pos = pos;
  c->forces = forces;
  c->virial_mode = virial_mode;
  c->walk_cut = s->rc_alg;
  pbc_set(&c->pbc, s->box, s->origin);
  sw_set(&c->sw, s->ron, s->rc_lj, s->rc_coul);
  c->nexcl = s->nexcl;
  c->excl = (excl_t *)malloc(sizeof(excl_t) * (size_t)(s->nexcl > 0 ? s->nexcl : 1));
  if (!c->excl) return PMO_ENOMEM;
  for (e = 0; e < s->nexcl; e++) {
    int a = s->excl[3 * e], b = s->excl[3 * e + 1];
    if (b < a) { int t = a; a = b; b = t; }
    c->excl[e].key = ((long long)a << 32) | (unsigned)b;
    c->excl[e].kind = s->excl[3 * e + 2];
    c->excl[e].order = e;
  }
  qsort(c->excl, (size_t)s->nexcl, sizeof(excl_t), excl_cmp);
  if (virial_mode >= 2) return build_molpos(c);
  return PMO_OK;
}

static void ctx_free(ctx_t *c) {
  free(c->excl);
  free(c->molpos);
}

int pmo_eval(const pmo_system *s, const double *pos, double *forces,
             double *energies, double *virial, double *molvirial,
             int virial_mode, int brute) {
  ctx_t c;
  int rc = ctx_init(&c, s, pos, forces, virial_mode), k;
  if (rc) { ctx_free(&c); return rc; }
  if (!forces || !energies) { ctx_free(&c); return PMO_EBADARG; }
  if (brute) {
    int i, j;
    for (i = 0; i < s->n; i++)
      for (j = i + 1; j < s->n; j++) one_pair(&c, i, j);
  } else {
    rc = walk_cells(&c);
  }
  energies[0] += c.e_coul;
  energies[1] += c.e_lj;
  if (virial && virial_mode >= 1)
    for (k = 0; k < 9; k++) virial[k] += c.vir[k];
  if (molvirial && virial_mode >= 2)
    for (k = 0; k < 9; k++) molvirial[k] += c.mvir[k];
  ctx_free(&c);
  return rc;
}

/* NonbondedFullEwaldSystemForce::initialize, the constants the real-space
 * term uses (force/nonbonded/NonbondedFullEwaldSystemForce.h:586-598):
 * default alpha sqrt(pi) (5.5 N / V^2)^(1/6), V = |(e1 x e2) . e3|
 * (topology/PeriodicBoundaryConditions.cpp:40), rc = sqrt(-log(accuracy)) /
 * alpha, 2 alpha / sqrt(pi). */
int pmo_ewald_constants(const pmo_system *s, double alpha, double accuracy,
                        double out[4]) {
  double v, p;
  if (!s || !out || !(accuracy > 0.0) || !(accuracy < 1.0)) return PMO_EBADARG;
  v = fabs((s->box[0] * s->box[1]) * s->box[2]);
  if (alpha <= 0.0) alpha = sqrt(M_PI) * pow(5.5 * (unsigned)s->n / (v * v), 1.0 / 6.0);
  p = -log(accuracy);
  out[0] = alpha;
  out[1] = sqrt(p) / alpha;
  out[2] = 2.0 * alpha / sqrt(M_PI);
  out[3] = alpha * alpha;
  return PMO_OK;
}

static int ewald_setup(ctx_t *c, const pmo_system *s, double alpha, double accuracy,
                       int exact_erfc) {
  double k[4];
  int a;
  if (pmo_ewald_constants(s, alpha, accuracy, k)) return PMO_EBADARG;
  for (a = 0; a < 3; a++)
    if (fabs(s->box[a]) < 2.0 * k[1]) return PMO_EBADARG; /* lattice images */
  c->form = exact_erfc ? 2 : 1;
  c->ew_alpha = k[0];
  c->ew_rc2 = k[1] * k[1];
  c->ew_2api = k[2];
  c->ew_alpha2 = k[3];
  c->walk_cut = k[1];
  return PMO_OK;
}

int pmo_eval_ewald_real(const pmo_system *s, double alpha, double accuracy,
                        int exact_erfc, const double *pos, double *forces,
                        double *energies, double *virial, double *molvirial,
                        int virial_mode, int brute) {
  ctx_t c;
  int rc = ctx_init(&c, s, pos, forces, virial_mode), k;
  if (!rc) rc = ewald_setup(&c, s, alpha, accuracy, exact_erfc);
  if (rc) { ctx_free(&c); return rc; }
  if (!forces || !energies) { ctx_free(&c); return PMO_EBADARG; }
  if (brute) {
    int i;
    for (i = 0; i < s->n; i++) ewald_atom(&c, i, i + 1 < s->n ? i + 1 : -1, NULL);
  } else {
    rc = walk_cells(&c);
  }
  energies[0] += c.e_coul;
  if (virial && virial_mode >= 1)
    for (k = 0; k < 9; k++) virial[k] += c.vir[k];
  if (molvirial && virial_mode >= 2)
    for (k = 0; k < 9; k++) molvirial[k] += c.mvir[k];
  ctx_free(&c);
  return rc;
}

long long pmo_count_pairs_ewald(const pmo_system *s, double alpha, double accuracy,
                                const double *pos) {
  ctx_t c;
  long long n;
  if (ctx_init(&c, s, pos, NULL, 0) || ewald_setup(&c, s, alpha, accuracy, 1)) {
    ctx_free(&c);
    return -1;
  }
  c.count_only = 1;
  if (walk_cells(&c)) { ctx_free(&c); return -1; }
  n = c.pairs;
  ctx_free(&c);
  return n;
}

long long pmo_count_pairs(const pmo_system *s, const double *pos) {
  ctx_t c;
  long long n;
  if (ctx_init(&c, s, pos, NULL, 0)) { ctx_free(&c); return -1; }
  c.count_only = 1;
  if (walk_cells(&c)) { ctx_free(&c); return -1; }
  n = c.pairs;
  ctx_free(&c);
  return n;
}

/* LeapfrogIntegrator::run / doKickdoDrift without modifiers
 * (integrator/leapfrog/LeapfrogIntegrator.cpp:58-105): h = dt *
 * INV_TIMEFACTOR, v += F h / m, x += v h. */
int pmo_leapfrog(const pmo_system *s, double *pos, double *vel,
                 const double *mass, double dt_fs, int nsteps,
                 double *energies) {
  const double h = dt_fs * PMO_INV_TIMEFACTOR;
  const int n = s->n;
  double *f = (double *)calloc((size_t)3 * (size_t)(n > 0 ? n : 1), sizeof(double));
  double e[2] = {0.0, 0.0};
  int step, i, k, rc;
  if (!f) return PMO_ENOMEM;
  rc = pmo_eval(s, pos, f, e, NULL, NULL, 0, 0);
  for (step = 0; step < nsteps && !rc; step++) {
    double kick = step == 0 ? 0.5 * h : h;
    for (i = 0; i < n; i++)
      for (k = 0; k < 3; k++) vel[3 * i + k] += f[3 * i + k] * kick / mass[i];
    for (i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
    for (i = 0; i < 3 * n; i++) f[i] = 0.0;
    e[0] = e[1] = 0.0;
    rc = pmo_eval(s, pos, f, e, NULL, NULL, 0, 0);
  }
  for (i = 0; i < n; i++)
    for (k = 0; k < 3; k++) vel[3 * i + k] += f[3 * i + k] * 0.5 * h / mass[i];
  if (energies) { energies[0] = e[0]; energies[1] = e[1]; }
  free(f);
  return rc;
}

/* ---------------------------------------------------------------------- */
/* SETTLE for one water: canonical triangle O (0, ra, 0), H1 (-rc, -rb, 0),
 * H2 (rc, -rb, 0) about the centre of mass; the new orientation is found in
 * the frame whose z axis is normal to the old molecular plane. */
static void cross3(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static void unit3(double a[3]) {
  double r = sqrt(dot3(a, a));
  a[0] /= r; a[1] /= r; a[2] /= r;
}

static void settle_one(double mo, double mh, double doh, double dhh,
                       const double *A0, const double *B0, const double *C0,
                       double *A1, double *B1, double *C1) {
  const double M = mo + 2.0 * mh;
  const double rc = 0.5 * dhh;
  const double t = sqrt(doh * doh - rc * rc);
  const double ra = 2.0 * mh * t / M, rb = t - ra;
  double com[3], a1[3], b1[3], c1[3], b0[3], c0[3], ex[3], ey[3], ez[3];
  int k;
  for (k = 0; k < 3; k++) {
    com[k] = (mo * A1[k] + mh * B1[k] + mh * C1[k]) / M;
    a1[k] = A1[k] - com[k];
    b1[k] = B1[k] - com[k];
    c1[k] = C1[k] - com[k];
    b0[k] = B0[k] - A0[k];
    c0[k] = C0[k] - A0[k];
  }
  cross3(b0, c0, ez);
  cross3(a1, ez, ex);
  cross3(ez, ex, ey);
  unit3(ex); unit3(ey); unit3(ez);
  {
    const double xb0 = dot3(ex, b0), yb0 = dot3(ey, b0);
    const double xc0 = dot3(ex, c0), yc0 = dot3(ey, c0);
    const double za1 = dot3(ez, a1);
    const double xb1 = dot3(ex, b1), yb1 = dot3(ey, b1), zb1 = dot3(ez, b1);
    const double xc1 = dot3(ex, c1), yc1 = dot3(ey, c1), zc1 = dot3(ez, c1);
    const double sphi = za1 / ra, cphi = sqrt(1.0 - sphi * sphi);
    const double spsi = (zb1 - zc1) / (2.0 * rc * cphi), cpsi = sqrt(1.0 - spsi * spsi);
    const double ya2 = ra * cphi, xb2 = -rc * cpsi;
    const double t1 = -rb * cphi, t2 = rc * spsi * sphi;
    const double yb2 = t1 - t2, yc2 = t1 + t2;
    /* rotation in the plane that conserves the old orientation's momentum */
    const double al = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
    const double be = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
    const double ga = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
    const double ab = al * al + be * be;
    const double sth = (al * ga - be * sqrt(ab - ga * ga)) / ab, cth = sqrt(1.0 - sth * sth);
    const double xa3 = -ya2 * sth, ya3 = ya2 * cth, za3 = za1;
    const double xb3 = xb2 * cth - yb2 * sth, yb3 = xb2 * sth + yb2 * cth, zb3 = zb1;
    const double xc3 = -xb2 * cth - yc2 * sth, yc3 = -xb2 * sth + yc2 * cth, zc3 = zc1;
    for (k = 0; k < 3; k++) {
      A1[k] = com[k] + xa3 * ex[k] + ya3 * ey[k] + za3 * ez[k];
      B1[k] = com[k] + xb3 * ex[k] + yb3 * ey[k] + zb3 * ez[k];
      C1[k] = com[k] + xc3 * ex[k] + yc3 * ey[k] + zc3 * ez[k];
    }
  }
}

void pmo_settle(int nwater, const int *widx, const double *mass, double doh,
                double dhh, const double *old_pos, double *new_pos) {
  int w;
  if (nwater <= 0) return;
  for (w = 0; w < nwater; w++) {
    const int a = widx[3 * w], b = widx[3 * w + 1], c = widx[3 * w + 2];
    settle_one(mass[widx[0]], mass[widx[1]], doh, dhh, old_pos + 3 * a, old_pos + 3 * b,
               old_pos + 3 * c, new_pos + 3 * a, new_pos + 3 * b, new_pos + 3 * c);
  }
}

int pmo_leapfrog_rigid(const pmo_system *s, double *pos, double *vel,
                       const double *mass, double dt_fs, int nsteps, int nwater,
                       const int *widx, double doh, double dhh,
                       double *energies) {
  const double h = dt_fs * PMO_INV_TIMEFACTOR;
  const int n = s->n;
  double *f = (double *)calloc((size_t)3 * (size_t)(n > 0 ? n : 1), sizeof(double));
  double *old = (double *)malloc(sizeof(double) * (size_t)3 * (size_t)(n > 0 ? n : 1));
  double e[2] = {0.0, 0.0};
  int step, i, k, rc;
  if (!f || !old) { free(f); free(old); return PMO_ENOMEM; }
  rc = pmo_eval(s, pos, f, e, NULL, NULL, 0, 0);
  for (step = 0; step < nsteps && !rc; step++) {
    double kick = step == 0 ? 0.5 * h : h;
    for (i = 0; i < 3 * n; i++) old[i] = pos[i];
    for (i = 0; i < n; i++)
      for (k = 0; k < 3; k++) vel[3 * i + k] += f[3 * i + k] * kick / mass[i];
    for (i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
    pmo_settle(nwater, widx, mass, doh, dhh, old, pos);
    for (i = 0; i < nwater; i++)
      for (k = 0; k < 3; k++) {
        const int a = widx[3 * i + k];
        vel[3 * a] = (pos[3 * a] - old[3 * a]) / h;
        vel[3 * a + 1] = (pos[3 * a + 1] - old[3 * a + 1]) / h;
        vel[3 * a + 2] = (pos[3 * a + 2] - old[3 * a + 2]) / h;
      }
    for (i = 0; i < 3 * n; i++) f[i] = 0.0;
    e[0] = e[1] = 0.0;
    rc = pmo_eval(s, pos, f, e, NULL, NULL, 0, 0);
  }
  for (i = 0; i < n; i++)
    for (k = 0; k < 3; k++) vel[3 * i + k] += f[3 * i + k] * 0.5 * h / mass[i];
  if (energies) { energies[0] = e[0]; energies[1] = e[1]; }
  free(f);
  free(old);
  return rc;
}
