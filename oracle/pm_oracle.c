/*
 * CPU oracle (test infrastructure only) -- plain-C FP64 restatement of ProtoMol 3's
 * nonbonded cutoff and particle-mesh-Ewald force path.  Each function names the reference
 * file:line it follows (paths relative to the ProtoMol 3 tree).  Nothing in the product links
 * this file; tests/ and bench.py's cpu_baseline load it as the checker.
 */
#include "pm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Constants: base/PMConstants.cpp:53-54, :67. */
static const double INV_TIMEFACTOR = 0.02045482828087295;

/* ---------------------------------------------------------------------------------------------
 * Periodic boundary conditions (topology/PeriodicBoundaryConditions.h:72-110, .cpp:32-77).
 * ------------------------------------------------------------------------------------------ */
typedef struct {
  double L[3], Lr[3], H[3], H2[3], D;
} pbc_t;

static void pbc_init(pbc_t *b, const double box[3], const double origin[3]) {
  /* myMin/myMax from origin -+ (e1+e2+e3)/2, myH = max - min, myD = min((Li/2)^2). */
  for (int k = 0; k < 3; k++) {
    double lo = origin[k] - box[k] * 0.5, hi = origin[k] + box[k] * 0.5;
    b->L[k] = box[k];
    b->Lr[k] = 1.0 / box[k];
    b->H[k] = hi - lo;
    b->H2[k] = b->H[k] * 0.5;
  }
  double dx = (box[0] * 0.5) * (box[0] * 0.5), dy = (box[1] * 0.5) * (box[1] * 0.5),
         dz = (box[2] * 0.5) * (box[2] * 0.5);
  b->D = fmin(dx, fmin(dy, dz));
}

/* minimalDifference(c1, c2, distSquared): diff = c2 - c1, single wrap, then rint. */
static double min_diff(const pbc_t *b, const double *c1, const double *c2, double d[3]) {
  for (int k = 0; k < 3; k++) d[k] = c2[k] - c1[k];
  double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  if (r2 > b->D) {
    for (int k = 0; k < 3; k++) {
      if (d[k] < -b->H2[k]) d[k] += b->H[k];
      else if (d[k] > b->H2[k]) d[k] -= b->H[k];
    }
    r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 > b->D) {
      for (int k = 0; k < 3; k++) d[k] -= b->L[k] * rint(b->Lr[k] * d[k]);
      r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    }
  }
  return r2;
}

static void add_virial(double *v, const double f[3], const double d[3]) {
  /* ScalarStructure::addVirial (type/ScalarStructure.cpp:36-53). */
  if (!v) return;
  double xy = f[0] * d[1], xz = f[0] * d[2], yz = f[1] * d[2];
  v[0] += f[0] * d[0]; v[1] += xy; v[2] += xz;
  v[3] += xy; v[4] += f[1] * d[1]; v[5] += yz;
  v[6] += xz; v[7] += yz; v[8] += f[2] * d[2];
}

/* ---------------------------------------------------------------------------------------------
 * Exclusions (topology/ExclusionTable.h:116-131): per-atom sorted partner lists.
 * ------------------------------------------------------------------------------------------ */
typedef struct {
  int *start, *partner, *kind;
} excl_t;

static void excl_build(excl_t *e, const orc_system *s) {
  int n = s->n;
  e->start = (int *)calloc((size_t)n + 1, sizeof(int));
  e->partner = (int *)malloc(sizeof(int) * (size_t)(2 * s->nexcl + 1));
  e->kind = (int *)malloc(sizeof(int) * (size_t)(2 * s->nexcl + 1));
  for (int k = 0; k < s->nexcl; k++) {
    e->start[s->excl_pairs[2 * k] + 1]++;
    e->start[s->excl_pairs[2 * k + 1] + 1]++;
  }
  for (int i = 0; i < n; i++) e->start[i + 1] += e->start[i];
  int *fill = (int *)calloc((size_t)n, sizeof(int));
  for (int k = 0; k < s->nexcl; k++) {
    int a = s->excl_pairs[2 * k], b = s->excl_pairs[2 * k + 1];
    e->partner[e->start[a] + fill[a]] = b; e->kind[e->start[a] + fill[a]++] = s->excl_kind[k];
    e->partner[e->start[b] + fill[b]] = a; e->kind[e->start[b] + fill[b]++] = s->excl_kind[k];
  }
  free(fill);
}

static int excl_check(const excl_t *e, int i, int j) {
  for (int k = e->start[i]; k < e->start[i + 1]; k++)
    if (e->partner[k] == j) return e->kind[k];
  return 0;
}

static void excl_free(excl_t *e) { free(e->start); free(e->partner); free(e->kind); }

/* ---------------------------------------------------------------------------------------------
 * Switching functions: C1 (switch/C1SwitchingFunction.h:41-50, .cpp:12-16),
 * C2 (switch/C2SwitchingFunction.h:42-53, .cpp:12-18), Cutoff (CutoffSwitchingFunction.h:41-44).
 * ------------------------------------------------------------------------------------------ */
typedef struct {
  int kind;
  double rc, rc2, ron2, s1, s2, s3, c15_1, c05_3, c15_3;
} sw_t;

static void sw_init(sw_t *w, int kind, double switchon, double cutoff) {
  w->kind = kind;
  w->rc = cutoff;
  w->rc2 = cutoff * cutoff;
  w->ron2 = switchon * switchon;
  double d = cutoff * cutoff - switchon * switchon;
  w->s1 = 1.0 / (d * d * d);
  w->s2 = cutoff * cutoff - 3.0 * switchon * switchon;
  w->s3 = 4.0 / (d * d * d);
  w->c15_1 = 1.5 / cutoff;
  w->c05_3 = 0.5 / (cutoff * cutoff * cutoff);
  w->c15_3 = 1.5 / (cutoff * cutoff * cutoff);
}

static void sw_eval(const sw_t *w, double r2, double *val, double *deriv) {
  if (w->kind == ORC_SWITCH_C2) {
    *deriv = 0.0;
    if (r2 > w->rc2) *val = 0.0;
    else if (r2 >= w->ron2) {
      double c2 = w->rc2 - r2;
      double c4 = c2 * (w->s2 + 2.0 * r2);
      *val = w->s1 * (c2 * c4);
      *deriv = w->s3 * (c2 * c2 - c4);
    } else *val = 1.0;
  } else if (w->kind == ORC_SWITCH_C1) {
    if (r2 > w->rc2) { *val = 0.0; *deriv = 0.0; return; }
    double dist = sqrt(r2);
    *val = 1.0 - dist * (w->c15_1 - r2 * w->c05_3);
    *deriv = -w->c15_1 / dist + dist * w->c15_3;
  } else {
    *deriv = 0.0;
    *val = (r2 > w->rc2 ? 0.0 : 1.0);
  }
}

/* Abramowitz & Stegun 7.1.26 polynomial (base/MathUtilities.cpp:39-49). */
static double poly5(double ar) {
  const double E1 = 0.254829592, E2 = -0.284496736, E3 = 1.421413741, E4 = -1.453152027,
               E5 = 1.061405429, PP = 0.3275911;
  double t = 1.0 / (1.0 + PP * ar);
  return t * (E1 + t * (E2 + t * (E3 + t * (E4 + t * E5))));
}

/* ---------------------------------------------------------------------------------------------
 * Unordered-pair enumeration with a periodic cell grid (cells >= cutoff).  Visits every pair
 * i<j whose minimal-image distance can be within the cutoff exactly once, which is the pair set
 * the reference's CellListEnumerator + NonbondedCutoffForce::doEvaluate produce
 * (topology/CellListEnumeratorPeriodicBoundaries.h:25-134, force/nonbonded/NonbondedCutoffForce.h:37-54).
 * ------------------------------------------------------------------------------------------ */
typedef void (*pair_fn)(void *ctx, int i, int j);

static void for_each_pair(const orc_system *s, const double *pos, double cutoff, pair_fn fn,
                          void *ctx) {
  int nc[3], brute = 0;
  for (int k = 0; k < 3; k++) {
    nc[k] = (int)floor(s->box[k] / cutoff);
    if (nc[k] < 3) brute = 1;
  }
  int n = s->n;
  if (brute || n < 64) {
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) fn(ctx, i, j);
    return;
  }
  int ncell = nc[0] * nc[1] * nc[2];
  int *head = (int *)malloc(sizeof(int) * (size_t)ncell), *next = (int *)malloc(sizeof(int) * (size_t)n);
  int *cell = (int *)malloc(sizeof(int) * (size_t)n);
  for (int c = 0; c < ncell; c++) head[c] = -1;
  for (int i = n - 1; i >= 0; i--) {
    int ci[3];
    for (int k = 0; k < 3; k++) {
      double u = pos[3 * i + k] / s->box[k];
      u -= floor(u);
      ci[k] = (int)(u * nc[k]);
      if (ci[k] >= nc[k]) ci[k] = nc[k] - 1;
      if (ci[k] < 0) ci[k] = 0;
    }
    int c = (ci[0] * nc[1] + ci[1]) * nc[2] + ci[2];
    cell[i] = c;
    next[i] = head[c];
    head[c] = i;
  }
  for (int cx = 0; cx < nc[0]; cx++)
    for (int cy = 0; cy < nc[1]; cy++)
      for (int cz = 0; cz < nc[2]; cz++) {
        int c = (cx * nc[1] + cy) * nc[2] + cz;
        for (int dx = -1; dx <= 1; dx++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dz = -1; dz <= 1; dz++) {
              int ox = (cx + dx + nc[0]) % nc[0], oy = (cy + dy + nc[1]) % nc[1],
                  oz = (cz + dz + nc[2]) % nc[2];
              int c2 = (ox * nc[1] + oy) * nc[2] + oz;
              for (int i = head[c]; i != -1; i = next[i])
                for (int j = head[c2]; j != -1; j = next[j])
                  if (i < j) fn(ctx, i, j);
            }
      }
  free(head); free(next); free(cell);
}

/* ---------------------------------------------------------------------------------------------
 * Cutoff LJ + Coulomb (force/OneAtomPairTwo.h:30-96, force/LennardJonesForce.h:28-60,
 * force/CoulombForce.h:29-40).
 * ------------------------------------------------------------------------------------------ */
typedef struct {
  const orc_system *s;
  const double *pos;
  const orc_cutoff_params *p;
  pbc_t b;
  excl_t ex;
  sw_t swl, swc;
  double cut2;
  double *f, elj, ecoul, *vir;
} cut_ctx;

static void cut_pair(void *vc, int i, int j) {
  cut_ctx *c = (cut_ctx *)vc;
  const orc_system *s = c->s;
  double d[3];
  double r2 = min_diff(&c->b, c->pos + 3 * i, c->pos + 3 * j, d);
  if (r2 > c->cut2) return;
  int ex = (s->molecule[i] == s->molecule[j]) ? excl_check(&c->ex, i, j) : 0;
  if (ex == 2) return;
  double rd2 = 1.0 / r2;
  double f1 = 0.0, e1 = 0.0, f2 = 0.0, e2 = 0.0, val, der;
  if (c->p->do_lj) {
    const double *lj = s->lj + 4 * (s->type[i] * s->ntypes + s->type[j]);
    double A = (ex != 1) ? lj[0] : lj[2], B = (ex != 1) ? lj[1] : lj[3];
    double r6 = rd2 * rd2 * rd2, r12 = r6 * r6, r6B = B * r6, r12A = A * r12;
    e1 = r12A - r6B;
    f1 = 12.0 * r12A * rd2 - 6.0 * r6B * rd2;
    sw_eval(&c->swl, r2, &val, &der);
    f1 = f1 * val - e1 * der;
    e1 = e1 * val;
  }
  if (c->p->do_coul) {
    e2 = s->charge[i] * s->charge[j] * sqrt(rd2);
    if (ex == 1) e2 *= s->coulomb_scaling;
    f2 = e2 * rd2;
    sw_eval(&c->swc, r2, &val, &der);
    f2 = f2 * val - e2 * der;
    e2 = e2 * val;
  }
  c->elj += e1;
  c->ecoul += e2;
  double ft = f1 + f2, fij[3] = {d[0] * ft, d[1] * ft, d[2] * ft};
  for (int k = 0; k < 3; k++) {
    c->f[3 * i + k] -= fij[k];
    c->f[3 * j + k] += fij[k];
  }
  add_virial(c->vir, fij, d);
}

int orc_cutoff(const orc_system *s, const double *pos, const orc_cutoff_params *p,
               double *forces, double *energies, double *virial) {
  cut_ctx c;
  memset(&c, 0, sizeof(c));
  c.s = s; c.pos = pos; c.p = p; c.f = forces; c.vir = virial;
  double zero[3] = {0, 0, 0};
  pbc_init(&c.b, s->box, zero);
  excl_build(&c.ex, s);
  sw_init(&c.swl, p->lj_switch, p->lj_switchon, p->lj_cutoff);
  sw_init(&c.swc, p->coul_switch, p->coul_switchon, p->coul_cutoff);
  double rc = 0.0;
  if (p->do_lj) rc = fmax(rc, p->lj_cutoff);
  if (p->do_coul) rc = fmax(rc, p->coul_cutoff);
  c.cut2 = rc * rc;
  for_each_pair(s, pos, rc, cut_pair, &c);
  energies[ORC_E_LJ] += c.elj;
  energies[ORC_E_COULOMB] += c.ecoul;
  excl_free(&c.ex);
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Complex FFT (mixed radix, unnormalised, in place on strided lines).  Stands in for the
 * reference's ZFFT backend (mdl/interface/force/nonbonded/fft.c); the PME energies and forces
 * do not depend on the transform sign because the influence function is even in m.
 * ------------------------------------------------------------------------------------------ */
static void fft_line(double *re, double *im, int n, int sign, double *tr, double *ti) {
  /* Recursive decimation-in-time on a contiguous copy. */
  if (n == 1) return;
  int p = 2;
  while (n % p) p++;
  int m = n / p;
  /* split into p decimated subsequences */
  for (int r = 0; r < p; r++)
    for (int k = 0; k < m; k++) {
      tr[r * m + k] = re[k * p + r];
      ti[r * m + k] = im[k * p + r];
    }
  memcpy(re, tr, sizeof(double) * (size_t)n);
  memcpy(im, ti, sizeof(double) * (size_t)n);
  for (int r = 0; r < p; r++) fft_line(re + r * m, im + r * m, m, sign, tr, ti);
  for (int k = 0; k < m; k++) {
    double xr[64], xi[64];
    for (int r = 0; r < p; r++) {
      double a = sign * 2.0 * M_PI * (double)r * (double)k / (double)n;
      double c = cos(a), sn = sin(a);
      double yr = re[r * m + k], yi = im[r * m + k];
      xr[r] = yr * c - yi * sn;
      xi[r] = yr * sn + yi * c;
    }
    for (int q = 0; q < p; q++) {
      double sr = 0, si = 0;
      for (int r = 0; r < p; r++) {
        double a = sign * 2.0 * M_PI * (double)((r * q) % p) / (double)p;
        double c = cos(a), sn = sin(a);
        sr += xr[r] * c - xi[r] * sn;
        si += xr[r] * sn + xi[r] * c;
      }
      tr[k + q * m] = sr;
      ti[k + q * m] = si;
    }
  }
  memcpy(re, tr, sizeof(double) * (size_t)n);
  memcpy(im, ti, sizeof(double) * (size_t)n);
}

static void fft3d(double *re, double *im, int nx, int ny, int nz, int sign) {
  int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  double *lr = (double *)malloc(sizeof(double) * (size_t)nmax * 4);
  double *li = lr + nmax, *tr = li + nmax, *ti = tr + nmax;
  /* z lines */
  for (int i = 0; i < nx * ny; i++) fft_line(re + (size_t)i * nz, im + (size_t)i * nz, nz, sign, tr, ti);
  /* y lines */
  for (int i = 0; i < nx; i++)
    for (int k = 0; k < nz; k++) {
      for (int j = 0; j < ny; j++) {
        size_t a = ((size_t)i * ny + j) * nz + k;
        lr[j] = re[a]; li[j] = im[a];
      }
      fft_line(lr, li, ny, sign, tr, ti);
      for (int j = 0; j < ny; j++) {
        size_t a = ((size_t)i * ny + j) * nz + k;
        re[a] = lr[j]; im[a] = li[j];
      }
    }
  /* x lines */
  for (int j = 0; j < ny; j++)
    for (int k = 0; k < nz; k++) {
      for (int i = 0; i < nx; i++) {
        size_t a = ((size_t)i * ny + j) * nz + k;
        lr[i] = re[a]; li[i] = im[a];
      }
      fft_line(lr, li, nx, sign, tr, ti);
      for (int i = 0; i < nx; i++) {
        size_t a = ((size_t)i * ny + j) * nz + k;
        re[a] = lr[i]; im[a] = li[i];
      }
    }
  free(lr);
}

/* ---------------------------------------------------------------------------------------------
 * B-spline weights (mdl/interface/force/nonbonded/BSpline.cpp:55-105).
 * ------------------------------------------------------------------------------------------ */
static void bspline(int p, double w, double *th, double *dth) {
  if (p == 1) { th[0] = 1; dth[0] = 0; return; }
  if (p == 2) { th[1] = w; th[0] = 1.0 - w; dth[1] = 1; dth[0] = -1; return; }
  th[p - 1] = 0.0;
  th[1] = w;
  th[0] = 1.0 - w;
  for (int k = 2; k < p - 1; k++) {
    double div = 1.0 / k;
    th[k] = div * w * th[k - 1];
    for (int j = 1; j < k; j++)
      th[k - j] = div * ((w + j) * th[k - j - 1] + ((double)(k + 1 - j) - w) * th[k - j]);
    th[0] = div * (1 - w) * th[0];
  }
  dth[0] = -th[0];
  for (int j = 1; j <= p - 1; j++) dth[j] = th[j - 1] - th[j];
  double div = 1.0 / (p - 1.0);
  th[p - 1] = div * w * th[p - 2];
  for (int j = 1; j < p - 1; j++)
    th[p - 1 - j] = div * ((w + j) * th[p - j - 2] + ((double)(p - j) - w) * th[p - 1 - j]);
  th[0] = div * (1 - w) * th[0];
}

double orc_pme_alpha(double rc, double accuracy) {
  /* NonbondedPMEwaldSystemForce.h:520-537. */
  double alpha = 1.0;
  while (erfc(alpha * rc) / rc >= accuracy) alpha *= 2.0;
  double low = 0.0, high = alpha;
  for (int i = 0; i < 100; ++i) {
    alpha = 0.5 * (low + high);
    if (erfc(alpha * rc) / rc >= accuracy) low = alpha;
    else high = alpha;
  }
  return alpha;
}

/* ---------------------------------------------------------------------------------------------
 * PME (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h, Grid.h).
 * ------------------------------------------------------------------------------------------ */
typedef struct {
  const orc_system *s;
  const double *pos;
  pbc_t b;
  excl_t ex;
  sw_t sw;
  double alpha, a2pi, rc2;
  int nlat;
  double *lat;
  double *f, ereal, *vir;
} real_ctx;

/* realTerm inner body for one (i, j) visit (NonbondedPMEwaldSystemForce.h:644-700). */
static void real_pair(real_ctx *c, int i, int j, double *fi) {
  const orc_system *s = c->s;
  double dmin[3];
  /* two-argument minimalDifference: same wrapping, distance not returned */
  min_diff(&c->b, c->pos + 3 * i, c->pos + 3 * j, dmin);
  int ex = (s->molecule[i] == s->molecule[j]) ? excl_check(&c->ex, i, j) : 0;
  if (i == j) ex = 2;
  double qi = s->charge[i], qj = s->charge[j];
  for (int k = 0; k < c->nlat; k++) {
    if (ex == 2) { ex = 0; continue; }
    double rij[3] = {dmin[0] + c->lat[3 * k], dmin[1] + c->lat[3 * k + 1], dmin[2] + c->lat[3 * k + 2]};
    double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
    if (r2 > c->rc2) continue;
    double r = sqrt(r2);
    double qq = qi * qj;
    if (ex == 1) qq *= s->coulomb_scaling;
    double rr = 1.0 / r, ar = c->alpha * r;
    double e = qq * exp(-ar * ar);
    double energy = poly5(ar) * e * rr;
    double force = (energy + c->a2pi * e) * rr * rr;
    double val, der;
    sw_eval(&c->sw, r2, &val, &der);
    force = force * val - energy * der;
    energy = energy * val;
    c->ereal += energy;
    double fij[3] = {rij[0] * force, rij[1] * force, rij[2] * force};
    for (int q = 0; q < 3; q++) {
      fi[q] -= fij[q];
      c->f[3 * j + q] += fij[q];
    }
    add_virial(c->vir, fij, rij);
    ex = 0;
  }
}

static void real_pair_cb(void *vc, int i, int j) {
  real_ctx *c = (real_ctx *)vc;
  double fi[3] = {0, 0, 0};
  real_pair(c, i, j, fi);
  for (int q = 0; q < 3; q++) c->f[3 * i + q] += fi[q];
}

/* PeriodicBoundaryConditions::buildLatticeVectors (PeriodicBoundaryConditions.cpp:79-106),
 * with (0,0,0) prepended (NonbondedPMEwaldSystemForce.h:577-578). */
static int build_lattice(const double box[3], double rc, double **out) {
  int bk = (int)floor(rc / box[0] + 1.0), bl = (int)floor(rc / box[1] + 1.0),
      bm = (int)floor(rc / box[2] + 1.0);
  int cap = (2 * bk + 1) * (2 * bl + 1) * (2 * bm + 1) + 1;
  double *v = (double *)malloc(sizeof(double) * 3 * (size_t)cap);
  double *nn = (double *)malloc(sizeof(double) * (size_t)cap);
  int cnt = 0;
  for (int k = -bk; k <= bk; k++)
    for (int l = -bl; l <= bl; l++)
      for (int m = -bm; m <= bm; m++)
        if (k || l || m) {
          double c[3] = {box[0] * k, box[1] * l, box[2] * m};
          double nrm = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
          if (nrm <= 2 * rc) {
            memcpy(v + 3 * cnt, c, sizeof(c));
            nn[cnt++] = nrm * nrm;
          }
        }
  /* stable insertion sort by squared norm */
  for (int a = 1; a < cnt; a++)
    for (int b2 = a; b2 > 0 && nn[b2] < nn[b2 - 1]; b2--) {
      double t = nn[b2]; nn[b2] = nn[b2 - 1]; nn[b2 - 1] = t;
      for (int q = 0; q < 3; q++) { t = v[3 * b2 + q]; v[3 * b2 + q] = v[3 * b2 - 3 + q]; v[3 * b2 - 3 + q] = t; }
    }
  double *o = (double *)malloc(sizeof(double) * 3 * (size_t)(cnt + 1));
  o[0] = o[1] = o[2] = 0.0;
  memcpy(o + 3, v, sizeof(double) * 3 * (size_t)cnt);
  free(v); free(nn);
  *out = o;
  return cnt + 1;
}

static void dftmod(int order, int n, const double *th, double *mod) {
  /* Grid::dftmod (Grid.h:588-600) */
  for (int i = 0; i < n; i++) {
    double sc = 0.0, ss = 0.0;
    for (int j = 0; j < order; j++) {
      double x = M_PI * 2.0 * i * j / (double)n;
      sc += th[j] * cos(x);
      ss += th[j] * sin(x);
    }
    mod[i] = 1.0 / (sc * sc + ss * ss);
  }
}

static double pme_recip(const orc_system *s, const double *pos, const orc_pme_params *p,
                        double alpha, double *forces, double *virial) {
  int nx = p->nx, ny = p->ny, nz = p->nz, P = p->order, n = s->n;
  double Lx = s->box[0], Ly = s->box[1], Lz = s->box[2];
  size_t K = (size_t)nx * ny * nz;
  double *re = (double *)calloc(K, sizeof(double)), *im = (double *)calloc(K, sizeof(double));
  /* Grid::initialize (Grid.h:498-586) */
  int offx = -(P - 1) / 2 + nx, offy = -(P - 1) / 2 + ny, offz = -(P - 1) / 2 + nz;
  double hxr = nx / Lx, hyr = ny / Ly, hzr = nz / Lz;
  double V = Lx * Ly * Lz, fac = M_PI * M_PI / (alpha * alpha);
  double *ex = (double *)malloc(sizeof(double) * (size_t)(nx + ny + nz));
  double *ey = ex + nx, *ez = ey + ny;
  for (int i = 0; i < nx; i++) { int i0 = i <= nx / 2 ? i : i - nx; double m = i0 * (1.0 / Lx); ex[i] = exp(-fac * (m * m)); }
  for (int j = 0; j < ny; j++) { int j0 = j <= ny / 2 ? j : j - ny; double m = j0 * (1.0 / Ly); ey[j] = exp(-fac * (m * m)); }
  for (int k = 0; k <= nz / 2; k++) { double m = k * (1.0 / Lz); ez[k] = exp(-fac * (m * m)); }
  double *modx = (double *)malloc(sizeof(double) * (size_t)(nx + ny + nz));
  double *mody = modx + nx, *modz = mody + ny;
  double th0[32], dth0[32];
  bspline(P, 0.0, th0, dth0);
  dftmod(P, nx, th0, modx);
  dftmod(P, ny, th0, mody);
  dftmod(P, nz, th0, modz);
  /* anterpolateCharge (Grid.h:107-154) */
  int *base = (int *)malloc(sizeof(int) * 3 * (size_t)n);
  double *th = (double *)malloc(sizeof(double) * 6 * (size_t)P * (size_t)n);
  for (int a = 0; a < n; a++) {
    double u[3] = {pos[3 * a] * hxr, pos[3 * a + 1] * hyr, pos[3 * a + 2] * hzr};
    int nn[3] = {nx, ny, nz}, off[3] = {offx, offy, offz};
    for (int d = 0; d < 3; d++) {
      while (u[d] < 0.0) u[d] += nn[d];
      while (u[d] >= nn[d]) u[d] -= nn[d];
      int iu = (int)u[d];
      base[3 * a + d] = iu + off[d];
      bspline(P, u[d] - iu, th + (size_t)(6 * a + 2 * d) * P, th + (size_t)(6 * a + 2 * d + 1) * P);
    }
    double q = s->charge[a];
    const double *tx = th + (size_t)(6 * a) * P, *ty = th + (size_t)(6 * a + 2) * P, *tz = th + (size_t)(6 * a + 4) * P;
    for (int i = 0; i < P; i++) {
      double aa = q * tx[i];
      int i1 = (i + base[3 * a]) % nx;
      for (int j = 0; j < P; j++) {
        double ab = aa * ty[j];
        int j1 = (j + base[3 * a + 1]) % ny;
        for (int k = 0; k < P; k++) {
          int k1 = (k + base[3 * a + 2]) % nz;
          re[((size_t)i1 * ny + j1) * nz + k1] += ab * tz[k];
        }
      }
    }
  }
  fft3d(re, im, nx, ny, nz, +1);
  /* scalarSum (Grid.h:236-341) */
  double energy = 0.0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  double piVr = 1.0 / (M_PI * V);
  for (int i = 0; i < nx; i++) {
    int i0 = i <= nx / 2 ? i : i - nx;
    double mi = i0 * (1.0 / Lx), exi = ex[i] * piVr;
    for (int j = 0; j < ny; j++) {
      int j0 = j <= ny / 2 ? j : j - ny;
      double modxy = modx[i] * mody[j], mj = j0 * (1.0 / Ly), mij = mi * mi + mj * mj;
      double exy = exi * ey[j];
      for (int k = (i != 0 || j != 0 ? 0 : 1); k <= nz / 2; k++) {
        double mk = k * (1.0 / Lz), m2 = mij + mk * mk;
        double theta = modxy * modz[k] * exy * ez[k] / m2;
        size_t a = ((size_t)i * ny + j) * nz + k;
        double q = re[a] * re[a] + im[a] * im[a];
        double e = q * theta, v = 2.0 * (1.0 / m2 + fac);
        if (k > 0 && ((k != nz / 2) || (nz & 1))) {
          e *= 2.0;
          size_t w = ((size_t)((nx - i) % nx) * ny + (ny - j) % ny) * nz + (nz - k) % nz;
          re[w] *= theta;
          im[w] *= theta;
        }
        energy += e;
        vxx += e * (1.0 - v * mi * mi); vxy -= e * (v * mi * mj); vxz -= e * (v * mi * mk);
        vyy += e * (1.0 - v * mj * mj); vyz -= e * (v * mj * mk); vzz += e * (1.0 - v * mk * mk);
        re[a] *= theta;
        im[a] *= theta;
      }
    }
  }
  re[0] = 0.0; im[0] = 0.0;
  if (virial) {
    virial[0] += vxx * 0.5; virial[1] += vxy * 0.5; virial[2] += vxz * 0.5;
    virial[3] += vxy * 0.5; virial[4] += vyy * 0.5; virial[5] += vyz * 0.5;
    virial[6] += vxz * 0.5; virial[7] += vyz * 0.5; virial[8] += vzz * 0.5;
  }
  fft3d(re, im, nx, ny, nz, -1);
  /* interpolateForce (Grid.h:158-189) */
  for (int a = 0; a < n; a++) {
    const double *tx = th + (size_t)(6 * a) * P, *dx = tx + P, *ty = tx + 2 * P, *dy = tx + 3 * P,
                 *tz = tx + 4 * P, *dz = tx + 5 * P;
    double fx = 0, fy = 0, fz = 0;
    for (int i = 0; i < P; i++) {
      int i1 = (i + base[3 * a]) % nx;
      for (int j = 0; j < P; j++) {
        int j1 = (j + base[3 * a + 1]) % ny;
        double xij = dx[i] * ty[j], yij = tx[i] * dy[j], zij = tx[i] * ty[j];
        for (int k = 0; k < P; k++) {
          int k1 = (k + base[3 * a + 2]) % nz;
          double term = re[((size_t)i1 * ny + j1) * nz + k1];
          fx -= term * xij * tz[k];
          fy -= term * yij * tz[k];
          fz -= term * zij * dz[k];
        }
      }
    }
    double q = s->charge[a];
    forces[3 * a] += fx * hxr * q;
    forces[3 * a + 1] += fy * hyr * q;
    forces[3 * a + 2] += fz * hzr * q;
  }
  free(re); free(im); free(ex); free(modx); free(base); free(th);
  return energy * 0.5;
}

int orc_pme(const orc_system *s, const double *pos, const orc_pme_params *p, double *forces,
            double *energies, double *virial, double *alpha_out, double *terms_out) {
  double alpha = p->alpha > 0.0 ? p->alpha : orc_pme_alpha(p->cutoff, p->accuracy);
  if (alpha_out) *alpha_out = alpha;
  double a2pi = 2.0 * alpha / sqrt(M_PI);
  double V = s->box[0] * s->box[1] * s->box[2];
  double intra = 0.0, self = 0.0, charged = 0.0, ereal = 0.0, erecip = 0.0;
  pbc_t b;
  double zero[3] = {0, 0, 0};
  pbc_init(&b, s->box, zero);
  excl_t ex;
  excl_build(&ex, s);
  if (p->do_corr) {
    /* correctionTerm (NonbondedPMEwaldSystemForce.h:874-911) */
    for (int k = 0; k < s->nexcl; k++) {
      int a1 = s->excl_pairs[2 * k], a2 = s->excl_pairs[2 * k + 1];
      double rij[3];
      double r2 = min_diff(&b, pos + 3 * a1, pos + 3 * a2, rij);
      double qq = s->charge[a1] * s->charge[a2];
      if (s->excl_kind[k] == 1) qq *= 1 - s->coulomb_scaling;
      double r = sqrt(r2), rr = 1 / r, e = erf(alpha * r) * rr;
      intra -= qq * e;
      double fs = qq * (a2pi * exp(-alpha * alpha * r2) - e) * rr * rr;
      double fij[3] = {rij[0] * fs, rij[1] * fs, rij[2] * fs};
      for (int q = 0; q < 3; q++) {
        forces[3 * a1 + q] -= fij[q];
        forces[3 * a2 + q] += fij[q];
      }
      add_virial(virial, fij, rij);
    }
    /* self and charged-system terms (NonbondedPMEwaldSystemForce.h:555-575) */
    double q2 = 0.0, q1 = 0.0;
    for (int i = 0; i < s->n; i++) q2 += s->charge[i] * s->charge[i];
    self = -q2 * alpha / sqrt(M_PI);
    for (int i = 0; i < s->n; i++) q1 += s->charge[i];
    if (fabs(q1 * 0.00268283) > 1.0e-5) charged = -M_PI / (2.0 * V * alpha * alpha) * q1 * q1;
    if (virial) { virial[0] += charged; virial[4] += charged; virial[8] += charged; }
  }
  if (p->do_real) {
    real_ctx c;
    memset(&c, 0, sizeof(c));
    c.s = s; c.pos = pos; c.b = b; c.ex = ex; c.alpha = alpha; c.a2pi = a2pi;
    c.rc2 = p->cutoff * p->cutoff; c.f = forces; c.vir = virial;
    sw_init(&c.sw, p->real_switch, 0.0, p->cutoff);
    c.nlat = build_lattice(s->box, p->cutoff, &c.lat);
    if (c.nlat == 1) {
      for_each_pair(s, pos, p->cutoff, real_pair_cb, &c);
    } else {
      for (int i = 0; i < s->n; i++) {
        double fi[3] = {0, 0, 0};
        for (int j = i; j < s->n; j++) real_pair(&c, i, j, fi);
        for (int q = 0; q < 3; q++) forces[3 * i + q] += fi[q];
      }
    }
    ereal = c.ereal;
    free(c.lat);
  }
  if (p->do_recip) erecip = pme_recip(s, pos, p, alpha, forces, virial);
  energies[ORC_E_COULOMB] += ereal + erecip + intra + 0.0 + self + charged;
  if (terms_out) {
    terms_out[0] = ereal; terms_out[1] = erecip; terms_out[2] = intra;
    terms_out[3] = self; terms_out[4] = charged;
  }
  excl_free(&ex);
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Bonds (force/bonded/BondSystemForce.h:78-117) and angles (AngleSystemForce.h:87-172).
 * ------------------------------------------------------------------------------------------ */
int orc_bonded(const orc_system *s, const double *pos, double *forces, double *energies,
               double *virial) {
  pbc_t b;
  double zero[3] = {0, 0, 0};
  pbc_init(&b, s->box, zero);
  for (int k = 0; k < s->nbonds; k++) {
    int a1 = s->bonds[2 * k], a2 = s->bonds[2 * k + 1];
    double r12[3];
    min_diff(&b, pos + 3 * a2, pos + 3 * a1, r12);
    double r = sqrt(r12[0] * r12[0] + r12[1] * r12[1] + r12[2] * r12[2]);
    double dpotdr = 2.0 * s->bond_k[k] * (r - s->bond_r0[k]);
    double f1[3] = {r12[0] * (-dpotdr / r), r12[1] * (-dpotdr / r), r12[2] * (-dpotdr / r)};
    for (int q = 0; q < 3; q++) { forces[3 * a1 + q] += f1[q]; forces[3 * a2 + q] -= f1[q]; }
    energies[ORC_E_BOND] += s->bond_k[k] * (r - s->bond_r0[k]) * (r - s->bond_r0[k]);
    add_virial(virial, f1, r12);
  }
  for (int k = 0; k < s->nangles; k++) {
    int a1 = s->angles[3 * k], a2 = s->angles[3 * k + 1], a3 = s->angles[3 * k + 2];
    double r12[3], r32[3], r13[3];
    min_diff(&b, pos + 3 * a2, pos + 3 * a1, r12);
    min_diff(&b, pos + 3 * a2, pos + 3 * a3, r32);
    min_diff(&b, pos + 3 * a3, pos + 3 * a1, r13);
    double d12 = sqrt(r12[0] * r12[0] + r12[1] * r12[1] + r12[2] * r12[2]);
    double d32 = sqrt(r32[0] * r32[0] + r32[1] * r32[1] + r32[2] * r32[2]);
    double d13 = sqrt(r13[0] * r13[0] + r13[1] * r13[1] + r13[2] * r13[2]);
    double cr[3] = {r12[1] * r32[2] - r12[2] * r32[1], r12[2] * r32[0] - r12[0] * r32[2],
                    r12[0] * r32[1] - r12[1] * r32[0]};
    double theta = atan2(sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]),
                         r12[0] * r32[0] + r12[1] * r32[1] + r12[2] * r32[2]);
    double sn = sin(theta), cs = cos(theta);
    double kth = s->angle_k[k], th0 = s->angle_theta0[k];
    double dpot = 2.0 * kth * (theta - th0);
    double ubk = s->ub_k[k], ubr = s->ub_r0[k];
    double f1[3], f3[3], f2[3];
    for (int q = 0; q < 3; q++) {
      double dr12 = r12[q] / d12, dr32 = r32[q] / d32, dr13 = r13[q] / d13;
      double dt1 = (dr12 * cs - dr32) / (sn * d12);
      double dt3 = (dr32 * cs - dr12) / (sn * d32);
      double ub1 = dr13 * (2.0 * ubk * (d13 - ubr));
      f1[q] = -dt1 * dpot - ub1;
      f3[q] = -dt3 * dpot - (-ub1);
      f2[q] = -f1[q] - f3[q];
      forces[3 * a1 + q] += f1[q];
      forces[3 * a2 + q] += f2[q];
      forces[3 * a3 + q] += f3[q];
    }
    energies[ORC_E_ANGLE] += kth * (theta - th0) * (theta - th0) + ubk * (d13 - ubr) * (d13 - ubr);
    if (virial) {
      double xy = f1[0] * r12[1] + f3[0] * r32[1], xz = f1[0] * r12[2] + f3[0] * r32[2],
             yz = f1[1] * r12[2] + f3[1] * r32[2];
      virial[0] += f1[0] * r12[0] + f3[0] * r32[0]; virial[1] += xy; virial[2] += xz;
      virial[3] += xy; virial[4] += f1[1] * r12[1] + f3[1] * r32[1]; virial[5] += yz;
      virial[6] += xz; virial[7] += yz; virial[8] += f1[2] * r12[2] + f3[2] * r32[2];
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Leapfrog (integrator/leapfrog/LeapfrogIntegrator.cpp:33-104; StandardIntegrator.cpp:45-78).
 * ------------------------------------------------------------------------------------------ */
static void all_forces(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                       int do_bonded, const double *pos, double *f, double *e) {
  memset(f, 0, sizeof(double) * 3 * (size_t)s->n);
  memset(e, 0, sizeof(double) * ORC_E_COUNT);
  if (do_bonded) orc_bonded(s, pos, f, e, NULL);
  if (cp && (cp->do_lj || cp->do_coul)) orc_cutoff(s, pos, cp, f, e, NULL);
  if (pme) orc_pme(s, pos, pme, f, e, NULL, NULL, NULL);
}

int orc_leapfrog(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                 int do_bonded, double dt_fs, int nsteps, double *pos, double *vel,
                 double *forces_out, double *energies_out) {
  int n = s->n;
  double *f = forces_out, e[ORC_E_COUNT];
  double h = dt_fs * INV_TIMEFACTOR;
  all_forces(s, cp, pme, do_bonded, pos, f, e);
  if (nsteps >= 1) {
    for (int i = 0; i < n; i++)
      for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h * 0.5 / s->mass[i];
    for (int i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
    all_forces(s, cp, pme, do_bonded, pos, f, e);
    for (int st = 1; st < nsteps; st++) {
      for (int i = 0; i < n; i++)
        for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h / s->mass[i];
      for (int i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
      all_forces(s, cp, pme, do_bonded, pos, f, e);
    }
    for (int i = 0; i < n; i++)
      for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h * 0.5 / s->mass[i];
  }
  memcpy(energies_out, e, sizeof(e));
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Langevin leapfrog (integrator/base/LangevinLeapfrogIntegrator.cpp:23-29 constructor units,
 * :36-41 doDrift, :44-71 doHalfKick; integrator/StandardIntegrator.cpp:27-37 run): every step is
 * a half kick, a drift, the forces and a half kick, where a half kick is
 *   v = v vdt + F fdt / m + g sqrt(2 kB T gamma / m) ndt,
 *   fdt = (1 - exp(-gamma h / 2)) / gamma, vdt = exp(-gamma h / 2),
 *   ndt = sqrt((1 - exp(-gamma h)) / (2 gamma)),
 * gamma in the reference's internal unit (gamma_ps / (1000 INV_TIMEFACTOR)) and h = dt
 * INV_TIMEFACTOR.  The operations are rounded in the reference's order (Vector3D * scalar,
 * then / mass).
 *
 * The Gaussian numbers g: the reference draws them from one serial generator
 * (base/MathUtilities.cpp:206-238) in atom order, which a device thread per atom cannot replay.
 * The device draws them from a counter-based generator keyed by the seed, with the counter (atom,
 * half-kick index); half kick j of a run (j = 0, 1, ... from the state set) uses stream j.  The
 * generator is restated here so that runs at T > 0 can be compared too: Philox4x32 with 10 rounds
 * (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011), 53-bit
 * uniforms (v + 1/2) 2^-53 in (0, 1), and the Box-Muller transform.  At T = 0 the noise term is
 * exactly zero whatever g, which is how the reference's own integrator pins this function.
 * ------------------------------------------------------------------------------------------ */
static const double BOLTZMANN = 0.001987191; /* base/PMConstants.cpp */

static void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

static double u01(uint32_t a, uint32_t b) {
  uint64_t v = (((uint64_t)a << 21) ^ (uint64_t)b) & ((1ull << 53) - 1);
  return ((double)v + 0.5) * (1.0 / 9007199254740992.0);
}

void orc_gauss3(unsigned long long seed, int atom, long long stream, double g[3]) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  uint32_t c0[4] = {(uint32_t)atom, (uint32_t)stream, (uint32_t)((uint64_t)stream >> 32), 0u};
  uint32_t c1[4] = {(uint32_t)atom, (uint32_t)stream, (uint32_t)((uint64_t)stream >> 32), 1u};
  philox10(c0, k0, k1);
  philox10(c1, k0, k1);
  double u1 = u01(c0[0], c0[1]), u2 = u01(c0[2], c0[3]), u3 = u01(c1[0], c1[1]), u4 = u01(c1[2], c1[3]);
  double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
  g[0] = r1 * cos(2.0 * M_PI * u2);
  g[1] = r1 * sin(2.0 * M_PI * u2);
  g[2] = r2 * cos(2.0 * M_PI * u4);
}

static void langevin_half_kick(const orc_system *s, const double *f, double h, double gamma,
                               double kT, unsigned long long seed, long long stream, double *vel) {
  const double fdt = (1.0 - exp(-0.5 * gamma * h)) / gamma;
  const double vdt = exp(-0.5 * gamma * h);
  const double ndt = sqrt((1.0 - exp(-gamma * h)) / (2.0 * gamma));
  const double fc = 2 * kT * gamma;
  for (int i = 0; i < s->n; i++) {
    double g[3], m = s->mass[i], sq = sqrt(fc / m);
    orc_gauss3(seed, i, stream, g);
    for (int q = 0; q < 3; q++)
      vel[3 * i + q] = vel[3 * i + q] * vdt + f[3 * i + q] * fdt / m + g[q] * sq * ndt;
  }
}

int orc_langevin(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                 int do_bonded, double dt_fs, double temperature, double gamma_ps,
                 unsigned long long seed, long long first_step, int nsteps, double *pos, double *vel,
                 double *forces_out, double *energies_out) {
  double *f = forces_out, e[ORC_E_COUNT];
  const double h = dt_fs * INV_TIMEFACTOR;
  const double gamma = gamma_ps / (1000 * INV_TIMEFACTOR);
  const double kT = BOLTZMANN * temperature;
  if (!(gamma > 0) || temperature < 0) return 1;
  all_forces(s, cp, pme, do_bonded, pos, f, e);
  for (int st = 0; st < nsteps; st++) {
    long long j = 2 * (first_step + st);
    langevin_half_kick(s, f, h, gamma, kT, seed, j, vel);
    for (int i = 0; i < 3 * s->n; i++) pos[i] += vel[i] * h;
    all_forces(s, cp, pme, do_bonded, pos, f, e);
    langevin_half_kick(s, f, h, gamma, kT, seed, j + 1, vel);
  }
  memcpy(energies_out, e, sizeof(e));
  return 0;
}

/* ------------------------------------------------------------------ SHAKE / RATTLE */
static const double TIMEFACTOR = 48.88821290839616; /* base/PMConstants.cpp:53 */

/* ModifierMetaShake::calcError (ModifierMetaShake.cpp:12-33): mean over the constraints of
 * |d^2 - l^2| / (2 l^2), with d = x[a2] - x[a1]. */
static double shake_error(const orc_constraints *c, const double *x) {
  double error = 0;
  for (int i = 0; i < c->n; i++) {
    const double *p1 = x + 3 * c->a1[i], *p2 = x + 3 * c->a2[i];
    const double l2 = c->len[i] * c->len[i];
    const double dx = p2[0] - p1[0], dy = p2[1] - p1[1], dz = p2[2] - p1[2];
    error += fabs(dx * dx + dy * dy + dz * dz - l2) / (2.0 * l2);
  }
  return error / c->n;
}

int orc_shake(const orc_constraints *c, const double *mass, int n_atoms, double dt_fs, double *pos,
              double *vel, double *last_pos) {
  /* ModifierShake::doExecute (ModifierShake.cpp:17-75); the virial term is not accumulated */
  double error = shake_error(c, pos);
  const double dt = dt_fs / TIMEFACTOR;
  int iter = 0;
  while (error > c->shake_eps) {
    for (int i = 0; i < c->n; i++) {
      const int a1 = c->a1[i], a2 = c->a2[i];
      double *p1 = pos + 3 * a1, *p2 = pos + 3 * a2, *v1 = vel + 3 * a1, *v2 = vel + 3 * a2;
      const double *q1 = last_pos + 3 * a1, *q2 = last_pos + 3 * a2;
      const double pab[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
      const double pabsq = pab[0] * pab[0] + pab[1] * pab[1] + pab[2] * pab[2];
      const double rabsq = c->len[i] * c->len[i];
      const double diffsq = rabsq - pabsq;
      const double rab[3] = {q1[0] - q2[0], q1[1] - q2[1], q1[2] - q2[2]};
      const double rpab = rab[0] * pab[0] + rab[1] * pab[1] + rab[2] * pab[2];
      const double rM1 = 1 / mass[a1], rM2 = 1 / mass[a2];
      const double gab = diffsq / (2 * (rM1 + rM2) * rpab);
      double dp[3];
      for (int q = 0; q < 3; q++) dp[q] = rab[q] * gab;
      for (int q = 0; q < 3; q++) {
        p1[q] += dp[q] * rM1;
        p2[q] -= dp[q] * rM2;
      }
      for (int q = 0; q < 3; q++) dp[q] /= dt;
      for (int q = 0; q < 3; q++) {
        v1[q] += dp[q] * rM1;
        v2[q] -= dp[q] * rM2;
      }
    }
    error = shake_error(c, pos);
    iter++;
    if (iter > c->shake_maxiter) break;
  }
  memcpy(last_pos, pos, sizeof(double) * 3 * (size_t)n_atoms);
  return iter;
}

/* ModifierMetaRattle::calcError (ModifierMetaRattle.cpp:12-31): mean |(x1 - x2).(v1 - v2)|. */
static double rattle_error(const orc_constraints *c, const double *x, const double *v) {
  double error = 0;
  for (int i = 0; i < c->n; i++) {
    const int a1 = c->a1[i], a2 = c->a2[i];
    const double vab[3] = {v[3 * a1] - v[3 * a2], v[3 * a1 + 1] - v[3 * a2 + 1], v[3 * a1 + 2] - v[3 * a2 + 2]};
    const double rab[3] = {x[3 * a1] - x[3 * a2], x[3 * a1 + 1] - x[3 * a2 + 1], x[3 * a1 + 2] - x[3 * a2 + 2]};
    error += fabs(rab[0] * vab[0] + rab[1] * vab[1] + rab[2] * vab[2]);
  }
  return error / c->n;
}

/* ModifierRattle::doExecute (ModifierRattle.cpp:17-64), with its virial term when virial is
 * not NULL: every constraint of every sweep adds (2 dp) x rab as ScalarStructure::addVirial does
 * (type/ScalarStructure.cpp:36-54), dp = rab gab. */
static int rattle_v(const orc_constraints *c, const double *mass, double dt_fs, const double *pos,
                    double *vel, double *virial) {
  double error = rattle_error(c, pos, vel);
  const double dt = dt_fs / TIMEFACTOR;
  int iter = 0;
  while (error > c->rattle_eps) {
    for (int i = 0; i < c->n; i++) {
      const int a1 = c->a1[i], a2 = c->a2[i];
      const double rM1 = 1 / mass[a1], rM2 = 1 / mass[a2];
      const double *p1 = pos + 3 * a1, *p2 = pos + 3 * a2;
      double *v1 = vel + 3 * a1, *v2 = vel + 3 * a2;
      const double rab[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
      const double rabsq = rab[0] * rab[0] + rab[1] * rab[1] + rab[2] * rab[2];
      const double vab[3] = {v1[0] - v2[0], v1[1] - v2[1], v1[2] - v2[2]};
      const double rvab = rab[0] * vab[0] + rab[1] * vab[1] + rab[2] * vab[2];
      const double gab = -rvab / (dt * (rM1 + rM2) * rabsq);
      double dp[3];
      for (int q = 0; q < 3; q++) {
        dp[q] = rab[q] * gab;
        v1[q] += dp[q] * dt * rM1;
        v2[q] -= dp[q] * dt * rM2;
      }
      if (virial) {
        const double f[3] = {dp[0] * 2, dp[1] * 2, dp[2] * 2};
        const double xy = f[0] * rab[1], xz = f[0] * rab[2], yz = f[1] * rab[2];
        virial[0] += f[0] * rab[0];
        virial[1] += xy;
        virial[2] += xz;
        virial[3] += xy;
        virial[4] += f[1] * rab[1];
        virial[5] += yz;
        virial[6] += xz;
        virial[7] += yz;
        virial[8] += f[2] * rab[2];
      }
    }
    error = rattle_error(c, pos, vel);
    iter++;
    if (iter > c->rattle_maxiter) break;
  }
  return iter;
}

int orc_rattle(const orc_constraints *c, const double *mass, double dt_fs, const double *pos,
               double *vel) {
  return rattle_v(c, mass, dt_fs, pos, vel, NULL);
}

int orc_leapfrog_constrained(const orc_system *s, const orc_cutoff_params *cp,
                             const orc_pme_params *pme, int do_bonded, const orc_constraints *c,
                             double dt_fs, int nsteps, double *pos, double *vel, double *last_pos,
                             double *forces_out, double *energies_out, double *rattle_virial) {
  const int n = s->n;
  const int shake = c && c->n > 0 && c->shake_eps > 0 && c->shake_maxiter > 0;
  const int rattle = c && c->n > 0 && c->rattle_eps > 0 && c->rattle_maxiter > 0;
  double *f = forces_out, e[ORC_E_COUNT];
  const double h = dt_fs * INV_TIMEFACTOR;
  all_forces(s, cp, pme, do_bonded, pos, f, e);
  if (nsteps >= 1) {
    /* doHalfKickdoDrift, fast path (no pre-drift modifier), then the post-drift SHAKE */
    for (int i = 0; i < n; i++)
      for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h * 0.5 / s->mass[i];
    for (int i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
    if (shake) orc_shake(c, s->mass, n, dt_fs, pos, vel, last_pos);
    all_forces(s, cp, pme, do_bonded, pos, f, e);
    for (int st = 1; st < nsteps; st++) {
      if (rattle) {
        /* doKickdoDrift with a post-step modifier: half kick, RATTLE, half kick, drift */
        for (int i = 0; i < n; i++)
          for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h * 0.5 / s->mass[i];
        orc_rattle(c, s->mass, dt_fs, pos, vel);
        for (int i = 0; i < n; i++)
          for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h * 0.5 / s->mass[i];
      } else {
        for (int i = 0; i < n; i++)
          for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h / s->mass[i];
      }
      for (int i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
      if (shake) orc_shake(c, s->mass, n, dt_fs, pos, vel, last_pos);
      all_forces(s, cp, pme, do_bonded, pos, f, e);
    }
    for (int i = 0; i < n; i++)
      for (int q = 0; q < 3; q++) vel[3 * i + q] += f[3 * i + q] * h * 0.5 / s->mass[i];
    if (rattle) {
      if (rattle_virial) memset(rattle_virial, 0, 9 * sizeof(double));
      rattle_v(c, s->mass, dt_fs, pos, vel, rattle_virial);
    }
  }
  memcpy(energies_out, e, sizeof(e));
  return 0;
}

/* LangevinLeapfrogIntegrator run(nsteps) with SHAKE as a post-drift modifier and RATTLE as a
 * post-step modifier (integrator/StandardIntegrator.cpp:27-37: half kick, doDriftOrNextIntegrator
 * = drift then the post-drift modifiers, forces, half kick, the post-step modifiers;
 * integrator/STSIntegrator.cpp:28-32), the half kicks as orc_langevin. */
int orc_langevin_constrained(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                             int do_bonded, const orc_constraints *c, double dt_fs, double temperature,
                             double gamma_ps, unsigned long long seed, long long first_step, int nsteps,
                             double *pos, double *vel, double *last_pos, double *forces_out,
                             double *energies_out, double *rattle_virial) {
  const int n = s->n;
  const int shake = c && c->n > 0 && c->shake_eps > 0 && c->shake_maxiter > 0;
  const int rattle = c && c->n > 0 && c->rattle_eps > 0 && c->rattle_maxiter > 0;
  double *f = forces_out, e[ORC_E_COUNT];
  const double h = dt_fs * INV_TIMEFACTOR;
  const double gamma = gamma_ps / (1000 * INV_TIMEFACTOR);
  const double kT = BOLTZMANN * temperature;
  if (!(gamma > 0) || temperature < 0) return 1;
  all_forces(s, cp, pme, do_bonded, pos, f, e);
  for (int st = 0; st < nsteps; st++) {
    long long j = 2 * (first_step + st);
    langevin_half_kick(s, f, h, gamma, kT, seed, j, vel);
    for (int i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
    if (shake) orc_shake(c, s->mass, n, dt_fs, pos, vel, last_pos);
    all_forces(s, cp, pme, do_bonded, pos, f, e);
    langevin_half_kick(s, f, h, gamma, kT, seed, j + 1, vel);
    if (rattle) {
      if (rattle_virial) memset(rattle_virial, 0, 9 * sizeof(double));
      rattle_v(c, s->mass, dt_fs, pos, vel, rattle_virial);
    }
  }
  memcpy(energies_out, e, sizeof(e));
  return 0;
}
