/* FP64 CPU restatement of ProtoMol's nonbonded hot path -- TEST
 * INFRASTRUCTURE ONLY (the checker for the CUDA library; never part of the
 * product).  Compiled with -ffp-contract=off so that every double operation
 * rounds exactly like the reference's own x86-64 build.  Citations are
 * file:line in the ProtoMol tree. */
#include "pmoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PM_EPSILON 1.0e-14              /* base/PMConstants.cpp:50 */
#define PM_INV_TIMEFACTOR 0.02045482828087295 /* base/PMConstants.cpp:54 */
#define PM_BOLTZMANN 0.001987191        /* base/PMConstants.cpp:70 */
#define PM_MAX_INT_2 (2147483647 / 2)   /* base/PMConstants.cpp:45 */

/* ------------------------------------------------------------------ */
/* Periodic boundary conditions, topology/PeriodicBoundaryConditions.cpp:32-78
 * and PeriodicBoundaryConditions.h:56-140 (orthogonal branch). */
typedef struct {
  int periodic;
  double e1[3], e2[3], e3[3], origin[3];
  double e1r[3], e2r[3], e3r[3];
  double min[3], max[3], H[3], H2[3];
  double D;
  double V;
} pbc_t;

static void cross3(const double *a, const double *b, double *o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static double norm2(const double *a) {
  return a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
}

static void pbc_set(const orc_system *s, pbc_t *p) {
  int c;
  double a1[3], a2[3], a3[3], sum[3], a[3], b[3], d1, d2, d3, t[3];
  memset(p, 0, sizeof(*p));
  p->periodic = s->periodic;
  if (!s->periodic) return;
  memcpy(p->e1, s->box + 0, 24);
  memcpy(p->e2, s->box + 3, 24);
  memcpy(p->e3, s->box + 6, 24);
  memcpy(p->origin, s->box + 9, 24);
  cross3(p->e1, p->e2, t);
  p->V = fabs(dot3(t, p->e3));
  cross3(p->e2, p->e3, a1);
  d1 = dot3(p->e1, a1);
  cross3(p->e3, p->e1, a2);
  d2 = dot3(p->e2, a2);
  cross3(p->e1, p->e2, a3);
  d3 = dot3(p->e3, a3);
  for (c = 0; c < 3; c++) {
    p->e1r[c] = a1[c] / d1;
    p->e2r[c] = a2[c] / d2;
    p->e3r[c] = a3[c] / d3;
    sum[c] = (p->e1[c] + p->e2[c]) + p->e3[c];
  }
  for (c = 0; c < 3; c++) {
    a[c] = p->origin[c] - sum[c] * 0.5;
    b[c] = p->origin[c] + sum[c] * 0.5;
    p->min[c] = a[c] < b[c] ? a[c] : b[c];
    p->max[c] = a[c] > b[c] ? a[c] : b[c];
  }
  {
    double dx = (p->e1[0] * 0.5) * (p->e1[0] * 0.5);
    double dy = (p->e2[1] * 0.5) * (p->e2[1] * 0.5);
    double dz = (p->e3[2] * 0.5) * (p->e3[2] * 0.5);
    p->D = dx < (dy < dz ? dy : dz) ? dx : (dy < dz ? dy : dz);
  }
  for (c = 0; c < 3; c++) {
    p->H[c] = p->max[c] - p->min[c];
    p->H2[c] = p->H[c] * 0.5;
  }
}

/* minimalDifference(c1, c2, distSquared), PeriodicBoundaryConditions.h:72-110. */
static void pbc_mindiff(const pbc_t *p, const double *c1, const double *c2,
                        double *d, double *r2) {
  int c;
  for (c = 0; c < 3; c++) d[c] = c2[c] - c1[c];
  *r2 = norm2(d);
  if (!p->periodic) return;
  if (*r2 > p->D) {
    for (c = 0; c < 3; c++) {
      if (d[c] < -p->H2[c])
        d[c] += p->H[c];
      else if (d[c] > p->H2[c])
        d[c] -= p->H[c];
    }
    *r2 = norm2(d);
    if (*r2 > p->D) {
      d[0] -= p->e1[0] * rint(p->e1r[0] * d[0]);
      d[1] -= p->e2[1] * rint(p->e2r[1] * d[1]);
      d[2] -= p->e3[2] * rint(p->e3r[2] * d[2]);
      *r2 = norm2(d);
    }
  }
}

/* minimalPosition(c), PeriodicBoundaryConditions.h:113-140. */
static void pbc_minpos(const pbc_t *p, const double *x, double *o) {
  int c;
  if (!p->periodic) {
    for (c = 0; c < 3; c++) o[c] = x[c];
    return;
  }
  for (c = 0; c < 3; c++) o[c] = x[c] - p->origin[c];
  if (norm2(o) <= p->D) return;
  for (c = 0; c < 3; c++) {
    if (o[c] < -p->H2[c])
      o[c] += p->H[c];
    else if (o[c] > p->H2[c])
      o[c] -= p->H[c];
  }
  if (norm2(o) <= p->D) return;
  o[0] = o[0] - p->e1[0] * rint(p->e1r[0] * o[0]);
  o[1] = o[1] - p->e2[1] * rint(p->e2r[1] * o[1]);
  o[2] = o[2] - p->e3[2] * rint(p->e3r[2] * o[2]);
}

/* ------------------------------------------------------------------ */
/* Cell list (Topology.h:44-86, CubicCellManager.cpp:40-65,
 * ArrayCellListStructure.cpp:22-152). */
typedef struct {
  int nx, ny, nz;
  long ncells;
  int *head;     /* ncells, first atom (ascending index) or -1 */
  int *next;     /* n, cellListNext */
  int *cell;     /* 3n */
  double cs[3];  /* cell size vector */
  int maxN[3], n1[3], maxN1[3];
} cells_t;

static void cells_free(cells_t *c) {
  free(c->head);
  free(c->next);
  free(c->cell);
}

static int cells_build(const orc_system *s, const pbc_t *p, double cellsize,
                       cells_t *cl) {
  int i, c, dims[3];
  double mn[3], mx[3], vdiff[3], vres[3], inv[3], delta[3], origin[3];
  memset(cl, 0, sizeof(*cl));
  if (p->periodic) {
    for (c = 0; c < 3; c++) { mn[c] = p->min[c]; mx[c] = p->max[c]; }
    for (c = 0; c < 3; c++) origin[c] = p->origin[c];
  } else {
    /* Vector3DBlock::boundingbox, type/Vector3DBlock.cpp:9-35 */
    for (c = 0; c < 3; c++) mn[c] = mx[c] = s->pos[c];
    for (i = 1; i < s->n; i++)
      for (c = 0; c < 3; c++) {
        double v = s->pos[3 * i + c];
        if (v < mn[c]) mn[c] = v;
        else if (v > mx[c]) mx[c] = v;
      }
    for (c = 0; c < 3; c++) origin[c] = 0.0;
  }
  for (c = 0; c < 3; c++) vdiff[c] = mx[c] - mn[c];
  if (p->periodic) {
    for (c = 0; c < 3; c++) {
      double f = floor(vdiff[c] / cellsize);
      cl->cs[c] = vdiff[c] / (1.0 > f ? 1.0 : f);
      vres[c] = vdiff[c];
    }
  } else {
    for (c = 0; c < 3; c++) {
      cl->cs[c] = cellsize;
      vres[c] = vdiff[c] + cellsize;
    }
  }
  for (c = 0; c < 3; c++) {
    int k = (int)floor(vres[c] / cl->cs[c] + PM_EPSILON);
    dims[c] = k > 1 ? k : 1;
    inv[c] = 1.0 / cl->cs[c];
  }
  cl->nx = dims[0]; cl->ny = dims[1]; cl->nz = dims[2];
  for (c = 0; c < 3; c++) {
    cl->maxN[c] = PM_MAX_INT_2 - PM_MAX_INT_2 % dims[c];
    cl->n1[c] = -dims[c] / 2;
    cl->maxN1[c] = cl->maxN[c] - cl->n1[c];
  }
  cl->ncells = (long)dims[0] * dims[1] * dims[2];
  cl->head = (int *)malloc(sizeof(int) * cl->ncells);
  cl->next = (int *)malloc(sizeof(int) * (s->n > 0 ? s->n : 1));
  cl->cell = (int *)malloc(sizeof(int) * 3 * (s->n > 0 ? s->n : 1));
  if (!cl->head || !cl->next || !cl->cell) return -1;
  for (i = 0; i < cl->ncells; i++) cl->head[i] = -1;
  for (c = 0; c < 3; c++) delta[c] = origin[c] - mn[c];
  /* reverse order, prepend: lists end up in ascending atom order */
  for (i = s->n - 1; i >= 0; i--) {
    double mp[3], q[3];
    int xyz[3];
    long idx;
    pbc_minpos(p, s->pos + 3 * i, mp);
    for (c = 0; c < 3; c++) {
      q[c] = delta[c] + mp[c];
      xyz[c] = (int)floor(q[c] * inv[c]);
      cl->cell[3 * i + c] = xyz[c];
    }
    /* Positions exactly on the upper box face map to index n in the
     * reference (an out-of-range array slot); clamp for the oracle. */
    for (c = 0; c < 3; c++) {
      if (xyz[c] >= dims[c]) xyz[c] = dims[c] - 1;
      if (xyz[c] < 0) xyz[c] = 0;
    }
    idx = ((long)xyz[0] * dims[1] + xyz[1]) * dims[2] + xyz[2];
    cl->next[i] = cl->head[idx];
    cl->head[idx] = i;
  }
  return 0;
}

int orc_cell_assign(const orc_system *s, double cellsize, int *cell_xyz,
                    int *dims) {
  pbc_t p;
  cells_t cl;
  pbc_set(s, &p);
  if (cells_build(s, &p, cellsize, &cl)) return -1;
  memcpy(cell_xyz, cl.cell, sizeof(int) * 3 * s->n);
  dims[0] = cl.nx; dims[1] = cl.ny; dims[2] = cl.nz;
  cells_free(&cl);
  return 0;
}

typedef struct { int x, y, z; } cell3;
static int cell_lt(const cell3 *a, const cell3 *b) {
  if (a->x < b->x) return 1;
  if (a->x > b->x) return 0;
  if (a->y < b->y) return 1;
  if (a->y > b->y) return 0;
  return a->z < b->z;
}
static int cell_cmp(const void *a, const void *b) {
  const cell3 *x = (const cell3 *)a, *y = (const cell3 *)b;
  if (cell_lt(x, y)) return -1;
  if (cell_lt(y, x)) return 1;
  return 0;
}

/* Delta list, CellListEnumeratorPeriodicBoundaries.h:25-86 and
 * CellListEnumeratorStandard.h:26-80. */
static int build_deltas(const cells_t *cl, int periodic, double cutoff,
                        cell3 **out) {
  int k, l, m, nd = 0, cap = 64;
  double cutoff2 = cutoff * cutoff;
  int nx = (int)(cutoff / cl->cs[0] + 1.0 + PM_EPSILON);
  int ny = (int)(cutoff / cl->cs[1] + 1.0 + PM_EPSILON);
  int nz = (int)(cutoff / cl->cs[2] + 1.0 + PM_EPSILON);
  int n0, n1, n2;
  double xx = cl->cs[0] * cl->cs[0], yy = cl->cs[1] * cl->cs[1],
         zz = cl->cs[2] * cl->cs[2];
  cell3 *d = (cell3 *)malloc(sizeof(cell3) * cap);
  if (periodic) {
    n0 = nx < cl->nx ? nx : cl->nx;
    n1 = ny < cl->ny ? ny : cl->ny;
    n2 = nz < cl->nz ? nz : cl->nz;
  } else {
    n0 = nx < cl->nx - 1 ? nx : cl->nx - 1;
    n1 = ny < cl->ny - 1 ? ny : cl->ny - 1;
    n2 = nz < cl->nz - 1 ? nz : cl->nz - 1;
  }
  for (k = -n0; k <= n0; k++) {
    int x = abs(k) - 1;
    double d0;
    if (x < 0) x = 0;
    d0 = (x * x) * xx;
    for (l = -n1; l <= n1; l++) {
      int y = abs(l) - 1;
      double d1;
      if (y < 0) y = 0;
      d1 = d0 + (y * y) * yy;
      for (m = -n2; m <= n2; m++) {
        int z = abs(m) - 1;
        cell3 c, bc;
        int have = 0, t;
        if (z < 0) z = 0;
        if (!(d1 + (z * z) * zz < cutoff2)) continue;
        c.x = k; c.y = l; c.z = m;
        if (periodic) {
          /* ArrayCellListStructure.h:118-122 basisCell */
          bc.x = (c.x + cl->maxN1[0]) % cl->nx + cl->n1[0];
          bc.y = (c.y + cl->maxN1[1]) % cl->ny + cl->n1[1];
          bc.z = (c.z + cl->maxN1[2]) % cl->nz + cl->n1[2];
          if (bc.x == 0 && bc.y == 0 && bc.z == 0) have = 1;
          for (t = 0; t < nd && !have; t++)
            if (d[t].x == bc.x && d[t].y == bc.y && d[t].z == bc.z) have = 1;
          if (have) continue;
        } else {
          cell3 zero = {0, 0, 0};
          if (!cell_lt(&zero, &c)) continue;
          bc = c;
        }
        if (nd == cap) {
          cap *= 2;
          d = (cell3 *)realloc(d, sizeof(cell3) * cap);
        }
        d[nd++] = bc;
      }
    }
  }
  qsort(d, nd, sizeof(cell3), cell_cmp);
  *out = d;
  return nd;
}

/* Calls visit(i, j) for every candidate pair in the reference's order:
 * NonbondedCutoffForce::doEvaluate (NonbondedCutoffForce.h:37-54) driving
 * the enumerator's next() (CellListEnumeratorPeriodicBoundaries.h:114-134). */
typedef void (*pair_visit)(void *ctx, int i, int j);
static int enumerate_cutoff(const orc_system *s, const pbc_t *p,
                            double cellsize, double cutoff, int self_too,
                            pair_visit visit, void *ctx) {
  cells_t cl;
  cell3 *deltas;
  int nd;
  long a;
  if (cells_build(s, p, cellsize, &cl)) return -1;
  nd = build_deltas(&cl, p->periodic, cutoff, &deltas);
  for (a = 0; a < cl.ncells; a++) {
    int ax, ay, az, t, i, j;
    if (cl.head[a] < 0) continue;
    ax = (int)(a / ((long)cl.ny * cl.nz));
    ay = (int)((a / cl.nz) % cl.ny);
    az = (int)(a % cl.nz);
    /* same-cell pair first */
    for (i = cl.head[a]; i != -1; i = cl.next[i])
      for (j = self_too ? i : cl.next[i]; j != -1; j = cl.next[j])
        visit(ctx, i, j);
    for (t = 0; t < nd; t++) {
      long b;
      int bx = ax + deltas[t].x, by = ay + deltas[t].y, bz = az + deltas[t].z;
      if (p->periodic) {
        bx = (bx + cl.maxN[0]) % cl.nx;
        by = (by + cl.maxN[1]) % cl.ny;
        bz = (bz + cl.maxN[2]) % cl.nz;
      } else if (bx < 0 || by < 0 || bz < 0 || bx >= cl.nx || by >= cl.ny ||
                 bz >= cl.nz)
        continue;
      b = ((long)bx * cl.ny + by) * cl.nz + bz;
      if (cl.head[b] < 0) continue;
      if (a > b) continue; /* while (i > j) */
      for (i = cl.head[a]; i != -1; i = cl.next[i])
        for (j = cl.head[b]; j != -1; j = cl.next[j]) visit(ctx, i, j);
    }
  }
  free(deltas);
  cells_free(&cl);
  return 0;
}

/* ExclusionTable::check (topology/ExclusionTable.h:116-130), as a sorted
 * lookup of the (a1 < a2) table. */
typedef struct {
  int n;
  int *start; /* n+1 */
  int *partner;
  int *cls;
} excl_t;

static int excl_build(const orc_system *s, excl_t *e) {
  int k, *cnt;
  e->n = s->n;
  e->start = (int *)calloc(s->n + 1, sizeof(int));
  e->partner = (int *)malloc(sizeof(int) * (2 * s->nexcl + 1));
  e->cls = (int *)malloc(sizeof(int) * (2 * s->nexcl + 1));
  cnt = (int *)calloc(s->n + 1, sizeof(int));
  for (k = 0; k < s->nexcl; k++) {
    e->start[s->excl[3 * k] + 1]++;
    e->start[s->excl[3 * k + 1] + 1]++;
  }
  for (k = 0; k < s->n; k++) e->start[k + 1] += e->start[k];
  for (k = 0; k < s->nexcl; k++) {
    int a = s->excl[3 * k], b = s->excl[3 * k + 1], c = s->excl[3 * k + 2];
    e->partner[e->start[a] + cnt[a]] = b;
    e->cls[e->start[a] + cnt[a]++] = c;
    e->partner[e->start[b] + cnt[b]] = a;
    e->cls[e->start[b] + cnt[b]++] = c;
  }
  free(cnt);
  return 0;
}
static void excl_free(excl_t *e) {
  free(e->start);
  free(e->partner);
  free(e->cls);
}
static int excl_check(const excl_t *e, int i, int j) {
  int k;
  for (k = e->start[i]; k < e->start[i + 1]; k++)
    if (e->partner[k] == j) return e->cls[k];
  return ORC_EXCL_NONE;
}

/* ------------------------------------------------------------------ */
/* Switching functions: value and derivative-over-distance. */
typedef struct {
  int kind;
  double cutoff, cutoff2, switchon2;
  double c1_15c1, c1_05c3, c1_15c3;      /* C1SwitchingFunction.cpp:12-17 */
  double s1, s2, s3;                     /* C2SwitchingFunction.cpp:12-19 */
  int ordInt, ordIdx;                    /* CnSwitchingFunction.cpp:41-60 */
  double irange[8];
  double compoff, compoff2, itrange[8];  /* CmpCnCnSwitchingFunction.cpp:11-25 */
  int complement;                        /* ComplementSwitchingFunction.h */
  double rough2;                         /* cutoffSquared() of the rough test */
} sw_t;

static const double CN_SW[5][7] = {     /* CnSwitchingFunction.cpp:9-15 */
    {10., -15., 6., 0, 0, 0, 0},
    {35., -84., 70., -20., 0, 0, 0},
    {126., -420., 540., -315., 70., 0, 0},
    {0, 0, 0, 0, 0, 0, 0},
    {1716., -9009., 20020., -24024., 16380., -6006., 924.0}};
static const double CN_DSW[5][7] = {    /* CnSwitchingFunction.cpp:17-23 */
    {30., -60., 30., 0, 0, 0, 0},
    {140., -420., 420., -140., 0, 0, 0},
    {630., -2520., 3780., -2520., 630., 0, 0},
    {0, 0, 0, 0, 0, 0, 0},
    {12012., -72072., 180180., -240240., 180180., -72072., 12012.0}};

static void sw_init(const orc_switch *in, sw_t *o) {
  int i;
  double rc = in->cutoff, rs = in->switchon;
  memset(o, 0, sizeof(*o));
  o->kind = in->kind & ~ORC_SW_COMPLEMENT;
  switch (o->kind) {
    case ORC_SW_UNIVERSAL:
      o->cutoff = 1e300;
      o->cutoff2 = 1e300; /* Constant::MAXREAL */
      break;
    case ORC_SW_CUTOFF:
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      break;
    case ORC_SW_C1:
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      o->c1_15c1 = 1.5 / rc;
      o->c1_05c3 = 0.5 / (rc * rc * rc);
      o->c1_15c3 = 1.5 / (rc * rc * rc);
      break;
    case ORC_SW_C2: {
      double d = rc * rc - rs * rs;
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      o->switchon2 = rs * rs;
      o->s1 = 1.0 / (d * d * d); /* power<3> */
      o->s2 = rc * rc - 3.0 * rs * rs;
      o->s3 = 4.0 / (d * d * d);
      break;
    }
    case ORC_SW_CN: {
      double mycut = in->switchoff != 0.0 ? in->switchoff : rc;
      o->cutoff = mycut;
      o->cutoff2 = mycut * mycut;
      o->switchon2 = rs * rs;
      o->ordInt = (int)in->order;
      o->ordIdx = o->ordInt - 2;
      if (o->ordInt == 5) o->ordInt = 2;
      o->irange[0] = pow(rs - rc, -(o->ordInt + 1));
      for (i = 1; i < o->ordInt + 1; i++)
        o->irange[i] = o->irange[i - 1] / (rs - rc);
      break;
    }
    case ORC_SW_CMPCNCN: { /* CmpCnCnSwitchingFunction.cpp:11-25 */
      double so = in->switchoff, ord = in->order;
      o->cutoff = rc;
      o->cutoff2 = rc * rc;
      o->switchon2 = rs * rs;
      o->compoff = so;
      o->compoff2 = so * so;
      if (ord == 5.0) ord = 2.0; /* the order is remapped before its index */
      o->ordInt = (int)ord;
      o->ordIdx = o->ordInt - 2;
      o->irange[0] = 1.0 / pow(rs - so, o->ordInt + 1);
      o->itrange[0] = 1.0 / pow(so - rc, o->ordInt + 1);
      for (i = 1; i < o->ordInt + 1; i++) {
        o->irange[i] = o->irange[i - 1] / (rs - so);
        o->itrange[i] = o->itrange[i - 1] / (so - rc);
      }
      break;
    }
  }
  o->rough2 = o->cutoff2;
  if (in->kind & ORC_SW_COMPLEMENT) {
    /* ComplementSwitchingFunction: no rough test, cutoff MAXREAL; the
     * original function keeps its own constants */
    o->complement = 1;
    o->rough2 = 1e300;
  }
}

static void sw_eval_base(const sw_t *w, double r2, double *val, double *der);
/* ComplementSwitchingFunction::operator() (ComplementSwitchingFunction.h:42-46):
 * 1 - value, -derivative of the original function. */
static void sw_eval(const sw_t *w, double r2, double *val, double *der) {
  sw_eval_base(w, r2, val, der);
  if (w->complement) {
    *val = 1.0 - *val;
    *der = -*der;
  }
}

static void sw_eval_base(const sw_t *w, double r2, double *val, double *der) {
  switch (w->kind) {
    case ORC_SW_UNIVERSAL: /* UniversalSwitchingFunction.h:45-48 */
      *val = 1.0;
      *der = 0.0;
      return;
    case ORC_SW_CUTOFF: /* CutoffSwitchingFunction.h:41-44 */
      *der = 0;
      *val = r2 > w->cutoff2 ? 0.0 : 1.0;
      return;
    case ORC_SW_C1: { /* C1SwitchingFunction.h:41-50 */
      double d;
      if (r2 > w->cutoff2) {
        *val = 0.0;
        *der = 0.0;
        return;
      }
      d = sqrt(r2);
      *val = 1.0 - d * (w->c1_15c1 - r2 * w->c1_05c3);
      *der = -w->c1_15c1 / d + d * w->c1_15c3;
      return;
    }
    case ORC_SW_C2: /* C2SwitchingFunction.h:42-52 */
      *der = 0.0;
      if (r2 > w->cutoff2)
        *val = 0.0;
      else if (r2 >= w->switchon2) {
        double c2 = w->cutoff2 - r2;
        double c4 = c2 * (w->s2 + 2.0 * r2);
        *val = w->s1 * (c2 * c4);
        *der = w->s3 * (c2 * c2 - c4);
      } else
        *val = 1.0;
      return;
    case ORC_SW_CN: { /* CnSwitchingFunction.cpp:149-175 */
      double c[9], sd, sq;
      int i;
      *der = 0.0;
      *val = 0.0;
      if (r2 > w->cutoff2) return;
      if (r2 < w->switchon2) {
        *val = 1.0;
        return;
      }
      sq = sqrt(r2);
      sd = sq - w->cutoff;
      c[0] = pow(sd, w->ordInt);
      for (i = 1; i < w->ordInt + 2; i++) c[i] = c[i - 1] * sd;
      for (i = 0; i < w->ordInt + 1; i++) {
        *val += CN_SW[w->ordIdx][i] * c[i + 1] * w->irange[i];
        *der += CN_DSW[w->ordIdx][i] * c[i] * w->irange[i];
      }
      *der /= sq;
      return;
    }
    case ORC_SW_CMPCNCN: { /* CmpCnCnSwitchingFunction.h:45-95 */
      double c[9], sd, sq;
      int i;
      *der = 0.0;
      if (r2 > w->cutoff2)
        *val = 0.0;
      else if (r2 > w->compoff2) {
        sq = sqrt(r2);
        sd = sq - w->cutoff;
        c[0] = pow(sd, w->ordInt);
        for (i = 1; i < w->ordInt + 2; i++) c[i] = c[i - 1] * sd;
        *val = *der = 0.0;
        for (i = 0; i < w->ordInt + 1; i++) {
          *val += CN_SW[w->ordIdx][i] * c[i + 1] * w->itrange[i];
          *der += CN_DSW[w->ordIdx][i] * c[i] * w->itrange[i];
        }
        *der /= sq;
      } else if (r2 >= w->switchon2) {
        sq = sqrt(r2);
        sd = sq - w->compoff;
        c[0] = pow(sd, w->ordInt);
        for (i = 1; i < w->ordInt + 2; i++) c[i] = c[i - 1] * sd;
        *val = *der = 0.0;
        for (i = 0; i < w->ordInt + 1; i++) {
          *val += CN_SW[w->ordIdx][i] * c[i + 1] * w->irange[i];
          *der -= CN_DSW[w->ordIdx][i] * c[i] * w->irange[i];
        }
        *val = 1.0 - *val;
        *der /= sq;
      } else
        *val = 0.0;
      return;
    }
  }
}

/* ------------------------------------------------------------------ */
/* Pair potentials. */
static void lj_eval(const orc_system *s, int i, int j, int excl, double rr2,
                    double *e, double *f) {
  /* LennardJonesForce.h:28-60 */
  const double *p = s->lj + 4 * (s->type[i] * s->ntypes + s->type[j]);
  double A = excl != ORC_EXCL_MODIFIED ? p[0] : p[2];
  double B = excl != ORC_EXCL_MODIFIED ? p[1] : p[3];
  double r6 = rr2 * rr2 * rr2;
  double r12 = r6 * r6;
  double r6B = B * r6;
  double r12A = A * r12;
  *e = r12A - r6B;
  *f = 12.0 * r12A * rr2 - 6.0 * r6B * rr2;
}
static void coul_eval(const orc_system *s, int i, int j, int excl, double rr2,
                      double *e, double *f) {
  /* CoulombForce.h:29-40 */
  *e = s->charge[i] * s->charge[j] * sqrt(rr2);
  if (excl == ORC_EXCL_MODIFIED) *e *= s->coulomb_scaling;
  *f = *e * rr2;
}

/* CoulombSCPISMForce::operator() (force/coulomb/CoulombSCPISMForce.h:
 * 33-71): the Coulomb energy over a distance-dependent dielectric; no
 * contribution when either atom's molecule is water. */
static void scpism_eval(const orc_system *s, const orc_scpism *p, double D, int i, int j,
                        int excl, double rr2, double *e, double *f) {
  double rDist, Dist, alpha_ij, Dp1, rDp1, Dm1, k, rEXP, DiElec, rDiElec, drDiElec;
  *e = 0.0;
  *f = 0.0;
  if (p->water[i] || p->water[j]) return;
  rDist = sqrt(rr2);
  Dist = 1.0 / rDist;
  alpha_ij = p->sqrtalpha[i] * p->sqrtalpha[j];
  Dp1 = D + 1.0;
  rDp1 = 1.0 / Dp1;
  Dm1 = D - 1.0;
  k = Dm1 * 0.5;
  rEXP = k * exp(-alpha_ij * Dist);
  DiElec = Dp1 / (1.0 + rEXP) - 1.0;
  rDiElec = 1.0 / DiElec;
  *e = s->charge[i] * s->charge[j] * rDist * rDiElec *
       (excl == ORC_EXCL_MODIFIED ? s->coulomb_scaling : 1);
  drDiElec = alpha_ij * rDp1 * (1.0 + DiElec) * (D - DiElec);
  *f = (rDiElec * drDiElec + rDist) * *e * rDist;
}

typedef struct {
  const orc_system *s;
  const pbc_t *p;
  const orc_scpism *scp;
  double scp_D;
  excl_t ex;
  int nterms;
  int pot[2];
  sw_t sw[2];
  int modify;
  double cut2;
  double *forces, *energies, *virial;
  int *pairs;
  int list_pairs;
  long npairs, cap;
} cutoff_ctx;

static void add_virial(double *v, const double *fij, const double *d) {
  /* ScalarStructure::addVirial(force, diff), type/ScalarStructure.cpp */
  int a, b;
  if (!v) return;
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) v[3 * a + b] += fij[a] * d[b];
}

/* OneAtomPairTwo::doOneAtomPair (force/OneAtomPairTwo.h:30-100) and
 * OneAtomPair::doOneAtomPair (force/OneAtomPair.h:47-107). */
static void cutoff_visit(void *vctx, int i, int j) {
  cutoff_ctx *c = (cutoff_ctx *)vctx;
  const orc_system *s = c->s;
  double d[3], r2, rr2, fsum = 0.0, fij[3];
  int t, excl;
  pbc_mindiff(c->p, s->pos + 3 * i, s->pos + 3 * j, d, &r2);
  if (r2 > c->cut2) return;
  excl = s->molecule[i] == s->molecule[j] ? excl_check(&c->ex, i, j)
                                          : ORC_EXCL_NONE;
  if (excl == ORC_EXCL_FULL) return;
  if (c->list_pairs) {
    if (c->pairs && c->npairs < c->cap) {
      c->pairs[3 * c->npairs] = i;
      c->pairs[3 * c->npairs + 1] = j;
      c->pairs[3 * c->npairs + 2] = excl;
    }
    c->npairs++;
    return;
  }
  rr2 = 1.0 / r2;
  for (t = 0; t < c->nterms; t++) {
    double e, f, sv = 1.0, sd = 0.0;
    if (c->pot[t] == ORC_POT_LJ)
      lj_eval(s, i, j, excl, rr2, &e, &f);
    else if (c->pot[t] == ORC_POT_SCPISM)
      scpism_eval(s, c->scp, c->scp_D, i, j, excl, rr2, &e, &f);
    else
      coul_eval(s, i, j, excl, rr2, &e, &f);
    /* MODIFY is set for C1/C2/Cn only (enums in the switch/ headers); OneAtomPairTwo
     * switches both terms when either modifies (OneAtomPairTwo.h:66-76). */
    if (c->modify) {
      sw_eval(&c->sw[t], r2, &sv, &sd);
      f = f * sv - e * sd;
      e = e * sv;
    }
    if (c->pot[t] == ORC_POT_LJ)
      c->energies[1] += e;
    else
      c->energies[0] += e;
    fsum += f;
  }
  for (t = 0; t < 3; t++) fij[t] = d[t] * fsum;
  for (t = 0; t < 3; t++) {
    c->forces[3 * i + t] -= fij[t];
    c->forces[3 * j + t] += fij[t];
  }
  add_virial(c->virial, fij, d);
}

static double sw_cut2(const sw_t *w) { return w->rough2; }
static int sw_modifies(int kind) {
  /* MODIFY = 1: C1, C2, Cn, CmpCnCn and every Complement (switch/ headers) */
  if (kind & ORC_SW_COMPLEMENT) return 1;
  return kind == ORC_SW_C1 || kind == ORC_SW_C2 || kind == ORC_SW_CN ||
         kind == ORC_SW_CMPCNCN;
}

long orc_cutoff_pairs(const orc_system *s, double cellsize, double alg_cutoff,
                      double pair_cutoff, int *pairs_out, long cap) {
  pbc_t p;
  cutoff_ctx c;
  memset(&c, 0, sizeof(c));
  pbc_set(s, &p);
  c.s = s;
  c.p = &p;
  excl_build(s, &c.ex);
  c.cut2 = pair_cutoff * pair_cutoff;
  c.pairs = pairs_out;
  c.list_pairs = 1;
  c.cap = cap;
  enumerate_cutoff(s, &p, cellsize, alg_cutoff, 0, cutoff_visit, &c);
  excl_free(&c.ex);
  return c.npairs;
}

int orc_cutoff_force(const orc_system *s, double cellsize, double alg_cutoff,
                     int nterms, const int *potentials, const orc_switch *sw,
                     double *forces, double *energies, double *virial) {
  pbc_t p;
  cutoff_ctx c;
  int t;
  if (nterms < 1 || nterms > 2) return -1;
  memset(&c, 0, sizeof(c));
  pbc_set(s, &p);
  c.s = s;
  c.p = &p;
  excl_build(s, &c.ex);
  c.nterms = nterms;
  c.cut2 = 0.0;
  for (t = 0; t < nterms; t++) {
    c.pot[t] = potentials[t];
    sw_init(&sw[t], &c.sw[t]);
    if (sw_cut2(&c.sw[t]) > c.cut2) c.cut2 = sw_cut2(&c.sw[t]);
    if (sw_modifies(sw[t].kind)) c.modify = 1;
  }
  c.forces = forces;
  c.energies = energies;
  c.virial = virial;
  enumerate_cutoff(s, &p, cellsize, alg_cutoff, 0, cutoff_visit, &c);
  excl_free(&c.ex);
  return 0;
}

/* NonbondedSimpleFullSystemForce::doEvaluate (blocks of 64, i < j) with
 * OneAtomPair (OneAtomPair.h:47-107); vacuum: plain difference. */
int orc_simplefull_force(const orc_system *s, int potential,
                         const orc_switch *sw, double *forces,
                         double *energies, double *virial) {
  return orc_simplefull_force_n(s, 1, &potential, sw, forces, energies, virial);
}

/* OneAtomPair / OneAtomPairTwo over every pair i < j in blocks of 64
 * (NonbondedSimpleFullSystemForce.h:125-150); the rough test is against
 * the larger switch cutoff (OneAtomPairTwo.h:40-44), minimal image in a
 * periodic box. */
static int allpairs_force(const orc_system *s, const orc_scpism *scp, double D, int nterms,
                          const int *potentials, const orc_switch *sw, double *forces,
                          double *energies, double *virial);

int orc_simplefull_force_n(const orc_system *s, int nterms, const int *potentials,
                           const orc_switch *sw, double *forces, double *energies,
                           double *virial) {
  return allpairs_force(s, NULL, 0.0, nterms, potentials, sw, forces, energies, virial);
}

int orc_scpism_pair_force(const orc_system *s, const orc_scpism *p, double D, int nterms,
                          const int *potentials, const orc_switch *sw, double *forces,
                          double *energies, double *virial) {
  if (!p) return -1;
  return allpairs_force(s, p, D, nterms, potentials, sw, forces, energies, virial);
}

static int allpairs_force(const orc_system *s, const orc_scpism *scp, double D, int nterms,
                          const int *potentials, const orc_switch *sw, double *forces,
                          double *energies, double *virial) {
  pbc_t p;
  cutoff_ctx c;
  int bi, bj, i, j, t;
  const int bs = 64;
  if (nterms < 1 || nterms > 2) return -1;
  memset(&c, 0, sizeof(c));
  pbc_set(s, &p);
  c.s = s;
  c.p = &p;
  c.scp = scp;
  c.scp_D = D;
  excl_build(s, &c.ex);
  c.nterms = nterms;
  c.cut2 = 0.0;
  for (t = 0; t < nterms; t++) {
    c.pot[t] = potentials[t];
    sw_init(&sw[t], &c.sw[t]);
    if (sw_cut2(&c.sw[t]) > c.cut2) c.cut2 = sw_cut2(&c.sw[t]);
    if (sw_modifies(sw[t].kind)) c.modify = 1;
  }
  c.forces = forces;
  c.energies = energies;
  c.virial = virial;
  for (bi = 0; bi < s->n; bi += bs)
    for (bj = bi; bj < s->n; bj += bs)
      for (i = bi; i < bi + bs && i < s->n; i++)
        for (j = (bj <= i ? i + 1 : bj); j < bj + bs && j < s->n; j++)
          cutoff_visit(&c, i, j);
  excl_free(&c.ex);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Ewald.  Parameters: NonbondedFullEwaldSystemForce.h:598-620. */
void orc_ewald_setup(const orc_system *s, double alpha, double accuracy,
                     int exact_erf, orc_ewald *o) {
  double pp = -log(accuracy);
  (void)s;
  o->alpha = alpha;
  o->accuracy = accuracy;
  o->rc = sqrt(pp) / alpha;
  o->kc = 2.0 * alpha * sqrt(pp);
  o->exact_erf = exact_erf;
}

/* poly5, base/MathUtilities.cpp:39-49 (Abramowitz & Stegun 7.1.26). */
static double poly5(double ar) {
  double t = 1.0 / (1.0 + 0.3275911 * ar);
  return t * (0.254829592 +
              t * (-0.284496736 +
                   t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
}
static int cmp_norm(const void *a, const void *b) {
  const double *x = (const double *)a, *y = (const double *)b;
  double nx = norm2(x), ny = norm2(y);
  return nx < ny ? -1 : (nx > ny ? 1 : 0);
}

/* buildLatticeVectors, PeriodicBoundaryConditions.cpp:80-104, with (0,0,0)
 * prepended (NonbondedFullEwaldSystemForce.h:716-717). */
static int build_lattice(const pbc_t *p, double cutoff, double **out) {
  double a[3];
  int c, k, l, m, n = 1, cap;
  int bk, bl, bm;
  double *lat;
  for (c = 0; c < 3; c++) a[c] = (p->e1[c] + p->e2[c]) + p->e3[c];
  bk = (int)floor(cutoff / fabs(a[0]) + 1.0);
  bl = (int)floor(cutoff / fabs(a[1]) + 1.0);
  bm = (int)floor(cutoff / fabs(a[2]) + 1.0);
  cap = (2 * bk + 1) * (2 * bl + 1) * (2 * bm + 1) + 1;
  lat = (double *)calloc(3 * cap, sizeof(double));
  for (k = -bk; k <= bk; k++)
    for (l = -bl; l <= bl; l++)
      for (m = -bm; m <= bm; m++)
        if (k != 0 || l != 0 || m != 0) {
          double v[3];
          for (c = 0; c < 3; c++)
            v[c] = (p->e1[c] * k + p->e2[c] * l) + p->e3[c] * m;
          if (sqrt(norm2(v)) <= 2 * cutoff) {
            memcpy(lat + 3 * n, v, 24);
            n++;
          }
        }
  qsort(lat + 3, n - 1, 3 * sizeof(double), cmp_norm);
  *out = lat;
  return n;
}

typedef struct {
  const orc_system *s;
  const pbc_t *p;
  const orc_ewald *e;
  excl_t ex;
  double *lat;
  int nlat;
  double rc2;
  double *forces, *energy, *virial;
} ewald_ctx;

/* realTerm inner body, NonbondedFullEwaldSystemForce.h:784-852. */
static void ewald_real_visit(void *vctx, int i, int j) {
  ewald_ctx *c = (ewald_ctx *)vctx;
  const orc_system *s = c->s;
  const double a2pi = 2.0 * c->e->alpha / sqrt(M_PI);
  double dmin[3], r2dummy;
  double qi = s->charge[i], qj = s->charge[j];
  int k, excl;
  pbc_mindiff(c->p, s->pos + 3 * i, s->pos + 3 * j, dmin, &r2dummy);
  excl = s->molecule[i] == s->molecule[j] ? excl_check(&c->ex, i, j)
                                          : ORC_EXCL_NONE;
  if (i == j) excl = ORC_EXCL_FULL;
  for (k = 0; k < c->nlat; k++) {
    double rij[3], r2, r, qq, energy, force, fij[3];
    int t;
    if (excl == ORC_EXCL_FULL) {
      excl = ORC_EXCL_NONE;
      continue;
    }
    for (t = 0; t < 3; t++) rij[t] = dmin[t] + c->lat[3 * k + t];
    r2 = norm2(rij);
    if (r2 > c->rc2) continue;
    r = sqrt(r2);
    qq = qi * qj;
    if (excl == ORC_EXCL_MODIFIED) qq *= s->coulomb_scaling;
    if (!c->e->exact_erf) {
      double rr = 1.0 / r;
      double ar = c->e->alpha * r;
      double ee = qq * exp(-ar * ar);
      energy = poly5(ar) * ee * rr;
      force = ((energy + a2pi * ee) * rr * rr);
    } else {
      double a = erfc(c->e->alpha * r) / r; /* libm erfc, as the exact-erf build resolves it */
      energy = qq * a;
      force = qq * (a + a2pi * exp(-(c->e->alpha * c->e->alpha) * r2)) / r2;
    }
    /* Cutoff switching: value 1 inside Rc, derivative 0 */
    *c->energy += energy;
    for (t = 0; t < 3; t++) fij[t] = rij[t] * force;
    for (t = 0; t < 3; t++) {
      c->forces[3 * i + t] -= fij[t];
      c->forces[3 * j + t] += fij[t];
    }
    add_virial(c->virial, fij, rij);
    excl = ORC_EXCL_NONE;
  }
}

int orc_ewald_real(const orc_system *s, const orc_ewald *e, double cellsize,
                   double *forces, double *energy, double *virial) {
  pbc_t p;
  ewald_ctx c;
  memset(&c, 0, sizeof(c));
  pbc_set(s, &p);
  if (!p.periodic) return -1;
  c.s = s;
  c.p = &p;
  c.e = e;
  excl_build(s, &c.ex);
  c.nlat = build_lattice(&p, e->rc, &c.lat);
  c.rc2 = e->rc * e->rc;
  c.forces = forces;
  c.energy = energy;
  c.virial = virial;
  *energy = 0.0;
  enumerate_cutoff(s, &p, cellsize, e->rc, 1, ewald_real_visit, &c);
  free(c.lat);
  excl_free(&c.ex);
  return 0;
}

/* reciprocalTerm, NonbondedFullEwaldSystemForce.h:868-1083: k-vector
 * half-space |k| < Kc (:640-660), energy 4pi/V sum b|S|^2 with
 * b = exp(-k^2/4a^2)/k^2, forces 8pi/V b k (sin_i C - cos_i S).  Evaluated
 * with direct sin/cos per atom rather than the reference's recurrence
 * table (identical to rounding). */
int orc_ewald_reciprocal(const orc_system *s, const orc_ewald *e,
                         double *forces, double *energy, double *virial) {
  pbc_t p;
  int h, k, l, i, n = s->n;
  double LX, LY, LZ, LXr, LYr, LZr, Vr, a2r, fac, kc2, en = 0.0;
  double vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  int hmax, kmax, lmax;
  double *mp, *sn, *cs;
  pbc_set(s, &p);
  if (!p.periodic) return -1;
  LX = p.e1[0]; LY = p.e2[1]; LZ = p.e3[2];
  LXr = p.e1r[0]; LYr = p.e2r[1]; LZr = p.e3r[2];
  Vr = 1.0 / p.V;
  a2r = 1.0 / (e->alpha * e->alpha);
  fac = 1.0 / (4.0 * e->alpha * e->alpha);
  kc2 = e->kc * e->kc;
  hmax = (int)floor(e->kc / (2.0 * M_PI) * LX);
  kmax = (int)floor(e->kc / (2.0 * M_PI) * LY);
  lmax = (int)floor(e->kc / (2.0 * M_PI) * LZ);
  mp = (double *)malloc(sizeof(double) * 3 * n);
  sn = (double *)malloc(sizeof(double) * n);
  cs = (double *)malloc(sizeof(double) * n);
  for (i = 0; i < n; i++) pbc_minpos(&p, s->pos + 3 * i, mp + 3 * i);
  for (h = 0; h <= hmax; h++) {
    double kx = 2.0 * M_PI * h * LXr;
    for (k = (h == 0 ? 0 : -kmax); k <= kmax; k++) {
      double ky = 2.0 * M_PI * k * LYr;
      for (l = (h == 0 && k == 0 ? 1 : -lmax); l <= lmax; l++) {
        double kz = 2.0 * M_PI * l * LZr;
        double ksq = kx * kx + ky * ky + kz * kz;
        double ss = 0.0, sc = 0.0, b, ee, a;
        if (!(ksq < kc2)) continue;
        for (i = 0; i < n; i++) {
          double arg = kx * mp[3 * i] + ky * mp[3 * i + 1] + kz * mp[3 * i + 2];
          sn[i] = s->charge[i] * sin(arg);
          cs[i] = s->charge[i] * cos(arg);
          ss += sn[i];
          sc += cs[i];
        }
        b = 1.0 / ksq * exp(-ksq * a2r / 4.0);
        ee = b * (ss * ss + sc * sc);
        en += ee;
        if (virial) {
          double c = 2.0 * (1.0 / ksq + fac);
          vxx += ee * (1.0 - c * kx * kx);
          vxy -= ee * c * kx * ky;
          vxz -= ee * c * kx * kz;
          vyy += ee * (1.0 - c * ky * ky);
          vyz -= ee * c * ky * kz;
          vzz += ee * (1.0 - c * kz * kz);
        }
        a = 8.0 * M_PI * Vr * b;
        for (i = 0; i < n; i++) {
          double g = a * (sn[i] * sc - cs[i] * ss);
          forces[3 * i] += kx * g;
          forces[3 * i + 1] += ky * g;
          forces[3 * i + 2] += kz * g;
        }
      }
    }
  }
  {
    double c = 4.0 * M_PI * Vr;
    *energy = c * en;
    if (virial) {
      virial[0] += c * vxx; virial[1] += c * vxy; virial[2] += c * vxz;
      virial[3] += c * vxy; virial[4] += c * vyy; virial[5] += c * vyz;
      virial[6] += c * vxz; virial[7] += c * vyz; virial[8] += c * vzz;
    }
  }
  free(mp);
  free(sn);
  free(cs);
  return 0;
}

/* correctionTerm, NonbondedFullEwaldSystemForce.h:1092-1131. */
int orc_ewald_correction(const orc_system *s, const orc_ewald *e,
                         double *forces, double *energy, double *virial) {
  pbc_t p;
  int k;
  const double a2pi = 2.0 * e->alpha / sqrt(M_PI);
  double en = 0.0;
  pbc_set(s, &p);
  for (k = 0; k < s->nexcl; k++) {
    int a1 = s->excl[3 * k], a2 = s->excl[3 * k + 1];
    int cl = s->excl_table_class ? s->excl_table_class[k] : s->excl[3 * k + 2];
    double rij[3], r2, qq, r, rr, ee, fij[3], g;
    int t;
    pbc_mindiff(&p, s->pos + 3 * a1, s->pos + 3 * a2, rij, &r2);
    qq = s->charge[a1] * s->charge[a2];
    if (cl == ORC_EXCL_MODIFIED) qq *= 1 - s->coulomb_scaling;
    r = sqrt(r2);
    rr = 1 / r;
    ee = erf(e->alpha * r) * rr; /* libm erf: the name resolves to ::erf here */
    en -= qq * ee;
    g = qq * (a2pi * exp(-(e->alpha * e->alpha) * r2) - ee) * rr * rr;
    for (t = 0; t < 3; t++) fij[t] = rij[t] * g;
    for (t = 0; t < 3; t++) {
      forces[3 * a1 + t] -= fij[t];
      forces[3 * a2 + t] += fij[t];
    }
    add_virial(virial, fij, rij);
  }
  *energy = en;
  return 0;
}

void orc_ewald_self(const orc_system *s, const orc_ewald *e, double *self,
                    double *charged) {
  pbc_t p;
  int i;
  double q2 = 0.0, q = 0.0;
  pbc_set(s, &p);
  for (i = 0; i < s->n; i++) q2 += s->charge[i] * s->charge[i];
  *self = -q2 * e->alpha / sqrt(M_PI);
  for (i = 0; i < s->n; i++) q += s->charge[i];
  *charged = 0.0;
  if (fabs(q * 0.00268283) > 1.0e-5)
    *charged = -M_PI / (2.0 * p.V * (e->alpha * e->alpha)) * q * q;
}

/* ------------------------------------------------------------------ */
/* GB, OBC.  Pairs i < j in the SimpleFull order, vacuum differences. */
/* ------------------------------------------------------------------ */
/* Lattice sum: NonbondedFullSystemForce::doEvaluate (force/nonbonded/
 * NonbondedFullSystemForce.h:38-62) with OneAtomPairFull::doOneAtomPair
 * (force/OneAtomPairFull.h:35-135). */
static void full_pot(const orc_system *s, int pot, int i, int j, int excl, double r2,
                     const sw_t *w, int modify, double *e, double *f) {
  double rr2 = 1.0 / r2, sv, sd;
  if (pot == ORC_POT_LJ)
    lj_eval(s, i, j, excl, rr2, e, f);
  else
    coul_eval(s, i, j, excl, rr2, e, f);
  if (modify) {
    sw_eval(w, r2, &sv, &sd);
    *f = *f * sv - *e * sd;
    *e = *e * sv;
  }
}

int orc_full_force(const orc_system *s, int potential, const orc_switch *sw,
                   double alg_cutoff, double *forces, double *energies, double *virial) {
  pbc_t p;
  sw_t w;
  excl_t ex;
  double *lat;
  int nlat, modify, bi, bj, i, j, k, t;
  const int bs = 64; /* defaultBlockSize */
  double *esum = energies + (potential == ORC_POT_LJ ? 1 : 0);
  pbc_set(s, &p);
  if (!p.periodic) return -1;
  sw_init(sw, &w);
  modify = sw_modifies(sw->kind);
  excl_build(s, &ex);
  nlat = build_lattice(&p, alg_cutoff, &lat); /* lat[0] is the zero vector */
  for (bi = 0; bi < s->n; bi += bs)
    for (bj = bi; bj < s->n; bj += bs)
      for (i = bi; i < bi + bs && i < s->n; i++)
        for (j = (bj <= i ? i : bj); j < bj + bs && j < s->n; j++) {
          const int same = i == j;
          double dmin[3], r2, e, f, fij[3];
          if (same && nlat == 1) continue;
          pbc_mindiff(&p, s->pos + 3 * i, s->pos + 3 * j, dmin, &r2);
          if (!same) {
            int excl;
            r2 = norm2(dmin);
            if (r2 > w.rough2) continue; /* roughTest fails: no image either */
            excl = excl_check(&ex, i, j);
            if (excl != ORC_EXCL_FULL) {
              full_pot(s, potential, i, j, excl, r2, &w, modify, &e, &f);
              *esum += e;
              for (t = 0; t < 3; t++) fij[t] = -dmin[t] * f;
              for (t = 0; t < 3; t++) {
                forces[3 * i + t] += fij[t];
                forces[3 * j + t] -= fij[t];
              }
              for (t = 0; t < 3; t++) dmin[t] = -dmin[t];
              add_virial(virial, fij, dmin);
              for (t = 0; t < 3; t++) dmin[t] = -dmin[t];
            }
          }
          for (k = 1; k < nlat; k++) {
            double d[3];
            for (t = 0; t < 3; t++) d[t] = dmin[t] + lat[3 * k + t];
            r2 = norm2(d);
            if (r2 > w.rough2) continue;
            full_pot(s, potential, i, j, ORC_EXCL_NONE, r2, &w, modify, &e, &f);
            if (same)
              e /= 2;
            else {
              for (t = 0; t < 3; t++) fij[t] = -d[t] * f;
              for (t = 0; t < 3; t++) {
                forces[3 * i + t] += fij[t];
                forces[3 * j + t] -= fij[t];
              }
              for (t = 0; t < 3; t++) d[t] = -d[t];
              add_virial(virial, fij, d);
            }
            *esum += e;
          }
        }
  free(lat);
  excl_free(&ex);
  return 0;
}

/* ------------------------------------------------------------------ */
/* SCPISM Born radii and self force (force/born/BornRadii.h:33-77,
 * force/born/BornSelfForce.h:31-118, force/born/BornSwitch.h). */
static double born_sw(int sw, double r) { /* BornSwitch::switchValue */
  double f;
  if (r >= 5.0) return 0.0;
  if (sw == 3) {
    f = (1 - .0016 * r * r * r * r);
    return f * f * f * f;
  } else if (sw == 1) {
    f = (1 - .04 * r * r);
    return f * f;
  } else if (sw == 2) {
    f = (1 - 0.008 * r * r * r);
    return f * f * f;
  }
  return 1.0;
}
static double born_swd(int sw, double r) { /* BornSwitch::switchDerivative */
  double f;
  if (r >= 5.0) return 0.0;
  if (sw == 3) {
    f = (1 - .0016 * r * r * r * r);
    return -16 * .0016 * r * r * r * f * f * f;
  } else if (sw == 1) {
    return -0.16 * (1 - 0.04 * r * r) * r;
  } else if (sw == 2) {
    return -9 * .008 * r * r * (1 - .008 * r * r * r) * (1 - .008 * r * r * r);
  }
  return 0.0;
}
/* The polar hydrogen term of atom a against atom b: g_a' g_b when a is a
 * polar H (1), b an acceptor (2) in another residue, with g_a' = -0.378
 * for an HN against an O (BornRadii.h:45-58). */
static int born_polar(const orc_scpism *p, int a, int b, double *gg) {
  double ga;
  if (!(p->hbond[a] == 1 && p->hbond[b] == 2 && p->residue[a] != p->residue[b])) return 0;
  ga = (p->name[a] == 1 && p->name[b] == 2) ? -0.378 : p->g[a];
  *gg = ga * p->g[b];
  return 1;
}

int orc_born_force(const orc_system *s, const orc_scpism *p, int radii_bornswitch,
                   double radii_cutoff, int self_bornswitch, double self_cutoff, double D,
                   double *born_out, double *forces, double *energies, double *virial) {
  pbc_t pb;
  excl_t ex;
  int i, j, t;
  const int n = s->n;
  const double E = 0.80; /* the polar H+ constant (BornRadii.h:51) */
  const double K = (D - 1.0) / 2;
  double *R = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  double *Ds = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  int *used = (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
  double self_total = 0.0;
  if (!p) return -1;
  pbc_set(s, &pb);
  excl_build(s, &ex);
  /* BornRadii: preForce (radius = zeta), then every pair op in cutoff */
  for (i = 0; i < n; i++) R[i] = p->zeta[i];
  for (i = 0; i < n; i++)
    for (j = i + 1; j < n; j++) {
      double d[3], r2, dist, f, gg;
      int excl;
      pbc_mindiff(&pb, s->pos + 3 * i, s->pos + 3 * j, d, &r2);
      if (r2 > radii_cutoff * radii_cutoff) continue;
      excl = s->molecule[i] == s->molecule[j] ? excl_check(&ex, i, j) : ORC_EXCL_NONE;
      if (excl == ORC_EXCL_FULL) continue;
      if (p->water[i] || p->water[j]) continue;
      dist = sqrt(r2);
      f = born_sw(radii_bornswitch, dist);
      R[i] += p->eta[i] * f * exp(-p->c[i] * dist);
      if (born_polar(p, i, j, &gg)) R[i] += gg * f * exp(-E * dist);
      R[j] += p->eta[j] * f * exp(-p->c[j] * dist);
      if (born_polar(p, j, i, &gg)) R[j] += gg * f * exp(-E * dist);
    }
  if (born_out)
    for (i = 0; i < n; i++) born_out[i] = R[i];
  /* BornSelf: the solvation factor D_s of each atom, computed once */
  for (i = 0; i < n; i++) Ds[i] = (1.0 + D) / (1 + K * exp(-p->alpha[i] * R[i])) - 1.0;
  for (i = 0; i < n; i++)
    for (j = i + 1; j < n; j++) {
      double d[3], r2, dist, rDist, f, fp, gg, force = 0.0, fij[3];
      int excl, side;
      pbc_mindiff(&pb, s->pos + 3 * i, s->pos + 3 * j, d, &r2);
      if (r2 > self_cutoff * self_cutoff) continue;
      excl = s->molecule[i] == s->molecule[j] ? excl_check(&ex, i, j) : ORC_EXCL_NONE;
      if (excl == ORC_EXCL_FULL) continue;
      dist = sqrt(r2);
      rDist = 1.0 / dist;
      f = born_sw(self_bornswitch, dist);
      fp = born_swd(self_bornswitch, dist);
      for (side = 0; side < 2; side++) {
        const int a = side ? j : i, b = side ? i : j;
        double dRs = p->eta[a] * (fp - f * p->c[a]) * exp(-p->c[a] * dist);
        double rR = 1.0 / R[a], rDs = 1.0 / Ds[a];
        double dDs = p->alpha[a] * (1.0 / (1.0 + D)) * (1 + Ds[a]) * (D - Ds[a]);
        double q = s->charge[a];
        if (born_polar(p, a, b, &gg)) dRs += gg * (fp - f * E) * exp(-E * dist);
        force += (-0.5 * q * q * rR * rR * (1.0 - rDs - R[a] * rDs * rDs * dDs) * dRs) * rDist;
      }
      used[i] = used[j] = 1;
      for (t = 0; t < 3; t++) fij[t] = d[t] * force;
      for (t = 0; t < 3; t++) {
        forces[3 * i + t] -= fij[t];
        forces[3 * j + t] += fij[t];
      }
      add_virial(virial, fij, d);
    }
  for (i = 0; i < n; i++)
    if (used[i]) self_total += 0.5 * s->charge[i] * s->charge[i] / R[i] * (1.0 / Ds[i] - 1);
  energies[0] += self_total;
  free(R);
  free(Ds);
  free(used);
  excl_free(&ex);
  return 0;
}

/* Burial sums, psi and Born radii (GBBornRadii pair op and postProcess). */
static void gb_burial_born(const orc_system *s, const orc_gb *g, double *burial, double *psi,
                           double *born) {
  int n = s->n, i, j;
  /* GBBornRadii pair op (GBBornRadii.cpp:15-128) */
  for (i = 0; i < n; i++)
    for (j = i + 1; j < n; j++) {
      double d[3], r2, dist, ri, rj, oi, oj, Si, Sj, L, U, C, iL, iU, term;
      int t;
      if (g->water[i] || g->water[j]) continue;
      for (t = 0; t < 3; t++) d[t] = s->pos[3 * j + t] - s->pos[3 * i + t];
      r2 = norm2(d);
      dist = sqrt(r2);
      ri = g->vdwr[i]; rj = g->vdwr[j];
      oi = ri - g->offset[i]; oj = rj - g->offset[j];
      Si = g->scale[i]; Sj = g->scale[j];
      if (oi >= dist + Sj * oj) {
        L = 1.0; U = 1.0;
      } else {
        L = (oi > fabs(dist - Sj * oj)) ? oi : fabs(dist - Sj * oj);
        U = dist + Sj * oj;
      }
      C = (oi < oj * Sj - dist) ? 2.0 * (1.0 / oi - 1.0 / L) : 0;
      iL = 1.0 / L; iU = 1.0 / U;
      term = (iL - iU) + (dist / 4.0) * (iU * iU - iL * iL) +
             (1.0 / (2.0 * dist)) * log(L / U) +
             ((Sj * Sj * oj * oj) / (4.0 * dist)) * (iL * iL - iU * iU) + C;
      burial[i] += term;
      if (oj >= dist + Si * oi) {
        L = 1.0; U = 1.0;
      } else {
        L = (oj > fabs(dist - Si * oi)) ? oj : fabs(dist - Si * oi);
        U = dist + Si * oi;
      }
      C = (oj < oi * Si - dist) ? 2.0 * (1.0 / oj - 1.0 / L) : 0;
      iL = 1.0 / L; iU = 1.0 / U;
      term = (iL - iU) + (dist / 4.0) * (iU * iU - iL * iL) +
             (1.0 / (2.0 * dist)) * log(L / U) +
             ((Si * Si * oi * oi) / (4.0 * dist)) * (iL * iL - iU * iU) + C;
      burial[j] += term;
    }
  /* GBBornRadii::postProcess (GBBornRadii.cpp:145-173) */
  for (i = 0; i < n; i++) {
    double ri = g->vdwr[i], oi = ri - g->offset[i], tp, inv;
    psi[i] = 0.5 * burial[i] * oi;
    tp = g->alpha_obc * psi[i] - g->beta_obc * psi[i] * psi[i] +
         g->gamma_obc * psi[i] * psi[i] * psi[i];
    inv = (1 / oi) - (1 / ri) * tanh(tp);
    born[i] = 1 / inv;
  }
}

int orc_gb_force(const orc_system *s, const orc_gb *g, double *born,
                 double *forces, double *energy) {
  int n = s->n, i, j;
  double *burial = (double *)calloc(n, sizeof(double));
  double *psi = (double *)calloc(n, sizeof(double));
  double *partial = (double *)calloc(n, sizeof(double));
  double *ptm = (double *)calloc((size_t)n * n, sizeof(double)); /* partialTerm[i][j] */
  int *selfcount = (int *)calloc(n, sizeof(int));
  double *selfE = (double *)calloc(n, sizeof(double));
  const double dielec = (1 / g->solute_dielec) - (1 / g->solvent_dielec);
  double en = 0.0;
  if (!burial || !psi || !partial || !ptm || !selfcount || !selfE) return -1;
  gb_burial_born(s, g, burial, psi, born);
  /* GBPartialSum (GBPartialSum.cpp:11-42) */
  for (i = 0; i < n; i++)
    for (j = i + 1; j < n; j++) {
      double d[3], r2, ril, ex, fil, part;
      int t;
      for (t = 0; t < 3; t++) d[t] = s->pos[3 * j + t] - s->pos[3 * i + t];
      r2 = norm2(d);
      ril = sqrt(r2);
      ex = exp(-(ril * ril) / (4.0 * born[i] * born[j]));
      fil = sqrt(ril * ril + born[i] * born[j] * ex);
      part = s->charge[i] * s->charge[j] * (1 / (fil * fil)) * 0.5 * (1 / fil) * ex;
      ptm[(size_t)i * n + j] = part * (born[j] + (ril * ril) / (4.0 * born[i]));
      ptm[(size_t)j * n + i] = part * (born[i] + (ril * ril) / (4.0 * born[j]));
      partial[i] += ptm[(size_t)i * n + j];
      partial[j] += ptm[(size_t)j * n + i];
    }
  /* GBForce (GBForce.cpp:14-176) */
  for (i = 0; i < n; i++)
    for (j = i + 1; j < n; j++) {
      double d[3], r2, dist, ri, rj, oi, oj, Si, Sj, bi, bj, psi_i, psi_j,
          tpi, tpj, ex, fGB, qi, qj, L, U, Lj, Uj, iL, dL, dU, dC, dLj, dUj,
          dCj, th_i, th_j, tdi, tdj, Sit, Sjt, dBTi, dRi, dBTj, dRj, force,
          fij[3];
      int t;
      for (t = 0; t < 3; t++) d[t] = s->pos[3 * j + t] - s->pos[3 * i + t];
      r2 = norm2(d);
      dist = sqrt(r2);
      ri = g->vdwr[i]; rj = g->vdwr[j];
      oi = ri - g->offset[i]; oj = rj - g->offset[j];
      psi_i = psi[i]; psi_j = psi[j];
      tpi = g->alpha_obc * psi_i - g->beta_obc * psi_i * psi_i +
            g->gamma_obc * psi_i * psi_i * psi_i;
      tpj = g->alpha_obc * psi_j - g->beta_obc * psi_j * psi_j +
            g->gamma_obc * psi_j * psi_j * psi_j;
      bi = born[i]; bj = born[j];
      ex = exp(-(dist * dist) / (4.0 * bi * bj));
      fGB = sqrt(dist * dist + bi * bj * ex);
      qi = s->charge[i]; qj = s->charge[j];
      en += -(qi * qj) * (1 / fGB) * dielec;
      if (!selfcount[i]) {
        selfE[i] = -0.5 * (qi * qi) * (1 / bi) * dielec;
        selfcount[i] = 1;
      }
      if (!selfcount[j]) {
        selfE[j] = -0.5 * (qj * qj) * (1 / bj) * dielec;
        selfcount[j] = 1;
      }
      Si = g->scale[i]; Sj = g->scale[j];
      if (oi >= dist + Sj * oj) {
        L = 1; U = 1;
      } else {
        L = (oi > fabs(dist - Sj * oj)) ? oi : fabs(dist - Sj * oj);
        U = dist + Sj * oj;
      }
      iL = 1 / L;
      dL = (oi <= (dist - Sj * oj)) ? 1 : 0;
      dU = (oi < (dist + Sj * oj)) ? 1 : 0;
      dC = (oi <= (Sj * oj - dist)) ? 2 * iL * iL * dL : 0;
      if (oj >= dist + Si * oi) {
        Lj = 1; Uj = 1;
      } else {
        Lj = (oj > fabs(dist - Si * oi)) ? oj : fabs(dist - Si * oi);
        Uj = dist + Si * oi;
      }
      dLj = (oj <= (dist - Si * oi)) ? 1 : 0;
      dUj = (oj < (dist + Si * oi)) ? 1 : 0;
      dCj = (oj <= (Si * oi - dist)) ? 2 * (1 / Lj) * (1 / Lj) * dLj : 0;
      th_i = tanh(tpi);
      th_j = tanh(tpj);
      tdi = (g->alpha_obc - 2 * g->beta_obc * psi_i + 3 * g->gamma_obc * psi_i * psi_i);
      tdj = (g->alpha_obc - 2 * g->beta_obc * psi_j + 3 * g->gamma_obc * psi_j * psi_j);
      Sit = (Si * oi) / dist;
      Sjt = (Sj * oj) / dist;
      dBTi = -0.5 * dL * (1 / (L * L)) + 0.5 * dU * (1 / (U * U)) +
             0.125 * ((1 / (U * U)) - (1 / (L * L))) +
             0.125 * dist * ((2 / (L * L * L)) * dL - (2 / (U * U * U)) * dU) -
             0.25 * (1 / (dist * dist)) * log(L / U) +
             (U / (4 * dist * L)) * ((1 / U) * dL - (L / (U * U)) * dU) -
             0.125 * (Sjt * Sjt) * ((1 / (L * L)) - (1 / (U * U))) +
             0.25 * ((Sj * Sj * oj * oj) / (dist * U * U * U)) * dU -
             0.25 * ((Sj * Sj * oj * oj) / (dist * L * L * L)) * dL + dC;
      dRi = (bi * bi) * oi * (1 - th_i * th_i) * tdi * (1 / ri) * dBTi;
      dBTj = -0.5 * dLj * (1 / (Lj * Lj)) + 0.5 * dUj * (1 / (Uj * Uj)) +
             0.125 * ((1 / (Uj * Uj)) - (1 / (Lj * Lj))) +
             0.125 * dist * ((2 / (Lj * Lj * Lj)) * dLj - (2 / (Uj * Uj * Uj)) * dUj) -
             0.25 * (1 / (dist * dist)) * log(Lj / Uj) +
             (Uj / (4 * dist * Lj)) * ((1 / Uj) * dLj - (Lj / (Uj * Uj)) * dUj) -
             0.125 * (Sit * Sit) * ((1 / (Lj * Lj)) - (1 / (Uj * Uj))) +
             0.25 * ((Si * Si * oi * oi) / (dist * Uj * Uj * Uj)) * dUj -
             0.25 * ((Si * Si * oi * oi) / (dist * Lj * Lj * Lj)) * dLj + dCj;
      dRj = (bj * bj) * oj * (1 - th_j * th_j) * tdj * (1 / rj) * dBTj;
      force = 0;
      force -= qi * qj * (1 / (fGB * fGB)) * 0.5 * (1 / fGB) *
               ((2 * dist - 0.5 * ex * dist) +
                ex * dRi * (bj + (dist * dist) / (4 * bi)) +
                ex * dRj * (bi + (dist * dist) / (4 * bj))) *
               (1 / dist);
      force -= 0.5 * qi * qi * dRi / (bi * bi) / dist;
      force -= 0.5 * qj * qj * dRj / (bj * bj) / dist;
      force -= (partial[i] - ptm[(size_t)i * n + j]) * (dRi / dist);
      force -= (partial[j] - ptm[(size_t)j * n + i]) * (dRj / dist);
      force *= dielec;
      for (t = 0; t < 3; t++) fij[t] = d[t] * force;
      for (t = 0; t < 3; t++) {
        forces[3 * i + t] -= fij[t];
        forces[3 * j + t] += fij[t];
      }
    }
  /* GBForce::postProcess (GBForce.cpp:230-242) */
  for (i = 0; i < n; i++) en += selfE[i];
  *energy = en;
  free(burial); free(psi); free(partial); free(ptm); free(selfcount);
  free(selfE);
  return 0;
}

/* ProtoMol's integer power, MathUtilities.cpp:114-134 (square and
 * multiply, so results round as the reference's do). */
static double pm_power(double x, int n) {
  double z = 1.0, y = x;
  int m = n;
  if (n == 0) return 1.0;
  if (n < 0) return 1.0 / pm_power(x, -n);
  while (m > 0) {
    if (m & 1) z *= y;
    y *= y;
    m >>= 1;
  }
  return z;
}

/* GBACEForce (force/GB/GBACEForce.cpp:17-209): the ACE nonpolar term on the
 * Born radii of GBBornRadii.  Energy: per atom 4 pi sigma (r_i + rho_s)^2
 * (r_i / R_i)^6, set once for every atom that takes part in a pair
 * (ACEPotentialCount, summed in postProcess :161-171); pair force
 * c1 (c_i R_i^-7 dR_i/dr + c_j R_j^-7 dR_j/dr) / d with c1 = 24 pi sigma and
 * c_i = (r_i + rho_s)^2 r_i^6, dR/dr as in GBForce.  "pi" is the
 * reference's own constant 3.14169 (GBACEForce.cpp:6).  Every unordered pair
 * once (NonbondedSimpleFull, OneAtomPairNoExclusion: exclusions ignored). */
#define ACE_PI 3.14169
int orc_gbace_force(const orc_system *s, const orc_gb *g, double sigma, double rho_s,
                    double *forces, double *energy) {
  int n = s->n, i, j;
  double *burial = (double *)calloc(n > 0 ? n : 1, sizeof(double));
  double *psi = (double *)calloc(n > 0 ? n : 1, sizeof(double));
  double *born = (double *)calloc(n > 0 ? n : 1, sizeof(double));
  double *ace = (double *)calloc(n > 0 ? n : 1, sizeof(double));
  int *acecount = (int *)calloc(n > 0 ? n : 1, sizeof(int));
  double en = 0.0;
  if (!burial || !psi || !born || !ace || !acecount) return -1;
  gb_burial_born(s, g, burial, psi, born);
  for (i = 0; i < n; i++)
    for (j = i + 1; j < n; j++) {
      double d[3], r2, dist, ri, rj, oi, oj, Si, Sj, psi_i, psi_j, tpi, tpj, bi, bj, c1, ci,
          cj, L, U, Lj, Uj, dL, dU, dC, dLj, dUj, dCj, th_i, th_j, tdi, tdj, Sit, Sjt, dBTi,
          dRi, dBTj, dRj, force;
      int t;
      for (t = 0; t < 3; t++) d[t] = s->pos[3 * j + t] - s->pos[3 * i + t];
      r2 = norm2(d);
      dist = sqrt(r2);
      ri = g->vdwr[i]; rj = g->vdwr[j];
      oi = ri - g->offset[i]; oj = rj - g->offset[j];
      Si = g->scale[i]; Sj = g->scale[j];
      psi_i = psi[i]; psi_j = psi[j];
      tpi = g->alpha_obc * psi_i - g->beta_obc * psi_i * psi_i +
            g->gamma_obc * psi_i * psi_i * psi_i;
      tpj = g->alpha_obc * psi_j - g->beta_obc * psi_j * psi_j +
            g->gamma_obc * psi_j * psi_j * psi_j;
      bi = born[i]; bj = born[j];
      if (!acecount[i]) {
        ace[i] = 4 * ACE_PI * sigma * (ri + rho_s) * (ri + rho_s) * pm_power(ri / bi, 6);
        acecount[i] = 1;
      }
      if (!acecount[j]) {
        ace[j] = 4 * ACE_PI * sigma * (rj + rho_s) * (rj + rho_s) * pm_power(rj / bj, 6);
        acecount[j] = 1;
      }
      c1 = 24 * ACE_PI * sigma;
      ci = (ri + rho_s) * (ri + rho_s) * pow(ri, 6);
      cj = (rj + rho_s) * (rj + rho_s) * pow(rj, 6);
      if (oi >= dist + Sj * oj) {
        L = 1; U = 1;
      } else {
        L = (oi > fabs(dist - Sj * oj)) ? oi : fabs(dist - Sj * oj);
        U = dist + Sj * oj;
      }
      if (oj >= dist + Si * oi) {
        Lj = 1; Uj = 1;
      } else {
        Lj = (oj > fabs(dist - Si * oi)) ? oj : fabs(dist - Si * oi);
        Uj = dist + Si * oi;
      }
      dL = (oi <= (dist - Sj * oj)) ? 1 : 0;
      dU = (oi < (dist + Sj * oj)) ? 1 : 0;
      dC = (oi <= (Sj * oj - dist)) ? 2 * (1 / L) * (1 / L) * dL : 0;
      dLj = (oj <= (dist - Si * oi)) ? 1 : 0;
      dUj = (oj < (dist + Si * oi)) ? 1 : 0;
      dCj = (oj <= (Si * oi - dist)) ? 2 * (1 / Lj) * (1 / Lj) * dLj : 0;
      th_i = tanh(tpi);
      th_j = tanh(tpj);
      tdi = (g->alpha_obc - 2 * g->beta_obc * psi_i + 3 * g->gamma_obc * psi_i * psi_i);
      tdj = (g->alpha_obc - 2 * g->beta_obc * psi_j + 3 * g->gamma_obc * psi_j * psi_j);
      Sit = (Si * oi) / dist;
      Sjt = (Sj * oj) / dist;
      dBTi = -0.5 * dL * (1 / (L * L)) + 0.5 * dU * (1 / (U * U)) +
             0.125 * ((1 / (U * U)) - (1 / (L * L))) +
             0.125 * dist * ((2 / (L * L * L)) * dL - (2 / (U * U * U)) * dU) -
             0.25 * (1 / (dist * dist)) * log(L / U) +
             (U / (4 * dist * L)) * ((1 / U) * dL - (L / (U * U)) * dU) -
             0.125 * pm_power(Sjt, 2) * ((1 / (L * L)) - (1 / (U * U))) +
             0.25 * ((Sj * Sj * oj * oj) / (dist * U * U * U)) * dU -
             0.25 * ((Sj * Sj * oj * oj) / (dist * L * L * L)) * dL + dC;
      dRi = pm_power(bi, 2) * oi * (1 - th_i * th_i) * tdi * (1 / ri) * dBTi;
      dBTj = -0.5 * dLj * (1 / (Lj * Lj)) + 0.5 * dUj * (1 / (Uj * Uj)) +
             0.125 * ((1 / (Uj * Uj)) - (1 / (Lj * Lj))) +
             0.125 * dist * ((2 / (Lj * Lj * Lj)) * dLj - (2 / (Uj * Uj * Uj)) * dUj) -
             0.25 * (1 / (dist * dist)) * log(Lj / Uj) +
             (Uj / (4 * dist * Lj)) * ((1 / Uj) * dLj - (Lj / (Uj * Uj)) * dUj) -
             0.125 * pm_power(Sit, 2) * ((1 / (Lj * Lj)) - (1 / (Uj * Uj))) +
             0.25 * ((Si * Si * oi * oi) / (dist * Uj * Uj * Uj)) * dUj -
             0.25 * ((Si * Si * oi * oi) / (dist * Lj * Lj * Lj)) * dLj + dCj;
      dRj = pm_power(bj, 2) * oj * (1 - th_j * th_j) * tdj * (1 / rj) * dBTj;
      force = 0;
      force += c1 * (ci * (1 / pm_power(bi, 7)) * dRi * (1 / dist) +
                     cj * (1 / pm_power(bj, 7)) * dRj * (1 / dist));
      for (t = 0; t < 3; t++) {
        forces[3 * i + t] -= d[t] * force;
        forces[3 * j + t] += d[t] * force;
      }
    }
  for (i = 0; i < n; i++) en += ace[i];
  *energy = en;
  free(burial); free(psi); free(born); free(ace); free(acecount);
  return 0;
}

/* ------------------------------------------------------------------ */
/* ---------------------------------------------------------- torsions */
static void cross_to(const double *u, const double *v, double *o) {
  o[0] = u[1] * v[2] - u[2] * v[1];
  o[1] = u[2] * v[0] - u[0] * v[2];
  o[2] = u[0] * v[1] - u[1] * v[0];
}

/* MTorsionSystemForce::calcTorsion (MTorsionSystemForce.h:40-204): the
 * dihedral angle from the normals of the (1,2,3) and (2,3,4) planes, and
 * the gradient through d cos(phi) when |sin phi| > 0.1, else through
 * d sin(phi), which avoids dividing by a small sine or cosine. */
int orc_torsion_force(const orc_system *s, int nt, const int *atoms,
                      const double *params, double *forces, double *energy,
                      double *virial) {
  pbc_t p;
  int t, c;
  double e = 0.0, v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  pbc_set(s, &p);
  for (t = 0; t < nt; t++) {
    const int a1 = atoms[4 * t], a2 = atoms[4 * t + 1], a3 = atoms[4 * t + 2],
              a4 = atoms[4 * t + 3];
    const double k = params[3 * t], delta = params[3 * t + 2];
    const int per = (int)params[3 * t + 1];
    double r12[3], r23[3], r34[3], na[3], nb[3], nc[3], r2;
    double f1[3], f2[3], f3[3];
    pbc_mindiff(&p, s->pos + 3 * a2, s->pos + 3 * a1, r12, &r2);
    pbc_mindiff(&p, s->pos + 3 * a3, s->pos + 3 * a2, r23, &r2);
    pbc_mindiff(&p, s->pos + 3 * a4, s->pos + 3 * a3, r34, &r2);
    cross_to(r12, r23, na);
    cross_to(r23, r34, nb);
    cross_to(r23, na, nc);
    const double ia = 1.0 / sqrt(norm2(na)), ib = 1.0 / sqrt(norm2(nb)),
                 ic = 1.0 / sqrt(norm2(nc));
    for (c = 0; c < 3; c++) {
      na[c] *= ia;
      nb[c] *= ib;
      nc[c] *= ic;
    }
    const double cphi = dot3(na, nb), sphi = dot3(nc, nb);
    const double phi = -atan2(sphi, cphi);
    double dvdphi;
    if (per > 0) {
      dvdphi = -per * k * sin(per * phi + delta);
      e += k * (1.0 + cos(per * phi + delta));
    } else {
      double diff = phi - delta;
      if (diff < -M_PI) diff += 2 * M_PI;
      else if (diff > M_PI) diff -= 2 * M_PI;
      dvdphi = 2.0 * k * diff;
      e += k * diff * diff;
    }
    if (fabs(sphi) > 0.1) {
      double ga[3], gb[3];
      const double g = dvdphi / sphi;
      for (c = 0; c < 3; c++) {
        ga[c] = (na[c] * cphi - nb[c]) * ia;
        gb[c] = (nb[c] * cphi - na[c]) * ib;
      }
      /* f1 = g (r23 x ga), f3 = g (gb x r23), f2 = g (ga x r12 + r34 x gb) */
      double t1[3], t2[3];
      cross_to(r23, ga, t1);
      cross_to(gb, r23, t2);
      for (c = 0; c < 3; c++) {
        f1[c] = g * t1[c];
        f3[c] = g * t2[c];
      }
      cross_to(ga, r12, t1);
      cross_to(r34, gb, t2);
      for (c = 0; c < 3; c++) f2[c] = g * (t1[c] + t2[c]);
    } else {
      double gc[3], gb[3], t1[3];
      const double g = -dvdphi / cphi;
      for (c = 0; c < 3; c++) {
        gc[c] = (nc[c] * sphi - nb[c]) * ic;
        gb[c] = (nb[c] * sphi - nc[c]) * ib;
      }
      /* f1 = g (|r23|^2 gc - r23 (r23 . gc)) */
      const double r23sq = norm2(r23), r23gc = dot3(r23, gc);
      for (c = 0; c < 3; c++) f1[c] = g * (r23sq * gc[c] - r23[c] * r23gc);
      cross_to(gb, r23, t1);
      for (c = 0; c < 3; c++) f3[c] = g * t1[c];
      /* f2 = g (-(r23 . r12) gc + 2 r23 (r12 . gc) - r12 (r23 . gc) + r34 x gb)
       *      with the diagonal terms as the reference groups them */
      for (c = 0; c < 3; c++) {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        f2[c] = g * (-(r23[c1] * r12[c1] + r23[c2] * r12[c2]) * gc[c] +
                     (2.0 * r23[c] * r12[c1] - r12[c] * r23[c1]) * gc[c1] +
                     (2.0 * r23[c] * r12[c2] - r12[c] * r23[c2]) * gc[c2] +
                     gb[c2] * r34[c1] - gb[c1] * r34[c2]);
      }
    }
    for (c = 0; c < 3; c++) {
      forces[3 * a1 + c] += f1[c];
      forces[3 * a2 + c] += f2[c] - f1[c];
      forces[3 * a3 + c] += f3[c] - f2[c];
      forces[3 * a4 + c] -= f3[c];
    }
    /* the upper triangle, mirrored (the reference adds xy to YX etc.) */
    for (int i = 0; i < 3; i++)
      for (int j = i; j < 3; j++) {
        const double w = f1[i] * r12[j] + f2[i] * r23[j] + f3[i] * r34[j];
        v[3 * i + j] += w;
        if (j != i) v[3 * j + i] += w;
      }
  }
  *energy = e;
  if (virial)
    for (c = 0; c < 9; c++) virial[c] = v[c];
  return 0;
}

/* ------------------------------------------------------- bonds, angles */
/* BondSystemForce::calcBond (force/bonded/BondSystemForce.h:89-124):
 * harmonic k (r - r0)^2 along the minimal difference r12 = x1 - x2 seen
 * from atom 2; the force on atom 1 is r12 (-dV/dr / r), atom 2 gets its
 * negative, the virial is addVirial(f1, r12). */
int orc_bond_force(const orc_system *s, int nb, const int *atoms, const double *params,
                   double *forces, double *energy, double *virial) {
  pbc_t p;
  int b, c;
  double e = 0.0, v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  pbc_set(s, &p);
  for (b = 0; b < nb; b++) {
    const int a1 = atoms[2 * b], a2 = atoms[2 * b + 1];
    const double k = params[2 * b], r0 = params[2 * b + 1];
    double r12[3], r2, f1[3];
    pbc_mindiff(&p, s->pos + 3 * a2, s->pos + 3 * a1, r12, &r2);
    const double r = sqrt(norm2(r12));
    const double dpdr = 2.0 * k * (r - r0);
    for (c = 0; c < 3; c++) {
      f1[c] = r12[c] * (-dpdr / r);
      forces[3 * a1 + c] += f1[c];
      forces[3 * a2 + c] -= f1[c];
    }
    e += k * (r - r0) * (r - r0);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) v[3 * i + j] += f1[i] * r12[j];
  }
  *energy = e;
  if (virial)
    for (c = 0; c < 9; c++) virial[c] = v[c];
  return 0;
}

/* AngleSystemForce::calcAngle (force/bonded/AngleSystemForce.h:86-171):
 * harmonic in theta = atan2(|r12 x r32|, r12 . r32) plus the Urey-Bradley
 * spring between atoms 1 and 3; d theta / d x1 = (u12 cos - u32) /
 * (sin d12) and likewise for atom 3, atom 2 takes minus their sum.
 * params: k_theta, theta0, k_ub, r_ub. */
int orc_angle_force(const orc_system *s, int na, const int *atoms, const double *params,
                    double *forces, double *energy, double *virial) {
  pbc_t p;
  int t, c;
  double e = 0.0, v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  pbc_set(s, &p);
  for (t = 0; t < na; t++) {
    const int a1 = atoms[3 * t], a2 = atoms[3 * t + 1], a3 = atoms[3 * t + 2];
    const double kt = params[4 * t], t0 = params[4 * t + 1], kub = params[4 * t + 2],
                 rub = params[4 * t + 3];
    double r12[3], r32[3], r13[3], r2, cr[3], f1[3], f3[3];
    pbc_mindiff(&p, s->pos + 3 * a2, s->pos + 3 * a1, r12, &r2);
    pbc_mindiff(&p, s->pos + 3 * a2, s->pos + 3 * a3, r32, &r2);
    pbc_mindiff(&p, s->pos + 3 * a3, s->pos + 3 * a1, r13, &r2);
    const double d12 = sqrt(norm2(r12)), d32 = sqrt(norm2(r32)), d13 = sqrt(norm2(r13));
    cross3(r12, r32, cr);
    const double theta = atan2(sqrt(norm2(cr)), dot3(r12, r32));
    const double st = sin(theta), ct = cos(theta);
    const double dpdt = 2.0 * kt * (theta - t0);
    const double ub = 2.0 * kub * (d13 - rub);
    for (c = 0; c < 3; c++) {
      const double u12 = r12[c] / d12, u32 = r32[c] / d32, u13 = r13[c] / d13;
      const double dt1 = (u12 * ct - u32) / (st * d12);
      const double dt3 = (u32 * ct - u12) / (st * d32);
      const double ub1 = u13 * ub;
      f1[c] = -dt1 * dpdt - ub1;
      f3[c] = -dt3 * dpdt - (-ub1);
    }
    for (c = 0; c < 3; c++) {
      forces[3 * a1 + c] += f1[c];
      forces[3 * a2 + c] += -f1[c] - f3[c];
      forces[3 * a3 + c] += f3[c];
    }
    e += kt * (theta - t0) * (theta - t0) + kub * (d13 - rub) * (d13 - rub);
    for (int i = 0; i < 3; i++)
      for (int j = i; j < 3; j++) {
        const double w = f1[i] * r12[j] + f3[i] * r32[j];
        v[3 * i + j] += w;
        if (j != i) v[3 * j + i] += w;
      }
  }
  *energy = e;
  if (virial)
    for (c = 0; c < 9; c++) virial[c] = v[c];
  return 0;
}

void orc_kick(int n, const double *mass, const double *forces, double h,
              double *vel) {
  int i, c;
  for (i = 0; i < n; i++)
    for (c = 0; c < 3; c++) vel[3 * i + c] += forces[3 * i + c] * h / mass[i];
}
void orc_drift(int n, const double *vel, double h, double *pos) {
  int i;
  for (i = 0; i < 3 * n; i++) pos[i] += vel[i] * h;
}
void orc_langevin_half_kick(int n, const double *mass, const double *forces,
                            double timestep_fs, double gamma_ps,
                            double temperature, const double *gauss,
                            double *vel) {
  int i, c;
  const double gamma = gamma_ps / (1000 * PM_INV_TIMEFACTOR);
  const double dt = timestep_fs * PM_INV_TIMEFACTOR;
  const double fdt = (1.0 - exp(-0.5 * gamma * dt)) / gamma;
  const double vdt = exp(-0.5 * gamma * dt);
  const double ndt = sqrt((1.0 - exp(-gamma * dt)) / (2.0 * gamma));
  const double fc = 2 * PM_BOLTZMANN * temperature * gamma;
  for (i = 0; i < n; i++) {
    double m = mass[i];
    double sq = sqrt(fc / m);
    for (c = 0; c < 3; c++)
      vel[3 * i + c] = vel[3 * i + c] * vdt + forces[3 * i + c] * fdt / m +
                       gauss[3 * i + c] * sq * ndt;
  }
}
