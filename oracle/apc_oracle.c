/*
 * Test infrastructure (oracle): plain-C restatement of the reference's per-timestep
 * gravity path.  It checks the CUDA path and is never part of the product.
 *
 * Each function cites the reference code it restates (paths relative to the
 * reference project root).  It reproduces the reference's sequential algorithms
 * and output orders, including:
 *   - the temp-node order of the selection;
 *   - the octant-0-only sort in the neighbour search;
 *   - the INSERT_VALUES matrix assembly.
 * Where the reference reads out of bounds, the restatement guards the read and says
 * so.  Its key sort orders equal keys by particle index, where the reference's
 * std::sort leaves that order unspecified (octree.cpp:148).
 */
#include "apc_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "gmres_petsc.h"
#include "lsq_householder.h"

typedef struct {
  uint64_t key;
  int index;
} keyidx;

typedef struct {
  /* Physical_particle (particle.h:5-21) */
  int n;
  double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
  /* configuration */
  int depth, bc, lm, maxnc;
  double box[6];
  double gfd_c;
  /* Octree members (octree.h:60-214) */
  keyidx *ki;
  int treelen;
  int *numnodes;
  uint64_t *nkey;
  int *ndepth, *nfirst, *ncount, *nfirstchild, *nnchild;
  double *lox, *loy, *loz, *upx, *upy, *upz;
  /* Computational_particle (particle.h:23-53) */
  int nc, nv, nb, size, nneigh;
  double *cx, *cy, *cz, *ch;
  int *cfirst, *ccount, *ctype, *cfneigh, *cnneigh, *neigh24;
  double *density, *potential, *deriv, *bcrhs;
  int *st_idx;
  double *st_dist;
  double t_select, t_solve, t_move;
} apcor;

static oracle_gmres_params g_gm = {30, 1e-5, 1e-50, 1e5, 10000, 0, 0.0, 0};
#define MAX_STATS 64
static struct {
  int its, reason;
  double rnorm, sec;
} g_stats[MAX_STATS];
static int g_nstats = 0;
static int g_keep_n[2];
static int *g_keep_rp[2], *g_keep_ci[2];
static double *g_keep_v[2];

static double wall(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ------------------------------------------------------------------ keys */

/* Octree::computeKey64 (octree.cpp:676-852): `depth` bisections of the bounding box,
 * 3 bits per level (x -> 4, y -> 2, z -> 1), level 1 most significant.  A NaN
 * coordinate matches none of the eight cases and leaves that level unshifted, as in
 * the reference's if-else chain. */
uint64_t apcor_key64(double x, double y, double z, const double *box, int depth) {
  uint64_t key = 0;
  double lx = box[0], rx = box[1], ly = box[2], ry = box[3], lz = box[4], rz = box[5];
  for (int i = 1; i <= depth; ++i) {
    double mx = (lx + rx) / 2.0, my = (ly + ry) / 2.0, mz = (lz + rz) / 2.0;
    int xl = x < mx, xh = x >= mx, yl = y < my, yh = y >= my, zl = z < mz, zh = z >= mz;
    if (!((xl || xh) && (yl || yh) && (zl || zh))) continue;
    key = (key << 3) + (uint64_t)(xh * 4 + yh * 2 + zh);
    if (xh) lx = mx; else rx = mx;
    if (yh) ly = my; else ry = my;
    if (zh) lz = mz; else rz = mz;
  }
  return key;
}

static int cmp_keyidx(const void *a, const void *b) {
  const keyidx *p = (const keyidx *)a, *q = (const keyidx *)b;
  if (p->key != q->key) return p->key < q->key ? -1 : 1;
  return (p->index > q->index) - (p->index < q->index);
}

static void free_octree(apcor *o) {
  free(o->ki); free(o->numnodes); free(o->nkey); free(o->ndepth); free(o->nfirst);
  free(o->ncount); free(o->nfirstchild); free(o->nnchild);
  free(o->lox); free(o->loy); free(o->loz); free(o->upx); free(o->upy); free(o->upz);
  o->ki = NULL; o->numnodes = NULL; o->nkey = NULL; o->ndepth = NULL; o->nfirst = NULL;
  o->ncount = NULL; o->nfirstchild = NULL; o->nnchild = NULL;
  o->lox = o->loy = o->loz = o->upx = o->upy = o->upz = NULL;
  o->treelen = 0;
}

/* Octree::buildOctree (octree.cpp:111-494) */
static void build_octree(apcor *o) {
  const int N = o->n, D = o->depth;
  free_octree(o);
  o->ki = (keyidx *)malloc(sizeof(keyidx) * (size_t)(N > 0 ? N : 1));
#pragma omp parallel for
  for (int i = 0; i < N; ++i) {
    o->ki[i].key = apcor_key64(o->x[i], o->y[i], o->z[i], o->box, D);
    o->ki[i].index = i;
  }
  qsort(o->ki, (size_t)N, sizeof(keyidx), cmp_keyidx);

  uint64_t *mask = (uint64_t *)malloc(sizeof(uint64_t) * (D + 1));
  int *base = (int *)malloc(sizeof(int) * (D + 1));
  o->numnodes = (int *)malloc(sizeof(int) * (D + 1));
  int *nn = o->numnodes;
  mask[D] = (D >= 21) ? (~(uint64_t)0 >> 1) : (((uint64_t)1 << (3 * D)) - 1);
  mask[0] = 0;
  for (int k = D - 1; k >= 1; --k) {
    int s = 3 * (D - k);
    mask[k] = (mask[D] >> s) << s;
  }
  nn[0] = 1;
  for (int k = 1; k <= D; ++k) {
    int count = 1;
    for (int i = 1; i < N; ++i)
      if ((o->ki[i].key & mask[k]) != (o->ki[i - 1].key & mask[k])) ++count;
    nn[k] = count;
  }
  base[0] = 0;
  if (D >= 1) base[1] = 1;
  for (int k = 2; k <= D; ++k) base[k] = base[k - 1] + nn[k - 1];
  int T = 0;
  for (int k = 0; k <= D; ++k) T += nn[k];
  o->treelen = T;
  o->nkey = (uint64_t *)malloc(sizeof(uint64_t) * T);
  o->ndepth = (int *)malloc(sizeof(int) * T);
  o->nfirst = (int *)malloc(sizeof(int) * T);
  o->ncount = (int *)malloc(sizeof(int) * T);
  o->nfirstchild = (int *)malloc(sizeof(int) * T);
  o->nnchild = (int *)malloc(sizeof(int) * T);
  o->lox = (double *)malloc(sizeof(double) * T);
  o->loy = (double *)malloc(sizeof(double) * T);
  o->loz = (double *)malloc(sizeof(double) * T);
  o->upx = (double *)malloc(sizeof(double) * T);
  o->upy = (double *)malloc(sizeof(double) * T);
  o->upz = (double *)malloc(sizeof(double) * T);
  if (N > 0) {
    /* deepest level (octree.cpp:232-267) */
    int b = base[D];
    o->nkey[b] = o->ki[0].key;
    o->ndepth[b] = D;
    o->nfirst[b] = 0;
    o->nnchild[b] = 0;
    o->nfirstchild[b] = -1;
    int j = 1, fix = 0;
    for (int i = 1; i < N; ++i) {
      if (o->ki[i].key != o->ki[i - 1].key) {
        o->nkey[b + j] = o->ki[i].key;
        o->ndepth[b + j] = D;
        o->nfirst[b + j] = i;
        o->nnchild[b + j] = 0;
        o->nfirstchild[b + j] = -1;
        o->ncount[b + j - 1] = i - fix;
        ++j;
        fix = i;
      }
    }
    o->ncount[b + j - 1] = N - fix;
    /* upper levels (octree.cpp:276-313) */
    for (int level = D - 1; level >= 0; --level) {
      int bl = base[level], bc = base[level + 1];
      j = 1;
      fix = 0;
      o->nkey[bl] = o->nkey[bc] & mask[level];
      o->ndepth[bl] = level;
      o->nfirst[bl] = 0;
      o->nfirstchild[bl] = bc;
      int sum = o->ncount[bc];
      o->ncount[bl] = sum;
      for (int i = 1; i < nn[level + 1]; ++i) {
        if ((o->nkey[bc + i] & mask[level]) != (o->nkey[bc + i - 1] & mask[level])) {
          o->nkey[bl + j] = o->nkey[bc + i] & mask[level];
          o->ndepth[bl + j] = level;
          o->nfirst[bl + j] = o->nfirst[bc + i];
          o->ncount[bl + j - 1] = sum;
          o->nfirstchild[bl + j] = bc + i;
          o->nnchild[bl + j - 1] = i - fix;
          ++j;
          fix = i;
          sum = o->ncount[bc + i];
        } else {
          sum += o->ncount[bc + i];
        }
      }
      o->nnchild[bl + j - 1] = nn[level + 1] - fix;
      o->ncount[bl + j - 1] = sum;
    }
    /* node bounds from the parent's (octree.cpp:331-437) */
    double xw = o->box[1] - o->box[0], yw = o->box[3] - o->box[2], zw = o->box[5] - o->box[4];
    o->lox[0] = o->box[0]; o->loy[0] = o->box[2]; o->loz[0] = o->box[4];
    o->upx[0] = o->box[1]; o->upy[0] = o->box[3]; o->upz[0] = o->box[5];
    for (int level = 0; level < D; ++level) {
      xw *= 0.5; yw *= 0.5; zw *= 0.5;
      for (int i = 0; i < nn[level]; ++i) {
        int p = base[level] + i;
        for (int c = o->nfirstchild[p]; c < o->nfirstchild[p] + o->nnchild[p]; ++c) {
          unsigned t = (unsigned)((o->nkey[c] >> (3 * (D - level - 1))) & 7u);
          o->lox[c] = (t & 4) ? o->lox[p] + xw : o->lox[p];
          o->upx[c] = (t & 4) ? o->upx[p] : o->upx[p] - xw;
          o->loy[c] = (t & 2) ? o->loy[p] + yw : o->loy[p];
          o->upy[c] = (t & 2) ? o->upy[p] : o->upy[p] - yw;
          o->loz[c] = (t & 1) ? o->loz[p] + zw : o->loz[p];
          o->upz[c] = (t & 1) ? o->upz[p] : o->upz[p] - zw;
        }
      }
    }
  }
  free(mask);
  free(base);
}

/* Octree::periodic_wrap (octree.cpp:3035-3062) */
static double owrap(const apcor *o, double x, int dim) {
  if (o->bc == 1) {
    double len = o->box[2 * dim + 1] - o->box[2 * dim];
    while (x >= 0.5 * len) x -= len;
    while (x < -(0.5 * len)) x += len;
  }
  return x;
}

/* ------------------------------------------------------------ selection */

typedef struct {
  double *tx, *ty, *tz;
  int *leaf, *n_p, *old_index, *particle_index, *parent, *level, *child, *neigh;
} temp_nodes;

static const int k_opp[6] = {1, 0, 3, 2, 5, 4};

/* which child of the direction-d neighbour is face-adjacent to child c */
static int adj_child(int c, int d) {
  switch (d) {
    case 0: return c & ~4; /* x+ */
    case 1: return c | 4;  /* x- */
    case 2: return c | 2;  /* y- */
    case 3: return c & ~2; /* y+ */
    case 4: return c & ~1; /* z+ */
    default: return c | 1; /* z- */
  }
}
/* sibling of child c in direction d, or -1 when the neighbour is outside the parent */
static int sibling(int c, int d) {
  int bx = (c >> 2) & 1, by = (c >> 1) & 1, bz = c & 1;
  switch (d) {
    case 0: return bx ? -1 : (c | 4);
    case 1: return bx ? (c & ~4) : -1;
    case 2: return by ? (c & ~2) : -1;
    case 3: return by ? -1 : (c | 2);
    case 4: return bz ? -1 : (c | 1);
    default: return bz ? (c & ~1) : -1;
  }
}

static double tdist2(const apcor *o, const temp_nodes *t, int a, int b) {
  double dx = owrap(o, t->tx[a] - t->tx[b], 0);
  double dy = owrap(o, t->ty[a] - t->ty[b], 1);
  double dz = owrap(o, t->tz[a] - t->tz[b], 2);
  return dx * dx + dy * dy + dz * dz;
}

/* the child of opened node i nearest to node q (octree.cpp:1803-1820) */
static int nearest_child(const apcor *o, const temp_nodes *t, int q, int i) {
  double mindis = tdist2(o, t, q, t->child[8 * i]);
  int best = 0;
  for (int c = 0; c < 8; ++c) {
    double dis = tdist2(o, t, q, t->child[8 * i + c]);
    if (dis < mindis) { mindis = dis; best = c; }
  }
  return t->child[8 * i + best];
}

/* Open temp node i: create its 8 children at j..j+7 in octant order ---, --+, -+-,
 * -++, +--, +-+, ++-, +++ (octree.cpp:1185-1779 top-down; 1827-2555 bottom-up).
 * `balance` selects the bottom-up linking rule (descend to the nearest same-level
 * node, back-link only at equal level) over the top-down one. */
static void open_node(const apcor *o, temp_nodes *t, int i, int j, double hx, double hy, double hz,
                      int balance) {
  int inode = t->old_index[i];
  int l = 0;
  if (inode >= 0) l = o->nnchild[inode];
  int np[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (!l) {
    for (int i1 = t->particle_index[i]; i1 < t->particle_index[i] + t->n_p[i]; ++i1) {
      int p = o->ki[i1].index;
      int bx = !(o->x[p] < t->tx[i]), by = !(o->y[p] < t->ty[i]), bz = !(o->z[p] < t->tz[i]);
      /* the reference tests x<tx / x>=tx pairs; a NaN coordinate counts in no octant */
      if ((o->x[p] < t->tx[i] || o->x[p] >= t->tx[i]) && (o->y[p] < t->ty[i] || o->y[p] >= t->ty[i]) &&
          (o->z[p] < t->tz[i] || o->z[p] >= t->tz[i]))
        np[bx * 4 + by * 2 + bz]++;
    }
  }
  int prefix = 0;
  for (int c = 0; c < 8; ++c) {
    int bx = (c >> 2) & 1, by = (c >> 1) & 1, bz = c & 1;
    int k = j + c;
    int i2 = -1;
    for (int i1 = (l ? o->nfirstchild[inode] : 0); i1 < (l ? o->nfirstchild[inode] + l : 0); ++i1) {
      double cxv = (o->upx[i1] + o->lox[i1]) / 2, cyv = (o->upy[i1] + o->loy[i1]) / 2,
             czv = (o->upz[i1] + o->loz[i1]) / 2;
      int okx = bx ? (cxv > t->tx[i]) : (cxv < t->tx[i]);
      int oky = by ? (cyv > t->ty[i]) : (cyv < t->ty[i]);
      int okz = bz ? (czv > t->tz[i]) : (czv < t->tz[i]);
      if (okx && oky && okz) { i2 = i1; break; }
    }
    if (i2 > 0) {
      t->old_index[k] = i2;
      t->particle_index[k] = o->nfirst[i2];
      t->n_p[k] = o->ncount[i2];
    } else {
      /* the reference indexes the octree arrays with the temp index i here
       * (octree.cpp:1258 and siblings); guarded against i >= tree length */
      t->old_index[k] = -1;
      t->particle_index[k] = (i < o->treelen ? o->nfirst[i] : 0) + prefix;
      t->n_p[k] = np[c];
    }
    prefix += np[c];
    t->parent[k] = i;
    t->level[k] = t->level[i] + 1;
    t->leaf[k] = -1;
    t->child[8 * i + c] = k;
    t->tx[k] = bx ? t->tx[i] + 0.25 * hx : t->tx[i] - 0.25 * hx;
    t->ty[k] = by ? t->ty[i] + 0.25 * hy : t->ty[i] - 0.25 * hy;
    t->tz[k] = bz ? t->tz[i] + 0.25 * hz : t->tz[i] - 0.25 * hz;
    for (int d = 0; d < 6; ++d) {
      int s = sibling(c, d);
      if (s >= 0) {
        t->neigh[6 * k + d] = j + s;
        continue;
      }
      int i1 = t->neigh[6 * i + d];
      if (!balance) {
        if (i1 >= 0 && t->leaf[i1] == 0) {
          i1 = t->child[8 * i1 + adj_child(c, d)];
          t->neigh[6 * k + d] = i1;
          t->neigh[6 * i1 + k_opp[d]] = k;
        } else {
          t->neigh[6 * k + d] = i1;
        }
      } else {
        while (i1 > 0 && t->leaf[i1] == 0 && t->level[i1] < t->level[k]) i1 = nearest_child(o, t, k, i1);
        t->neigh[6 * k + d] = i1;
        /* the reference reads level[-1] here when i1 == -1 (non-periodic); guarded */
        if (i1 >= 0 && t->level[i1] == t->level[k]) t->neigh[6 * i1 + k_opp[d]] = k;
      }
    }
  }
}

static void halve(double h0, int lev, double *h) {
  double v = h0;
  for (int i = 0; i < lev; ++i) v = 0.5 * v;
  *h = v;
}

/* Octree::select_computational_particles_2to1_3d (octree.cpp:1050-3001).
 * Returns the number of output cells, or -1 when nmax temp nodes do not suffice. */
static int select_2to1(apcor *o, double c, int order, int nmax, int mindepth, int maxdepth) {
  temp_nodes t;
  t.tx = (double *)malloc(sizeof(double) * nmax);
  t.ty = (double *)malloc(sizeof(double) * nmax);
  t.tz = (double *)malloc(sizeof(double) * nmax);
  t.leaf = (int *)malloc(sizeof(int) * nmax);
  t.n_p = (int *)malloc(sizeof(int) * nmax);
  t.old_index = (int *)malloc(sizeof(int) * nmax);
  t.particle_index = (int *)malloc(sizeof(int) * nmax);
  t.parent = (int *)malloc(sizeof(int) * nmax);
  t.level = (int *)malloc(sizeof(int) * nmax);
  t.child = (int *)malloc(sizeof(int) * 8 * (size_t)nmax);
  t.neigh = (int *)malloc(sizeof(int) * 6 * (size_t)nmax);
  int rc = -1;
  int i = 0, j = 1;
  t.tx[0] = (o->upx[0] + o->lox[0]) / 2;
  t.ty[0] = (o->upy[0] + o->loy[0]) / 2;
  t.tz[0] = (o->upz[0] + o->loz[0]) / 2;
  t.n_p[0] = o->ncount[0];
  t.old_index[0] = 0;
  t.particle_index[0] = o->nfirst[0];
  t.parent[0] = -1;
  t.level[0] = o->ndepth[0];
  double hx0 = o->upx[0] - o->lox[0], hy0 = o->upy[0] - o->loy[0], hz0 = o->upz[0] - o->loz[0];
  double h0 = pow(hx0 * hy0 * hz0, 1.0 / 3);
  for (int d = 0; d < 6; ++d) t.neigh[d] = (o->bc == 1) ? 0 : -1;
  if (o->bc == 1)
    for (int k = 0; k < 8; ++k) t.child[k] = k + 1;

  /* top-down sweep (octree.cpp:1161-1790) */
  while (j - i > 0) {
    double temp = 1.0 * t.n_p[i], h, hx, hy, hz;
    halve(h0, t.level[i], &h);
    halve(hx0, t.level[i], &hx);
    halve(hy0, t.level[i], &hy);
    halve(hz0, t.level[i], &hz);
    for (int i1 = 0; i1 < 2 * order - 2; ++i1) temp = temp * h;
    if ((temp > c || t.level[i] < mindepth) && t.level[i] < maxdepth) {
      t.leaf[i] = 0;
      open_node(o, &t, i, j, hx, hy, hz, 0);
      j += 8;
      if (j + 8 > nmax) goto done;
    } else {
      t.leaf[i] = 1;
    }
    ++i;
  }

  /* bottom-up 2:1 balance (octree.cpp:1793-2718) */
  {
    int ml = t.level[i - 1];
    for (int ln = ml; ln > 1; --ln) {
      for (int i0 = 0; j > i0; ++i0) {
        if (t.level[i0] != ln) continue;
        for (int di = 0; di < 6; ++di) {
          int q = t.neigh[6 * i0 + di];
          while (q > 0 && t.leaf[q] == 0 && t.level[q] < ln) {
            q = nearest_child(o, &t, i0, q);
            t.neigh[6 * i0 + di] = q;
          }
          while (q > 0 && t.level[q] < ln - 1) {
            double hx, hy, hz;
            t.leaf[q] = 0;
            halve(hx0, t.level[q], &hx);
            halve(hy0, t.level[q], &hy);
            halve(hz0, t.level[q], &hz);
            open_node(o, &t, q, j, hx, hy, hz, 1);
            j += 8;
            if (j + 8 > nmax) goto done;
            q = t.neigh[6 * i0 + di];
            while (q > 0 && t.leaf[q] == 0 && t.level[q] < ln) {
              q = nearest_child(o, &t, i0, q);
              t.neigh[6 * i0 + di] = q;
            }
          }
        }
      }
      for (int i0 = 0; j > i0; ++i0) {
        if (t.level[i0] != ln) continue;
        for (int di = 0; di < 6; ++di) {
          int q = t.neigh[6 * i0 + di];
          while (q > 0 && t.leaf[q] == 0 && t.level[q] < ln) {
            q = nearest_child(o, &t, i0, q);
            t.neigh[6 * i0 + di] = q;
          }
        }
      }
    }
  }

  /* output (octree.cpp:2720-3000) */
  {
    int nleaf = 0, nbmax = 0;
    for (int k = 0; k < j; ++k)
      if (t.leaf[k]) {
        ++nleaf;
        for (int d = 0; d < 6; ++d) nbmax += t.neigh[6 * k + d] == -1;
      }
    int cap = nleaf + nbmax;
    free(o->cx); free(o->cy); free(o->cz); free(o->ch); free(o->cfirst); free(o->ccount);
    free(o->ctype); free(o->cfneigh); free(o->cnneigh); free(o->neigh24);
    o->cx = (double *)malloc(sizeof(double) * (cap + 1));
    o->cy = (double *)malloc(sizeof(double) * (cap + 1));
    o->cz = (double *)malloc(sizeof(double) * (cap + 1));
    o->ch = (double *)malloc(sizeof(double) * (cap + 1));
    o->cfirst = (int *)malloc(sizeof(int) * (cap + 1));
    o->ccount = (int *)malloc(sizeof(int) * (cap + 1));
    o->ctype = (int *)malloc(sizeof(int) * (cap + 1));
    o->cfneigh = (int *)malloc(sizeof(int) * (cap + 1));
    o->cnneigh = (int *)malloc(sizeof(int) * (cap + 1));
    o->neigh24 = (int *)malloc(sizeof(int) * (24 * (size_t)nleaf + 1));
    int nc = 0, nv = 0, nb = 0, m = 0;
    for (int pass = 0; pass < 2; ++pass) {
      int want = pass == 0 ? 1 : -1;
      for (int k = 0; k < j; ++k) {
        if (t.leaf[k] != want) continue;
        o->cx[m] = t.tx[k];
        o->cy[m] = t.ty[k];
        o->cz[m] = t.tz[k];
        halve(h0, t.level[k], &o->ch[m]);
        o->ccount[m] = t.n_p[k];
        o->cfirst[m] = t.particle_index[k];
        o->ctype[m] = pass == 0 ? 0 : -1;
        t.particle_index[k] = m;
        ++m;
        if (pass == 0) ++nc; else ++nv;
      }
    }
    static const int dir_order[6] = {0, 1, 3, 2, 4, 5};
    static const int quad[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {2, 3, 6, 7},
                                   {0, 1, 4, 5}, {0, 2, 4, 6}, {1, 3, 5, 7}};
    int total = 0, row = 0;
    for (int k = 0; k < j; ++k) {
      if (!t.leaf[k]) continue;
      o->cfneigh[row] = total;
      int i2 = 0;
      for (int dd = 0; dd < 6; ++dd) {
        int d = dir_order[dd];
        int q = t.neigh[6 * k + d];
        if (q == -1) {
          int b = nc + nv + nb;
          o->cx[b] = (d == 0) ? 1 : (d == 1) ? -1 : t.tx[k];
          o->cy[b] = (d == 3) ? 1 : (d == 2) ? -1 : t.ty[k];
          o->cz[b] = (d == 4) ? 1 : (d == 5) ? -1 : t.tz[k];
          halve(h0, t.level[k], &o->ch[b]);
          o->ccount[b] = 0;
          o->cfirst[b] = -1;
          o->neigh24[total + i2] = b;
          ++i2;
          ++nb;
        } else if (t.leaf[q]) {
          o->neigh24[total + i2] = t.particle_index[q];
          ++i2;
        } else {
          for (int a = 0; a < 4; ++a) o->neigh24[total + i2 + a] = t.particle_index[t.child[8 * q + quad[d][a]]];
          i2 += 4;
        }
      }
      total += i2;
      o->cnneigh[row] = i2;
      ++row;
    }
    for (int b = nc + nv; b < nc + nv + nb; ++b) {
      o->cnneigh[b] = 0;
      o->cfneigh[b] = total;
      o->ctype[b] = 1;
    }
    o->nc = nc;
    o->nv = nv;
    o->nb = nb;
    o->size = nc + nv + nb;
    o->nneigh = total;
    free(o->density); free(o->potential); free(o->deriv); free(o->bcrhs); free(o->st_idx); free(o->st_dist);
    o->density = (double *)calloc((size_t)o->size + 1, sizeof(double));
    o->potential = (double *)calloc((size_t)o->size + 1, sizeof(double));
    o->deriv = (double *)calloc(9 * (size_t)o->size + 1, sizeof(double));
    o->bcrhs = (double *)calloc((size_t)o->size + 1, sizeof(double));
    o->st_idx = (int *)calloc((size_t)o->lm * (o->size + 1), sizeof(int));
    o->st_dist = (double *)calloc((size_t)o->lm * (o->size + 1), sizeof(double));
    rc = o->size;
  }
done:
  free(t.tx); free(t.ty); free(t.tz); free(t.leaf); free(t.n_p); free(t.old_index);
  free(t.particle_index); free(t.parent); free(t.level); free(t.child); free(t.neigh);
  return rc;
}

/* -------------------------------------------------------------- solver */

/* Solver::periodic_wrap (solver.cpp:574-594) */
static double swrap(const apcor *o, double x, int dim) { return owrap(o, x, dim); }

/* Solver::get_squared_distance (solver.cpp:596-598) */
static double sqdist(const apcor *o, double dx, double dy, double dz) {
  return swrap(o, dx, 0) * swrap(o, dx, 0) + swrap(o, dy, 1) * swrap(o, dy, 1) +
         swrap(o, dz, 2) * swrap(o, dz, 2);
}

/* apartition / aquickSort (solver.cpp:600-632) */
static int apartition(double *a, int *b, int l, int r) {
  double pivot = a[l], t;
  int i = l, j = r + 1, ti;
  for (;;) {
    do ++i; while (i <= r && a[i] <= pivot);
    do --j; while (a[j] > pivot);
    if (i >= j) break;
    t = a[i]; a[i] = a[j]; a[j] = t;
    ti = b[i]; b[i] = b[j]; b[j] = ti;
  }
  t = a[l]; a[l] = a[j]; a[j] = t;
  ti = b[l]; b[l] = b[j]; b[j] = ti;
  return j;
}
static void aquicksort(double *a, int *b, int l, int r) {
  if (l < r) {
    int j = apartition(a, b, l, r);
    aquicksort(a, b, l, j - 1);
    aquicksort(a, b, j + 1, r);
  }
}

/* rotation used to bucket neighbours into octants (solver.cpp:464-475) */
static void rotation(double A[9]) {
  double al = 0.01, be = 0.001, ga = 0.0001;
  A[0] = cos(al) * cos(ga) - sin(al) * sin(be) * sin(ga);
  A[1] = -sin(al) * cos(be);
  A[2] = -cos(al) * sin(ga) - sin(al) * sin(be) * cos(ga);
  A[3] = cos(al) * sin(be) * sin(ga) + sin(al) * cos(ga);
  A[4] = cos(al) * cos(be);
  A[5] = cos(al) * sin(be) * cos(ga) - sin(al) * sin(ga);
  A[6] = cos(be) * sin(ga);
  A[7] = -sin(be);
  A[8] = cos(be) * cos(ga);
}

/* Solver::searchneighboroctant (solver.cpp:456-570).  Writes lm neighbour indices and
 * true distances.  Returns 0, or a negative code where the reference calls exit():
 * -1 too many neighbours in an octant (solver.cpp:535-539), -2 not enough neighbours
 * after 5 expansions (solver.cpp:544-550), -3 invalid neighbour index (511-519). */
static int search_octant(const apcor *o, int i0, int *neigh, double *distance, int nbuf,
                         const double A[9]) {
  const int lm = o->lm, nq = 10 * lm;
  int nn[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int *tn = (int *)calloc(8 * (size_t)nq + 1, sizeof(int));
  double *td = (double *)calloc(8 * (size_t)nq + 1, sizeof(double));
  int rc = 0, l;
  for (int q = o->cfneigh[i0]; q < o->cfneigh[i0] + o->cnneigh[i0]; ++q) {
    int m = o->neigh24[q];
    double wx = swrap(o, o->cx[m] - o->cx[i0], 0), wy = swrap(o, o->cy[m] - o->cy[i0], 1),
           wz = swrap(o, o->cz[m] - o->cz[i0], 2);
    double xt = A[0] * wx + A[1] * wy + A[2] * wz;
    double yt = A[3] * wx + A[4] * wy + A[5] * wz;
    double zt = A[6] * wx + A[7] * wy + A[8] * wz;
    int oct = (xt > 0) + 2 * (yt > 0) + 4 * (zt > 0);
    tn[oct * nq + nn[oct]] = m;
    td[oct * nq + nn[oct]] = sqdist(o, o->cx[m] - o->cx[i0], o->cy[m] - o->cy[i0], o->cz[m] - o->cz[i0]);
    nn[oct]++;
  }
  int ite = 0;
  for (l = nn[0] + nn[1] + nn[2] + nn[3] + nn[4] + nn[5] + nn[6] + nn[7]; l < lm;
       l = nn[0] + nn[1] + nn[2] + nn[3] + nn[4] + nn[5] + nn[6] + nn[7]) {
    int k = 0;
    for (int b = 0; b < 8; ++b)
      for (int e = 0; e < nn[b]; ++e) {
        if (k < nbuf) neigh[k] = tn[b * nq + e];
        ++k;
      }
    for (int a = 0; a < l; ++a) {
      int p = neigh[a];
      for (int q = o->cfneigh[p]; q < o->cfneigh[p] + o->cnneigh[p]; ++q) {
        int m = o->neigh24[q];
        if (m > o->nc + o->nv + o->nb) { rc = -3; goto out; }
        double wx = swrap(o, o->cx[m] - o->cx[i0], 0), wy = swrap(o, o->cy[m] - o->cy[i0], 1),
               wz = swrap(o, o->cz[m] - o->cz[i0], 2);
        double xt = A[0] * wx + A[1] * wy + A[2] * wz;
        double yt = A[3] * wx + A[4] * wy + A[5] * wz;
        double zt = A[6] * wx + A[7] * wy + A[8] * wz;
        int oct = (xt > 0) + 2 * (yt > 0) + 4 * (zt > 0);
        int flag = 0;
        for (int e = 0; e < nn[oct]; ++e)
          if (m == tn[oct * nq + e]) flag = 1;
        if (flag == 0 && m != i0) {
          tn[oct * nq + nn[oct]] = m;
          td[oct * nq + nn[oct]] = sqdist(o, o->cx[m] - o->cx[i0], o->cy[m] - o->cy[i0], o->cz[m] - o->cz[i0]);
          nn[oct]++;
          if (nn[oct] > nq) { rc = -1; goto out; } /* solver.cpp:533-539 */
        }
      }
    }
    if (++ite > 5) { rc = -2; goto out; }
  }
  if (l > nbuf) { rc = -1; goto out; }
  {
    int k = 0;
    for (int b = 0; b < 8; ++b) {
      double penalty = 1.0;
      /* sorts [k, k+nn[b]-1] of the bucketed storage: bucket 0 only for b == 0 */
      aquicksort(td, tn, k, k + nn[b] - 1);
      for (int e = 0; e < nn[b]; ++e) {
        neigh[k] = tn[b * nq + e];
        distance[k] = penalty * td[b * nq + e];
        penalty = penalty * 10000.0;
        ++k;
      }
    }
    aquicksort(distance, neigh, 0, l - 1);
    for (int a = 0; a < lm; ++a)
      distance[a] = sqrt(sqdist(o, o->cx[neigh[a]] - o->cx[i0], o->cy[neigh[a]] - o->cy[i0],
                                o->cz[neigh[a]] - o->cz[i0]));
  }
out:
  free(tn);
  free(td);
  return rc;
}

/* weighted monomial rows for one cell (solver.cpp:75-103 / 307-332) */
static void gfd_rows(const apcor *o, int i, const int *neigh, const double *distance, double *B,
                     double *w) {
  const int lm = o->lm, ln = 9;
  double maxdis = 0;
  for (int j = 0; j < lm; ++j)
    if (distance[j] > maxdis) maxdis = distance[j];
  maxdis = maxdis * 0.7;
  for (int j = 0; j < lm; ++j) {
    double weight = (exp(-distance[j] * distance[j] / maxdis / maxdis) - exp(-4)) / (1 - exp(-4));
    double p1 = swrap(o, o->cx[neigh[j]] - o->cx[i], 0) / o->ch[i];
    double p2 = swrap(o, o->cy[neigh[j]] - o->cy[i], 1) / o->ch[i];
    double p3 = swrap(o, o->cz[neigh[j]] - o->cz[i], 2) / o->ch[i];
    double *r = B + j * ln;
    r[0] = p1; r[1] = p2; r[2] = p3;
    r[3] = p1 * p1 / 2.0; r[4] = p2 * p2 / 2.0; r[5] = p3 * p3 / 2.0;
    r[6] = p1 * p2; r[7] = p1 * p3; r[8] = p2 * p3;
    for (int k = 0; k < ln; ++k) r[k] = r[k] * weight;
    w[j] = weight;
  }
}

typedef struct {
  int n;
  int *cnt;
  int *col; /* n x cap */
  double *val;
  int cap;
} rowmat;

static void rm_init(rowmat *a, int n, int cap) {
  a->n = n;
  a->cap = cap;
  a->cnt = (int *)calloc((size_t)n + 1, sizeof(int));
  a->col = (int *)malloc(sizeof(int) * (size_t)n * cap + 1);
  a->val = (double *)malloc(sizeof(double) * (size_t)n * cap + 1);
}
/* MatSetValues(..., INSERT_VALUES): overwrite an existing (row, col) entry */
static void rm_insert(rowmat *a, int r, int c, double v) {
  int *cc = a->col + (size_t)r * a->cap;
  double *vv = a->val + (size_t)r * a->cap;
  for (int k = 0; k < a->cnt[r]; ++k)
    if (cc[k] == c) { vv[k] = v; return; }
  if (a->cnt[r] < a->cap) {
    cc[a->cnt[r]] = c;
    vv[a->cnt[r]] = v;
    a->cnt[r]++;
  }
}
/* AIJ assembly: CSR with columns sorted per row */
static void rm_to_csr(const rowmat *a, int **rp, int **ci, double **v) {
  int nnz = 0;
  for (int r = 0; r < a->n; ++r) nnz += a->cnt[r];
  *rp = (int *)malloc(sizeof(int) * ((size_t)a->n + 1));
  *ci = (int *)malloc(sizeof(int) * ((size_t)nnz + 1));
  *v = (double *)malloc(sizeof(double) * ((size_t)nnz + 1));
  int k = 0;
  (*rp)[0] = 0;
  for (int r = 0; r < a->n; ++r) {
    int *cc = a->col + (size_t)r * a->cap;
    double *vv = a->val + (size_t)r * a->cap;
    int c = a->cnt[r];
    for (int s = 1; s < c; ++s) {
      int key = cc[s];
      double kv = vv[s];
      int t = s - 1;
      while (t >= 0 && cc[t] > key) { cc[t + 1] = cc[t]; vv[t + 1] = vv[t]; --t; }
      cc[t + 1] = key;
      vv[t + 1] = kv;
    }
    for (int s = 0; s < c; ++s) { (*ci)[k] = cc[s]; (*v)[k] = vv[s]; ++k; }
    (*rp)[r + 1] = k;
  }
}
static void rm_free(rowmat *a) { free(a->cnt); free(a->col); free(a->val); }

static void keep_matrix(int slot, int n, int *rp, int *ci, double *v) {
  free(g_keep_rp[slot]); free(g_keep_ci[slot]); free(g_keep_v[slot]);
  g_keep_n[slot] = n;
  g_keep_rp[slot] = rp;
  g_keep_ci[slot] = ci;
  g_keep_v[slot] = v;
}

static void run_gmres(int n, const int *rp, const int *ci, const double *v, const double *b, double *x) {
  oracle_gmres_params p = g_gm;
  double t0 = wall();
  oracle_gmres_csr(n, rp, ci, v, b, x, &p);
  if (g_nstats < MAX_STATS) {
    g_stats[g_nstats].its = p.its;
    g_stats[g_nstats].reason = p.reason;
    g_stats[g_nstats].rnorm = p.rnorm;
    g_stats[g_nstats].sec = wall() - t0;
    ++g_nstats;
  }
}

/* Solver::solve (solver.cpp:382-454): Build_Linear_System (24-180), Solve_Density
 * (182-218), Solve_Potential (220-293), Differentiate (295-362).  Returns 0, or the
 * negative code of the neighbour search / a positive LAPACK info where the reference
 * calls exit(). */
/* Solver::Differentiate (solver.cpp:295-362) of a given potential: per cell the search
 * and the weighted rows again, then the least-squares solve (dgels) for the differences
 * (phi_j - phi_i) c_field; deriv9 gets the gradient / h and the Hessian / h^2.  Work
 * buffers as in solve_all (b needs lm doubles here). */
static int differentiate(apcor *o, const double *phi, double c_field, double *deriv9, int *neigh,
                         double *distance, int nbuf, const double *A, double *B, double *b, double *w) {
  const int lm = o->lm, ln = 9, M = o->nc + o->nv;
  for (int i = 0; i < M; ++i) {
    int s = search_octant(o, i, neigh, distance, nbuf, A);
    if (s) return s;
    gfd_rows(o, i, neigh, distance, B, w);
    double p4 = phi[i];
    for (int j = 0; j < lm; ++j) {
      int k = neigh[j];
      double p1 = k < M ? phi[k] : 0.0;
      b[j] = w[j] * (p1 - p4) * c_field;
    }
    int info = oracle_dgels_rowmajor(lm, ln, 1, B, ln, b, 1);
    if (info > 0) return info;
    double h = o->ch[i];
    double *d = deriv9 + 9 * (size_t)i;
    d[0] = b[0] / h; d[1] = b[1] / h; d[2] = b[2] / h;
    d[3] = b[3] / h / h; d[4] = b[4] / h / h; d[5] = b[5] / h / h;
    d[6] = b[6] / h / h; d[7] = b[7] / h / h; d[8] = b[8] / h / h;
  }
  return 0;
}

static int solve_all(apcor *o, double c_dens, double c_pot, double c_field) {
  const int lm = o->lm, ln = 9, M = o->nc + o->nv;
  double A[9];
  rotation(A);
  int nbuf = 16 * lm > 8 * 10 * lm ? 16 * lm : 8 * 10 * lm;
  int *neigh = (int *)calloc((size_t)nbuf, sizeof(int));
  double *distance = (double *)calloc((size_t)nbuf, sizeof(double));
  double *B = (double *)malloc(sizeof(double) * lm * ln);
  double *b = (double *)malloc(sizeof(double) * lm * lm);
  double *w = (double *)malloc(sizeof(double) * lm);
  double *rhs = (double *)calloc((size_t)M + 1, sizeof(double));
  rowmat A1, A2;
  rm_init(&A1, M, lm + 1);
  rm_init(&A2, M, lm + 1);
  int rc = 0;
  for (int i = 0; i < M; ++i) {
    int s = search_octant(o, i, neigh, distance, nbuf, A);
    if (s) { rc = s; goto fail; }
    memcpy(o->st_idx + (size_t)i * lm, neigh, sizeof(int) * lm);
    memcpy(o->st_dist + (size_t)i * lm, distance, sizeof(double) * lm);
    gfd_rows(o, i, neigh, distance, B, w);
    for (int j = 0; j < lm; ++j) {
      for (int k = 0; k < lm; ++k) b[j * lm + k] = 0.0;
      b[j * lm + j] = w[j];
    }
    int info = oracle_dgels_rowmajor(lm, ln, lm, B, ln, b, lm);
    if (info > 0) { rc = info; goto fail; }
    double p1, p2 = 0.0, p3;
    for (int j = 0; j < lm; ++j) {
      p1 = (b[3 * lm + j] + b[4 * lm + j] + b[5 * lm + j]) / 24.0;
      p2 = p2 - p1;
      if (neigh[j] < M) rm_insert(&A1, i, neigh[j], p1);
    }
    p2 = p2 + 1;
    rm_insert(&A1, i, i, p2);
    rhs[i] = 1.0 * o->ccount[i] / o->ch[i] / o->ch[i] / o->ch[i] * c_dens;
    if (i == 0 && o->bc == 1) {
      p3 = 0.0;
      rm_insert(&A2, i, i, 1.0);
    } else {
      p2 = 0.0;
      p3 = 0.0;
      for (int j = 0; j < lm; ++j) {
        p1 = (b[3 * lm + j] + b[4 * lm + j] + b[5 * lm + j]) / o->ch[i] / o->ch[i];
        p2 = p2 - p1;
        if (o->ctype[neigh[j]] < 1) rm_insert(&A2, i, neigh[j], p1);
        else p3 = p3 - 0.0 * p1; /* Dirichlet value 0 moved to the rhs (solver.cpp:164-170) */
      }
      rm_insert(&A2, i, i, p2);
    }
    o->bcrhs[i] = p3;
  }
  {
    int *rp1, *ci1, *rp2, *ci2;
    double *v1, *v2;
    rm_to_csr(&A1, &rp1, &ci1, &v1);
    rm_to_csr(&A2, &rp2, &ci2, &v2);
    /* Solve_Density */
    run_gmres(M, rp1, ci1, v1, rhs, o->density);
    /* Solve_Potential: mean-subtracted rhs for periodic boxes (solver.cpp:236-259) */
    if (o->bc == 0) {
      for (int i = 0; i < M; ++i) rhs[i] = (o->density[i] + o->bcrhs[i]) * c_pot;
    } else {
      double s2 = 0, s3 = 0;
      for (int i = 0; i < M; ++i) {
        s2 = s2 + o->density[i] * o->ch[i] * o->ch[i] * o->ch[i];
        s3 = s3 + o->ch[i] * o->ch[i] * o->ch[i];
      }
      s2 = s2 / s3;
      for (int i = 0; i < M; ++i) rhs[i] = (o->density[i] - s2) * c_pot;
    }
    run_gmres(M, rp2, ci2, v2, rhs, o->potential);
    keep_matrix(0, M, rp1, ci1, v1);
    keep_matrix(1, M, rp2, ci2, v2);
  }
  /* Differentiate (solver.cpp:295-362) */
  rc = differentiate(o, o->potential, c_field, o->deriv, neigh, distance, nbuf, A, B, b, w);
fail:
  rm_free(&A1);
  rm_free(&A2);
  free(neigh); free(distance); free(B); free(b); free(w); free(rhs);
  return rc;
}

/* ------------------------------------------------------------------ API */

void *apcor_create(int n, const double *x, const double *y, const double *z, const double *vx,
                   const double *vy, const double *vz, int depth, int bc, const double *box,
                   double gfd_c, int lm) {
  apcor *o = (apcor *)calloc(1, sizeof(apcor));
  o->n = n;
  double **arr[9] = {&o->x, &o->y, &o->z, &o->vx, &o->vy, &o->vz, &o->ax, &o->ay, &o->az};
  for (int k = 0; k < 9; ++k) *arr[k] = (double *)calloc((size_t)n + 1, sizeof(double));
  memcpy(o->x, x, sizeof(double) * n);
  memcpy(o->y, y, sizeof(double) * n);
  memcpy(o->z, z, sizeof(double) * n);
  memcpy(o->vx, vx, sizeof(double) * n);
  memcpy(o->vy, vy, sizeof(double) * n);
  memcpy(o->vz, vz, sizeof(double) * n);
  o->depth = depth;
  o->bc = bc;
  o->lm = lm;
  o->gfd_c = gfd_c;
  o->maxnc = 10000; /* controller.cpp:76 */
  memcpy(o->box, box, sizeof(double) * 6);
  return o;
}

void apcor_destroy(void *h) {
  apcor *o = (apcor *)h;
  if (!o) return;
  free_octree(o);
  free(o->x); free(o->y); free(o->z); free(o->vx); free(o->vy); free(o->vz);
  free(o->ax); free(o->ay); free(o->az);
  free(o->cx); free(o->cy); free(o->cz); free(o->ch); free(o->cfirst); free(o->ccount);
  free(o->ctype); free(o->cfneigh); free(o->cnneigh); free(o->neigh24);
  free(o->density); free(o->potential); free(o->deriv); free(o->bcrhs); free(o->st_idx); free(o->st_dist);
  free(o);
}

void apcor_set_gmres(int restart, double rtol, double atol, double dtol, int max_it) {
  g_gm.restart = restart;
  g_gm.rtol = rtol;
  g_gm.atol = atol;
  g_gm.dtol = dtol;
  g_gm.max_it = max_it;
}

void apcor_set_maxnc(void *h, int maxnc) { ((apcor *)h)->maxnc = maxnc; }

/* Mover::select_computational_particles (mover.cpp:17-49): rebuild the octree, then
 * retry the selection with a doubled temp-node budget while it is below 1e6 */
int apcor_select(void *h) {
  apcor *o = (apcor *)h;
  double t0 = wall();
  build_octree(o);
  int number = -1;
  const int MAXNC = 1000000;
  while (number < 0 && o->maxnc < MAXNC) {
    number = o->n > 0 ? select_2to1(o, o->gfd_c, 2, o->maxnc, 0, o->depth) : -1;
    if (number < 0) o->maxnc = o->maxnc * 2;
  }
  o->t_select += wall() - t0;
  return number;
}

int apcor_cell_counts(void *h, int *nc, int *nv, int *nb, int *nneigh) {
  apcor *o = (apcor *)h;
  *nc = o->nc;
  *nv = o->nv;
  *nb = o->nb;
  *nneigh = o->nneigh;
  return o->size;
}

int apcor_get_cells(void *h, double *x, double *y, double *z, double *len, int *first, int *count,
                    int *type, int *firstneigh, int *numneigh, int *neigh24) {
  apcor *o = (apcor *)h;
  for (int i = 0; i < o->size; ++i) {
    x[i] = o->cx[i]; y[i] = o->cy[i]; z[i] = o->cz[i]; len[i] = o->ch[i];
    first[i] = o->cfirst[i]; count[i] = o->ccount[i]; type[i] = o->ctype[i];
    firstneigh[i] = o->cfneigh[i]; numneigh[i] = o->cnneigh[i];
  }
  memcpy(neigh24, o->neigh24, sizeof(int) * o->nneigh);
  return o->size;
}

int apcor_get_keys(void *h, uint64_t *keys, int *index) {
  apcor *o = (apcor *)h;
  if (!o->ki) return -1;
  for (int i = 0; i < o->n; ++i) {
    keys[i] = o->ki[i].key;
    index[i] = o->ki[i].index;
  }
  return o->n;
}

int apcor_octree_levels(void *h, int *numnodes) {
  apcor *o = (apcor *)h;
  if (!o->numnodes) return -1;
  memcpy(numnodes, o->numnodes, sizeof(int) * (o->depth + 1));
  return o->treelen;
}

int apcor_solve(void *h, double c_dens, double c_pot, double c_field) {
  apcor *o = (apcor *)h;
  double t0 = wall();
  int rc = solve_all(o, c_dens, c_pot, c_field);
  o->t_solve += wall() - t0;
  return rc;
}

int apcor_differentiate(void *h, const double *potential, double c_field, double *deriv9) {
  apcor *o = (apcor *)h;
  const int lm = o->lm;
  double A[9];
  rotation(A);
  int nbuf = 16 * lm > 8 * 10 * lm ? 16 * lm : 8 * 10 * lm;
  int *neigh = (int *)calloc((size_t)nbuf, sizeof(int));
  double *distance = (double *)calloc((size_t)nbuf, sizeof(double));
  double *B = (double *)malloc(sizeof(double) * lm * 9);
  double *b = (double *)malloc(sizeof(double) * lm * lm);
  double *w = (double *)malloc(sizeof(double) * lm);
  int rc = differentiate(o, potential, c_field, deriv9, neigh, distance, nbuf, A, B, b, w);
  free(neigh); free(distance); free(B); free(b); free(w);
  return rc;
}

int apcor_get_fields(void *h, double *density, double *potential, double *deriv9) {
  apcor *o = (apcor *)h;
  int M = o->nc + o->nv;
  memcpy(density, o->density, sizeof(double) * M);
  memcpy(potential, o->potential, sizeof(double) * M);
  memcpy(deriv9, o->deriv, sizeof(double) * 9 * M);
  return M;
}

int apcor_get_stencils(void *h, int *idx, double *dist) {
  apcor *o = (apcor *)h;
  int M = o->nc + o->nv;
  memcpy(idx, o->st_idx, sizeof(int) * (size_t)o->lm * M);
  memcpy(dist, o->st_dist, sizeof(double) * (size_t)o->lm * M);
  return M;
}

int apcor_solve_stats(int k, int *its, double *rnorm, int *reason, double *seconds) {
  if (k < 0 || k >= g_nstats) return -1;
  *its = g_stats[k].its;
  *rnorm = g_stats[k].rnorm;
  *reason = g_stats[k].reason;
  *seconds = g_stats[k].sec;
  return 0;
}
int apcor_solve_count(void) { return g_nstats; }
void apcor_reset_solve_stats(void) { g_nstats = 0; }

int apcor_last_matrix(int which, int *n, int *nnz, int *rp, int *ci, double *v) {
  if (which < 0 || which > 1 || !g_keep_rp[which]) return -1;
  int nn = g_keep_n[which], nz = g_keep_rp[which][nn];
  if (n) *n = nn;
  if (nnz) *nnz = nz;
  if (rp) memcpy(rp, g_keep_rp[which], sizeof(int) * (nn + 1));
  if (ci) memcpy(ci, g_keep_ci[which], sizeof(int) * nz);
  if (v) memcpy(v, g_keep_v[which], sizeof(double) * nz);
  return 0;
}

/* Mover::move_velocity (mover.cpp:51-89) with the interpolation of
 * Octree::interpolation_from_node_to_particle_2to1_3d (octree.cpp:3003-3031) */
double apcor_move_velocity(void *h, double dt, double c_vel) {
  apcor *o = (apcor *)h;
  double t0 = wall();
  for (int i = 0; i < o->nc + o->nv; ++i) {
    const double *d = o->deriv + 9 * (size_t)i;
    for (int k = o->cfirst[i]; k < o->cfirst[i] + o->ccount[i]; ++k) {
      int l = o->ki[k].index;
      double dx = o->x[l] - o->cx[i], dy = o->y[l] - o->cy[i], dz = o->z[l] - o->cz[i];
      o->ax[l] = d[0] + dx * d[3] + dy * d[6] + dz * d[7];
      o->ay[l] = d[1] + dx * d[6] + dy * d[4] + dz * d[8];
      o->az[l] = d[2] + dx * d[7] + dy * d[8] + dz * d[5];
    }
  }
  double mx = 0.0;
  for (int i = 0; i < o->n; ++i) {
    o->vx[i] = o->vx[i] + o->ax[i] * c_vel * dt;
    o->vy[i] = o->vy[i] + o->ay[i] * c_vel * dt;
    o->vz[i] = o->vz[i] + o->az[i] * c_vel * dt;
    double ch = (o->ax[i] * o->ax[i] + o->ay[i] * o->ay[i] + o->az[i] * o->az[i]) * c_vel * c_vel * dt * dt;
    if (ch > mx) mx = ch;
  }
  o->t_move += wall() - t0;
  return sqrt(mx);
}

/* Mover::periodic_wrap (mover.cpp:123-153) */
static double mwrap(const apcor *o, double x, int dim) {
  if (o->bc == 1) {
    double lo = o->box[2 * dim], hi = o->box[2 * dim + 1];
    while (x >= hi) x -= hi - lo;
    while (x < lo) x += hi - lo;
  }
  return x;
}

/* Mover::move_position (mover.cpp:91-121) */
double apcor_move_position(void *h, double dt, double c_pos) {
  apcor *o = (apcor *)h;
  double t0 = wall();
  double mx = 0.0;
  for (int i = 0; i < o->n; ++i) {
    o->x[i] = mwrap(o, o->x[i] + o->vx[i] * c_pos * dt, 0);
    o->y[i] = mwrap(o, o->y[i] + o->vy[i] * c_pos * dt, 1);
    o->z[i] = mwrap(o, o->z[i] + o->vz[i] * c_pos * dt, 2);
    double ch = (o->vx[i] * o->vx[i] + o->vy[i] * o->vy[i] + o->vz[i] * o->vz[i]) * c_pos * c_pos * dt * dt;
    if (ch > mx) mx = ch;
  }
  o->t_move += wall() - t0;
  return sqrt(mx);
}

int apcor_get_particles(void *h, double *x, double *y, double *z, double *vx, double *vy,
                        double *vz, double *ax, double *ay, double *az) {
  apcor *o = (apcor *)h;
  size_t s = sizeof(double) * o->n;
  if (x) memcpy(x, o->x, s);
  if (y) memcpy(y, o->y, s);
  if (z) memcpy(z, o->z, s);
  if (vx) memcpy(vx, o->vx, s);
  if (vy) memcpy(vy, o->vy, s);
  if (vz) memcpy(vz, o->vz, s);
  if (ax) memcpy(ax, o->ax, s);
  if (ay) memcpy(ay, o->ay, s);
  if (az) memcpy(az, o->az, s);
  return o->n;
}

void apcor_phase_times(void *h, double *t3) {
  apcor *o = (apcor *)h;
  t3[0] = o->t_select;
  t3[1] = o->t_solve;
  t3[2] = o->t_move;
}
