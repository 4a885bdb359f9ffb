/*
 * CPU restatement of the CAC reference's per-timestep force path.
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE (see cac_oracle.h).
 *
 * Reference citations are to tcphan0601/CAC V3.2.0/src.
 */
#define _POSIX_C_SOURCE 200809L
#include "cac_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NC 9          /* lattice sites per element edge */
#define NU 729        /* lattice sites per element */
#define NPE 8
#define NG 8

/* ------------------------------------------------------------------ tables */

/* Element::shape_function, Hex branch (element.cpp:2988-2997), at the lattice
 * sites of ElementVecCAC::setup_interpolate_element (element_vec_cac.cpp:
 * 1881-1899): px = dx_pc*i - 1, site n = (i*ny + j)*nz + k. */
void oracle_shape_array(double *shape)
{
  double dx = 2.0 / (NC - 1), dy = 2.0 / (NC - 1), dz = 2.0 / (NC - 1);
  int n = 0;
  for (int i = 0; i < NC; i++) {
    double px = dx * i - 1.0;
    for (int j = 0; j < NC; j++) {
      double py = dy * j - 1.0;
      for (int k = 0; k < NC; k++) {
        double pz = dz * k - 1.0;
        double *s = shape + 8 * n;
        s[0] = 0.125 * (1 - px) * (1 - py) * (1 - pz);
        s[1] = 0.125 * (1 + px) * (1 - py) * (1 - pz);
        s[2] = 0.125 * (1 + px) * (1 + py) * (1 - pz);
        s[3] = 0.125 * (1 - px) * (1 + py) * (1 - pz);
        s[4] = 0.125 * (1 - px) * (1 - py) * (1 + pz);
        s[5] = 0.125 * (1 + px) * (1 - py) * (1 + pz);
        s[6] = 0.125 * (1 + px) * (1 + py) * (1 + pz);
        s[7] = 0.125 * (1 - px) * (1 + py) * (1 + pz);
        n++;
      }
    }
  }
}

/* setup_integration_point, Hex with 2x2x2 Gauss cells and UNIFORM weights
 * wscale 1 1 1 1 (element_vec_cac.cpp:2401-2558): igcell = (i*2+j)*2+k at
 * px, py, pz in {0, ncell-1}; every cell is a node with weight
 * nucell/8; CONSISTENT weighted shape = shape*weight/nucell and g2n from the
 * shape value 1 (element_vec_cac.cpp:3248-3270). */
void oracle_gauss_tables(int *g2u, int *g2n, double *wsa, double *nodal_weight)
{
  static double shape[NU * 8];
  oracle_shape_array(shape);
  double w_node = (double) NU / (1.0 * 8 + 1.0 * 0 + 1.0 * 0 + 1.0 * 0) * 1.0;
  int g = 0;
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++)
      for (int k = 0; k < 2; k++) {
        int px = i ? NC - 1 : 0, py = j ? NC - 1 : 0, pz = k ? NC - 1 : 0;
        g2u[g] = px * NC * NC + py * NC + pz;
        g++;
      }
  for (g = 0; g < NG; g++) {
    g2n[g] = -1;
    for (int n = 0; n < NPE; n++) {
      wsa[g * 8 + n] = shape[g2u[g] * 8 + n] * w_node / NU;
      if (fabs(shape[g2u[g] * 8 + n] - 1.0) < 1e-6) g2n[g] = n;
    }
  }
  *nodal_weight = (double) NU / (double) NPE;   /* element_vec_cac.cpp:1732 */
}

/* Hex inverse consistent mass matrix (element.cpp:1784-1850): the tensor
 * product over the three natural axes of [[4, -2], [-2, 4]]. */
void oracle_inverse_mass_hex(double *minv)
{
  static const int sgn[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}};
  for (int a = 0; a < 8; a++)
    for (int b = 0; b < 8; b++) {
      double v = 1.0;
      for (int d = 0; d < 3; d++) v *= (sgn[a][d] == sgn[b][d]) ? 4.0 : -2.0;
      minv[a * 8 + b] = v;
    }
}

static double g_shape[NU * 8];
static int g_g2u[NG], g_g2n[NG], g_n2g[NPE], g_u2g[NU];
static double g_wsa[NG * 8], g_nodal_weight, g_minv[64];
/* Pair::nodal_energy_weight (pair.cpp:38); minimize sets it to 1 (minimize.cpp:37) */
static double g_nodal_energy_weight = -1.0;
static int g_tables_ready = 0;
/* neigh_modify check yes for the minimiser: a due rebuild only after a move
 * past half the skin (Neighbor::decide / check_distance, neighbor.cpp:1584-1683) */
static int g_neigh_check = 0;

void oracle_set_neighbor_check(int check) { g_neigh_check = check != 0; }

/* Neighbor::check_distance for a fixed box (neighbor.cpp:1617-1683):
 * 1 when an atom or node lies farther than sqrt(triggersq) from its position
 * at the last build, triggersq = 0.25 skin^2 (neighbor.cpp:240). */
static int moved_past_trigger(const oracle_state *s, const double *xhold, const double *nodexhold,
                              double skin)
{
  const double triggersq = 0.25 * skin * skin;
  int flag = 0;
  for (int i = 0; i < s->natoms; i++) {
    double delx = s->x[3 * i] - xhold[3 * i], dely = s->x[3 * i + 1] - xhold[3 * i + 1];
    double delz = s->x[3 * i + 2] - xhold[3 * i + 2];
    if (delx * delx + dely * dely + delz * delz > triggersq) flag = 1;
  }
  for (int k = 0; k < 8 * s->nelements; k++) {
    double delx = s->nodex[3 * k] - nodexhold[3 * k], dely = s->nodex[3 * k + 1] - nodexhold[3 * k + 1];
    double delz = s->nodex[3 * k + 2] - nodexhold[3 * k + 2];
    if (delx * delx + dely * dely + delz * delz > triggersq) flag = 1;
  }
  return flag;
}

static void tables(void)
{
  if (g_tables_ready) return;
  oracle_shape_array(g_shape);
  oracle_gauss_tables(g_g2u, g_g2n, g_wsa, &g_nodal_weight);
  oracle_inverse_mass_hex(g_minv);
  for (int u = 0; u < NU; u++) g_u2g[u] = -1;
  for (int g = 0; g < NG; g++) {
    g_u2g[g_g2u[g]] = g;
    g_n2g[g_g2n[g]] = g;
  }
  g_tables_ready = 1;
}

/* ------------------------------------------------------------ geometry */

static double prd(const oracle_state *s, int d) { return s->boxhi[d] - s->boxlo[d]; }

/* element centre as ElementVecCAC::update_center_coord (element_vec_cac.cpp:3740-3765) */
static void center(const oracle_state *s, int e, double c[3])
{
  const double *nx = s->nodex + (size_t) e * 24;
  c[0] = c[1] = c[2] = 0.0;
  for (int k = 0; k < NPE; k++) {
    c[0] += nx[3 * k + 0];
    c[1] += nx[3 * k + 1];
    c[2] += nx[3 * k + 2];
  }
  for (int d = 0; d < 3; d++) c[d] = c[d] / NPE / 1;
}

/* position of an i-site: an atom, or a Gauss point interpolated as in
 * npair_half_bin_newton.cpp:284-289 (sequential sum from 0.0) */
static void isite_pos(const oracle_state *s, int i, double p[3])
{
  if (i < s->natoms) {
    memcpy(p, s->x + 3 * (size_t) i, 3 * sizeof(double));
    return;
  }
  int e = (i - s->natoms) / NG, g = (i - s->natoms) % NG;
  const double *sh = g_shape + 8 * g_g2u[g];
  const double *nx = s->nodex + (size_t) e * 24;
  p[0] = p[1] = p[2] = 0.0;
  for (int k = 0; k < NPE; k++) {
    p[0] += sh[k] * nx[3 * k + 0];
    p[1] += sh[k] * nx[3 * k + 1];
    p[2] += sh[k] * nx[3 * k + 2];
  }
}

/* delx for a neighbour in the reference's arithmetic: a ghost copy's
 * coordinate is owner + pbc*prd (atom_vec pack_border), a lattice site is
 * subtracted node by node (npair_half_bin_newton.cpp:116-119, 194-199). */
static void pair_delta(const oracle_state *s, const double xi[3], int kind, int idx, int site,
                       const int8_t img[3], double del[3])
{
  double shift[3];
  for (int d = 0; d < 3; d++) shift[d] = img[d] * prd(s, d);
  if (kind == 0) {
    const double *xj = s->x + 3 * (size_t) idx;
    for (int d = 0; d < 3; d++) del[d] = xi[d] - (img[d] ? xj[d] + shift[d] : xj[d]);
    return;
  }
  const double *sh = g_shape + 8 * site;
  const double *nx = s->nodex + (size_t) idx * 24;
  del[0] = xi[0];
  del[1] = xi[1];
  del[2] = xi[2];
  for (int k = 0; k < NPE; k++)
    for (int d = 0; d < 3; d++)
      del[d] -= sh[k] * (img[d] ? nx[3 * k + d] + shift[d] : nx[3 * k + d]);
}

/* ------------------------------------------------------ atom bins (half rule) */

/* NBinStandard::setup_bins atom part (nbin_standard.cpp:84-128) and
 * NBin::coord2atombin (nbin.cpp:126-170) for an orthogonal box. */
typedef struct {
  double lo[3], hi[3], inv[3];
  int nbin[3];
} binning;

static void setup_atom_bins(const oracle_state *s, double cutneighmax, binning *b)
{
  double binsize_optimal = 0.5 * cutneighmax;
  double binsizeinv = 1.0 / binsize_optimal;
  for (int d = 0; d < 3; d++) {
    double bbox = s->boxhi[d] - s->boxlo[d];
    b->lo[d] = s->boxlo[d];
    b->hi[d] = s->boxhi[d];
    b->nbin[d] = (int) (bbox * binsizeinv);
    if (b->nbin[d] == 0) b->nbin[d] = 1;
    double binsize = bbox / b->nbin[d];
    b->inv[d] = 1.0 / binsize;
  }
}

static int coord2bin1(const binning *b, int d, double x)
{
  int ix;
  if (x >= b->hi[d]) ix = (int) ((x - b->hi[d]) * b->inv[d]) + b->nbin[d];
  else if (x >= b->lo[d]) {
    ix = (int) ((x - b->lo[d]) * b->inv[d]);
    if (ix > b->nbin[d] - 1) ix = b->nbin[d] - 1;
  } else ix = (int) ((x - b->lo[d]) * b->inv[d]) - 1;
  return ix;
}

/* lexicographic (z, y, x) comparison of the bins of two points: >0 if the
 * second is in the upper half stencil of the first (nstencil_half_bin_3d.cpp:18-24) */
static int bin_order(const binning *b, const double p[3], const double q[3])
{
  for (int d = 2; d >= 0; d--) {
    int a = coord2bin1(b, d, p[d]), c = coord2bin1(b, d, q[d]);
    if (c != a) return c > a ? 1 : -1;
  }
  return 0;
}

/* "above and to the right" (npair_half_bin_newton.cpp:105-111, 351-355) */
static int above_right(const double q[3], const double p[3])
{
  if (q[2] < p[2]) return 0;
  if (q[2] == p[2]) {
    if (q[1] < p[1]) return 0;
    if (q[1] == p[1] && q[0] < p[0]) return 0;
  }
  return 1;
}

/* ----------------------------------------------------------- candidate cells */

typedef struct {
  int kind, idx, site;   /* point identity */
  double w[3];           /* wrapped approximate position */
  int t[3];              /* wrap count: w = raw + t*prd */
} point;

typedef struct {
  int nc[3];
  double csize[3];
  int *head, *next;
  point *pts;
  int npts;
} cells;

static void wrap_point(const oracle_state *s, const double raw[3], point *p)
{
  for (int d = 0; d < 3; d++) {
    double L = prd(s, d);
    double f = floor((raw[d] - s->boxlo[d]) / L);
    p->t[d] = -(int) f;
    p->w[d] = raw[d] - f * L;
    if (p->w[d] >= s->boxhi[d]) { p->w[d] -= L; p->t[d] -= 1; }
    if (p->w[d] < s->boxlo[d]) { p->w[d] += L; p->t[d] += 1; }
  }
}

static int build_cells(const oracle_state *s, double cut, cells *c)
{
  tables();
  int n = s->natoms + s->nelements * NU;
  c->pts = (point *) malloc(sizeof(point) * (size_t) (n > 0 ? n : 1));
  c->npts = n;
  for (int d = 0; d < 3; d++) {
    double L = prd(s, d);
    c->nc[d] = (int) (L / cut);
    if (c->nc[d] < 1) c->nc[d] = 1;
    c->csize[d] = L / c->nc[d];
  }
  size_t ncell = (size_t) c->nc[0] * c->nc[1] * c->nc[2];
  c->head = (int *) malloc(sizeof(int) * ncell);
  c->next = (int *) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
  if (!c->pts || !c->head || !c->next) return -1;
  for (size_t i = 0; i < ncell; i++) c->head[i] = -1;
  int m = 0;
  for (int i = 0; i < s->natoms; i++, m++) {
    c->pts[m].kind = 0;
    c->pts[m].idx = i;
    c->pts[m].site = -1;
    wrap_point(s, s->x + 3 * (size_t) i, &c->pts[m]);
  }
  for (int e = 0; e < s->nelements; e++) {
    const double *nx = s->nodex + (size_t) e * 24;
    for (int u = 0; u < NU; u++, m++) {
      double raw[3] = {0, 0, 0};
      for (int k = 0; k < NPE; k++)
        for (int d = 0; d < 3; d++) raw[d] += g_shape[8 * u + k] * nx[3 * k + d];
      c->pts[m].kind = 1;
      c->pts[m].idx = e;
      c->pts[m].site = u;
      wrap_point(s, raw, &c->pts[m]);
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    int ci[3];
    for (int d = 0; d < 3; d++) {
      ci[d] = (int) ((c->pts[i].w[d] - s->boxlo[d]) / c->csize[d]);
      if (ci[d] >= c->nc[d]) ci[d] = c->nc[d] - 1;
      if (ci[d] < 0) ci[d] = 0;
    }
    size_t id = ((size_t) ci[2] * c->nc[1] + ci[1]) * c->nc[0] + ci[0];
    c->next[i] = c->head[id];
    c->head[id] = i;
  }
  return 0;
}

static void free_cells(cells *c)
{
  free(c->pts);
  free(c->head);
  free(c->next);
}

/* ------------------------------------------------------------------ lists */

typedef struct {
  int64_t n, cap;
  int32_t *jidx, *jsite;
  int8_t *jkind, *img;
} growbuf;

static int push(growbuf *g, int kind, int idx, int site, const int8_t img[3])
{
  if (g->n == g->cap) {
    int64_t cap = g->cap ? 2 * g->cap : 1 << 16;
    g->jidx = (int32_t *) realloc(g->jidx, sizeof(int32_t) * cap);
    g->jsite = (int32_t *) realloc(g->jsite, sizeof(int32_t) * cap);
    g->jkind = (int8_t *) realloc(g->jkind, cap);
    g->img = (int8_t *) realloc(g->img, 3 * cap);
    if (!g->jidx || !g->jsite || !g->jkind || !g->img) return -1;
    g->cap = cap;
  }
  g->jidx[g->n] = idx;
  g->jsite[g->n] = site;
  g->jkind[g->n] = (int8_t) kind;
  memcpy(g->img + 3 * g->n, img, 3);
  g->n++;
  return 0;
}

typedef struct {
  int kind, idx, site, img[3];
} cand;

static int cand_cmp(const void *a, const void *b)
{
  const cand *x = (const cand *) a, *y = (const cand *) b;
  if (x->kind != y->kind) return x->kind - y->kind;
  if (x->idx != y->idx) return x->idx - y->idx;
  if (x->site != y->site) return x->site - y->site;
  for (int d = 0; d < 3; d++)
    if (x->img[d] != y->img[d]) return x->img[d] - y->img[d];
  return 0;
}

/* NPairHalfBinNewton::build (npair_half_bin_newton.cpp:25-392) and
 * NPairFullBin::build (npair_full_bin.cpp:23-358), restated as: every
 * (i, j, image) whose distance in the reference's arithmetic satisfies
 * rsq <= cutneighsq, filtered by the list's storage rules.  The reference's
 * bin, bounding-box and sub-element tests only prune candidates (the
 * sub-element radius is padded, element.cpp:1472-1743), so they are replaced
 * by an exhaustive cell search.
 *
 * half: atoms keep atom j once (same bin: owned j after i, ghost j above-right;
 *       other bins: upper half stencil) and every lattice site; Gauss points
 *       keep no atoms, every non-Gauss site, and a Gauss site once
 *       (owned: element i < j, or same element and igcell < jgcell;
 *       ghost: element centre above-right).
 * full: everything except the site itself. */
int oracle_build_list(const oracle_state *s, double cutneigh_in, int half, oracle_list *out)
{
  tables();
  double cutoff = cutneigh_in;
  double cutneighsq = cutoff * cutoff;
  cells c;
  if (build_cells(s, cutoff, &c)) return -1;
  binning bins;
  setup_atom_bins(s, cutoff, &bins);

  int nsites = s->natoms + NG * s->nelements;
  out->nsites = nsites;
  out->offset = (int64_t *) malloc(sizeof(int64_t) * (nsites + 1));
  growbuf g = {0, 0, NULL, NULL, NULL, NULL};
  double *ecent = (double *) malloc(sizeof(double) * 3 * (size_t) (s->nelements + 1));
  for (int e = 0; e < s->nelements; e++) center(s, e, ecent + 3 * e);

  int maxcand = 4096;
  cand *cl = (cand *) malloc(sizeof(cand) * maxcand);

  for (int i = 0; i < nsites; i++) {
    out->offset[i] = g.n;
    double xi[3];
    isite_pos(s, i, xi);
    int iatom = i < s->natoms;
    int ie = iatom ? -1 : (i - s->natoms) / NG;
    int ig = iatom ? -1 : (i - s->natoms) % NG;
    int iu = iatom ? -1 : g_g2u[ig];
    point pi;
    wrap_point(s, xi, &pi);
    int ci[3];
    for (int d = 0; d < 3; d++) {
      ci[d] = (int) ((pi.w[d] - s->boxlo[d]) / c.csize[d]);
      if (ci[d] >= c.nc[d]) ci[d] = c.nc[d] - 1;
      if (ci[d] < 0) ci[d] = 0;
    }
    int ncand = 0;
    for (int oz = -1; oz <= 1; oz++)
      for (int oy = -1; oy <= 1; oy++)
        for (int ox = -1; ox <= 1; ox++) {
          int o[3] = {ox, oy, oz}, cj[3], wrapc[3];
          for (int d = 0; d < 3; d++) {
            int v = ci[d] + o[d];
            wrapc[d] = 0;
            while (v < 0) { v += c.nc[d]; wrapc[d] -= 1; }
            while (v >= c.nc[d]) { v -= c.nc[d]; wrapc[d] += 1; }
            cj[d] = v;
          }
          /* skip (cell, wrap) combinations already visited */
          int dup = 0;
          for (int pz = -1; pz <= oz && !dup; pz++)
            for (int py = -1; py <= 1 && !dup; py++)
              for (int px = -1; px <= 1 && !dup; px++) {
                if (pz == oz && (py > oy || (py == oy && px >= ox))) continue;
                int q[3] = {px, py, pz}, same = 1;
                for (int d = 0; d < 3 && same; d++) {
                  int v = ci[d] + q[d], w = 0;
                  while (v < 0) { v += c.nc[d]; w -= 1; }
                  while (v >= c.nc[d]) { v -= c.nc[d]; w += 1; }
                  if (v != cj[d] || w != wrapc[d]) same = 0;
                }
                if (same) dup = 1;
              }
          if (dup) continue;
          size_t id = ((size_t) cj[2] * c.nc[1] + cj[1]) * c.nc[0] + cj[0];
          for (int m = c.head[id]; m >= 0; m = c.next[m]) {
            const point *pj = &c.pts[m];
            /* image of the neighbour's owner: raw_i - (raw_j + s L) = w_i - (w_j + wrapc L) */
            int8_t img[3];
            for (int d = 0; d < 3; d++) img[d] = (int8_t) (wrapc[d] - pi.t[d] + pj->t[d]);
            /* never the site itself */
            if (pj->kind == 1 && !iatom && pj->idx == ie && pj->site == iu &&
                img[0] == 0 && img[1] == 0 && img[2] == 0)
              continue;
            if (pj->kind == 0 && iatom && pj->idx == i && img[0] == 0 && img[1] == 0 && img[2] == 0)
              continue;
            /* cheap prefilter on wrapped positions */
            double dd = 0.0;
            for (int d = 0; d < 3; d++) {
              double t = pi.w[d] - (pj->w[d] + wrapc[d] * prd(s, d));
              dd += t * t;
            }
            if (dd > (cutoff + 1e-6) * (cutoff + 1e-6)) continue;
            double del[3];
            pair_delta(s, xi, pj->kind, pj->idx, pj->site, img, del);
            double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
            if (!(rsq <= cutneighsq)) continue;

            if (half) {
              if (iatom && pj->kind == 0) {
                double q[3];
                const double *xj = s->x + 3 * (size_t) pj->idx;
                for (int d = 0; d < 3; d++) q[d] = img[d] ? xj[d] + img[d] * prd(s, d) : xj[d];
                int ghost = img[0] || img[1] || img[2];
                int ord = bin_order(&bins, xi, q);
                if (ord < 0) continue;
                if (ord == 0) {
                  if (!ghost && pj->idx <= i) continue;
                  if (ghost && !above_right(q, xi)) continue;
                }
              } else if (!iatom && pj->kind == 0) {
                continue;   /* Gauss-point lists keep no atoms */
              } else if (!iatom && pj->kind == 1 && g_u2g[pj->site] >= 0) {
                int jg = g_u2g[pj->site];
                int ghost = img[0] || img[1] || img[2];
                if (!ghost) {
                  if (ie > pj->idx) continue;
                  if (ie == pj->idx && ig >= jg) continue;
                } else {
                  double q[3];
                  for (int d = 0; d < 3; d++) q[d] = ecent[3 * pj->idx + d] + img[d] * prd(s, d);
                  if (!above_right(q, ecent + 3 * ie)) continue;
                }
              }
            }
            if (ncand == maxcand) {
              maxcand *= 2;
              cl = (cand *) realloc(cl, sizeof(cand) * maxcand);
            }
            cl[ncand].kind = pj->kind;
            cl[ncand].idx = pj->idx;
            cl[ncand].site = pj->site;
            for (int d = 0; d < 3; d++) cl[ncand].img[d] = img[d];
            ncand++;
          }
        }
    qsort(cl, ncand, sizeof(cand), cand_cmp);
    for (int k = 0; k < ncand; k++) {
      int8_t im[3] = {(int8_t) cl[k].img[0], (int8_t) cl[k].img[1], (int8_t) cl[k].img[2]};
      if (push(&g, cl[k].kind, cl[k].idx, cl[k].site, im)) return -1;
    }
  }
  out->offset[nsites] = g.n;
  out->nentries = g.n;
  out->jidx = g.jidx;
  out->jsite = g.jsite;
  out->jkind = g.jkind;
  out->img = g.img;
  free(cl);
  free(ecent);
  free_cells(&c);
  return 0;
}

void oracle_free_list(oracle_list *l)
{
  free(l->offset);
  free(l->jidx);
  free(l->jsite);
  free(l->jkind);
  free(l->img);
  memset(l, 0, sizeof(*l));
}

/* -------------------------------------------------------------- ev helpers */

static void ev_zero(const oracle_state *s, oracle_ev *ev)
{
  if (!ev) return;
  ev->energy = 0.0;
  memset(ev->virial, 0, sizeof(ev->virial));
  if (ev->eatom) memset(ev->eatom, 0, sizeof(double) * s->natoms);
  if (ev->vatom) memset(ev->vatom, 0, sizeof(double) * 6 * s->natoms);
  if (ev->enode) memset(ev->enode, 0, sizeof(double) * 8 * s->nelements);
  if (ev->vnode) memset(ev->vnode, 0, sizeof(double) * 48 * s->nelements);
}

/* Pair::ev_tally (pair.cpp:428-482) for one pair: global energy and virial
 * scaled by (iescale + jescale); per-site halves to i and to j when j carries
 * energy (atom or node). */
static void ev_tally(oracle_ev *ev, double escale, double vscale, double *ie, double *je,
                     double *iv, double *jv, double evdwl, double fpair, const double del[3])
{
  if (!ev) return;
  ev->energy += evdwl * escale;
  double epairhalf = 0.5 * evdwl;
  if (ie) *ie += epairhalf;
  if (je) *je += epairhalf;
  double v[6];
  v[0] = del[0] * del[0] * fpair;
  v[1] = del[1] * del[1] * fpair;
  v[2] = del[2] * del[2] * fpair;
  v[3] = del[0] * del[1] * fpair;
  v[4] = del[0] * del[2] * fpair;
  v[5] = del[1] * del[2] * fpair;
  for (int k = 0; k < 6; k++) ev->virial[k] += v[k] * vscale;
  if (iv)
    for (int k = 0; k < 6; k++) iv[k] += 0.5 * v[k];
  if (jv)
    for (int k = 0; k < 6; k++) jv[k] += 0.5 * v[k];
}

/* ---------------------------------------------------------------------- LJ */

static void zero_forces(oracle_state *s)
{
  memset(s->f, 0, sizeof(double) * 3 * s->natoms);
  memset(s->nodef, 0, sizeof(double) * 24 * s->nelements);
  memset(s->gaussf, 0, sizeof(double) * 24 * s->nelements);
}

/* PairLJCut::compute (pair_lj_cut.cpp:227-417) with newton_pair on over a
 * half list; ghost reactions land on their owners (the reverse communication
 * of comm_brick.cpp:658-740).  init_one: pair_lj_cut.cpp:142-160. */
int oracle_lj_compute(oracle_state *s, const oracle_list *L, double epsilon, double sigma,
                      double cut, oracle_ev *ev)
{
  tables();
  double lj1 = 48.0 * epsilon * pow(sigma, 12.0);
  double lj2 = 24.0 * epsilon * pow(sigma, 6.0);
  double lj3 = 4.0 * epsilon * pow(sigma, 12.0);
  double lj4 = 4.0 * epsilon * pow(sigma, 6.0);
  double offset = 0.0;
  double cutsq = cut * cut;
  zero_forces(s);
  ev_zero(s, ev);
  for (int i = 0; i < L->nsites; i++) {
    double xi[3];
    isite_pos(s, i, xi);
    double *fi, iescale, *ie = NULL, *iv = NULL;
    if (i < s->natoms) {
      fi = s->f + 3 * (size_t) i;
      iescale = 0.5;
      if (ev && ev->eatom) ie = ev->eatom + i;
      if (ev && ev->vatom) iv = ev->vatom + 6 * (size_t) i;
    } else {
      int e = (i - s->natoms) / NG, g = (i - s->natoms) % NG, node = g_g2n[g];
      fi = s->gaussf + (size_t) e * 24 + 3 * g;
      iescale = g_nodal_weight / 2.0;
      if (ev && ev->enode) ie = ev->enode + 8 * (size_t) e + node;
      if (ev && ev->vnode) iv = ev->vnode + 48 * (size_t) e + 6 * node;
    }
    for (int64_t k = L->offset[i]; k < L->offset[i + 1]; k++) {
      int kind = L->jkind[k], j = L->jidx[k], site = L->jsite[k];
      double del[3];
      pair_delta(s, xi, kind, j, site, L->img + 3 * k, del);
      double *fj = NULL, jescale = 0.0, *je = NULL, *jv = NULL;
      if (kind == 0) {
        fj = s->f + 3 * (size_t) j;
        jescale = 0.5;
        if (ev && ev->eatom) je = ev->eatom + j;
        if (ev && ev->vatom) jv = ev->vatom + 6 * (size_t) j;
      } else if (g_u2g[site] >= 0) {
        int jg = g_u2g[site], jn = g_g2n[jg];
        fj = s->gaussf + (size_t) j * 24 + 3 * jg;
        jescale = g_nodal_weight / 2.0;
        if (ev && ev->enode) je = ev->enode + 8 * (size_t) j + jn;
        if (ev && ev->vnode) jv = ev->vnode + 48 * (size_t) j + 6 * jn;
      }
      double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
      if (rsq < cutsq) {
        double r2inv = 1.0 / rsq;
        double r6inv = r2inv * r2inv * r2inv;
        double forcelj = r6inv * (lj1 * r6inv - lj2);
        double fpair = forcelj * r2inv;
        for (int d = 0; d < 3; d++) fi[d] += del[d] * fpair;
        if (fj)
          for (int d = 0; d < 3; d++) fj[d] -= del[d] * fpair;
        double evdwl = r6inv * (lj3 * r6inv - lj4) - offset;
        ev_tally(ev, iescale + jescale, iescale + jescale, ie, je, iv, jv, evdwl, fpair, del);
      }
    }
  }
  return 0;
}

/* --------------------------------------------------------------------- EAM */

/* PairEAM::interpolate (pair_eam.cpp:580-616): 7 coefficients per knot */
static void interpolate(int n, double delta, const double *f, double *spline)
{
#define SP(m, c) spline[(m) * 7 + (c)]
  for (int m = 1; m <= n; m++) SP(m, 6) = f[m];
  SP(1, 5) = SP(2, 6) - SP(1, 6);
  SP(2, 5) = 0.5 * (SP(3, 6) - SP(1, 6));
  SP(n - 1, 5) = 0.5 * (SP(n, 6) - SP(n - 2, 6));
  SP(n, 5) = SP(n, 6) - SP(n - 1, 6);
  for (int m = 3; m <= n - 2; m++)
    SP(m, 5) = ((SP(m - 2, 6) - SP(m + 2, 6)) + 8.0 * (SP(m + 1, 6) - SP(m - 1, 6))) / 12.0;
  for (int m = 1; m <= n - 1; m++) {
    SP(m, 4) = 3.0 * (SP(m + 1, 6) - SP(m, 6)) - 2.0 * SP(m, 5) - SP(m + 1, 5);
    SP(m, 3) = SP(m, 5) + SP(m + 1, 5) - 2.0 * (SP(m + 1, 6) - SP(m, 6));
  }
  SP(n, 4) = 0.0;
  SP(n, 3) = 0.0;
  for (int m = 1; m <= n; m++) {
    SP(m, 2) = SP(m, 5) / delta;
    SP(m, 1) = 2.0 * SP(m, 4) / delta;
    SP(m, 0) = 3.0 * SP(m, 3) / delta;
  }
#undef SP
}

static int grab(FILE *fp, int n, double *dst)
{
  for (int i = 0; i < n; i++)
    if (fscanf(fp, "%lg", &dst[i]) != 1) return -1;
  return 0;
}

/* PairEAMAlloy::read_file (pair_eam_alloy.cpp:100-190) for one element,
 * file2array (pair_eam_alloy.cpp:196-240: setfl arrays used directly,
 * rhomax = (nrho-1) drho) and array2spline (pair_eam.cpp:561-578). */
int oracle_eam_load_setfl(const char *path, oracle_eam *eam)
{
  FILE *fp = fopen(path, "r");
  if (!fp) return -1;
  char line[4096];
  for (int i = 0; i < 3; i++)
    if (!fgets(line, sizeof line, fp)) { fclose(fp); return -1; }
  int nel = 0;
  if (!fgets(line, sizeof line, fp) || sscanf(line, "%d", &nel) != 1 || nel != 1) {
    fclose(fp);
    return -2;
  }
  if (!fgets(line, sizeof line, fp) ||
      sscanf(line, "%d %lg %d %lg %lg", &eam->nrho, &eam->drho, &eam->nr, &eam->dr, &eam->cut) != 5) {
    fclose(fp);
    return -3;
  }
  if (!fgets(line, sizeof line, fp)) { fclose(fp); return -4; }   /* Z mass a lattice */
  double *frho = (double *) calloc(eam->nrho + 1, sizeof(double));
  double *rhor = (double *) calloc(eam->nr + 1, sizeof(double));
  double *z2r = (double *) calloc(eam->nr + 1, sizeof(double));
  int rc = grab(fp, eam->nrho, frho + 1) || grab(fp, eam->nr, rhor + 1) || grab(fp, eam->nr, z2r + 1);
  fclose(fp);
  if (rc) { free(frho); free(rhor); free(z2r); return -5; }
  eam->rhomax = (eam->nrho - 1) * eam->drho;
  eam->frho_spline = (double *) calloc((size_t) (eam->nrho + 1) * 7, sizeof(double));
  eam->rhor_spline = (double *) calloc((size_t) (eam->nr + 1) * 7, sizeof(double));
  eam->z2r_spline = (double *) calloc((size_t) (eam->nr + 1) * 7, sizeof(double));
  interpolate(eam->nrho, eam->drho, frho, eam->frho_spline);
  interpolate(eam->nr, eam->dr, rhor, eam->rhor_spline);
  interpolate(eam->nr, eam->dr, z2r, eam->z2r_spline);
  free(frho); free(rhor); free(z2r);
  return 0;
}

void oracle_eam_free(oracle_eam *eam)
{
  free(eam->frho_spline);
  free(eam->rhor_spline);
  free(eam->z2r_spline);
  memset(eam, 0, sizeof(*eam));
}

/* PairEAM::compute_fp (pair_eam.cpp:1160-1169) with the coefficient row
 * returned to the caller (the patched form), so F(rho) is evaluated on the
 * same row as F'(rho). */
static double compute_fp(const oracle_eam *eam, double rho, const double **coeff, double *p)
{
  double rdrho = 1.0 / eam->drho;
  *p = rho * rdrho + 1.0;
  int m = (int) (*p);
  if (m > eam->nrho - 1) m = eam->nrho - 1;
  if (m < 1) m = 1;
  *p -= m;
  if (*p > 1.0) *p = 1.0;
  *coeff = eam->frho_spline + 7 * (size_t) m;
  return ((*coeff)[0] * *p + (*coeff)[1]) * *p + (*coeff)[2];
}

/* PairEAM::compute (pair_eam.cpp:618-1031) over a half list with newton on.
 * Pass 1 accumulates density at atoms and at node Gauss points
 * (:707-812; every Gauss point is a node here); the reverse communication of
 * rho (:815) is implicit because ghost contributions land on owners.
 * Embedding at atoms (:819-833).  Pass 2 (:845-1028) recomputes F' at node
 * Gauss points from nodal rho and at every lattice-site neighbour from the
 * shape-interpolated nodal rho.  Energies use the patched compute_fp. */
int oracle_eam_compute(oracle_state *s, const oracle_list *L, const oracle_eam *eam,
                       oracle_ev *ev, double *rho_atom_out, double *rho_node_out)
{
  tables();
  double rdr = 1.0 / eam->dr;
  double cutforcesq = eam->cut * eam->cut;
  int nr = eam->nr;
  double *arho = (double *) calloc((size_t) s->natoms + 1, sizeof(double));
  double *afp = (double *) calloc((size_t) s->natoms + 1, sizeof(double));
  double *nrho = (double *) calloc((size_t) s->nelements * 8 + 1, sizeof(double));
  zero_forces(s);
  ev_zero(s, ev);

  for (int i = 0; i < L->nsites; i++) {
    double xi[3];
    isite_pos(s, i, xi);
    double *irho;
    if (i < s->natoms) irho = arho + i;
    else {
      int e = (i - s->natoms) / NG, g = (i - s->natoms) % NG;
      irho = nrho + 8 * (size_t) e + g_g2n[g];
    }
    for (int64_t k = L->offset[i]; k < L->offset[i + 1]; k++) {
      int kind = L->jkind[k], j = L->jidx[k], site = L->jsite[k];
      double del[3];
      pair_delta(s, xi, kind, j, site, L->img + 3 * k, del);
      double *jrho = NULL;
      if (kind == 0) jrho = arho + j;
      else if (g_u2g[site] >= 0) jrho = nrho + 8 * (size_t) j + g_g2n[g_u2g[site]];
      double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
      if (rsq < cutforcesq) {
        double p = sqrt(rsq) * rdr + 1.0;
        int m = (int) p;
        if (m > nr - 1) m = nr - 1;
        p -= m;
        if (p > 1.0) p = 1.0;
        const double *c = eam->rhor_spline + 7 * (size_t) m;
        *irho += ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
        if (jrho) *jrho += ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
      }
    }
  }

  for (int i = 0; i < s->natoms; i++) {
    const double *coeff;
    double p;
    afp[i] = compute_fp(eam, arho[i], &coeff, &p);
    double phi = ((coeff[3] * p + coeff[4]) * p + coeff[5]) * p + coeff[6];
    if (arho[i] > eam->rhomax) phi += afp[i] * (arho[i] - eam->rhomax);
    if (ev) {
      ev->energy += phi;
      if (ev->eatom) ev->eatom[i] += phi;
    }
  }

  for (int i = 0; i < L->nsites; i++) {
    double xi[3];
    isite_pos(s, i, xi);
    double *fi, iescale, fpi, *ie = NULL, *iv = NULL;
    if (i < s->natoms) {
      fi = s->f + 3 * (size_t) i;
      fpi = afp[i];
      iescale = 0.5;
      if (ev && ev->eatom) ie = ev->eatom + i;
      if (ev && ev->vatom) iv = ev->vatom + 6 * (size_t) i;
    } else {
      int e = (i - s->natoms) / NG, g = (i - s->natoms) % NG, node = g_g2n[g];
      fi = s->gaussf + (size_t) e * 24 + 3 * g;
      double rhoi = nrho[8 * (size_t) e + node];
      iescale = g_nodal_weight / 2.0;
      if (ev && ev->enode) ie = ev->enode + 8 * (size_t) e + node;
      if (ev && ev->vnode) iv = ev->vnode + 48 * (size_t) e + 6 * node;
      const double *coeff;
      double p;
      if (g_nodal_energy_weight >= 0.0) iescale = g_nodal_energy_weight / 2.0;
      fpi = compute_fp(eam, rhoi, &coeff, &p);
      double phi = ((coeff[3] * p + coeff[4]) * p + coeff[5]) * p + coeff[6];
      if (rhoi > eam->rhomax) phi += fpi * (rhoi - eam->rhomax);
      if (ev) {
        ev->energy += phi * iescale * 2.0;
        if (ev->enode) ev->enode[8 * (size_t) e + node] += phi;
      }
    }
    for (int64_t k = L->offset[i]; k < L->offset[i + 1]; k++) {
      int kind = L->jkind[k], j = L->jidx[k], site = L->jsite[k];
      double del[3];
      pair_delta(s, xi, kind, j, site, L->img + 3 * k, del);
      double *fj = NULL, jescale = 0.0, fpj, *je = NULL, *jv = NULL;
      if (kind == 0) {
        fpj = afp[j];
        fj = s->f + 3 * (size_t) j;
        jescale = 0.5;
        if (ev && ev->eatom) je = ev->eatom + j;
        if (ev && ev->vatom) jv = ev->vatom + 6 * (size_t) j;
      } else {
        const double *sh = g_shape + 8 * site;
        double rhoj = 0.0;
        for (int n = 0; n < NPE; n++) rhoj += sh[n] * nrho[8 * (size_t) j + n];
        const double *coeff;
        double p;
        fpj = compute_fp(eam, rhoj, &coeff, &p);
        if (g_u2g[site] >= 0) {
          int jg = g_u2g[site], jn = g_g2n[jg];
          fj = s->gaussf + (size_t) j * 24 + 3 * jg;
          jescale = g_nodal_energy_weight >= 0.0 ? g_nodal_energy_weight / 2.0 : g_nodal_weight / 2.0;
          if (ev && ev->enode) je = ev->enode + 8 * (size_t) j + jn;
          if (ev && ev->vnode) jv = ev->vnode + 48 * (size_t) j + 6 * jn;
        }
      }
      double rsq = del[0] * del[0] + del[1] * del[1] + del[2] * del[2];
      if (rsq < cutforcesq) {
        double r = sqrt(rsq);
        double p = r * rdr + 1.0;
        int m = (int) p;
        if (m > nr - 1) m = nr - 1;
        p -= m;
        if (p > 1.0) p = 1.0;
        const double *c = eam->rhor_spline + 7 * (size_t) m;
        double rhoip = (c[0] * p + c[1]) * p + c[2];
        double rhojp = (c[0] * p + c[1]) * p + c[2];
        c = eam->z2r_spline + 7 * (size_t) m;
        double z2p = (c[0] * p + c[1]) * p + c[2];
        double z2 = ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
        double recip = 1.0 / r;
        double phi = z2 * recip;
        double phip = z2p * recip - phi * recip;
        double psip = fpi * rhojp + fpj * rhoip + phip;
        double fpair = -psip * recip;
        for (int d = 0; d < 3; d++) fi[d] += del[d] * fpair;
        if (fj)
          for (int d = 0; d < 3; d++) fj[d] -= del[d] * fpair;
        ev_tally(ev, iescale + jescale, iescale + jescale, ie, je, iv, jv, phi, fpair, del);
      }
    }
  }
  if (rho_atom_out) memcpy(rho_atom_out, arho, sizeof(double) * s->natoms);
  if (rho_node_out) memcpy(rho_node_out, nrho, sizeof(double) * 8 * s->nelements);
  free(arho);
  free(afp);
  free(nrho);
  return 0;
}

/* ------------------------------------------------- assembly and integration */

/* Element::compute_nodef, CONSISTENT (element.cpp:2178-2210) */
void oracle_compute_nodef(oracle_state *s)
{
  tables();
  for (int e = 0; e < s->nelements; e++) {
    double fc[8][3];
    memset(fc, 0, sizeof fc);
    const double *gf = s->gaussf + (size_t) e * 24;
    for (int g = 0; g < NG; g++)
      for (int n = 0; n < NPE; n++)
        for (int d = 0; d < 3; d++) fc[n][d] += g_wsa[g * 8 + n] * gf[3 * g + d];
    double *nf = s->nodef + (size_t) e * 24;
    for (int a = 0; a < NPE; a++)
      for (int b = 0; b < NPE; b++)
        for (int d = 0; d < 3; d++) nf[3 * a + d] += g_minv[a * 8 + b] * fc[b][d];
  }
}

/* FixNVE::initial_integrate / final_integrate (fix_nve.cpp:62-219) with
 * dtf = 0.5 dt ftm2v (metal units, update.cpp:161-164) and node mass equal
 * to the atom mass of its type; element centres refreshed afterwards. */
void oracle_nve_initial(oracle_state *s, double dt)
{
  double dtf = 0.5 * dt * (1.0 / 1.0364269e-4);
  double dtfm = dtf / s->mass;
  for (size_t i = 0; i < 3 * (size_t) s->natoms; i++) {
    s->v[i] += dtfm * s->f[i];
    s->x[i] += dt * s->v[i];
  }
  for (size_t i = 0; i < 24 * (size_t) s->nelements; i++) {
    s->nodev[i] += dtfm * s->nodef[i];
    s->nodex[i] += dt * s->nodev[i];
  }
}

void oracle_nve_final(oracle_state *s, double dt)
{
  double dtf = 0.5 * dt * (1.0 / 1.0364269e-4);
  double dtfm = dtf / s->mass;
  for (size_t i = 0; i < 3 * (size_t) s->natoms; i++) s->v[i] += dtfm * s->f[i];
  for (size_t i = 0; i < 24 * (size_t) s->nelements; i++) s->nodev[i] += dtfm * s->nodef[i];
}

/* Domain::pbc (domain.cpp:526-700): owned atoms and element centres back into
 * the box; an element moves with all of its nodes. */
void oracle_pbc(oracle_state *s)
{
  for (int i = 0; i < s->natoms; i++)
    for (int d = 0; d < 3; d++) {
      double *x = s->x + 3 * (size_t) i + d;
      double L = prd(s, d);
      if (*x < s->boxlo[d]) *x += L;
      if (*x >= s->boxhi[d]) {
        *x -= L;
        if (*x < s->boxlo[d]) *x = s->boxlo[d];
      }
    }
  for (int e = 0; e < s->nelements; e++) {
    double c[3];
    center(s, e, c);
    for (int d = 0; d < 3; d++) {
      double L = prd(s, d), sh = 0.0;
      if (c[d] < s->boxlo[d]) sh = L;
      if (c[d] >= s->boxhi[d]) sh = -L;
      if (sh != 0.0)
        for (int k = 0; k < NPE; k++) s->nodex[(size_t) e * 24 + 3 * k + d] += sh;
    }
  }
}

/* Verlet::setup + Verlet::run (verlet.cpp:64-152, 218-360) with fix nve and
 * neigh_modify every N delay 0 check no */
int oracle_run_nve(oracle_state *s, int pair, double p0, double p1, double p2,
                   const oracle_eam *eam, double skin, double dt, int nsteps, int every)
{
  double cut = pair == 0 ? p2 : eam->cut;
  double cutoff = sqrt(cut * cut);
  double cutneigh = cutoff + skin;
  oracle_list L;
  oracle_pbc(s);
  if (oracle_build_list(s, cutneigh, 1, &L)) return -1;
#define FORCE()                                                    \
  do {                                                             \
    if (pair == 0) oracle_lj_compute(s, &L, p0, p1, p2, NULL);     \
    else oracle_eam_compute(s, &L, eam, NULL, NULL, NULL);         \
    oracle_compute_nodef(s);                                       \
  } while (0)
  FORCE();
  for (int step = 1; step <= nsteps; step++) {
    oracle_nve_initial(s, dt);
    if (every > 0 && step % every == 0) {
      oracle_free_list(&L);
      oracle_pbc(s);
      if (oracle_build_list(s, cutneigh, 1, &L)) return -1;
    }
    FORCE();
    oracle_nve_final(s, dt);
  }
#undef FORCE
  oracle_free_list(&L);
  return 0;
}


/* ------------------------------------------------------------------ FIRE */

/* FIRE 2.0 (Guenole et al., Comput. Mater. Sci. 175, 109584 (2020),
 * Algorithm 2, semi-implicit Euler) over atoms then nodes, with the
 * parameters of the reference's Min (min.h:61-72, defaults min.cpp:33-47) and
 * its stopping tests; the reference has no FIRE iterate of its own.
 * par: delaystep dtgrow dtshrink alpha0 alphashrink tmax tmin dmax halfstepback
 *      delaystep_start max_vdotf_negatif. */
static double fire_energy(oracle_state *s, const oracle_list *L, int pair, double p0, double p1,
                          double p2, const oracle_eam *eam)
{
  oracle_ev ev;
  memset(&ev, 0, sizeof ev);
  if (pair == 0) oracle_lj_compute(s, L, p0, p1, p2, &ev);
  else oracle_eam_compute(s, L, eam, &ev, NULL, NULL);
  oracle_compute_nodef(s);
  return ev.energy;
}

int oracle_minimize_fire(oracle_state *s, int pair, double p0, double p1, double p2,
                         const oracle_eam *eam, double skin, double dt0, double etol, double ftol,
                         int maxiter, int normstyle, int every, const double *par, int *code,
                         int *niter, double *energy, double *fnorm)
{
  const double FTM2V = 1.0 / 1.0364269e-4, EPS_ENERGY = 1.0e-8;
  int delaystep = (int) par[0];
  double dtgrow = par[1], dtshrink = par[2], alpha0 = par[3], alphashrink = par[4];
  double dtmax = par[5] * dt0, dtmin = par[6] * dt0, dmax = par[7];
  int halfstepback = (int) par[8], delaystep_start = (int) par[9], max_vdotf_negatif = (int) par[10];
  double cut = pair == 0 ? p2 : eam->cut;
  double cutneigh = sqrt(cut * cut) + skin;
  double saved_w = g_nodal_energy_weight;
  g_nodal_energy_weight = 1.0;
  oracle_list L;
  oracle_pbc(s);
  if (oracle_build_list(s, cutneigh, 1, &L)) return -1;
  size_t na3 = 3 * (size_t) s->natoms, nn3 = 24 * (size_t) s->nelements;
  /* positions at the last build (Neighbor::build keeps xhold / nodexhold) */
  double *xhold = malloc(sizeof(double) * (na3 ? na3 : 1));
  double *nodexhold = malloc(sizeof(double) * (nn3 ? nn3 : 1));
  if (!xhold || !nodexhold) {
    free(xhold);
    free(nodexhold);
    oracle_free_list(&L);
    return -1;
  }
  memcpy(xhold, s->x, sizeof(double) * na3);
  memcpy(nodexhold, s->nodex, sizeof(double) * nn3);
  memset(s->v, 0, sizeof(double) * na3);
  memset(s->nodev, 0, sizeof(double) * nn3);
  double ecur = fire_energy(s, &L, pair, p0, p1, p2, eam), eprev = ecur;
  double dt = dt0, alpha = alpha0, dtv = dt0;
  long long step = 0, last_negative = 0, start = 0, last_build = 0;
  int vdotf_neg = 0, iter = 0, status = -1;
  double fn = 0.0;
  while (1) {
    /* reductions over atoms then nodes */
    double vdotf = 0, vdotv = 0, fdotf = 0, vmax = 0, fmaxd = 0, fmax2 = 0;
    for (int pass = 0; pass < 2; pass++) {
      size_t n = pass ? nn3 : na3;
      const double *v = pass ? s->nodev : s->v, *f = pass ? s->nodef : s->f;
      for (size_t k = 0; k < n; k += 3) {
        double f2 = 0.0;
        for (int d = 0; d < 3; d++) {
          vdotf += v[k + d] * f[k + d];
          vdotv += v[k + d] * v[k + d];
          fdotf += f[k + d] * f[k + d];
          if (fabs(v[k + d]) > vmax) vmax = fabs(v[k + d]);
          if (fabs(f[k + d]) > fmaxd) fmaxd = fabs(f[k + d]);
          f2 += f[k + d] * f[k + d];
        }
        if (f2 > fmax2) fmax2 = f2;
      }
    }
    fn = normstyle == 1 ? fmax2 : (normstyle == 2 ? fmaxd * fmaxd : fdotf);
    if (iter > 0) {
      if (etol > 0.0 && step - last_negative > delaystep &&
          fabs(ecur - eprev) < etol * 0.5 * (fabs(ecur) + fabs(eprev) + EPS_ENERGY)) {
        status = 2;
        break;
      }
      if (ftol > 0.0 && fn < ftol * ftol) {
        status = 3;
        break;
      }
    }
    if (iter >= maxiter) {
      status = 0;
      break;
    }
    iter++;
    step++;
    int reset = 0;
    if (vdotf > 0.0) {
      vdotf_neg = 0;
      if (step - last_negative > delaystep) {
        dt = dt * dtgrow < dtmax ? dt * dtgrow : dtmax;
        alpha *= alphashrink;
      }
    } else {
      last_negative = step;
      int delayed = !(delaystep_start && step - start < delaystep);
      if (delayed) {
        alpha = alpha0;
        if (dt * dtshrink >= dtmin) dt *= dtshrink;
      }
      vdotf_neg++;
      if (max_vdotf_negatif > 0 && vdotf_neg > max_vdotf_negatif) {
        status = 11;
        break;
      }
      reset = 1;
    }
    double vest = reset ? dt * FTM2V / s->mass * fmaxd : vmax;
    double dtnew = dt;
    if (dtnew * vest > dmax && vest > 0.0) dtnew = dmax / vest;
    double hb = (reset && halfstepback) ? 0.5 * dtv : 0.0;
    dtv = dtnew;
    int mix = vdotf > 0.0;
    double s1 = 1.0 - alpha, s2 = fdotf <= 1e-20 ? 0.0 : alpha * sqrt(vdotv / fdotf);
    double dtfm = dtv * FTM2V / s->mass;
    for (int pass = 0; pass < 2; pass++) {
      size_t n = pass ? nn3 : na3;
      double *x = pass ? s->nodex : s->x, *v = pass ? s->nodev : s->v;
      const double *f = pass ? s->nodef : s->f;
      for (size_t k = 0; k < n; k++) {
        double vd = v[k];
        if (reset) {
          x[k] -= hb * vd;
          vd = 0.0;
        }
        vd += dtfm * f[k];
        if (mix) vd = s1 * vd + s2 * f[k];
        x[k] += dtv * vd;
        v[k] = vd;
      }
    }
    if (every > 0 && (step - last_build) % every == 0 &&
        (!g_neigh_check || moved_past_trigger(s, xhold, nodexhold, skin))) {
      oracle_free_list(&L);
      oracle_pbc(s);
      if (oracle_build_list(s, cutneigh, 1, &L)) {
        free(xhold);
        free(nodexhold);
        return -1;
      }
      last_build = step;
      memcpy(xhold, s->x, sizeof(double) * na3);
      memcpy(nodexhold, s->nodex, sizeof(double) * nn3);
    }
    eprev = ecur;
    ecur = fire_energy(s, &L, pair, p0, p1, p2, eam);
  }
  free(xhold);
  free(nodexhold);
  oracle_free_list(&L);
  g_nodal_energy_weight = saved_w;
  *code = status;
  *niter = iter;
  *energy = ecur;
  *fnorm = fn;
  return 0;
}
