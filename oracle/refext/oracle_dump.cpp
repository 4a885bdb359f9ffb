/*
 * Oracle read-out commands (see oracle_dump.h).  Test infrastructure only.
 *
 * Output is plain text with every double printed as %.17g so that a reader
 * recovers the exact binary value, or with `binary` the same values as raw
 * float64 (for systems of millions of sites).
 */
#include "oracle_dump.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "atom.h"
#include "comm.h"
#include "domain.h"
#include "element.h"
#include "error.h"
#include "force.h"
#include "modify.h"
#include "neigh_list.h"
#include "neighbor.h"
#include "pair.h"
#include "cac.h"
#include "update.h"

using namespace CAC_NS;

namespace {

void ensure_maps(Atom *atom, Element *element)
{
  if (atom->map_style == 0) {
    atom->map_init();
    atom->map_set();
  }
  if (element->map_style == 0) {
    element->map_init();
    element->map_set();
  }
}

int image_of(double xg, double xo, double prd)
{
  return (int) std::lround((xg - xo) / prd);
}

}  // namespace

/* ---------------------------------------------------------------------- */

OracleDump::OracleDump(CAC *cac) : Pointers(cac) {}

void OracleDump::command(int narg, char **arg)
{
  if (narg != 2 && narg != 3) error->all(FLERR, "Illegal oracle_dump command: oracle_dump FILE state|compute [binary]");
  int compute = 0;
  if (strcmp(arg[1], "compute") == 0) compute = 1;
  else if (strcmp(arg[1], "state") != 0) error->all(FLERR, "Illegal oracle_dump mode");
  int binary = 0;
  if (narg == 3) {
    if (strcmp(arg[2], "binary") != 0) error->all(FLERR, "Illegal oracle_dump format");
    binary = 1;
  }
  if (compute) setup_and_compute();
  write(arg[0], compute, binary);
}

/* ----------------------------------------------------------------------
   the setup sequence of Verlet::setup (verlet.cpp:90-152) with the pair style
   evaluated for global and per-site energy and virial
   ------------------------------------------------------------------------- */

void OracleDump::setup_and_compute()
{
  if (force->pair == nullptr) error->all(FLERR, "oracle_dump compute needs a pair style");
  cac->init();
  update->setupflag = 1;
  neighbor->lastcall = -1;
  atom->setup();
  element->setup();
  modify->setup_pre_exchange();
  domain->pbc();
  domain->reset_box();
  comm->setup_exchange();
  comm->exchange();
  comm->setup_borders();
  if (neighbor->style) neighbor->setup_bins();
  comm->borders();
  domain->image_check();
  domain->box_too_small_check();
  modify->setup_pre_neighbor();
  neighbor->build();
  force->setup();

  // force_clear (verlet.cpp:192-215) with newton on
  size_t nbytes = sizeof(double) * (atom->nlocal + atom->nghost);
  if (nbytes) memset(&atom->f[0][0], 0, 3 * nbytes);
  nbytes = sizeof(double) * (element->nlocal + element->nghost);
  if (nbytes) {
    memset(&element->nodef[0][0][0][0], 0, 3 * element->maxapc * element->maxnpe * nbytes);
    memset(&element->gaussf[0][0][0][0], 0, 3 * element->maxgcell * element->maxapc * nbytes);
  }

  const int eflag = ENERGY_GLOBAL | ENERGY_ATOM;
  const int vflag = VIRIAL_PAIR | VIRIAL_ATOM;
  force->pair->compute(eflag, vflag);
  if (force->newton) comm->reverse_comm();
  if (element->nelements) element->compute_nodef();
  update->setupflag = 0;

  // fold ghost per-site energy and virial into their owners
  ensure_maps(atom, element);
  Pair *pair = force->pair;
  int nlocal = atom->nlocal, nall = atom->nlocal + atom->nghost;
  for (int j = nlocal; j < nall; j++) {
    int o = atom->map(atom->tag[j]);
    if (o < 0 || o >= nlocal) error->one(FLERR, "oracle_dump: ghost atom without owner");
    pair->eatom[o] += pair->eatom[j];
    for (int k = 0; k < 6; k++) pair->vatom[o][k] += pair->vatom[j][k];
  }
  int nelocal = element->nlocal, neall = element->nlocal + element->nghost;
  for (int j = nelocal; j < neall; j++) {
    int o = element->map(element->tag[j]);
    if (o < 0 || o >= nelocal) error->one(FLERR, "oracle_dump: ghost element without owner");
    int t = element->etype[j];
    for (int b = 0; b < element->apc[t]; b++)
      for (int n = 0; n < element->npe[t]; n++) {
        pair->enode[o][b][n] += pair->enode[j][b][n];
        for (int k = 0; k < 6; k++) pair->vnode[o][b][n][k] += pair->vnode[j][b][n][k];
      }
  }
}

// Text (one line per header field, atom and node) or binary: the magic
// "CACODMP1", then float64 values: step, box (lo/hi x, y, z), natoms,
// nelements, energy, virial[6], then natoms rows of 17 and 8 x nelements
// rows of 21 values, the columns of the text form.
void OracleDump::write(const char *file, int with_energy, int binary)
{
  FILE *fp = fopen(file, binary ? "wb" : "w");
  if (!fp) error->one(FLERR, "oracle_dump: cannot open file");
  Pair *pair = force->pair;
  const bool ev = with_energy && pair;
  const double energy = ev ? pair->eng_vdwl : 0.0;
  double virial[6] = {0, 0, 0, 0, 0, 0};
  if (ev)
    for (int k = 0; k < 6; k++) virial[k] = pair->virial[k];
  if (binary) {
    fwrite("CACODMP1", 1, 8, fp);
    const double head[15] = {(double) update->ntimestep, domain->boxlo[0], domain->boxhi[0], domain->boxlo[1],
                             domain->boxhi[1], domain->boxlo[2], domain->boxhi[2], (double) atom->nlocal,
                             (double) element->nlocal, energy, virial[0], virial[1], virial[2], virial[3],
                             virial[4]};
    fwrite(head, sizeof(double), 15, fp);
    fwrite(&virial[5], sizeof(double), 1, fp);
  } else {
    fprintf(fp, "# cac oracle dump v1\n");
    fprintf(fp, "step %ld\n", (long) update->ntimestep);
    fprintf(fp, "box %.17g %.17g %.17g %.17g %.17g %.17g\n", domain->boxlo[0], domain->boxhi[0],
            domain->boxlo[1], domain->boxhi[1], domain->boxlo[2], domain->boxhi[2]);
    fprintf(fp, "natoms %d nelements %d\n", atom->nlocal, element->nlocal);
    if (ev) {
      fprintf(fp, "energy %.17g\n", energy);
      fprintf(fp, "virial %.17g %.17g %.17g %.17g %.17g %.17g\n", virial[0], virial[1], virial[2], virial[3],
              virial[4], virial[5]);
    } else {
      fprintf(fp, "energy 0\nvirial 0 0 0 0 0 0\n");
    }
  }

  std::vector<int> order(atom->nlocal);
  for (int i = 0; i < atom->nlocal; i++) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return atom->tag[a] < atom->tag[b]; });
  if (!binary) fprintf(fp, "atoms\n");
  for (int i : order) {
    double e = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
    if (ev) {
      e = pair->eatom[i];
      for (int k = 0; k < 6; k++) v[k] = pair->vatom[i][k];
    }
    const double row[17] = {(double) atom->tag[i], atom->x[i][0], atom->x[i][1], atom->x[i][2],
                            atom->v[i][0], atom->v[i][1], atom->v[i][2], atom->f[i][0], atom->f[i][1],
                            atom->f[i][2], e, v[0], v[1], v[2], v[3], v[4], v[5]};
    if (binary) {
      fwrite(row, sizeof(double), 17, fp);
    } else {
      fprintf(fp, "%d", (int) atom->tag[i]);
      for (int k = 1; k < 17; k++) fprintf(fp, " %.17g", row[k]);
      fprintf(fp, "\n");
    }
  }

  std::vector<int> eorder(element->nlocal);
  for (int i = 0; i < element->nlocal; i++) eorder[i] = i;
  std::sort(eorder.begin(), eorder.end(),
            [&](int a, int b) { return element->tag[a] < element->tag[b]; });
  if (!binary) fprintf(fp, "nodes\n");
  for (int i : eorder) {
    int t = element->etype[i];
    for (int b = 0; b < element->apc[t]; b++)
      for (int n = 0; n < element->npe[t]; n++) {
        int g = element->n2g[t][n];
        double *gf = element->gaussf[i][b][g];
        double e = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
        if (ev) {
          e = pair->enode[i][b][n];
          for (int k = 0; k < 6; k++) v[k] = pair->vnode[i][b][n][k];
        }
        const double row[21] = {(double) element->tag[i], (double) n,
                                element->nodex[i][b][n][0], element->nodex[i][b][n][1], element->nodex[i][b][n][2],
                                element->nodev[i][b][n][0], element->nodev[i][b][n][1], element->nodev[i][b][n][2],
                                element->nodef[i][b][n][0], element->nodef[i][b][n][1], element->nodef[i][b][n][2],
                                gf[0], gf[1], gf[2], e, v[0], v[1], v[2], v[3], v[4], v[5]};
        if (binary) {
          fwrite(row, sizeof(double), 21, fp);
        } else {
          fprintf(fp, "%d %d", (int) element->tag[i], n);
          for (int k = 2; k < 21; k++) fprintf(fp, " %.17g", row[k]);
          fprintf(fp, "\n");
        }
      }
  }
  fclose(fp);
}

/* ---------------------------------------------------------------------- */

OracleDumpNeigh::OracleDumpNeigh(CAC *cac) : Pointers(cac) {}

void OracleDumpNeigh::command(int narg, char **arg)
{
  if (narg != 1 && narg != 2)
    error->all(FLERR, "Illegal oracle_dump_neigh command: oracle_dump_neigh FILE [binary]");
  int binary = 0;
  if (narg == 2) {
    if (strcmp(arg[1], "binary") != 0) error->all(FLERR, "Illegal oracle_dump_neigh mode");
    binary = 1;
  }
  if (force->pair == nullptr) error->all(FLERR, "oracle_dump_neigh needs a pair style");
  NeighList *list = force->pair->get_list();
  if (list == nullptr) error->all(FLERR, "oracle_dump_neigh: no neighbour list (run 0 first)");
  ensure_maps(atom, element);

  double prd[3] = {domain->prd[0], domain->prd[1], domain->prd[2]};
  double **ax = atom->x;
  double **ex = element->x;
  int nalocal = atom->nlocal;
  int nelocal = element->nlocal;

  struct Key {
    int kind;  // 0 atom, 1 virtual site
    int tag, site, sx, sy, sz;
    bool operator<(const Key &o) const {
      if (kind != o.kind) return kind < o.kind;
      if (tag != o.tag) return tag < o.tag;
      if (site != o.site) return site < o.site;
      if (sx != o.sx) return sx < o.sx;
      if (sy != o.sy) return sy < o.sy;
      return sz < o.sz;
    }
  };
  struct Entry {
    Key i;
    std::vector<Key> js;
  };
  std::vector<Entry> entries(list->inum);

  for (int ii = 0; ii < list->inum; ii++) {
    int i = list->ilist[ii];
    int iindex = list->iindexlist[ii];
    Entry &en = entries[ii];
    if (iindex < 0) en.i = {0, (int) atom->tag[i], -1, 0, 0, 0};
    else en.i = {1, (int) element->tag[i], iindex, 0, 0, 0};
    int *jl = list->firstneigh[ii];
    int *jx = list->firstneighindex[ii];
    for (int jj = 0; jj < list->numneigh[ii]; jj++) {
      int j = jl[jj];
      Key k;
      if (jx[jj] < 0) {
        int o = (j < nalocal) ? j : atom->map(atom->tag[j]);
        k = {0, (int) atom->tag[j], -1, image_of(ax[j][0], ax[o][0], prd[0]),
             image_of(ax[j][1], ax[o][1], prd[1]), image_of(ax[j][2], ax[o][2], prd[2])};
      } else {
        int o = (j < nelocal) ? j : element->map(element->tag[j]);
        k = {1, (int) element->tag[j], jx[jj], image_of(ex[j][0], ex[o][0], prd[0]),
             image_of(ex[j][1], ex[o][1], prd[1]), image_of(ex[j][2], ex[o][2], prd[2])};
      }
      en.js.push_back(k);
    }
    std::sort(en.js.begin(), en.js.end());
  }
  std::sort(entries.begin(), entries.end(),
            [](const Entry &a, const Entry &b) { return a.i < b.i; });

  if (binary) {
    // rows of 7 int32 in canonical numbering, already in sorted order:
    // i-site (atom tag-1, or natoms + 8*(element tag-1) + Gauss point),
    // j kind, j tag-1, j site, image sx, sy, sz
    FILE *fb = fopen(arg[0], "wb");
    if (!fb) error->one(FLERR, "oracle_dump_neigh: cannot open file");
    const long natoms = (long) atom->natoms;
    std::vector<int> buf;
    for (auto &en : entries) {
      long isite = en.i.kind == 0 ? en.i.tag - 1L : natoms + 8L * (en.i.tag - 1) + en.i.site;
      buf.clear();
      for (auto &k : en.js) {
        int row[7] = {(int) isite, k.kind, k.tag - 1, k.site, k.sx, k.sy, k.sz};
        buf.insert(buf.end(), row, row + 7);
      }
      if (!buf.empty() && fwrite(buf.data(), sizeof(int), buf.size(), fb) != buf.size())
        error->one(FLERR, "oracle_dump_neigh: write failed");
    }
    fclose(fb);
    return;
  }

  FILE *fp = fopen(arg[0], "w");
  if (!fp) error->one(FLERR, "oracle_dump_neigh: cannot open file");
  fprintf(fp, "# cac oracle neighbour list v1: I kind tag site n / J kind tag site sx sy sz\n");
  fprintf(fp, "inum %d\n", list->inum);
  for (auto &en : entries) {
    fprintf(fp, "I %d %d %d %d\n", en.i.kind, en.i.tag, en.i.site, (int) en.js.size());
    for (auto &k : en.js)
      fprintf(fp, "J %d %d %d %d %d %d\n", k.kind, k.tag, k.site, k.sx, k.sy, k.sz);
  }
  fclose(fp);
}
