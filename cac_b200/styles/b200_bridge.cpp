/*
 * B200Bridge: the reference's host arrays <-> one cacb200 context.
 * See b200_bridge.h.
 */
#include "b200_bridge.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <cmath>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "atom.h"
#include "comm.h"
#include "compute_b200.h"
#include "domain.h"
#include "element.h"
#include "element_vec.h"
#include "error.h"
#include "force.h"
#include "modify.h"
#include "my_page.h"
#include "neigh_list.h"
#include "neighbor.h"
#include "output.h"
#include "pair.h"
#include "thermo.h"
#include "update.h"

#include "cacb200.h"
#include "pair_eam_alloy_b200.h"
#include "pair_lj_cut_b200.h"

using namespace CAC_NS;

B200Bridge::B200Bridge(CAC *cac) : Pointers(cac) {}

B200Bridge::~B200Bridge()
{
  if (ctx) cacb200_ctx_destroy(ctx);
}

void B200Bridge::status(int rc, const char *what)
{
  if (rc == CACB200_OK) return;
  std::string msg = std::string("b200: ") + what + " failed: " + (ctx ? cacb200_last_error(ctx) : "no context");
  error->all(FLERR, msg.c_str());
}

void B200Bridge::set_lj(double epsilon, double sigma, double cut)
{
  pair_style = CACB200_PAIR_LJ;
  lj = {epsilon, sigma, cut};
  uploaded_na = uploaded_ne = -1;
}

void B200Bridge::set_eam(int nrho, double drho, int nr, double dr, double cut, const double *frho,
                         const double *rhor, const double *z2r)
{
  pair_style = CACB200_PAIR_EAM;
  eam_nrho = nrho;
  eam_nr = nr;
  eam_drho = drho;
  eam_dr = dr;
  eam_cut = cut;
  eam_frho.assign(frho, frho + nrho);
  eam_rhor.assign(rhor, rhor + nr);
  eam_z2r.assign(z2r, z2r + nr);
  uploaded_na = uploaded_ne = -1;
}

/* the subset of CAC this package implements: one rank, orthogonal fully
   periodic box, one atom type, Hex elements with apc 1, 9 lattice sites per
   edge, 2x2x2 Gauss points, UNIFORM weights and CONSISTENT nodal forces */
void B200Bridge::check_system()
{
  if (comm->nprocs != 1) error->all(FLERR, "b200 styles run on one MPI rank");
  if (domain->triclinic) error->all(FLERR, "b200 styles need an orthogonal box");
  if (!domain->xperiodic || !domain->yperiodic || !domain->zperiodic)
    error->all(FLERR, "b200 styles need a periodic box");
  if (atom->ntypes != 1) error->all(FLERR, "b200 styles support one atom type");
  if (element->nelements) {
    if (element->maxapc != 1 || element->maxnpe != 8)
      error->all(FLERR, "b200 styles need element_style cac 8 1");
    if (element->nodal_force_style != Element::CONSISTENT)
      error->all(FLERR, "b200 styles need CONSISTENT nodal forces");
    if (element->weight_scale_flag != Element::UNIFORM)
      error->all(FLERR, "b200 styles need element_style ... wscale (UNIFORM weights)");
    for (int i = 0; i < element->nlocal; i++) {
      int t = element->etype[i];
      if (element->npe[t] != 8 || element->apc[t] != 1 || element->nucell[t] != 729 ||
          element->ngcell[t] != 8)
        error->all(FLERR, "b200 styles need Hex elements with 9x9x9 sites and 2x2x2 Gauss points");
    }
  }
  if (!ctx) {
    const char *dev = getenv("CACB200_DEVICE");
    status(cacb200_ctx_create(dev ? atoi(dev) : 0, &ctx), "context creation");
  }
}

void B200Bridge::configure_pair()
{
  if (pair_style == CACB200_PAIR_LJ) status(cacb200_set_lj(ctx, lj[0], lj[1], lj[2]), "set_lj");
  else if (pair_style == CACB200_PAIR_EAM)
    status(cacb200_set_eam(ctx, eam_nrho, eam_drho, eam_nr, eam_dr, eam_cut, eam_frho.data(),
                           eam_rhor.data(), eam_z2r.data()),
           "set_eam");
  else error->all(FLERR, "b200: no pair style configured");
}

void B200Bridge::upload(bool with_velocities)
{
  int na = atom->nlocal, ne = element->nlocal;
  const double *x = na ? &atom->x[0][0] : nullptr;
  const double *nx = ne ? &element->nodex[0][0][0][0] : nullptr;
  std::vector<double> zv;
  const double *v = nullptr, *nv = nullptr;
  if (with_velocities) {
    v = na ? &atom->v[0][0] : nullptr;
    nv = ne ? &element->nodev[0][0][0][0] : nullptr;
  } else {
    zv.assign(3 * (size_t)std::max(na, 1) + 24 * (size_t)std::max(ne, 1), 0.0);
    v = zv.data();
    nv = zv.data() + 3 * (size_t)std::max(na, 1);
  }
  status(cacb200_upload_system(ctx, domain->boxlo, domain->boxhi, na, x, v, ne, nx, nv, atom->mass[1]),
         "upload_system");
  configure_pair();
  uploaded_na = na;
  uploaded_ne = ne;
  for (int d = 0; d < 3; d++) {
    uploaded_lo[d] = domain->boxlo[d];
    uploaded_hi[d] = domain->boxhi[d];
  }
}

void B200Bridge::compute(Pair *pair)
{
  check_system();
  int na = atom->nlocal, ne = element->nlocal;
  bool rebuild = (uploaded_na != na || uploaded_ne != ne || neighbor->ago == 0);
  if (rebuild) {
    upload(false);
    status(cacb200_set_neighbor(ctx, neighbor->skin, 0), "set_neighbor");
    status(cacb200_build_lists(ctx, 0), "build_lists");
  } else {
    // a box the reference changed since the last rebuild (fix deform): the
    // device's periodic images follow it
    bool moved = false;
    for (int d = 0; d < 3; d++)
      moved = moved || domain->boxlo[d] != uploaded_lo[d] || domain->boxhi[d] != uploaded_hi[d];
    if (moved) {
      status(cacb200_set_box(ctx, domain->boxlo, domain->boxhi), "set_box");
      for (int d = 0; d < 3; d++) {
        uploaded_lo[d] = domain->boxlo[d];
        uploaded_hi[d] = domain->boxhi[d];
      }
    }
    status(cacb200_set_state(ctx, na ? &atom->x[0][0] : nullptr, nullptr,
                             ne ? &element->nodex[0][0][0][0] : nullptr, nullptr),
           "set_state");
  }
  int ef = (pair->eflag_global ? CACB200_ENERGY_GLOBAL : 0) | (pair->eflag_atom ? CACB200_ENERGY_ATOM : 0);
  int vf = (pair->vflag_global ? CACB200_VIRIAL_GLOBAL : 0) | (pair->vflag_atom ? CACB200_VIRIAL_ATOM : 0);
  status(cacb200_compute_forces(ctx, ef, vf), "compute_forces");

  fbuf.resize(3 * (size_t)std::max(na, 1));
  gbuf.resize(24 * (size_t)std::max(ne, 1));
  status(cacb200_get_forces(ctx, fbuf.data(), nullptr, gbuf.data()), "get_forces");
  double **f = atom->f;
  for (int i = 0; i < na; i++)
    for (int d = 0; d < 3; d++) f[i][d] += fbuf[3 * (size_t)i + d];
  double ****gf = element->gaussf;
  for (int e = 0; e < ne; e++)
    for (int g = 0; g < 8; g++)
      for (int d = 0; d < 3; d++) gf[e][0][g][d] += gbuf[24 * (size_t)e + 3 * g + d];

  if (ef || vf) {
    double energy = 0.0, vir[6];
    ebuf.resize(std::max(na, 1));
    vbuf.resize(6 * (size_t)std::max(na, 1));
    enbuf.resize(8 * (size_t)std::max(ne, 1));
    vnbuf.resize(48 * (size_t)std::max(ne, 1));
    status(cacb200_get_energy(ctx, &energy, vir, pair->eflag_atom ? ebuf.data() : nullptr,
                              pair->vflag_atom ? vbuf.data() : nullptr,
                              pair->eflag_atom ? enbuf.data() : nullptr,
                              pair->vflag_atom ? vnbuf.data() : nullptr),
           "get_energy");
    if (pair->eflag_global) pair->eng_vdwl += energy;
    if (pair->vflag_global)
      for (int k = 0; k < 6; k++) pair->virial[k] += vir[k];
    if (pair->eflag_atom) {
      for (int i = 0; i < na; i++) pair->eatom[i] += ebuf[i];
      for (int e = 0; e < ne; e++)
        for (int n = 0; n < 8; n++) pair->enode[e][0][n] += enbuf[8 * (size_t)e + n];
    }
    if (pair->vflag_atom) {
      for (int i = 0; i < na; i++)
        for (int k = 0; k < 6; k++) pair->vatom[i][k] += vbuf[6 * (size_t)i + k];
      for (int e = 0; e < ne; e++)
        for (int n = 0; n < 8; n++)
          for (int k = 0; k < 6; k++) pair->vnode[e][0][n][k] += vnbuf[48 * (size_t)e + 6 * n + k];
    }
  }
}

B200ThermoNow CAC_NS::b200_thermo_now;

void B200Bridge::run_device(int nsteps, double dt, int every, const B200Fixes &fx, bool step0_output)
{
  check_system();
  upload(true);
  status(cacb200_set_neighbor(ctx, neighbor->skin, every), "set_neighbor");
  status(cacb200_set_neighbor_modify(ctx, neighbor->delay, neighbor->dist_check), "set_neighbor_modify");
  if (fx.langevin) {
    status(cacb200_set_langevin(ctx, fx.t_start, fx.t_stop, fx.t_period, fx.seed, fx.zero), "set_langevin");
    status(cacb200_set_langevin_stream(ctx, fx.draws), "set_langevin_stream");
  }
  if (fx.deform)
    status(cacb200_set_deform(ctx, fx.deform_every, fx.deform_style, fx.deform_a, fx.deform_b,
                              fx.deform_remap_x),
           "set_deform");
  // thermo and dumps that read only what the device output path provides
  // need no state copy at thermo-only steps
  output_copies_state = !b200_device_output_safe(cac);
  const long long copies0 = state_copies;
  // per-site tallies at output steps only when a dump may read them
  const int ev_out = CACB200_ENERGY_GLOBAL | (output->ndump ? CACB200_ENERGY_ATOM : 0);
  const int vv_out = CACB200_VIRIAL_GLOBAL | (output->ndump ? CACB200_VIRIAL_ATOM : 0);
  const bigint step0 = update->ntimestep, end = step0 + nsteps;
  status(cacb200_run_begin(ctx, nsteps, dt, step0_output ? ev_out : 0, step0_output ? vv_out : 0), "run_begin");
  if (step0_output) output_step(step0, fx.deform, true);
  // Verlet::run's loop (verlet.cpp:218-360): the device advances to the next
  // step with output (Output::next), then the reference writes it
  while (update->ntimestep < end) {
    const bigint stop = std::min<bigint>(output->next, end);
    const bool out = stop == output->next;
    const int k = (int)(stop - update->ntimestep);
    status(cacb200_run_steps(ctx, k, dt, out ? ev_out : 0, out ? vv_out : 0), "run_steps");
    update->ntimestep = stop;
    if (out) output_step(stop, fx.deform, false);
  }
  download_state(fx.deform);
  download_forces();
  uploaded_na = uploaded_ne = -1;   // the reference must set up again (ghosts are stale)
  const long long copies = state_copies - copies0;
  for (FILE *fp : {screen, logfile})
    if (fp)
      fprintf(fp, "b200 device run: %d steps, %lld output steps with a host copy of the state\n", nsteps, copies);
}

// Forces of the last evaluation into atom->f, element->nodef and
// element->gaussf.
void B200Bridge::download_forces()
{
  int na = atom->nlocal, ne = element->nlocal;
  fbuf.resize(3 * (size_t)std::max(na, 1));
  gbuf.resize(24 * (size_t)std::max(ne, 1));
  std::vector<double> nf(24 * (size_t)std::max(ne, 1));
  status(cacb200_get_forces(ctx, fbuf.data(), nf.data(), gbuf.data()), "get_forces");
  for (int i = 0; i < na; i++)
    for (int d = 0; d < 3; d++) atom->f[i][d] = fbuf[3 * (size_t)i + d];
  for (int e = 0; e < ne; e++)
    for (int n = 0; n < 8; n++)
      for (int d = 0; d < 3; d++) {
        element->nodef[e][0][n][d] = nf[24 * (size_t)e + 3 * n + d];
        element->gaussf[e][0][n][d] = gbuf[24 * (size_t)e + 3 * n + d];
      }
}

void B200Bridge::minimize_fire(double etol, double ftol, int maxiter, double dt, int normstyle,
                               const B200Fire &p, int &stop, int &niter, double &energy, double &fnorm)
{
  check_system();
  upload(false);
  status(cacb200_set_neighbor(ctx, neighbor->skin, neighbor->every), "set_neighbor");
  status(cacb200_set_neighbor_modify(ctx, neighbor->delay, neighbor->dist_check), "set_neighbor_modify");
  status(cacb200_set_fire_params(ctx, p.delaystep, p.dtgrow, p.dtshrink, p.alpha0, p.alphashrink, p.tmax,
                                 p.tmin, p.dmax, p.halfstepback, p.delaystep_start, p.max_vdotf_negatif),
         "set_fire_params");
  status(cacb200_minimize_fire(ctx, etol, ftol, maxiter, dt, normstyle, &stop, &niter, &energy, &fnorm),
         "minimize_fire");
  int na = atom->nlocal, ne = element->nlocal;
  status(cacb200_get_state(ctx, na ? &atom->x[0][0] : nullptr, nullptr, ne ? &element->nodex[0][0][0][0] : nullptr,
                           nullptr),
         "get_state");
  // element centres follow the nodes (ElementVecCAC::update_center_coord)
  if (ne) element->evec->update_center_coord();
  uploaded_na = uploaded_ne = -1;   // the reference sets up again (ghosts are stale)
}

B200Bridge *CAC_NS::b200_bridge_of(Pair *pair)
{
  if (auto *p = dynamic_cast<PairLJCutB200 *>(pair)) return p->bridge;
  if (auto *p = dynamic_cast<PairEAMAlloyB200 *>(pair)) return p->bridge;
  return nullptr;
}

// Positions and velocities (and the box, when it deforms) from the device
// into the reference's arrays.
void B200Bridge::download_state(bool box)
{
  int na = atom->nlocal, ne = element->nlocal;
  status(cacb200_get_state(ctx, na ? &atom->x[0][0] : nullptr, na ? &atom->v[0][0] : nullptr,
                           ne ? &element->nodex[0][0][0][0] : nullptr,
                           ne ? &element->nodev[0][0][0][0] : nullptr),
         "get_state");
  // element centres follow the nodes, as after FixNVE::initial_integrate
  // (fix_nve.cpp:143)
  if (ne) element->evec->update_center_coord();
  if (box) {
    // the box the device ended with (FixDeform::update_domain)
    double lo[3], hi[3], m = 0.0;
    status(cacb200_get_box(ctx, lo, hi, &m), "get_box");
    for (int d = 0; d < 3; d++) {
      domain->boxlo[d] = lo[d];
      domain->boxhi[d] = hi[d];
    }
    domain->set_global_box();
    domain->set_local_box();
  }
}

// One output step of a device run, written by the reference's own Output
// (Output::setup on `first`, else Output::write): the box, the pair's
// global tallies and the device thermo read-out for compute temp/b200, all
// of a few doubles; a dump that may be due at this step (or computes that
// read host per-site data) also get the state, the forces and the per-site
// tallies in the reference's arrays.
void B200Bridge::output_step(bigint step, bool box, bool first)
{
  const bool dump_due = output->ndump && (first || output->next_dump_any == step);
  const bool copy = dump_due || output_copies_state;
  if (copy) {
    download_state(box);
    download_forces();
    state_copies++;
  } else if (box) {
    double lo[3], hi[3], m = 0.0;
    status(cacb200_get_box(ctx, lo, hi, &m), "get_box");
    for (int d = 0; d < 3; d++) {
      domain->boxlo[d] = lo[d];
      domain->boxhi[d] = hi[d];
    }
    domain->set_global_box();
    domain->set_local_box();
  }
  Pair *pair = force->pair;
  double e = 0.0, vir[6];
  if (dump_due) {
    // the per-site tallies of this step for per-atom computes (pe/atom,
    // stress/atom), as Pair::compute leaves them
    const int na = atom->nlocal, ne = element->nlocal;
    ebuf.resize(std::max(na, 1));
    vbuf.resize(6 * (size_t)std::max(na, 1));
    enbuf.resize(8 * (size_t)std::max(ne, 1));
    vnbuf.resize(48 * (size_t)std::max(ne, 1));
    status(cacb200_get_energy(ctx, &e, vir, ebuf.data(), vbuf.data(), enbuf.data(), vnbuf.data()), "get_energy");
    if (pair->eatom && pair->vatom) {
      for (int i = 0; i < na; i++) {
        pair->eatom[i] = ebuf[i];
        for (int k = 0; k < 6; k++) pair->vatom[i][k] = vbuf[6 * (size_t)i + k];
      }
      for (int i = na; i < na + atom->nghost; i++) {
        pair->eatom[i] = 0.0;
        for (int k = 0; k < 6; k++) pair->vatom[i][k] = 0.0;
      }
    }
    if (pair->enode && pair->vnode) {
      for (int el = 0; el < ne; el++)
        for (int n = 0; n < 8; n++) {
          pair->enode[el][0][n] = enbuf[8 * (size_t)el + n];
          for (int k = 0; k < 6; k++) pair->vnode[el][0][n][k] = vnbuf[48 * (size_t)el + 6 * n + k];
        }
      for (int el = ne; el < ne + element->nghost; el++)
        for (int n = 0; n < 8; n++) {
          pair->enode[el][0][n] = 0.0;
          for (int k = 0; k < 6; k++) pair->vnode[el][0][n][k] = 0.0;
        }
    }
    update->eflag_atom = update->vflag_atom = step;
  } else {
    status(cacb200_get_energy(ctx, &e, vir, nullptr, nullptr, nullptr, nullptr), "get_energy");
  }
  pair->eng_vdwl = e;
  pair->eng_coul = 0.0;
  for (int k = 0; k < 6; k++) pair->virial[k] = vir[k];
  b200_thermo_now.step = step;
  status(cacb200_thermo(ctx, strcmp(update->unit_style, "metal") == 0 ? CACB200_UNITS_METAL : CACB200_UNITS_METALGPA,
                        b200_thermo_now.v),
         "thermo");
  b200_thermo_now.active = true;
  update->ntimestep = step;
  update->eflag_global = update->vflag_global = step;
  modify->clearstep_compute();
  if (first) output->setup(0);
  else output->write(step);
  b200_thermo_now.active = false;
}

void B200Bridge::fill_host_list(NeighList *list)
{
  check_system();
  upload(false);
  status(cacb200_set_neighbor(ctx, neighbor->skin, 0), "set_neighbor");
  status(cacb200_build_lists(ctx, 1), "build_lists");
  int64_t n = 0;
  int nsites = 0;
  status(cacb200_list_size(ctx, 1, &n, &nsites), "list_size");
  std::vector<int64_t> off(nsites + 1);
  std::vector<int8_t> kind(std::max<int64_t>(n, 1)), img(3 * std::max<int64_t>(n, 1));
  std::vector<int32_t> idx(std::max<int64_t>(n, 1)), site(std::max<int64_t>(n, 1));
  status(cacb200_get_list(ctx, 1, off.data(), kind.data(), idx.data(), site.data(), img.data()), "get_list");

  // (owner, periodic image) -> the reference's local or ghost index: owners
  // by tag, each ghost's image from its position relative to its owner
  const int na = atom->nlocal, nag = na + atom->nghost;
  const int ne = element->nlocal, neg = ne + element->nghost;
  const double *prd = domain->prd;
  auto key = [](long owner, int sx, int sy, int sz) {
    return ((owner * 5 + (sx + 2)) * 5 + (sy + 2)) * 5 + (sz + 2);
  };
  auto image = [&](const double *xg, const double *xo, int d) {
    return (int) std::lround((xg[d] - xo[d]) / prd[d]);
  };
  std::unordered_map<tagint, int> aown, eown;
  for (int i = 0; i < na; i++) aown[atom->tag[i]] = i;
  for (int i = 0; i < ne; i++) eown[element->tag[i]] = i;
  std::unordered_map<long, int> aimg, eimg;
  for (int g = na; g < nag; g++) {
    auto it = aown.find(atom->tag[g]);
    if (it == aown.end()) continue;
    const double *xg = atom->x[g], *xo = atom->x[it->second];
    aimg[key(it->second, image(xg, xo, 0), image(xg, xo, 1), image(xg, xo, 2))] = g;
  }
  for (int g = ne; g < neg; g++) {
    auto it = eown.find(element->tag[g]);
    if (it == eown.end()) continue;
    const double *xg = element->x[g], *xo = element->x[it->second];
    eimg[key(it->second, image(xg, xo, 0), image(xg, xo, 1), image(xg, xo, 2))] = g;
  }

  MyPage<int> *ipage = list->ipage, *indexpage = list->indexpage;
  ipage->reset();
  indexpage->reset();
  int inum = 0;
  for (int i = 0; i < nsites; i++) {
    int *nptr = ipage->vget();
    int *iptr = indexpage->vget();
    int m = 0;
    for (int64_t k = off[i]; k < off[i + 1]; k++) {
      const int sx = img[3 * k], sy = img[3 * k + 1], sz = img[3 * k + 2];
      int j = idx[k];
      if (sx || sy || sz) {
        auto &tab = kind[k] == 0 ? aimg : eimg;
        auto it = tab.find(key(idx[k], sx, sy, sz));
        if (it == tab.end()) error->one(FLERR, "b200: a device list neighbour has no ghost copy on this rank");
        j = it->second;
      }
      nptr[m] = j;
      iptr[m] = kind[k] == 0 ? -1 : site[k];   // jucell * apc + jbasis with apc 1
      m++;
    }
    list->firstneigh[inum] = nptr;
    list->firstneighindex[inum] = iptr;
    list->numneigh[inum] = m;
    ipage->vgot(m);
    indexpage->vgot(m);
    if (ipage->status() || indexpage->status())
      error->one(FLERR, "Neighbor list overflow, boost neigh_modify one");
    list->ilist[inum] = i < na ? i : (i - na) / 8;
    list->iindexlist[inum] = i < na ? -1 : (i - na) % 8;   // igcell * apc + ibasis
    inum++;
  }
  list->ainum = na;
  list->einum = list->ninum = 0;
  list->ginum = inum - na;
  list->inum = inum;
}

void B200Bridge::dump_list(const char *file, int half)
{
  check_system();
  upload(false);
  status(cacb200_set_neighbor(ctx, neighbor->skin, 0), "set_neighbor");
  status(cacb200_build_lists(ctx, half), "build_lists");
  int64_t n = 0;
  int nsites = 0;
  status(cacb200_list_size(ctx, half, &n, &nsites), "list_size");
  std::vector<int64_t> off(nsites + 1);
  std::vector<int8_t> kind(std::max<int64_t>(n, 1)), img(3 * std::max<int64_t>(n, 1));
  std::vector<int32_t> idx(std::max<int64_t>(n, 1)), site(std::max<int64_t>(n, 1));
  status(cacb200_get_list(ctx, half, off.data(), kind.data(), idx.data(), site.data(), img.data()),
         "get_list");
  int na = atom->nlocal;
  typedef std::tuple<int, int, int, int, int, int> Key;
  std::vector<std::pair<Key, std::vector<Key>>> rows(nsites);
  for (int i = 0; i < nsites; i++) {
    Key ik = i < na ? Key(0, (int)atom->tag[i], -1, 0, 0, 0)
                    : Key(1, (int)element->tag[(i - na) / 8], (i - na) % 8, 0, 0, 0);
    rows[i].first = ik;
    for (int64_t k = off[i]; k < off[i + 1]; k++) {
      int t = kind[k] == 0 ? (int)atom->tag[idx[k]] : (int)element->tag[idx[k]];
      rows[i].second.emplace_back(kind[k], t, site[k], img[3 * k], img[3 * k + 1], img[3 * k + 2]);
    }
    std::sort(rows[i].second.begin(), rows[i].second.end());
  }
  std::sort(rows.begin(), rows.end(),
            [](const std::pair<Key, std::vector<Key>> &a, const std::pair<Key, std::vector<Key>> &b) {
              return a.first < b.first;
            });
  FILE *fp = fopen(file, "w");
  if (!fp) error->one(FLERR, "write_b200_neighbor: cannot open file");
  fprintf(fp, "# cac b200 neighbour list v1: I kind tag site n / J kind tag site sx sy sz\n");
  fprintf(fp, "inum %d\n", nsites);
  for (auto &r : rows) {
    fprintf(fp, "I %d %d %d %d\n", std::get<0>(r.first), std::get<1>(r.first), std::get<2>(r.first),
            (int)r.second.size());
    for (auto &k : r.second)
      fprintf(fp, "J %d %d %d %d %d %d\n", std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k),
              std::get<4>(k), std::get<5>(k));
  }
  fclose(fp);
}
