/*
 * pair_style lj/cut/fulllist (see pair_lj_cut_fulllist.h).  Test
 * infrastructure only.  Pair arithmetic as in PairLJCut::compute
 * (pair_lj_cut.cpp:227-417); every i accumulates its own force only.
 */
#include "pair_lj_cut_fulllist.h"

#include "atom.h"
#include "element.h"
#include "neigh_list.h"
#include "neigh_request.h"
#include "neighbor.h"

using namespace CAC_NS;

void PairLJCutFullList::init_style()
{
  int irequest = neighbor->request(this, instance_me);
  neighbor->requests[irequest]->half = 0;
  neighbor->requests[irequest]->full = 1;
  cut_respa = nullptr;
}

void PairLJCutFullList::compute(int eflag, int vflag)
{
  ev_init(eflag, vflag);
  double **ax = atom->x, **af = atom->f;
  int *atype = atom->type;
  int *npe = element->npe, *apc = element->apc, *etype = element->etype;
  int **ctype = element->ctype, **g2n = element->g2n;
  double ****nodex = element->nodex, ****gaussf = element->gaussf;
  double ***shape_array = element->shape_array;
  double *nodal_weight = element->nodal_weight;

  for (int ii = 0; ii < list->inum; ii++) {
    int i = list->ilist[ii];
    int iindex = list->iindexlist[ii];
    double xtmp, ytmp, ztmp, *fi, iescale = 0.0;
    int ictype;
    if (iindex < 0) {
      xtmp = ax[i][0]; ytmp = ax[i][1]; ztmp = ax[i][2];
      ictype = atype[i];
      fi = af[i];
      iescale = 0.5;
    } else {
      int t = etype[i];
      int igcell = iindex / apc[t], ibasis = iindex % apc[t];
      int inode = g2n[t][igcell];
      ictype = ctype[i][ibasis];
      fi = gaussf[i][ibasis][igcell];
      xtmp = nodex[i][ibasis][inode][0];
      ytmp = nodex[i][ibasis][inode][1];
      ztmp = nodex[i][ibasis][inode][2];
      iescale = nodal_weight[t] / 2.0;
    }
    int *jlist = list->firstneigh[ii];
    int *jindexlist = list->firstneighindex[ii];
    for (int jj = 0; jj < list->numneigh[ii]; jj++) {
      int j = jlist[jj];
      int jindex = jindexlist[jj];
      double delx = xtmp, dely = ytmp, delz = ztmp;
      int jctype;
      if (jindex < 0) {
        delx -= ax[j][0]; dely -= ax[j][1]; delz -= ax[j][2];
        jctype = atype[j];
      } else {
        int t = etype[j];
        int jucell = jindex / apc[t], jbasis = jindex % apc[t];
        jctype = ctype[j][jbasis];
        for (int node = 0; node < npe[t]; node++) {
          delx -= shape_array[t][jucell][node] * nodex[j][jbasis][node][0];
          dely -= shape_array[t][jucell][node] * nodex[j][jbasis][node][1];
          delz -= shape_array[t][jucell][node] * nodex[j][jbasis][node][2];
        }
      }
      double rsq = delx * delx + dely * dely + delz * delz;
      if (rsq < cutsq[ictype][jctype]) {
        double r2inv = 1.0 / rsq;
        double r6inv = r2inv * r2inv * r2inv;
        double forcelj = r6inv * (lj1[ictype][jctype] * r6inv - lj2[ictype][jctype]);
        double fpair = forcelj * r2inv;
        fi[0] += delx * fpair;
        fi[1] += dely * fpair;
        fi[2] += delz * fpair;
        if (eflag_global)
          eng_vdwl += iescale * (r6inv * (lj3[ictype][jctype] * r6inv - lj4[ictype][jctype]) -
                                 offset[ictype][jctype]);
      }
    }
  }
}
