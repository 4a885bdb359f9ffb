/*
 * CPU restatement of the CAC reference's per-timestep force path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE: only the tests, the smoke check and
 * the benchmark's CPU-baseline leg load this library, and only as the checker.
 *
 * Scope: one periodic orthogonal box, one atom type, 8-node Hex elements with
 * apc = 1, 9 lattice sites per edge and 2x2x2 Gauss points (the nodes), UNIFORM
 * weights, CONSISTENT nodal forces.  Every function cites the reference
 * (tcphan0601/CAC, V3.2.0/src) file:line that it restates.  Arithmetic keeps
 * the reference's FP64 operation order wherever it decides list membership
 * (distance tests); force sums may be accumulated in a different order.
 *
 * Site numbering ("i-sites"): atoms 0..natoms-1, then the Gauss points of
 * element e at natoms + 8*e + igcell.  Neighbour entries name an atom
 * (kind 0, idx = atom index, site = -1) or a lattice site of an element
 * (kind 1, idx = element index, site = jucell) plus the periodic image
 * (sx, sy, sz) in {-1, 0, 1}.
 */
#ifndef CAC_ORACLE_H
#define CAC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double boxlo[3], boxhi[3];
  int natoms, nelements;
  double *x, *v, *f;                 /* [natoms][3] */
  double *nodex, *nodev, *nodef;     /* [nelements][8][3] */
  double *gaussf;                    /* [nelements][8 igcell][3] */
  double mass;
} oracle_state;

typedef struct {
  int nsites;
  int64_t nentries;
  int64_t *offset;                   /* [nsites + 1] */
  int32_t *jidx;                     /* atom or element index */
  int32_t *jsite;                    /* -1 for atoms, jucell for lattice sites */
  int8_t *jkind;                     /* 0 atom, 1 lattice site */
  int8_t *img;                       /* [nentries][3] */
} oracle_list;

typedef struct {
  double energy;                     /* eng_vdwl */
  double virial[6];                  /* global pairwise virial (xx yy zz xy xz yz) */
  double *eatom;                     /* [natoms] or NULL */
  double *vatom;                     /* [natoms][6] or NULL */
  double *enode;                     /* [nelements][8] or NULL */
  double *vnode;                     /* [nelements][8][6] or NULL */
} oracle_ev;

typedef struct {
  int nrho, nr;
  double drho, dr, cut, rhomax;
  double *frho_spline;               /* [nrho+1][7] */
  double *rhor_spline;               /* [nr+1][7] */
  double *z2r_spline;                /* [nr+1][7] */
} oracle_eam;

/* element-type tables (Hex, 9x9x9 sites, 2x2x2 Gauss points) */
void oracle_shape_array(double *shape /* [729][8] */);
void oracle_gauss_tables(int *g2u /* [8] */, int *g2n /* [8] */,
                         double *weighted_shape /* [8][8] */, double *nodal_weight);
void oracle_inverse_mass_hex(double *minv /* [8][8] */);

/* neighbour lists: half = 1 for half/bin/newton, 0 for full/bin */
int oracle_build_list(const oracle_state *s, double cutneigh, int half, oracle_list *out);
void oracle_free_list(oracle_list *l);

/* pair styles over a half list (as the reference evaluates them) */
int oracle_lj_compute(oracle_state *s, const oracle_list *half, double epsilon,
                      double sigma, double cut, oracle_ev *ev);
int oracle_eam_load_setfl(const char *path, oracle_eam *eam);
void oracle_eam_free(oracle_eam *eam);
int oracle_eam_compute(oracle_state *s, const oracle_list *half, const oracle_eam *eam,
                       oracle_ev *ev, double *rho_atom, double *rho_node);

/* nodal force assembly (CONSISTENT) and velocity-Verlet halves */
void oracle_compute_nodef(oracle_state *s);
void oracle_nve_initial(oracle_state *s, double dt);
void oracle_nve_final(oracle_state *s, double dt);
void oracle_pbc(oracle_state *s);

/* whole run: setup forces, then nsteps of velocity Verlet with a list rebuild
 * every `every` steps.  pair = 0 LJ (p0 = epsilon, p1 = sigma, p2 = cut),
 * 1 EAM (eam).  On return the state holds the last step's x, v, f. */
int oracle_run_nve(oracle_state *s, int pair, double p0, double p1, double p2,
                   const oracle_eam *eam, double skin, double dt, int nsteps, int every);

/* neigh_modify check yes|no for oracle_minimize_fire (default no): a rebuild
 * due by `every` happens only after an atom or node moved past half the skin */
void oracle_set_neighbor_check(int check);

/* FIRE minimisation (see cac_oracle.c); par holds the 11 Min parameters */
int oracle_minimize_fire(oracle_state *s, int pair, double p0, double p1, double p2,
                         const oracle_eam *eam, double skin, double dt0, double etol, double ftol,
                         int maxiter, int normstyle, int every, const double *par, int *code,
                         int *niter, double *energy, double *fnorm);

#ifdef __cplusplus
}
#endif

#endif
