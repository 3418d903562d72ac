/*
 * FP64 CPU oracle for one AGBNP3 energy+gradient evaluation.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain double-precision restatement of
 * the reference's agbnp3_ener() path (agbnp3.c:492-566 ->
 * agbnp3_total_energy, agbnp3.c:1221-1816) used as the checker by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline leg.  The
 * product (agbnp3_b200) never links, loads or calls it.
 *
 * Parity is pinned against the reference library itself: tests/golden holds
 * outputs of the unmodified reference (built from its sources by
 * oracle/Makefile) on seeded globules, and tests compare this oracle with
 * those fixtures at FP32 tolerance (the reference computes in float,
 * agbnp3_private.h:40-45).
 *
 * All arrays are in the engine's internal atom order: heavy atoms first,
 * hydrogens last (agbnp3.c:739-779).
 */
#ifndef AGBNP3_ORACLE_H
#define AGBNP3_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_ORDER 5

typedef struct {
  int natoms, nheavy;
  const double *x, *y, *z;  /* coordinates */
  const double *r;          /* radii, already enlarged by 0.5 A */
  const double *charge;
  const double *igamma, *sgamma, *ialpha, *salpha;
  const int *hbtype;
  const double *hbcorr;
  const int *conn_offset; /* natoms+1, connection table in internal indices */
  const int *conn_list;
  double eps_in, eps_out;
  int compat; /* 1: reproduce two reference behaviours: the spe index read in
                 the water-site free-volume loop
                 (agbnp3_cpu_simd_kernels.c:2854) and the sign of the second
                 curvature term of the spline derivative
                 (agbnp3_utils.c:250-251, agbnp3_cpu_simd_kernels.c:966-967).
                 0: the consistent model (forces = -grad E). */
} orc_in;

typedef struct {
  /* energies */
  double egb, evdw, ecorr_vdw, ecav, ecorr_cav, ehb, mol_volume;
  /* outputs, caller-allocated (natoms or 3*natoms), internal order */
  double *sp, *br, *surf_area, *dgbdr, *dvwdr, *decav, *dehb;
  /* optional per-atom intermediates (NULL to skip) */
  double *volumep, *surf_raw, *spe, *br1, *dera, *deru, *derv, *derh;
  double *q2ab, *abrw, *psvol, *gammap, *derus, *dervs;
  /* optional near list: counts per heavy atom + concatenated neighbours */
  int *nl_count, *nl_list;
  int nl_cap, nl_total;
  /* optional overlap candidates of all tree levels, in the reference's
     enumeration order: order, parents (5 per candidate), raw volume,
     switched volume */
  int cand_cap, cand_total;
  int *cand_order, *cand_parents;
  double *cand_gvol, *cand_gvolp;
  int n_kept[ORC_MAX_ORDER + 1];
  /* optional water sites */
  int ws_cap, nws;
  double *ws_pos, *ws_sp;
  int *ws_parent0, *ws_type;
  /* optional Q4 spline tables: ntypes^2 tables of 512 nodes */
  int tab_cap, ntypes;
  double *tab_y, *tab_y2;
  int *rtype;
} orc_out;

/* returns 0 on success; on a water-site topology that the reference rejects
   with an error (trigonal out-of-plane) returns -2 */
int agbnp3_oracle_eval(const orc_in *in, orc_out *out);

#ifdef __cplusplus
}
#endif
#endif
