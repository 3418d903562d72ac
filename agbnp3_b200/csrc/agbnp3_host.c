/*
 * AGBNP3 public C API on top of the CUDA device layer.
 *
 * Host-side work mirrors the reference's agbnp3_new / agbnp3_ener
 * (agbnp3.c:121-566): the instance registry, the heavy-first atom reorder,
 * the copy of the parameters and of the connection table, the radius types
 * and the Q4 spline tables, and the water-site topology.  Everything that
 * depends on coordinates runs on the device (agbnp3_dev.cu).
 */
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "agbnp3.h"
#include "agbnp3_b200.h"
#include "agbnp3_dev.h"

#define H_PI 3.14159265359
#define H_KFC 2.5
#define H_PFC 2.97354
#define H_RINC 0.5
#define H_AMAX 20.0
#define H_HBRAD 1.4
#define MAX_RTYPES 256

static char last_error[1024];

static void errprint(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(last_error, sizeof(last_error), fmt, ap);
  va_end(ap);
  fprintf(stderr, "%s\n", last_error);
}

const char *agbnp3_last_error(void) { return last_error; }

/* for the library's CUDA translation units: record a message as the last
   error and print it, as errprint does */
void agb_host_set_error(const char *msg) { errprint("%s", msg); }

typedef struct {
  int in_use;
  int natoms, nheavy;
  int *int2ext, *ext2int;
  /* internal order */
  double *r, *charge, *igamma, *sgamma, *ialpha, *salpha, *hbcorr;
  int *hbtype;
  int *conn_off, *conn_list;
  int *rtype, ntypes;
  double *tab; /* ntypes^2 x AGB_NA x {y, y2} */
  int nws, ws_error;
  int *ws_kind, *ws_parent, *ws_nparent, *ws_prev;
  double *ws_khb;
  double eps_in, eps_out;
  float cell;
  int precision, compat, device, verbose;
  agb_dev *dev;
  double *stage; /* float interface: double copies of coordinates and outputs (15 natoms) */
} inst_t;

typedef struct {
  int in_use;
  int n;
  int *tags;
  int natoms;
  int precision, compat;
  agb_dev *dev;
} batch_t;

static int initialized = 0;
static inst_t **insts = NULL;
static int ninsts = 0;
static batch_t **batches = NULL;
static int nbatches = 0;
static int next_device = -1;

static int default_device(void) {
  if (next_device >= 0) return next_device;
  const char *e = getenv("AGBNP3_DEVICE");
  if (!e) e = getenv("LOCAL_RANK");
  return e ? atoi(e) : 0;
}

static void default_mode(int *prec, int *compat) {
  const char *p = getenv("AGBNP3_PRECISION");
  const char *c = getenv("AGBNP3_COMPAT");
  *prec = (p && (strcmp(p, "fp64") == 0 || strcmp(p, "0") == 0)) ? AGBNP3_PREC_FP64 : AGBNP3_PREC_MIXED;
  *compat = c ? atoi(c) != 0 : 1;
}

/* ------------------------------------------------------------------ */
/* registry (agbnp3.c:54-118, 568-578)                                 */
/* ------------------------------------------------------------------ */
int agbnp3_initialize(void) {
  if (initialized) return AGBNP_OK;
  initialized = 1;
  return AGBNP_OK;
}

int agbnp_initialize(void) { return agbnp3_initialize(); }

static inst_t *get_inst(int tag, const char *who) {
  if (!initialized) {
    errprint("%s: agbnp library is not initialized.", who);
    return NULL;
  }
  if (tag < 0 || tag >= ninsts || !insts[tag] || !insts[tag]->in_use) {
    errprint("%s: invalid tag %d.", who, tag);
    return NULL;
  }
  return insts[tag];
}

static void inst_free(inst_t *I) {
  if (!I) return;
  if (I->dev) agb_dev_destroy(I->dev);
  void *ps[] = {I->int2ext, I->ext2int, I->r,       I->charge,    I->igamma,  I->sgamma,   I->ialpha,
                I->salpha,  I->hbcorr,  I->hbtype,  I->conn_off,  I->conn_list, I->rtype,  I->tab,
                I->ws_kind, I->ws_parent, I->ws_nparent, I->ws_prev, I->ws_khb, I->stage};
  for (size_t k = 0; k < sizeof(ps) / sizeof(ps[0]); k++) free(ps[k]);
  free(I);
}

/* ------------------------------------------------------------------ */
/* Q4 tables (agbnp3_utils.c:148-227, 380-422, 808-883;               */
/* agbnp3.c:3886-3975)                                                 */
/* ------------------------------------------------------------------ */

/* integral of 1/r^4 over the part of a sphere (radius Rj, centre at
   distance rij) that lies outside a sphere of radius Ri; *dr = d/drij */
static double i4_integral(double rij, double Ri, double Rj, double *dr) {
  const double tp = 2.0 * H_PI;
  const double r2 = rij * rij;
  if (rij > Ri + Rj) { /* disjoint */
    double p = (rij + Rj) * (rij - Rj), l = 0.5 * log((rij + Rj) / (rij - Rj));
    *dr = tp * ((Rj / (rij * p)) * (1.0 - 2.0 * r2 / p) + l / r2);
    return tp * (Rj / p - l / rij);
  }
  if (r2 > (Rj - Ri) * (Rj - Ri)) { /* intersecting */
    double up = rij + Rj, p = up * (rij - Rj);
    double a = 1.0 / up, b = 1.0 / Ri, l = 0.5 * log(up / Ri);
    *dr = tp * (0.5 * (1.0 - 0.5 * p / r2) * (a * a - b * b) + l / r2);
    return tp * (b - a + (0.25 * p * (a * a - b * b) - l) / rij);
  }
  if (Ri > Rj) { /* descreener inside the excluded sphere */
    *dr = 0.0;
    return 0.0;
  }
  double p = -(rij + Rj) * (Rj - rij);
  if (rij < 0.001 * Rj) { /* removable singularity at rij = 0 */
    double t = rij / Rj;
    *dr = -(2.0 * tp * t / (Rj * Rj)) * (1.0 / (t * t - 1.0) + 2.0 / 3.0);
    return tp * (2.0 / Ri + Rj / p - (1.0 + 2.0 / 3.0 * t * t) / Rj);
  }
  double l = 0.5 * log((rij + Rj) / (Rj - rij));
  *dr = tp * (-(Rj / p) * (2.0 * rij / p - 1.0 / rij) + l / r2);
  return tp * (2.0 / Ri + Rj / p - l / rij);
}

/* the descreener's radius grown by twice its Gaussian overlap with the
   descreened atom; both Gaussian exponents use Ri, as the reference does */
static double i4_inflated(double rij, double Ri, double Rj, double *dr) {
  double a = H_KFC / (Ri * Ri), s = 2.0 * a;
  double g = H_PFC * H_PFC * exp(-a * a * rij * rij / s) * pow(H_PI / s, 1.5);
  double vj = 4.0 * H_PI * Rj * Rj * Rj / 3.0;
  return i4_integral(rij, Ri, Rj * pow((vj + 2.0 * g) / vj, 1.0 / 3.0), dr);
}

/* one spline table: nodes a_k = k h on [0, 20] of i4_inflated(a, b, 1),
   clamped spline with slope of the integral at 0 and zero slope (and
   value) at 20; stores {y, y2} pairs */
static void build_table(double b, double *out) {
  const int n = AGB_NA;
  const double h = H_AMAX / (n - 1);
  double y[AGB_NA], m[AGB_NA], w[AGB_NA];
  double a = 0.0, slope0 = 0.0, dr;
  for (int k = 0; k < n - 1; k++) {
    y[k] = i4_inflated(a, b, 1.0, &dr);
    if (k == 0) slope0 = dr;
    a += h;
  }
  y[n - 1] = 0.0;
  /* tridiagonal system for the second derivatives (uniform grid); the end
     conditions are those of agbnp3_cspline_setup (agbnp3_utils.c:193-227) */
  m[0] = -0.5;
  w[0] = (3.0 / h) * ((y[1] - y[0]) / h - slope0);
  for (int k = 1; k < n - 1; k++) {
    double piv = 0.5 * m[k - 1] + 2.0;
    m[k] = -0.5 / piv;
    double jump = (y[k + 1] - y[k]) / h - (y[k] - y[k - 1]) / h;
    w[k] = (3.0 * jump / h - 0.5 * w[k - 1]) / piv;
  }
  double tail = (3.0 / h) * (0.0 - (y[n - 1] - y[n - 2]) / (2.0 * h));
  m[n - 1] = (tail - 0.5 * w[n - 2]) / (0.5 * m[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; k--) m[k] = m[k] * m[k + 1] + w[k];
  for (int k = 0; k < n; k++) {
    out[2 * k] = y[k];
    out[2 * k + 1] = m[k];
  }
}

/* radius types: one per distinct radius (agbnp3_utils.c:808-838 groups
   equal float radii; distinct double radii are kept apart here, so that a
   type has one exact radius, while each type's table is built from its
   float radius as in the reference) */
static int build_tables(inst_t *I) {
  double radii[MAX_RTYPES];
  int nt = 0;
  I->rtype = (int *)malloc(sizeof(int) * I->natoms);
  if (!I->rtype) return -1;
  for (int i = 0; i < I->natoms; i++) {
    double ri = I->r[i];
    int t = -1;
    for (int k = 0; k < nt; k++)
      if (ri == radii[k]) {
        t = k;
        break;
      }
    if (t < 0) {
      if (nt == MAX_RTYPES) {
        errprint("agbnp3_new(): more than %d distinct atomic radii.", MAX_RTYPES);
        return -1;
      }
      radii[nt] = ri;
      t = nt++;
    }
    I->rtype[i] = t;
  }
  I->ntypes = nt;
  I->tab = (double *)malloc(sizeof(double) * (size_t)nt * nt * AGB_NA * 2);
  if (!I->tab) return -1;
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++)
      build_table(((double)(float)radii[a] - H_RINC) / (double)(float)radii[b],
                  I->tab + (size_t)(a * nt + b) * AGB_NA * 2);
  return 0;
}

/* ------------------------------------------------------------------ */
/* water-site topology: the dispatch of agbnp3_create_ws_ofatom       */
/* (agbnp3.c:1920-2012) and the parent lookups of the create_ws_*     */
/* functions; positions are computed on the device every call         */
/* ------------------------------------------------------------------ */
typedef struct {
  int kind, np, par[4];
} ws_desc;

/* returns the number of sites of atom iat (0..4), -1 when the reference
   aborts the evaluation (trigonal out-of-plane with != 3 bonds) */
static int ws_of_atom(const inst_t *I, int iat, ws_desc *o) {
  const int *off = I->conn_off, *lst = I->conn_list + I->conn_off[iat];
  int nne = off[iat + 1] - off[iat];
  int t = I->hbtype[iat];
  switch (t) {
    case AGBNP_HB_POLARH: {
      for (int q = 0; q < nne; q++)
        if (lst[q] < I->nheavy) {
          o[0] = (ws_desc){WK_POLARH, 2, {iat, lst[q], -1, -1}};
          return 1;
        }
      return 0; /* isolated or no heavy parent: no site */
    }
    case AGBNP_HB_TRIGONAL:
    case AGBNP_HB_TRIGONAL_S: {
      if (t == AGBNP_HB_TRIGONAL && nne == 2) {
        o[0] = (ws_desc){WK_BIS2, 3, {iat, lst[0], lst[1], -1}};
        return 1;
      }
      if (nne != 1) return 0;
      int ir = lst[0];
      int nr = off[ir + 1] - off[ir];
      const int *lr = I->conn_list + off[ir];
      if (nr != 3) return 0;
      int r1 = -1, r2 = -1;
      for (int q = 0; q < nr && r1 < 0; q++)
        if (lr[q] != iat) r1 = lr[q];
      for (int q = 0; q < nr && r2 < 0; q++)
        if (lr[q] != iat && lr[q] != r1) r2 = lr[q];
      if (r1 < 0 || r2 < 0) return 0;
      o[0] = (ws_desc){WK_TRIG1_A, 4, {iat, ir, r1, r2}};
      o[1] = (ws_desc){WK_TRIG1_B, 4, {iat, ir, r1, r2}};
      if (t == AGBNP_HB_TRIGONAL) return 2;
      o[2] = (ws_desc){WK_TRIGS_A, 4, {iat, ir, r1, r2}};
      o[3] = (ws_desc){WK_TRIGS_B, 4, {iat, ir, r1, r2}};
      return 4;
    }
    case AGBNP_HB_TRIGONAL_OOP:
      if (nne != 3) return -1;
      o[0] = (ws_desc){WK_OOP_A, 4, {iat, lst[0], lst[1], lst[2]}};
      o[1] = (ws_desc){WK_OOP_B, 4, {iat, lst[0], lst[1], lst[2]}};
      return 2;
    case AGBNP_HB_TETRAHEDRAL:
      if (nne == 2) {
        o[0] = (ws_desc){WK_TET2_A, 3, {iat, lst[0], lst[1], -1}};
        o[1] = (ws_desc){WK_TET2_B, 3, {iat, lst[0], lst[1], -1}};
        return 2;
      }
      if (nne == 3) {
        o[0] = (ws_desc){WK_BIS3, 4, {iat, lst[0], lst[1], lst[2]}};
        return 1;
      }
      if (nne == 1) {
        int ir = lst[0];
        int nr = off[ir + 1] - off[ir];
        const int *lr = I->conn_list + off[ir];
        if (nr != 4) return 0;
        int m = 0;
        for (int q = 0; q < 4; q++)
          if (lr[q] != iat) o[m++] = (ws_desc){WK_TET1, 3, {iat, ir, lr[q], -1}};
        return m == 3 ? 3 : 0;
      }
      return 0;
    default:
      return 0;
  }
}

static int build_ws(inst_t *I) {
  int cap = 16, n = 0;
  ws_desc *all = (ws_desc *)malloc(sizeof(ws_desc) * cap);
  if (!all) return -1;
  I->ws_error = 0;
  for (int i = 0; i < I->natoms; i++) {
    if (I->hbtype[i] == AGBNP_HB_INACTIVE) continue;
    ws_desc tmp[4];
    int k = ws_of_atom(I, i, tmp);
    if (k < 0) {
      I->ws_error = 1;
      continue;
    }
    if (n + k > cap) {
      cap = 2 * (n + k);
      all = (ws_desc *)realloc(all, sizeof(ws_desc) * cap);
      if (!all) return -1;
    }
    memcpy(all + n, tmp, sizeof(ws_desc) * k);
    n += k;
  }
  I->nws = n;
  int m = n > 0 ? n : 1;
  I->ws_kind = (int *)malloc(sizeof(int) * m);
  I->ws_parent = (int *)malloc(sizeof(int) * 4 * m);
  I->ws_nparent = (int *)malloc(sizeof(int) * m);
  I->ws_prev = (int *)malloc(sizeof(int) * m);
  I->ws_khb = (double *)malloc(sizeof(double) * m);
  if (!I->ws_kind || !I->ws_parent || !I->ws_nparent || !I->ws_prev || !I->ws_khb) return -1;
  for (int w = 0; w < n; w++) {
    I->ws_kind[w] = all[w].kind;
    I->ws_nparent[w] = all[w].np;
    for (int q = 0; q < 4; q++) I->ws_parent[4 * w + q] = all[w].par[q] >= 0 ? all[w].par[q] : all[w].par[0];
    I->ws_khb[w] = I->hbcorr[all[w].par[0]];
    /* the atom index the reference's free-volume loop carries into this
       site: the previous site's last parent (agbnp3_cpu_simd_kernels.c:
       2927-2933); before the first site it is nheavy, a hydrogen, whose
       spe is 0 */
    I->ws_prev[w] = w == 0 ? -1 : all[w - 1].par[all[w - 1].np - 1];
  }
  free(all);
  return 0;
}

/* ------------------------------------------------------------------ */
/* device systems                                                      */
/* ------------------------------------------------------------------ */
static int make_dev(inst_t **L, int n, int precision, int compat, int device, agb_dev **out) {
  int N = 0, NW = 0, nt = L[0]->ntypes;
  for (int k = 0; k < n; k++) {
    N += L[k]->natoms;
    NW += L[k]->nws;
    if (L[k]->ntypes != nt) nt = -1;
  }
  agb_dev_desc d;
  memset(&d, 0, sizeof(d));
  d.ninst = n;
  d.natoms = N;
  d.nws = NW;
  d.precision = precision;
  d.compat = compat;
  d.device = device;
  int *inst_begin = (int *)malloc(sizeof(int) * (n + 1)), *inst_nheavy = (int *)malloc(sizeof(int) * n);
  int *ws_begin = (int *)malloc(sizeof(int) * (n + 1));
  double *inst_df = (double *)malloc(sizeof(double) * n);
  float *inst_cell = (float *)malloc(sizeof(float) * n);
  int *ext_of = (int *)malloc(sizeof(int) * N), *rtype = (int *)malloc(sizeof(int) * N);
  double *arr[6];
  for (int k = 0; k < 6; k++) arr[k] = (double *)malloc(sizeof(double) * N);
  int m = NW > 0 ? NW : 1;
  int *ws_kind = (int *)malloc(sizeof(int) * m), *ws_parent = (int *)malloc(sizeof(int) * 4 * m);
  int *ws_nparent = (int *)malloc(sizeof(int) * m), *ws_prev = (int *)malloc(sizeof(int) * m);
  double *ws_khb = (double *)malloc(sizeof(double) * m);

  /* radius types shared by all members: map each member's types onto a
     common list (first appearance across members) */
  double radii[MAX_RTYPES];
  int ntot = 0;
  int *tmap = (int *)malloc(sizeof(int) * MAX_RTYPES * n);
  for (int k = 0; k < n; k++) {
    inst_t *I = L[k];
    double loc[MAX_RTYPES];
    for (int i = 0; i < I->natoms; i++) loc[I->rtype[i]] = I->r[i];
    for (int t = 0; t < I->ntypes; t++) {
      int f = -1;
      for (int q = 0; q < ntot; q++)
        if (loc[t] == radii[q]) f = q;
      if (f < 0) {
        if (ntot == MAX_RTYPES) {
          errprint("batch: more than %d distinct atomic radii", MAX_RTYPES);
          return -1;
        }
        radii[ntot] = loc[t];
        f = ntot++;
      }
      tmap[k * MAX_RTYPES + t] = f;
    }
  }
  nt = ntot;
  double *tab = (double *)malloc(sizeof(double) * (size_t)nt * nt * AGB_NA * 2);
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++)
      build_table(((double)(float)radii[a] - H_RINC) / (double)(float)radii[b],
                  tab + (size_t)(a * nt + b) * AGB_NA * 2);

  int g = 0, w = 0;
  for (int k = 0; k < n; k++) {
    inst_t *I = L[k];
    inst_begin[k] = g;
    ws_begin[k] = w;
    inst_nheavy[k] = I->nheavy;
    inst_df[k] = -0.5 * (1.0 / I->eps_in - 1.0 / I->eps_out);
    inst_cell[k] = I->cell;
    for (int i = 0; i < I->natoms; i++) {
      ext_of[g + i] = g + I->int2ext[i];
      rtype[g + i] = tmap[k * MAX_RTYPES + I->rtype[i]];
      arr[0][g + i] = I->r[i];
      arr[1][g + i] = I->charge[i];
      arr[2][g + i] = I->igamma[i];
      arr[3][g + i] = I->sgamma[i];
      arr[4][g + i] = I->ialpha[i];
      arr[5][g + i] = I->salpha[i];
    }
    for (int s = 0; s < I->nws; s++) {
      ws_kind[w + s] = I->ws_kind[s];
      ws_nparent[w + s] = I->ws_nparent[s];
      for (int q = 0; q < 4; q++) ws_parent[4 * (w + s) + q] = g + I->ws_parent[4 * s + q];
      ws_prev[w + s] = I->ws_prev[s] >= 0 ? g + I->ws_prev[s] : -1;
      ws_khb[w + s] = I->ws_khb[s];
    }
    g += I->natoms;
    w += I->nws;
  }
  inst_begin[n] = g;
  ws_begin[n] = w;
  d.inst_begin = inst_begin;
  d.inst_nheavy = inst_nheavy;
  d.inst_df = inst_df;
  d.inst_cell = inst_cell;
  d.ext_of = ext_of;
  d.r = arr[0];
  d.charge = arr[1];
  d.igamma = arr[2];
  d.sgamma = arr[3];
  d.ialpha = arr[4];
  d.salpha = arr[5];
  d.rtype = rtype;
  d.ntypes = nt;
  d.tab = tab;
  d.ws_kind = ws_kind;
  d.ws_parent = ws_parent;
  d.ws_nparent = ws_nparent;
  d.ws_prev = ws_prev;
  d.ws_khb = ws_khb;
  d.ws_begin = ws_begin;
  int rc = agb_dev_create(&d, out);
  if (rc != 0) errprint("device setup failed: %s", agb_dev_last_error());
  free(inst_begin); free(inst_nheavy); free(ws_begin); free(inst_df); free(inst_cell); free(ext_of); free(rtype);
  for (int k = 0; k < 6; k++) free(arr[k]);
  free(ws_kind); free(ws_parent); free(ws_nparent); free(ws_prev); free(ws_khb); free(tmap); free(tab);
  return rc;
}

/* ------------------------------------------------------------------ */
/* agbnp3_new / agbnp3_delete / agbnp3_terminate                       */
/* ------------------------------------------------------------------ */
int agbnp3_new(int *tag, int natoms, float_i *x, float_i *y, float_i *z, float_i *r, float_i *charge,
               float_i dielectric_in, float_i dielectric_out, float_i *igamma, float_i *sgamma, float_i *ialpha,
               float_i *salpha, int *hbtype, float_i *hbcorr, int nhydrogen, int *ihydrogen, NeighList *conntbl,
               int verbose) {
  (void)x;
  (void)y;
  (void)z;
  if (!initialized) {
    errprint("agbnp3_new(): agbnp library is not initialized.");
    return AGBNP_ERR;
  }
  if (!tag || natoms <= 0 || !r || !charge || !igamma || !sgamma || !ialpha || !salpha || !hbtype || !hbcorr ||
      nhydrogen < 0 || nhydrogen > natoms || (nhydrogen > 0 && !ihydrogen)) {
    errprint("agbnp3_new(): invalid arguments.");
    return AGBNP_ERR;
  }
  if (!conntbl) {
    errprint("agbnp3_new(): error: NULL connection table. AGBNP v.3 requires a connection table.");
    return AGBNP_ERR;
  }
  if (conntbl->natoms < natoms || !conntbl->nne || !conntbl->neighl) {
    errprint("agbnp3_new(): connection table covers %d atoms, expected %d.", conntbl->natoms, natoms);
    return AGBNP_ERR;
  }
  inst_t *I = (inst_t *)calloc(1, sizeof(inst_t));
  if (!I) {
    errprint("agbnp3_new(): out of memory.");
    return AGBNP_ERR;
  }
  int N = natoms;
  I->natoms = N;
  I->verbose = verbose;
  I->eps_in = dielectric_in;
  I->eps_out = dielectric_out;
  default_mode(&I->precision, &I->compat);
  I->device = default_device();

  /* heavy atoms first, hydrogens last, each in caller order
     (agbnp3.c:739-779) */
  char *ish = (char *)calloc(N, 1);
  I->int2ext = (int *)malloc(sizeof(int) * N);
  I->ext2int = (int *)malloc(sizeof(int) * N);
  if (!ish || !I->int2ext || !I->ext2int) goto oom;
  for (int k = 0; k < nhydrogen; k++) {
    if (ihydrogen[k] < 0 || ihydrogen[k] >= N) {
      errprint("agbnp3_new(): hydrogen index %d out of range.", ihydrogen[k]);
      free(ish);
      inst_free(I);
      return AGBNP_ERR;
    }
    ish[ihydrogen[k]] = 1;
  }
  int nh = 0;
  for (int i = 0; i < N; i++) nh += ish[i];
  I->nheavy = N - nh;
  {
    int c = 0, h = I->nheavy;
    for (int i = 0; i < N; i++) {
      int k = ish[i] ? h++ : c++;
      I->int2ext[k] = i;
      I->ext2int[i] = k;
    }
  }
  free(ish);

  double **dst[] = {&I->r, &I->charge, &I->igamma, &I->sgamma, &I->ialpha, &I->salpha, &I->hbcorr};
  const float_i *src[] = {r, charge, igamma, sgamma, ialpha, salpha, hbcorr};
  for (int k = 0; k < 7; k++) {
    *dst[k] = (double *)malloc(sizeof(double) * N);
    if (!*dst[k]) goto oom;
    for (int i = 0; i < N; i++) (*dst[k])[i] = (double)src[k][I->int2ext[i]];
  }
  /* the radius increment of agbnp3.c:210 */
  for (int i = 0; i < N; i++) I->r[i] += H_RINC;
  I->hbtype = (int *)malloc(sizeof(int) * N);
  if (!I->hbtype) goto oom;
  for (int i = 0; i < N; i++) I->hbtype[i] = hbtype[I->int2ext[i]];

  /* connection table in internal indices (agbnp3.c:308-317) */
  I->conn_off = (int *)malloc(sizeof(int) * (N + 1));
  if (!I->conn_off) goto oom;
  I->conn_off[0] = 0;
  for (int i = 0; i < N; i++) {
    int e = I->int2ext[i];
    if (conntbl->nne[e] < 0) {
      errprint("agbnp3_new(): negative connection count for atom %d.", e);
      inst_free(I);
      return AGBNP_ERR;
    }
    I->conn_off[i + 1] = I->conn_off[i] + conntbl->nne[e];
  }
  I->conn_list = (int *)malloc(sizeof(int) * (I->conn_off[N] + 1));
  if (!I->conn_list) goto oom;
  for (int i = 0; i < N; i++) {
    int e = I->int2ext[i];
    for (int q = 0; q < conntbl->nne[e]; q++) {
      int j = conntbl->neighl[e][q];
      if (j < 0 || j >= N) {
        errprint("agbnp3_new(): connection table of atom %d names atom %d, outside 0..%d.", e, j, N - 1);
        inst_free(I);
        return AGBNP_ERR;
      }
      I->conn_list[I->conn_off[i] + q] = I->ext2int[j];
    }
  }

  if (build_tables(I) != 0) {
    errprint("agbnp3_new(): error building the Q4 lookup tables.");
    inst_free(I);
    return AGBNP_ERR;
  }
  if (build_ws(I) != 0) goto oom;

  /* cell edge of the neighbour grid: the largest near-list cutoff
     1.6 (ri + rj) and water-site cutoff 1.6 (ri + 1.4), with margin */
  {
    double rmax = 0.0;
    for (int i = 0; i < I->nheavy; i++)
      if (I->r[i] > rmax) rmax = I->r[i];
    double cut = 1.6 * (2.0 * rmax > rmax + H_HBRAD ? 2.0 * rmax : rmax + H_HBRAD);
    I->cell = (float)(cut * 1.001 + 0.01);
  }

  if (make_dev(&I, 1, I->precision, I->compat, I->device, &I->dev) != 0) {
    inst_free(I);
    return AGBNP_ERR;
  }

  /* slot table (agbnp3.c:143-170) */
  int slot = -1;
  for (int k = 0; k < ninsts; k++)
    if (!insts[k]) {
      slot = k;
      break;
    }
  if (slot < 0) {
    inst_t **p = (inst_t **)realloc(insts, sizeof(inst_t *) * (ninsts + 1));
    if (!p) goto oom;
    insts = p;
    slot = ninsts++;
  }
  I->in_use = 1;
  insts[slot] = I;
  *tag = slot;
  if (verbose)
    fprintf(stderr, "agbnp3_new(): instance %d: %d atoms (%d heavy), %d radius types, %d water sites, device %d\n",
            slot, N, I->nheavy, I->ntypes, I->nws, I->device);
  return AGBNP_OK;
oom:
  errprint("agbnp3_new(): out of host memory.");
  inst_free(I);
  return AGBNP_ERR;
}

int agbnp3_delete(int tag) {
  inst_t *I = get_inst(tag, "agbnp3_delete()");
  if (!I) return AGBNP_ERR;
  inst_free(I);
  insts[tag] = NULL;
  return AGBNP_OK;
}

int agbnp_delete(int tag) { return agbnp3_delete(tag); }

int agbnp3_batch_delete(int btag);

void agbnp3_terminate(void) {
  if (!initialized) {
    errprint("agbnp3_terminate(): agbnp library is not initialized.");
    return;
  }
  for (int k = 0; k < nbatches; k++)
    if (batches[k]) agbnp3_batch_delete(k);
  free(batches);
  batches = NULL;
  nbatches = 0;
  for (int k = 0; k < ninsts; k++)
    if (insts[k]) agbnp3_delete(k);
  free(insts);
  insts = NULL;
  ninsts = 0;
  initialized = 0;
}

void agbnp_terminate(void) { agbnp3_terminate(); }

/* ------------------------------------------------------------------ */
/* evaluation                                                          */
/* ------------------------------------------------------------------ */
static int eval_dev(agb_dev *dev, const char *who) {
  if (agb_dev_evaluate(dev) != 0) {
    errprint("%s: %s", who, agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_ener(int tag, int init, float_i *x, float_i *y, float_i *z, float_i *sp, float_i *br,
                float_i *mol_volume, float_i *surf_area, float_i *egb, float_i (*dgbdr)[3], float_i *evdw,
                float_i *ecorr_vdw, float_i (*dvwdr)[3], float_i *ecav, float_i *ecorr_cav, float_i (*decav)[3],
                float_i *ehb, float_i (*dehb)[3]) {
  (void)init;
  inst_t *I = get_inst(tag, "agbnp3_ener()");
  if (!I) return AGBNP_ERR;
  if (I->ws_error) {
    errprint("agbnp3_ener(): a trigonal out-of-plane acceptor does not have three bonded atoms.");
    return AGBNP_ERR;
  }
  if (!x || !y || !z) {
    errprint("agbnp3_ener(): NULL coordinates.");
    return AGBNP_ERR;
  }
  double e[7];
#ifdef SINGLE_PREC_INTERFACE
  /* float arrays in and out through double copies */
  const int N = I->natoms;
  if (!I->stage && !(I->stage = (double *)malloc(sizeof(double) * 15 * (size_t)N))) {
    errprint("agbnp3_ener(): out of memory.");
    return AGBNP_ERR;
  }
  double *sx = I->stage, *sy = sx + N, *sz = sy + N;
  for (int i = 0; i < N; i++) {
    sx[i] = x[i];
    sy[i] = y[i];
    sz[i] = z[i];
  }
  if (agb_dev_upload_coords(I->dev, sx, sy, sz) != 0) {
    errprint("agbnp3_ener(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  if (eval_dev(I->dev, "agbnp3_ener()") != AGBNP_OK) return AGBNP_ERR;
  double *osp = I->stage, *obr = osp + N, *osa = obr + N, *ogb = osa + N, *ogv = ogb + 3 * (size_t)N,
         *ogc = ogv + 3 * (size_t)N, *ogh = ogc + 3 * (size_t)N;
  if (agb_dev_download(I->dev, e, sp ? osp : NULL, br ? obr : NULL, surf_area ? osa : NULL, dgbdr ? ogb : NULL,
                       dvwdr ? ogv : NULL, decav ? ogc : NULL, dehb ? ogh : NULL) != 0) {
    errprint("agbnp3_ener(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  float_i *o1[] = {sp, br, surf_area};
  const double *d1[] = {osp, obr, osa};
  for (int k = 0; k < 3; k++)
    if (o1[k])
      for (int i = 0; i < N; i++) o1[k][i] = (float_i)d1[k][i];
  float_i(*o3[])[3] = {dgbdr, dvwdr, decav, dehb};
  const double *d3[] = {ogb, ogv, ogc, ogh};
  for (int k = 0; k < 4; k++)
    if (o3[k])
      for (int i = 0; i < N; i++)
        for (int c = 0; c < 3; c++) o3[k][i][c] = (float_i)d3[k][3 * i + c];
#else
  if (agb_dev_upload_coords(I->dev, x, y, z) != 0) {
    errprint("agbnp3_ener(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  if (eval_dev(I->dev, "agbnp3_ener()") != AGBNP_OK) return AGBNP_ERR;
  if (agb_dev_download(I->dev, e, sp, br, surf_area, (double *)dgbdr, (double *)dvwdr, (double *)decav,
                       (double *)dehb) != 0) {
    errprint("agbnp3_ener(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
#endif
  if (egb) *egb = e[0];
  if (evdw) *evdw = e[1];
  if (ecorr_vdw) *ecorr_vdw = e[2];
  if (ecav) *ecav = e[3];
  if (ecorr_cav) *ecorr_cav = e[4];
  if (ehb) *ehb = e[5];
  if (mol_volume) *mol_volume = e[6];
  return AGBNP_OK;
}

/* ------------------------------------------------------------------ */
/* extensions                                                          */
/* ------------------------------------------------------------------ */
int agbnp3_set_mode(int tag, int precision, int compat) {
  inst_t *I = get_inst(tag, "agbnp3_set_mode()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_set_mode(I->dev, precision, compat) != 0) {
    errprint("agbnp3_set_mode(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  I->precision = precision;
  I->compat = compat != 0;
  return AGBNP_OK;
}

int agbnp3_pair_order(int tag, int mode) {
  inst_t *I = get_inst(tag, "agbnp3_pair_order()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_set_pair_order(I->dev, mode) != 0) {
    errprint("agbnp3_pair_order(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_set_nblist_skin(int tag, double skin) {
  inst_t *I = get_inst(tag, "agbnp3_set_nblist_skin()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_set_skin(I->dev, skin) != 0) {
    errprint("agbnp3_set_nblist_skin(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_shard_unique_id(void *id, int nbytes) {
  int n = agb_dev_shard_unique_id(id, nbytes);
  if (n < 0) errprint("agbnp3_shard_unique_id(): %s", agb_dev_last_error());
  return n < 0 ? AGBNP_ERR : n;
}

int agbnp3_shard(int tag, int rank, int nranks, const void *id, int nbytes) {
  inst_t *I = get_inst(tag, "agbnp3_shard()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_shard(I->dev, rank, nranks, id, nbytes) != 0) {
    errprint("agbnp3_shard(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_shard_segment(int tag, int k) {
  inst_t *I = get_inst(tag, "agbnp3_shard_segment()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_shard_segment(I->dev, k) != 0) {
    errprint("agbnp3_shard_segment(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

long long agbnp3_shard_buffers(int tag, int k, double *host, int store) {
  inst_t *I = get_inst(tag, "agbnp3_shard_buffers()");
  if (!I) return AGBNP_ERR;
  long long n = agb_dev_shard_buffers(I->dev, k, host, store);
  if (n < 0) errprint("agbnp3_shard_buffers(): %s", agb_dev_last_error());
  return n;
}

int agbnp3_get_mode(int tag, int *precision, int *compat) {
  inst_t *I = get_inst(tag, "agbnp3_get_mode()");
  if (!I) return AGBNP_ERR;
  if (precision) *precision = I->precision;
  if (compat) *compat = I->compat;
  return AGBNP_OK;
}

int agbnp3_set_device(int device) {
  if (device < 0) {
    errprint("agbnp3_set_device(): invalid device %d.", device);
    return AGBNP_ERR;
  }
  next_device = device;
  return AGBNP_OK;
}

int agbnp3_set_coords(int tag, const double *x, const double *y, const double *z) {
  inst_t *I = get_inst(tag, "agbnp3_set_coords()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_upload_coords(I->dev, x, y, z) != 0) {
    errprint("agbnp3_set_coords(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_ener_resident(int tag) {
  inst_t *I = get_inst(tag, "agbnp3_ener_resident()");
  if (!I) return AGBNP_ERR;
  if (I->ws_error) {
    errprint("agbnp3_ener_resident(): a trigonal out-of-plane acceptor does not have three bonded atoms.");
    return AGBNP_ERR;
  }
  return eval_dev(I->dev, "agbnp3_ener_resident()");
}

int agbnp3_get_results(int tag, double *energies, double *sp, double *br, double *surf_area, double (*dgbdr)[3],
                       double (*dvwdr)[3], double (*decav)[3], double (*dehb)[3]) {
  inst_t *I = get_inst(tag, "agbnp3_get_results()");
  if (!I) return AGBNP_ERR;
  if (agb_dev_download(I->dev, energies, sp, br, surf_area, (double *)dgbdr, (double *)dvwdr, (double *)decav,
                       (double *)dehb) != 0) {
    errprint("agbnp3_get_results(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

/* one evaluation from and into device arrays: coordinates in, outputs out,
   no host copies; ordered after the work queued on `stream` */
static int ener_device(agb_dev *dev, const char *who, const double *x, const double *y, const double *z,
                       double *energies, double *sp, double *br, double *surf_area, double *dgbdr, double *dvwdr,
                       double *decav, double *dehb, void *stream) {
  if (!x || !y || !z) {
    errprint("%s: coordinate arrays must not be NULL.", who);
    return AGBNP_ERR;
  }
  if (agb_dev_upload_coords_dev(dev, x, y, z, stream) != 0) {
    errprint("%s: %s", who, agb_dev_last_error());
    return AGBNP_ERR;
  }
  if (eval_dev(dev, who) != AGBNP_OK) return AGBNP_ERR;
  if (agb_dev_download_dev(dev, energies, sp, br, surf_area, dgbdr, dvwdr, decav, dehb, stream) != 0) {
    errprint("%s: %s", who, agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_ener_device(int tag, const double *x, const double *y, const double *z, double *energies, double *sp,
                       double *br, double *surf_area, double *dgbdr, double *dvwdr, double *decav, double *dehb,
                       void *stream) {
  inst_t *I = get_inst(tag, "agbnp3_ener_device()");
  if (!I) return AGBNP_ERR;
  if (I->ws_error) {
    errprint("agbnp3_ener_device(): a trigonal out-of-plane acceptor does not have three bonded atoms.");
    return AGBNP_ERR;
  }
  return ener_device(I->dev, "agbnp3_ener_device()", x, y, z, energies, sp, br, surf_area, dgbdr, dvwdr, decav,
                     dehb, stream);
}

int agbnp3_surrogate_classes(int tag, const double *class_radii, int nclass, int *unmatched) {
  inst_t *I = get_inst(tag, "agbnp3_surrogate_classes()");
  if (!I) return AGBNP_ERR;
  int u = 0;
  if (agb_dev_surrogate_classes(I->dev, class_radii, nclass, &u) != 0) {
    errprint("agbnp3_surrogate_classes(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  if (unmatched) *unmatched = u;
  return AGBNP_OK;
}

int agbnp3_surrogate_features(int tag, const float *mean, const float *invstd, void *out) {
  inst_t *I = get_inst(tag, "agbnp3_surrogate_features()");
  if (!I) return AGBNP_ERR;
  if (!out) {
    errprint("agbnp3_surrogate_features(): NULL output.");
    return AGBNP_ERR;
  }
  if (agb_dev_surrogate_features(I->dev, mean, invstd, out) != 0) {
    errprint("agbnp3_surrogate_features(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

void *agbnp3_stream(int tag) {
  inst_t *I = get_inst(tag, "agbnp3_stream()");
  return I ? agb_dev_stream(I->dev) : NULL;
}

int agbnp3_stage_timing(int tag, int enable) {
  inst_t *I = get_inst(tag, "agbnp3_stage_timing()");
  if (!I) return AGBNP_ERR;
  agb_dev_set_timing(I->dev, enable);
  return AGBNP_OK;
}

int agbnp3_stage_times(int tag, double *ms, int n) {
  inst_t *I = get_inst(tag, "agbnp3_stage_times()");
  return I ? agb_dev_stage_times(I->dev, ms, n) : AGBNP_ERR;
}

const char *agbnp3_stage_name(int stage) { return agb_dev_stage_name(stage); }

int agbnp3_stats(int tag, long long *out, int n) {
  inst_t *I = get_inst(tag, "agbnp3_stats()");
  return I ? agb_dev_stats(I->dev, out, n) : AGBNP_ERR;
}

long long agbnp3_debug_fetch(int tag, int what, void *out, long long cap) {
  inst_t *I = get_inst(tag, "agbnp3_debug_fetch()");
  return I ? agb_dev_debug_fetch(I->dev, what, out, cap) : -1;
}

/* ------------------------------------------------------------------ */
/* batches                                                             */
/* ------------------------------------------------------------------ */
static batch_t *get_batch(int btag, const char *who) {
  if (!initialized || btag < 0 || btag >= nbatches || !batches[btag]) {
    errprint("%s: invalid batch %d.", who, btag);
    return NULL;
  }
  return batches[btag];
}

int agbnp3_batch_new(int *btag, int ntags, const int *tags) {
  if (!initialized || !btag || ntags <= 0 || !tags) {
    errprint("agbnp3_batch_new(): invalid arguments.");
    return AGBNP_ERR;
  }
  inst_t **L = (inst_t **)malloc(sizeof(inst_t *) * ntags);
  if (!L) return AGBNP_ERR;
  int natoms = 0;
  for (int k = 0; k < ntags; k++) {
    L[k] = get_inst(tags[k], "agbnp3_batch_new()");
    if (!L[k]) {
      free(L);
      return AGBNP_ERR;
    }
    if (L[k]->ws_error) {
      errprint("agbnp3_batch_new(): member %d has an invalid trigonal out-of-plane acceptor.", tags[k]);
      free(L);
      return AGBNP_ERR;
    }
    natoms += L[k]->natoms;
  }
  batch_t *B = (batch_t *)calloc(1, sizeof(batch_t));
  if (!B) {
    free(L);
    return AGBNP_ERR;
  }
  B->n = ntags;
  B->natoms = natoms;
  B->tags = (int *)malloc(sizeof(int) * ntags);
  memcpy(B->tags, tags, sizeof(int) * ntags);
  B->precision = L[0]->precision;
  B->compat = L[0]->compat;
  if (make_dev(L, ntags, B->precision, B->compat, L[0]->device, &B->dev) != 0) {
    free(L);
    free(B->tags);
    free(B);
    return AGBNP_ERR;
  }
  free(L);
  int slot = -1;
  for (int k = 0; k < nbatches; k++)
    if (!batches[k]) {
      slot = k;
      break;
    }
  if (slot < 0) {
    batch_t **p = (batch_t **)realloc(batches, sizeof(batch_t *) * (nbatches + 1));
    if (!p) return AGBNP_ERR;
    batches = p;
    slot = nbatches++;
  }
  B->in_use = 1;
  batches[slot] = B;
  *btag = slot;
  return AGBNP_OK;
}

int agbnp3_batch_delete(int btag) {
  batch_t *B = get_batch(btag, "agbnp3_batch_delete()");
  if (!B) return AGBNP_ERR;
  agb_dev_destroy(B->dev);
  free(B->tags);
  free(B);
  batches[btag] = NULL;
  return AGBNP_OK;
}

int agbnp3_batch_natoms(int btag) {
  batch_t *B = get_batch(btag, "agbnp3_batch_natoms()");
  return B ? B->natoms : AGBNP_ERR;
}

int agbnp3_batch_set_coords(int btag, const double *x, const double *y, const double *z) {
  batch_t *B = get_batch(btag, "agbnp3_batch_set_coords()");
  if (!B) return AGBNP_ERR;
  if (agb_dev_upload_coords(B->dev, x, y, z) != 0) {
    errprint("agbnp3_batch_set_coords(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_batch_ener_resident(int btag) {
  batch_t *B = get_batch(btag, "agbnp3_batch_ener_resident()");
  return B ? eval_dev(B->dev, "agbnp3_batch_ener_resident()") : AGBNP_ERR;
}

int agbnp3_batches_ener_resident(int nb, const int *btags) {
  agb_dev *devs[64];
  if (nb <= 0 || nb > 64 || !btags) {
    errprint("agbnp3_batches_ener_resident(): %d batches (1 to 64).", nb);
    return AGBNP_ERR;
  }
  for (int k = 0; k < nb; k++) {
    batch_t *B = get_batch(btags[k], "agbnp3_batches_ener_resident()");
    if (!B) return AGBNP_ERR;
    for (int q = 0; q < k; q++)
      if (btags[q] == btags[k]) {
        errprint("agbnp3_batches_ener_resident(): batch %d given twice.", btags[k]);
        return AGBNP_ERR;
      }
    devs[k] = B->dev;
  }
  if (agb_dev_evaluate_many(devs, nb) != 0) {
    errprint("agbnp3_batches_ener_resident(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_batch_get_results(int btag, double *energies, double *sp, double *br, double *surf_area,
                             double (*dgbdr)[3], double (*dvwdr)[3], double (*decav)[3], double (*dehb)[3]) {
  batch_t *B = get_batch(btag, "agbnp3_batch_get_results()");
  if (!B) return AGBNP_ERR;
  if (agb_dev_download(B->dev, energies, sp, br, surf_area, (double *)dgbdr, (double *)dvwdr, (double *)decav,
                       (double *)dehb) != 0) {
    errprint("agbnp3_batch_get_results(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_batch_ener_device(int btag, const double *x, const double *y, const double *z, double *energies,
                             double *sp, double *br, double *surf_area, double *dgbdr, double *dvwdr, double *decav,
                             double *dehb, void *stream) {
  batch_t *B = get_batch(btag, "agbnp3_batch_ener_device()");
  if (!B) return AGBNP_ERR;
  return ener_device(B->dev, "agbnp3_batch_ener_device()", x, y, z, energies, sp, br, surf_area, dgbdr, dvwdr,
                     decav, dehb, stream);
}

int agbnp3_batch_set_mode(int btag, int precision, int compat) {
  batch_t *B = get_batch(btag, "agbnp3_batch_set_mode()");
  if (!B) return AGBNP_ERR;
  if (agb_dev_set_mode(B->dev, precision, compat) != 0) {
    errprint("agbnp3_batch_set_mode(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  B->precision = precision;
  B->compat = compat;
  return AGBNP_OK;
}

int agbnp3_batch_pair_order(int btag, int mode) {
  batch_t *B = get_batch(btag, "agbnp3_batch_pair_order()");
  if (!B) return AGBNP_ERR;
  if (agb_dev_set_pair_order(B->dev, mode) != 0) {
    errprint("agbnp3_batch_pair_order(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

int agbnp3_batch_stats(int btag, long long *out, int n) {
  batch_t *B = get_batch(btag, "agbnp3_batch_stats()");
  return B ? agb_dev_stats(B->dev, out, n) : AGBNP_ERR;
}

int agbnp3_batch_set_nblist_skin(int btag, double skin) {
  batch_t *B = get_batch(btag, "agbnp3_batch_set_nblist_skin()");
  if (!B) return AGBNP_ERR;
  if (agb_dev_set_skin(B->dev, skin) != 0) {
    errprint("agbnp3_batch_set_nblist_skin(): %s", agb_dev_last_error());
    return AGBNP_ERR;
  }
  return AGBNP_OK;
}

void *agbnp3_batch_stream(int btag) {
  batch_t *B = get_batch(btag, "agbnp3_batch_stream()");
  return B ? agb_dev_stream(B->dev) : NULL;
}

int agbnp3_batch_stage_timing(int btag, int enable) {
  batch_t *B = get_batch(btag, "agbnp3_batch_stage_timing()");
  if (!B) return AGBNP_ERR;
  agb_dev_set_timing(B->dev, enable);
  return AGBNP_OK;
}

int agbnp3_batch_stage_times(int btag, double *ms, int n) {
  batch_t *B = get_batch(btag, "agbnp3_batch_stage_times()");
  return B ? agb_dev_stage_times(B->dev, ms, n) : AGBNP_ERR;
}

/* ------------------------------------------------------------------ */
/* autotuner with an optional cache file ($AGBNP3_TUNE_CACHE): one line */
/* per key "<instances>:<size bucket> <nch> <jb>"                       */
/* ------------------------------------------------------------------ */
static void tune_key(char *key, size_t n, int ninst, int natoms) {
  int bucket = (int)floor(4.0 * log2((double)natoms > 1 ? (double)natoms : 1.0));
  snprintf(key, n, "%d:%d", ninst, bucket);
}

static int tune_lookup(const char *key, int *p) {
  const char *path = getenv("AGBNP3_TUNE_CACHE");
  if (!path) return 0;
  FILE *f = fopen(path, "r");
  if (!f) return 0;
  char k[64];
  int a, b, found = 0;
  while (fscanf(f, "%63s %d %d", k, &a, &b) == 3)
    if (strcmp(k, key) == 0) {
      p[0] = a;
      p[1] = b;
      found = 1;
    }
  fclose(f);
  return found;
}

static void tune_store(const char *key, const int *p) {
  const char *path = getenv("AGBNP3_TUNE_CACHE");
  if (!path) return;
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d\n", key, p[0], p[1]);
  fclose(f);
}

static int autotune_dev(agb_dev *dev, int ninst, int natoms, int *params, int n, const char *who) {
  char key[64];
  int p[4] = {0, 0, -1, -1}, rc;
  tune_key(key, sizeof(key), ninst, natoms);
  if (tune_lookup(key, p))
    rc = agb_dev_autotune(dev, 0, p, p);
  else {
    rc = agb_dev_autotune(dev, 3, NULL, p);
    if (rc == 0) tune_store(key, p);
  }
  if (rc != 0) {
    errprint("%s: %s", who, agb_dev_last_error());
    return AGBNP_ERR;
  }
  for (int k = 0; k < n && k < 4; k++) params[k] = p[k];
  return AGBNP_OK;
}

int agbnp3_autotune(int tag, int *params, int n) {
  inst_t *I = get_inst(tag, "agbnp3_autotune()");
  if (!I) return AGBNP_ERR;
  return autotune_dev(I->dev, 1, I->natoms, params, n, "agbnp3_autotune()");
}

int agbnp3_batch_autotune(int btag, int *params, int n) {
  batch_t *B = get_batch(btag, "agbnp3_batch_autotune()");
  if (!B) return AGBNP_ERR;
  return autotune_dev(B->dev, B->n, B->natoms, params, n, "agbnp3_batch_autotune()");
}

