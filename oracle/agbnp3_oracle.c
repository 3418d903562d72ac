/*
 * FP64 CPU oracle for one AGBNP3 energy+gradient evaluation.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, smoke() and bench.py's
 * cpu_baseline leg.  The product never links or calls this file.
 *
 * A double-precision restatement of the reference's agbnp3_total_energy()
 * (agbnp3.c:1221-1816).  Each stage cites the reference function it
 * follows.  Index-set decisions that the reference makes in float (near-list
 * membership and ordering) are made here with the same float arithmetic so
 * that the sets are identical; everything else is double.  Overlap-tree
 * enumeration follows the reference's level order exactly, so candidate k
 * here is candidate k of the reference's Gaussian buffers.
 */
#include "agbnp3_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* constants of the model (agbnp3_private.h:97-137, 680-684) */
#define O_PI 3.14159265359
#define O_KFC 2.5
#define O_PFC 2.97354
#define O_VOLA 0.01
#define O_VOLB 0.1
#define O_RINC 0.5
#define O_NBOFF 1.6f
#define O_HBLEN 2.5
#define O_HBRAD 1.4
#define O_HBSWA 0.65
#define O_HBSWB 1.00
#define O_HBSWA0 0.60
#define O_NA 512
#define O_AMAX 20.0
#define O_RW 1.4
#define O_TOKCAL 332.0

typedef double m33[3][3];

/* ------------------------------------------------------------------ */
/* Q4 descreening integral and its spline tables                       */
/* ------------------------------------------------------------------ */

/* volume integral of 1/r^4 over a sphere of radius Rj at distance rij,
   excluding the part inside radius Ri (agbnp3.c:3886-3944) */
static double o_i4(double rij, double Ri, double Rj, double *dr) {
  const double tp = 2.0 * O_PI;
  double rij2 = rij * rij;
  if (rij > Ri + Rj) {
    double up = rij + Rj, um = rij - Rj, prod = up * um;
    double lg = 0.5 * log(up / um);
    *dr = tp * ((Rj / (rij * prod)) * (1.0 - 2.0 * rij2 / prod) + lg / rij2);
    return tp * (Rj / prod - lg / rij);
  }
  double gap = Rj - Ri;
  if (rij2 > gap * gap) { /* partial overlap of the two spheres */
    double up = rij + Rj, um = rij - Rj, prod = up * um;
    double iu = 1.0 / up, iri = 1.0 / Ri;
    double dsq = iu * iu - iri * iri;
    double lg = 0.5 * log(up / Ri);
    *dr = tp * (0.5 * (1.0 - 0.5 * prod / rij2) * dsq + lg / rij2);
    return tp * (-(iu - iri) + (0.25 * prod * dsq - lg) / rij);
  }
  if (Ri > Rj) { /* descreened sphere engulfs the descreener */
    *dr = 0.0;
    return 0.0;
  }
  double up = rij + Rj, dn = Rj - rij, prod = -up * dn;
  if (rij < 0.001 * Rj) { /* series form near the removable singularity */
    double t = rij / Rj;
    *dr = -(2.0 * tp * t / (Rj * Rj)) * (1.0 / (t * t - 1.0) + 2.0 / 3.0);
    return tp * (2.0 / Ri + Rj / prod - (1.0 + (2.0 / 3.0) * t * t) / Rj);
  }
  double lg = 0.5 * log(up / dn);
  *dr = tp * (-(Rj / prod) * (2.0 * rij / prod - 1.0 / rij) + lg / rij2);
  return tp * (2.0 / Ri + Rj / prod - lg / rij);
}

/* i4 with the descreener inflated by twice its Gaussian overlap with the
   descreened atom (agbnp3.c:3946-3975; both exponents use Ri as there) */
static double o_i4ov(double rij, double Ri, double Rj, double *dr) {
  double ai = O_KFC / (Ri * Ri), aj = ai;
  double s = ai + aj;
  double gvol = O_PFC * O_PFC * exp(-ai * aj * rij * rij / s) * pow(O_PI / s, 1.5);
  double volj = 4.0 * O_PI * Rj * Rj * Rj / 3.0;
  double rnew = pow((volj + 2.0 * gvol) / volj, 1.0 / 3.0) * Rj;
  return o_i4(rij, Ri, rnew, dr);
}

/* clamped cubic spline on a uniform grid (agbnp3_utils.c:193-227):
   forward elimination of the tridiagonal second-derivative system, with the
   end conditions of the reference, then back substitution */
static void o_spline(double h, int n, const double *y, double d0, double dn, double *m) {
  double *w = (double *)malloc(sizeof(double) * n);
  m[0] = -0.5;
  w[0] = (3.0 / h) * ((y[1] - y[0]) / h - d0);
  for (int i = 1; i < n - 1; i++) {
    double piv = 0.5 * m[i - 1] + 2.0;
    m[i] = -0.5 / piv;
    double jump = (y[i + 1] - y[i]) / h - (y[i] - y[i - 1]) / h;
    w[i] = (6.0 * jump / (2.0 * h) - 0.5 * w[i - 1]) / piv;
  }
  double tail = (3.0 / h) * (dn - (y[n - 1] - y[n - 2]) / (2.0 * h));
  m[n - 1] = (tail - 0.5 * w[n - 2]) / (0.5 * m[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; k--) m[k] = m[k] * m[k + 1] + w[k];
  free(w);
}

/* one table of Q4(a)*Rj for a = d/Rj on [0, 20], descreened radius ratio b
   (agbnp3_utils.c:380-422) */
static void o_build_table(double b, double *y, double *y2) {
  double h = O_AMAX / (O_NA - 1);
  double a = 0.0, d0 = 0.0, dr;
  for (int i = 0; i < O_NA - 1; i++) {
    y[i] = o_i4ov(a, b, 1.0, &dr);
    if (i == 0) d0 = dr;
    a += h;
  }
  y[O_NA - 1] = 0.0;
  o_spline(h, O_NA, y, d0, 0.0, y2);
}

typedef struct {
  int ntypes;
  double *y, *y2; /* ntypes^2 * O_NA */
  double h, hinv;
  int ref_sign;
} o_tables;

/* cubic-spline evaluation (agbnp3_utils.c:229-252, 331-377).  The
   derivative of the spline has +(3B^2-1)h/6 y2[k+1]; the reference
   subtracts that term, which `ref_sign` reproduces. */
static void o_interp(const o_tables *t, int slot, double x, double *f, double *fp) {
  double xh = x * t->hinv;
  int k = (int)xh;
  if (k > O_NA - 2) {
    *f = 0.0;
    *fp = 0.0;
    return;
  }
  const double *y = t->y + (size_t)slot * O_NA, *y2 = t->y2 + (size_t)slot * O_NA;
  double dp1 = t->h / 6.0, dp2 = t->h * dp1;
  double A = (k + 1.0) - xh, B = xh - k;
  *f = A * y[k] + B * y[k + 1] + ((A * A * A - A) * y2[k] + (B * B * B - B) * y2[k + 1]) * dp2;
  double s2 = t->ref_sign ? 1.0 : -1.0;
  *fp = (y[k + 1] - y[k]) * t->hinv - ((3.0 * A * A - 1.0) * y2[k] + s2 * (3.0 * B * B - 1.0) * y2[k + 1]) * dp1;
}

/* Q4 of the atom with radius type `td` descreened by a heavy atom of type
   `ts` and radius Rs at distance d; *dq = dQ4/dd (agbnp3_utils.c:297-326) */
static double o_q4(const o_tables *t, int td, int ts, double d, double Rs, double *dq) {
  double f, fp;
  o_interp(t, td * t->ntypes + ts, d / Rs, &f, &fp);
  *dq = fp / (Rs * Rs);
  return f / Rs;
}

/* ------------------------------------------------------------------ */
/* switching functions (agbnp3.c:1104-1188)                            */
/* ------------------------------------------------------------------ */
static double o_swf_area(double x, double *fp) {
  if (x < 0.0) {
    *fp = 0.0;
    return 0.0;
  }
  double t = x / (64.0 + x * x);
  double f = x * t;
  *fp = 2.0 * t * (1.0 - f);
  return f;
}

static double o_poly_switch(double x, double xa, double xb, double *fp, double *fpp) {
  if (x > xb) {
    if (fp) *fp = 0.0;
    if (fpp) *fpp = 0.0;
    return 1.0;
  }
  if (x < xa) {
    if (fp) *fp = 0.0;
    if (fpp) *fpp = 0.0;
    return 0.0;
  }
  double d = 1.0 / (xb - xa), u = (x - xa) * d, u2 = u * u;
  if (fp) *fp = d * 30.0 * u2 * (1.0 - 2.0 * u + u2);
  if (fpp) *fpp = d * d * 60.0 * u * (1.0 - 3.0 * u + 2.0 * u2);
  return u * u2 * (10.0 - 15.0 * u + 6.0 * u2);
}

static double o_swf_invbr(double beta, double *fp) {
  if (beta < 0.0) {
    *fp = 0.0;
    return 0.02;
  }
  double t = sqrt(0.02 * 0.02 + beta * beta);
  *fp = beta / t;
  return t;
}

/* ------------------------------------------------------------------ */
/* Gaussian overlap of two Gaussians (agbnp3_cpu_simd_kernels.c:2418-2477) */
/* ------------------------------------------------------------------ */
typedef struct {
  double a, p, c[3];
} o_gauss;

typedef struct {
  o_gauss g;   /* product Gaussian */
  double gvol; /* raw overlap volume */
  double gvolp, fp, fpp;
} o_ovl;

static void o_ogauss(const o_gauss *g1, const o_gauss *g2, o_ovl *o) {
  double dx = g2->c[0] - g1->c[0], dy = g2->c[1] - g1->c[1], dz = g2->c[2] - g1->c[2];
  double d2 = dx * dx + dy * dy + dz * dz;
  double s = g1->a + g2->a, inv = 1.0 / s;
  double p12 = g1->p * g2->p * exp(-g1->a * g2->a * d2 * inv);
  o->gvol = p12 * pow(O_PI * inv, 1.5);
  for (int k = 0; k < 3; k++) o->g.c[k] = inv * (g1->a * g1->c[k] + g2->a * g2->c[k]);
  o->g.a = s;
  o->g.p = p12;
  double sp, spp;
  double sw = o_poly_switch(o->gvol, O_VOLA, O_VOLB, &sp, &spp);
  o->gvolp = sw * o->gvol;
  o->fp = sw + o->gvol * sp;
  o->fpp = 2.0 * sp + o->gvol * spp;
}

/* ------------------------------------------------------------------ */
/* small 3-vector helpers for the water-site geometry                 */
/* ------------------------------------------------------------------ */
static void v_sub(const double a[3], const double b[3], double c[3]) {
  for (int k = 0; k < 3; k++) c[k] = a[k] - b[k];
}
static double v_norm(const double a[3]) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static void v_cross(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
/* d(unit vector)/d(vector): (I - u u^T)/|r| */
static void m_unit_der(const double u[3], double inv, m33 D) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[i][j] = inv * ((i == j ? 1.0 : 0.0) - u[i] * u[j]);
}
static void m_mul(m33 A, m33 B, m33 C) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
      for (int k = 0; k < 3; k++) s += A[i][k] * B[k][j];
      C[i][j] = s;
    }
}
static void m_zero(m33 A) { memset(A, 0, sizeof(m33)); }
static void m_eye(m33 A) {
  m_zero(A);
  A[0][0] = A[1][1] = A[2][2] = 1.0;
}
/* d(a x b)/da and d(a x b)/db, row i = component i */
static void m_cross_der(const double a[3], const double b[3], m33 Da, m33 Db) {
  m_zero(Da);
  m_zero(Db);
  Da[0][1] = b[2]; Da[0][2] = -b[1];
  Da[1][0] = -b[2]; Da[1][2] = b[0];
  Da[2][0] = b[1]; Da[2][1] = -b[0];
  Db[0][1] = -a[2]; Db[0][2] = a[1];
  Db[1][0] = a[2]; Db[1][2] = -a[0];
  Db[2][0] = -a[1]; Db[2][1] = a[0];
}

typedef struct {
  double pos[3];
  int nparents;
  int parent[4];
  m33 dpos[4]; /* dpos[p][i][j] = d pos_i / d x_{parent p, j} */
  double khb;
  int type;
} o_ws;

#define WS_POLARH 1
#define WS_TRIGONAL 10
#define WS_TRIGONAL_S 30
#define WS_TETRAHEDRAL 20
#define WS_TRIGONAL1 11
#define WS_TRIGONAL2 12
#define WS_TRIGONAL_OOP 13
#define WS_TETRAHEDRAL1 21
#define WS_TETRAHEDRAL2 22
#define WS_TETRAHEDRAL3 23

/* site along the donor-hydrogen bond (agbnp3.c:2107-2150) */
static void g_polarh(const double *xd, const double *xh, o_ws *w) {
  double b[3];
  v_sub(xh, xd, b);
  double L = v_norm(b), s = O_HBLEN / L, u[3];
  for (int k = 0; k < 3; k++) {
    w->pos[k] = xd[k] + s * b[k];
    u[k] = b[k] / L;
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double proj = (i == j ? 1.0 : 0.0) - u[i] * u[j];
      w->dpos[0][i][j] = s * proj;                          /* hydrogen */
      w->dpos[1][i][j] = (i == j ? 1.0 : 0.0) - s * proj;  /* heavy atom */
    }
}

/* two in-plane sites of a trigonal acceptor A-R(R1)(R2), each opposite one
   of the R-R1 / R-R2 bonds (agbnp3.c:2310-2380) */
static void g_trigonal1(const double *A, const double *R, const double *R1, const double *R2, o_ws *w1,
                        o_ws *w2) {
  const double *Rk[2] = {R1, R2};
  o_ws *ws[2] = {w1, w2};
  for (int s = 0; s < 2; s++) {
    double b[3], u[3];
    v_sub(Rk[s], R, b);
    double L = v_norm(b);
    for (int k = 0; k < 3; k++) {
      u[k] = b[k] / L;
      ws[s]->pos[k] = A[k] - O_HBLEN * u[k];
    }
    for (int p = 0; p < 4; p++) m_zero(ws[s]->dpos[p]);
    m_eye(ws[s]->dpos[0]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double g = (O_HBLEN / L) * ((i == j ? 1.0 : 0.0) - u[i] * u[j]);
        ws[s]->dpos[1][i][j] = g;
        ws[s]->dpos[2 + s][i][j] = -g;
      }
  }
}

/* two out-of-plane sites at 60 degrees from the A-R axis
   (agbnp3.c:2600-2697) */
static void g_trigonal_s(const double *A, const double *R, const double *R1, o_ws *w1, o_ws *w2) {
  const double cth = 0.5, sth = 0.866025;
  double e0[3], e1[3], n[3], uin[3], uout[3];
  v_sub(A, R, e0);
  v_sub(R1, R, e1);
  double l0 = v_norm(e0);
  for (int k = 0; k < 3; k++) uin[k] = e0[k] / l0;
  v_cross(e1, e0, n);
  double ln = v_norm(n);
  for (int k = 0; k < 3; k++) uout[k] = n[k] / ln;
  for (int k = 0; k < 3; k++) {
    w1->pos[k] = A[k] + O_HBLEN * (cth * uin[k] + sth * uout[k]);
    w2->pos[k] = A[k] + O_HBLEN * (cth * uin[k] - sth * uout[k]);
  }
  m33 Din, Dout, Dn_e1, Dn_e0, G0, G1;
  m_unit_der(uin, 1.0 / l0, Din);
  m_unit_der(uout, 1.0 / ln, Dout);
  m_cross_der(e1, e0, Dn_e1, Dn_e0);
  m_mul(Dout, Dn_e0, G0); /* d uout / d e0 */
  m_mul(Dout, Dn_e1, G1); /* d uout / d e1 */
  o_ws *ws[2] = {w1, w2};
  for (int s = 0; s < 2; s++) {
    double sg = s == 0 ? 1.0 : -1.0;
    for (int p = 0; p < 4; p++) m_zero(ws[s]->dpos[p]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double gin = O_HBLEN * cth * Din[i][j];
        double g0 = sg * O_HBLEN * sth * G0[i][j];
        double g1 = sg * O_HBLEN * sth * G1[i][j];
        ws[s]->dpos[0][i][j] = gin + g0 + (i == j ? 1.0 : 0.0); /* A  (e0 = A - R)  */
        ws[s]->dpos[1][i][j] = -gin - g0 - g1;                 /* R                */
        ws[s]->dpos[2][i][j] = g1;                             /* R1 (e1 = R1 - R) */
      }
  }
}

/* two sites along the normal of the R1 R2 R3 plane through A, at 2.7 A
   (agbnp3.c:2815-2942) */
static void g_trigonal_oop(const double *A, const double *R1, const double *R2, const double *R3, o_ws *w1,
                           o_ws *w2) {
  double dist = (double)(float)(O_HBLEN + 0.2);
  double v1[3], v2[3], n[3], nu[3];
  v_sub(R2, R1, v1);
  v_sub(R3, R1, v2);
  v_cross(v2, v1, n);
  double ln = v_norm(n);
  for (int k = 0; k < 3; k++) nu[k] = n[k] / ln;
  for (int k = 0; k < 3; k++) {
    w1->pos[k] = A[k] + dist * nu[k];
    w2->pos[k] = A[k] - dist * nu[k];
  }
  m33 P, Dv2, Dv1, G1, G2;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) P[i][j] = (i == j ? 1.0 : 0.0) - nu[i] * nu[j];
  m_cross_der(v2, v1, Dv2, Dv1);
  m_mul(P, Dv1, G1);
  m_mul(P, Dv2, G2);
  double sc = dist / ln;
  o_ws *ws[2] = {w1, w2};
  for (int s = 0; s < 2; s++) {
    double sg = s == 0 ? sc : -sc;
    m_eye(ws[s]->dpos[0]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        ws[s]->dpos[2][i][j] = sg * G1[i][j];
        ws[s]->dpos[3][i][j] = sg * G2[i][j];
        ws[s]->dpos[1][i][j] = -(ws[s]->dpos[2][i][j] + ws[s]->dpos[3][i][j]);
      }
  }
}

/* site opposite the bisector of two or three bonds of A: trigonal2
   (agbnp3.c:3027-3090) for n=2, tetrahedral3 (agbnp3.c:3477-3556) for n=3 */
static void g_bisector(const double *A, const double **Rk, int n, o_ws *w) {
  double u[3][3], inv[3], s[3] = {0, 0, 0};
  for (int q = 0; q < n; q++) {
    double b[3];
    v_sub(Rk[q], A, b);
    double L = v_norm(b);
    inv[q] = 1.0 / L;
    for (int k = 0; k < 3; k++) {
      u[q][k] = b[k] / L;
      s[k] += u[q][k];
    }
  }
  double ls = v_norm(s), us[3];
  for (int k = 0; k < 3; k++) {
    us[k] = s[k] / ls;
    w->pos[k] = A[k] - O_HBLEN * us[k];
  }
  m33 Ds;
  m_unit_der(us, 1.0 / ls, Ds);
  for (int p = 0; p < 4; p++) m_zero(w->dpos[p]);
  m_eye(w->dpos[0]);
  for (int q = 0; q < n; q++) {
    m33 Dq, G;
    m_unit_der(u[q], inv[q], Dq);
    m_mul(Ds, Dq, G);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        w->dpos[q + 1][i][j] = -O_HBLEN * G[i][j];
        w->dpos[0][i][j] += O_HBLEN * G[i][j];
      }
  }
}

/* two lone-pair sites of an sp3 acceptor with two bonds
   (agbnp3.c:3266-3390) */
static void g_tetrahedral2(const double *A, const double *R1, const double *R2, o_ws *w1, o_ws *w2) {
  const double cth = -0.577350269, sth = 0.816496581;
  double r1[3], r2[3], u1[3], u2[3], s[3], n[3], uin[3], uout[3];
  v_sub(R1, A, r1);
  v_sub(R2, A, r2);
  double l1 = v_norm(r1), l2 = v_norm(r2);
  for (int k = 0; k < 3; k++) {
    u1[k] = r1[k] / l1;
    u2[k] = r2[k] / l2;
    s[k] = u1[k] + u2[k];
  }
  double ls = v_norm(s);
  for (int k = 0; k < 3; k++) uin[k] = s[k] / ls;
  v_cross(r2, r1, n);
  double ln = v_norm(n);
  for (int k = 0; k < 3; k++) uout[k] = n[k] / ln;
  for (int k = 0; k < 3; k++) {
    w1->pos[k] = A[k] + O_HBLEN * (cth * uin[k] + sth * uout[k]);
    w2->pos[k] = A[k] + O_HBLEN * (cth * uin[k] - sth * uout[k]);
  }
  m33 Ds, D1, D2, Gin1, Gin2, Dout, Dn_r2, Dn_r1, Go1, Go2;
  m_unit_der(uin, 1.0 / ls, Ds);
  m_unit_der(u1, 1.0 / l1, D1);
  m_unit_der(u2, 1.0 / l2, D2);
  m_mul(Ds, D1, Gin1);
  m_mul(Ds, D2, Gin2);
  m_unit_der(uout, 1.0 / ln, Dout);
  m_cross_der(r2, r1, Dn_r2, Dn_r1);
  m_mul(Dout, Dn_r1, Go1);
  m_mul(Dout, Dn_r2, Go2);
  o_ws *ws[2] = {w1, w2};
  for (int s2 = 0; s2 < 2; s2++) {
    double sg = s2 == 0 ? 1.0 : -1.0;
    for (int p = 0; p < 4; p++) m_zero(ws[s2]->dpos[p]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double a1 = O_HBLEN * cth * Gin1[i][j] + sg * O_HBLEN * sth * Go1[i][j];
        double a2 = O_HBLEN * cth * Gin2[i][j] + sg * O_HBLEN * sth * Go2[i][j];
        ws[s2]->dpos[1][i][j] = a1;
        ws[s2]->dpos[2][i][j] = a2;
        ws[s2]->dpos[0][i][j] = -(a1 + a2) + (i == j ? 1.0 : 0.0);
      }
  }
}

/* one site of an sp3 acceptor bonded to a four-connected centre R,
   anti-parallel to the R-R1 bond (agbnp3.c:3704-3761) */
static void g_tetrahedral1(const double *A, const double *R, const double *R1, o_ws *w) {
  double b[3], u[3];
  v_sub(R1, R, b);
  double L = v_norm(b);
  for (int k = 0; k < 3; k++) {
    u[k] = b[k] / L;
    w->pos[k] = A[k] - O_HBLEN * u[k];
  }
  for (int p = 0; p < 4; p++) m_zero(w->dpos[p]);
  m_eye(w->dpos[0]);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double g = (O_HBLEN / L) * ((i == j ? 1.0 : 0.0) - u[i] * u[j]);
      w->dpos[1][i][j] = g;
      w->dpos[2][i][j] = -g;
    }
}

/* water sites of one atom, in the reference's order; returns the number of
   sites, or -1 when the reference aborts the evaluation
   (agbnp3.c:1920-2012 and the create_ws_atoms_* functions) */
static int o_make_ws(const orc_in *in, int iat, o_ws *out) {
  const int *off = in->conn_offset, *nb = in->conn_list;
  int nne = off[iat + 1] - off[iat];
  const int *lst = nb + off[iat];
#define XYZ(i, v) double v[3] = {in->x[i], in->y[i], in->z[i]}
  XYZ(iat, A);
  double khb = in->hbcorr[iat];
  int t = in->hbtype[iat];
  int n = 0;
  if (t == WS_POLARH) {
    if (nne <= 0) return 0;
    int jat = -1;
    for (int q = 0; q < nne; q++)
      if (lst[q] < in->nheavy) {
        jat = lst[q];
        break;
      }
    if (jat < 0) return 0;
    XYZ(jat, D);
    g_polarh(D, A, &out[0]);
    out[0].nparents = 2;
    out[0].parent[0] = iat;
    out[0].parent[1] = jat;
    out[0].type = WS_POLARH;
    n = 1;
  } else if (t == WS_TRIGONAL || t == WS_TRIGONAL_S) {
    if (t == WS_TRIGONAL && nne == 2) {
      XYZ(lst[0], R1);
      XYZ(lst[1], R2);
      const double *Rk[2] = {R1, R2};
      g_bisector(A, Rk, 2, &out[0]);
      out[0].nparents = 3;
      out[0].parent[0] = iat;
      out[0].parent[1] = lst[0];
      out[0].parent[2] = lst[1];
      out[0].type = WS_TRIGONAL2;
      n = 1;
    } else if (nne == 1) {
      int ir = lst[0];
      int nr = off[ir + 1] - off[ir];
      const int *lr = nb + off[ir];
      if (nr != 3) return 0;
      int ir1 = -1, ir2 = -1;
      for (int q = 0; q < nr; q++)
        if (lr[q] != iat) {
          ir1 = lr[q];
          break;
        }
      for (int q = 0; q < nr; q++)
        if (lr[q] != iat && lr[q] != ir1) {
          ir2 = lr[q];
          break;
        }
      if (ir1 < 0 || ir2 < 0) return 0;
      XYZ(ir, R);
      XYZ(ir1, R1);
      XYZ(ir2, R2);
      int ty = t == WS_TRIGONAL ? WS_TRIGONAL1 : WS_TRIGONAL_S;
      g_trigonal1(A, R, R1, R2, &out[0], &out[1]);
      n = 2;
      if (t == WS_TRIGONAL_S) {
        g_trigonal_s(A, R, R1, &out[2], &out[3]);
        n = 4;
      }
      for (int s = 0; s < n; s++) {
        out[s].nparents = 4;
        out[s].parent[0] = iat;
        out[s].parent[1] = ir;
        out[s].parent[2] = ir1;
        out[s].parent[3] = ir2;
        out[s].type = ty;
      }
    }
  } else if (t == WS_TRIGONAL_OOP) {
    if (nne != 3) return -1;
    XYZ(lst[0], R1);
    XYZ(lst[1], R2);
    XYZ(lst[2], R3);
    g_trigonal_oop(A, R1, R2, R3, &out[0], &out[1]);
    for (int s = 0; s < 2; s++) {
      out[s].nparents = 4;
      out[s].parent[0] = iat;
      for (int q = 0; q < 3; q++) out[s].parent[q + 1] = lst[q];
      out[s].type = WS_TRIGONAL_OOP;
    }
    n = 2;
  } else if (t == WS_TETRAHEDRAL) {
    if (nne == 2) {
      XYZ(lst[0], R1);
      XYZ(lst[1], R2);
      g_tetrahedral2(A, R1, R2, &out[0], &out[1]);
      for (int s = 0; s < 2; s++) {
        out[s].nparents = 3;
        out[s].parent[0] = iat;
        out[s].parent[1] = lst[0];
        out[s].parent[2] = lst[1];
        out[s].type = WS_TETRAHEDRAL2;
      }
      n = 2;
    } else if (nne == 3) {
      XYZ(lst[0], R1);
      XYZ(lst[1], R2);
      XYZ(lst[2], R3);
      const double *Rk[3] = {R1, R2, R3};
      g_bisector(A, Rk, 3, &out[0]);
      out[0].nparents = 4;
      out[0].parent[0] = iat;
      for (int q = 0; q < 3; q++) out[0].parent[q + 1] = lst[q];
      out[0].type = WS_TETRAHEDRAL3;
      n = 1;
    } else if (nne == 1) {
      int ir = lst[0];
      int nr = off[ir + 1] - off[ir];
      const int *lr = nb + off[ir];
      if (nr != 4) return 0;
      int irr[4], m = 0;
      for (int q = 0; q < 4; q++)
        if (lr[q] != iat) irr[m++] = lr[q];
      if (m != 3) return 0;
      XYZ(ir, R);
      for (int s = 0; s < 3; s++) {
        XYZ(irr[s], R1);
        g_tetrahedral1(A, R, R1, &out[s]);
        out[s].nparents = 3;
        out[s].parent[0] = iat;
        out[s].parent[1] = ir;
        out[s].parent[2] = irr[s];
        out[s].type = WS_TETRAHEDRAL1;
      }
      n = 3;
    }
  }
  for (int s = 0; s < n; s++) out[s].khb = khb;
  return n;
#undef XYZ
}

/* ------------------------------------------------------------------ */
/* the evaluation                                                     */
/* ------------------------------------------------------------------ */
typedef struct {
  int order;
  int par[ORC_MAX_ORDER];
  int group; /* index of the generating overlap one level down, or root atom */
  o_ovl o;
} o_node;

typedef struct {
  o_node *v;
  int n, cap;
} o_level;

static void lvl_push(o_level *L, const o_node *nd) {
  if (L->n == L->cap) {
    L->cap = L->cap ? 2 * L->cap : 1024;
    L->v = (o_node *)realloc(L->v, sizeof(o_node) * L->cap);
  }
  L->v[L->n++] = *nd;
}

typedef struct {
  float d2;
  int j;
} o_nb;

static int nb_cmp(const void *a, const void *b) {
  const o_nb *p = (const o_nb *)a, *q = (const o_nb *)b;
  if (p->d2 < q->d2) return -1;
  if (p->d2 > q->d2) return 1;
  return (p->j > q->j) - (p->j < q->j);
}

int agbnp3_oracle_eval(const orc_in *in, orc_out *out) {
  const int N = in->natoms, NH = in->nheavy;
  const double *x = in->x, *y = in->y, *z = in->z, *r = in->r;
  const double df = -0.5 * (1.0 / in->eps_in - 1.0 / in->eps_out);
  const double fourpi1 = 1.0 / (4.0 * O_PI);

#define ALLOC(n) ((double *)calloc((size_t)(n) + 1, sizeof(double)))
  double *vols = ALLOC(N), *volumep = ALLOC(N), *surf = ALLOC(N), *br1 = ALLOC(N);
  double *sp = ALLOC(N), *spe = ALLOC(N), *psvol = ALLOC(N), *surf_f = ALLOC(N), *gammap = ALLOC(N);
  double *bfil = ALLOC(N), *bder = ALLOC(N), *br = ALLOC(N), *brw = ALLOC(N);
  double *dera = ALLOC(N), *q2ab = ALLOC(N), *abrw = ALLOC(N);
  double *deru = ALLOC(N), *derv = ALLOC(N), *derh = ALLOC(N), *derus = ALLOC(N), *dervs = ALLOC(N);
  double *ga = ALLOC(N);
  double(*gb)[3] = (double(*)[3])ALLOC(3 * N);
  double(*gv)[3] = (double(*)[3])ALLOC(3 * N);
  double(*gc)[3] = (double(*)[3])ALLOC(3 * N);
  double(*gh)[3] = (double(*)[3])ALLOC(3 * N);
  int *rtype = (int *)calloc(N + 1, sizeof(int));

  /* reset (agbnp3_utils.c:477-519) and Gaussian parameters
     (agbnp3.c:1063-1102) */
  for (int i = 0; i < N; i++) {
    vols[i] = 4.0 * O_PI / 3.0 * r[i] * r[i] * r[i];
    br1[i] = 1.0 / (r[i] - O_RINC);
    ga[i] = O_KFC / (r[i] * r[i]);
  }
  for (int i = 0; i < NH; i++) {
    volumep[i] = vols[i];
    surf[i] = 4.0 * O_PI * r[i] * r[i];
  }

  /* radius types in order of first appearance (agbnp3_utils.c:808-838) and
     one Q4 table per ordered type pair (agbnp3_utils.c:840-883) */
  float radii[64];
  int nt = 0;
  for (int i = 0; i < N; i++) {
    float ri = (float)r[i];
    int f = -1;
    for (int k = 0; k < nt; k++)
      if (fabsf(ri - radii[k]) < FLT_MIN) {
        f = k;
        break;
      }
    if (f < 0) {
      if (nt == 64) return -3;
      radii[nt] = ri;
      f = nt++;
    }
    rtype[i] = f;
  }
  o_tables T;
  T.ntypes = nt;
  T.ref_sign = in->compat;
  T.h = O_AMAX / (O_NA - 1);
  T.hinv = 1.0 / T.h;
  T.y = (double *)malloc(sizeof(double) * nt * nt * O_NA);
  T.y2 = (double *)malloc(sizeof(double) * nt * nt * O_NA);
  for (int a = 0; a < nt; a++)
    for (int b = 0; b < nt; b++) {
      double ratio = ((double)radii[a] - O_RINC) / (double)radii[b];
      o_build_table(ratio, T.y + (size_t)(a * nt + b) * O_NA, T.y2 + (size_t)(a * nt + b) * O_NA);
    }

  /* near list of heavy atoms: float membership test and float d^2 ordering
     exactly as agbnp3.c:4041-4066 */
  int *nl_off = (int *)calloc(NH + 1, sizeof(int));
  int nl_cap = 64 * NH + 16, nl_n = 0;
  int *nl = (int *)malloc(sizeof(int) * nl_cap);
  o_nb *buf = (o_nb *)malloc(sizeof(o_nb) * (NH + 1));
  for (int i = 0; i < NH; i++) {
    int m = 0;
    float xi = (float)x[i], yi = (float)y[i], zi = (float)z[i], ri = (float)r[i];
    for (int j = i + 1; j < NH; j++) {
      float dx = (float)x[j] - xi, dy = (float)y[j] - yi, dz = (float)z[j] - zi;
      float dxx = dx * dx, dyy = dy * dy, dzz = dz * dz;
      float d2 = (dxx + dyy) + dzz;
      float u = (ri + (float)r[j]) * O_NBOFF;
      if (d2 < u * u) {
        buf[m].d2 = d2;
        buf[m].j = j;
        m++;
      }
    }
    qsort(buf, m, sizeof(o_nb), nb_cmp);
    if (nl_n + m > nl_cap) {
      nl_cap = 2 * (nl_n + m);
      nl = (int *)realloc(nl, sizeof(int) * nl_cap);
    }
    for (int k = 0; k < m; k++) nl[nl_n++] = buf[k].j;
    nl_off[i + 1] = nl_n;
  }
  free(buf);

  /* overlap tree, levels 2..5 (agbnp3_cpu_simd_kernels.c:1064-1598) */
  o_level lev[ORC_MAX_ORDER + 1];
  memset(lev, 0, sizeof(lev));
  double vcoef[ORC_MAX_ORDER + 1];
  for (int m = 1; m <= ORC_MAX_ORDER; m++) vcoef[m] = ((m % 2) ? 1.0 : -1.0) / m;
  int ncand = 0;
  o_gauss *atg = (o_gauss *)malloc(sizeof(o_gauss) * (NH + 1));
  for (int i = 0; i < NH; i++) {
    atg[i].a = ga[i];
    atg[i].p = O_PFC;
    atg[i].c[0] = x[i];
    atg[i].c[1] = y[i];
    atg[i].c[2] = z[i];
  }
#define RECORD_CAND(ord, pars, ovp)                                                      \
  do {                                                                                 \
    if (out->cand_order && ncand < out->cand_cap) {                                     \
      out->cand_order[ncand] = (ord);                                                   \
      for (int q_ = 0; q_ < ORC_MAX_ORDER; q_++)                                        \
        out->cand_parents[ORC_MAX_ORDER * ncand + q_] = q_ < (ord) ? (pars)[q_] : -1;    \
      out->cand_gvol[ncand] = (ovp)->gvol;                                              \
      out->cand_gvolp[ncand] = (ovp)->gvolp;                                            \
    }                                                                                  \
    ncand++;                                                                           \
  } while (0)
  for (int i = 0; i < NH; i++) {
    for (int k = nl_off[i]; k < nl_off[i + 1]; k++) {
      int j = nl[k];
      o_node nd;
      nd.order = 2;
      nd.par[0] = i;
      nd.par[1] = j;
      nd.group = i;
      o_ogauss(&atg[i], &atg[j], &nd.o);
      RECORD_CAND(2, nd.par, &nd.o);
      if (nd.o.gvolp > FLT_MIN) lvl_push(&lev[2], &nd);
    }
  }
  for (int m = 3; m <= ORC_MAX_ORDER && lev[m - 1].n > 0; m++) {
    o_level *P = &lev[m - 1];
    for (int a = 0; a < P->n; a++) {
      for (int b = a + 1; b < P->n && P->v[b].group == P->v[a].group; b++) {
        int jat = P->v[b].par[m - 2];
        o_node nd;
        nd.order = m;
        memcpy(nd.par, P->v[a].par, sizeof(int) * (m - 1));
        nd.par[m - 1] = jat;
        nd.group = a;
        o_ogauss(&P->v[a].o.g, &atg[jat], &nd.o);
        RECORD_CAND(m, nd.par, &nd.o);
        if (nd.o.gvolp > FLT_MIN) lvl_push(&lev[m], &nd);
      }
    }
  }
  out->cand_total = ncand;
  for (int m = 0; m <= ORC_MAX_ORDER; m++) out->n_kept[m] = lev[m].n;

  /* self volumes and surface areas from every kept overlap */
  for (int m = 2; m <= ORC_MAX_ORDER; m++) {
    double sgn = (m % 2) ? 1.0 : -1.0; /* order * volpcoeff */
    for (int q = 0; q < lev[m].n; q++) {
      o_node *nd = &lev[m].v[q];
      double h3 = sgn * nd->o.fp * 3.0 / nd->o.g.a, h4 = 0.5 * sgn * nd->o.fp;
      for (int ii = 0; ii < m; ii++) {
        int k = nd->par[ii];
        volumep[k] += vcoef[m] * nd->o.gvolp;
        double u1 = ga[k] * nd->o.gvol, u2 = -2.0 * u1;
        double v0 = u2 * (x[k] - nd->o.g.c[0]), v1 = u2 * (y[k] - nd->o.g.c[1]), v2 = u2 * (z[k] - nd->o.g.c[2]);
        double d2 = v0 * v0 + v1 * v1 + v2 * v2;
        surf[k] += (h3 * u1 + h4 * d2 / u1) / r[k];
      }
    }
  }

  /* scaling factors, cavity energy, molecular volume
     (agbnp3_utils.c:524-613, agbnp3.c:1390-1411) */
  out->ecav = out->ecorr_cav = out->mol_volume = 0.0;
  for (int i = 0; i < NH; i++) {
    double fp, f = o_swf_area(surf[i], &fp);
    surf_f[i] = surf[i] * f;
    gammap[i] = (in->igamma[i] + in->sgamma[i]) * (f + surf[i] * fp);
    spe[i] = volumep[i] / vols[i];
    double rv = r[i] - O_RINC, q = rv / r[i];
    double pr = r[i] * (1.0 - q * q * q) / 3.0;
    psvol[i] = (fp * surf[i] + f) * pr;
    volumep[i] = volumep[i] - surf_f[i] * pr;
    sp[i] = volumep[i] / vols[i];
    out->ecav += in->igamma[i] * surf_f[i];
    out->ecorr_cav += in->sgamma[i] * surf_f[i];
    out->mol_volume += volumep[i];
  }

  /* inverse Born radii (agbnp3_cpu_simd_kernels.c:500-678) */
  for (int i = 0; i < NH; i++)
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      double d = sqrt((x[j] - x[i]) * (x[j] - x[i]) + (y[j] - y[i]) * (y[j] - y[i]) + (z[j] - z[i]) * (z[j] - z[i]));
      double dq;
      double q = o_q4(&T, rtype[j], rtype[i], d, r[i], &dq); /* j descreened by i */
      br1[j] -= fourpi1 * q * sp[i];
    }

  /* Born radii and vdW energy (agbnp3_utils.c:615-670, agbnp3.c:1466-1487) */
  out->evdw = out->ecorr_vdw = 0.0;
  for (int i = 0; i < N; i++) {
    double fp;
    bfil[i] = o_swf_invbr(br1[i], &fp);
    bder[i] = fp;
    br[i] = 1.0 / bfil[i];
    double t = br[i] + O_RW;
    brw[i] = 3.0 * br[i] * br[i] / (t * t * t * t);
    double a3 = 1.0 / (t * t * t);
    out->evdw += in->ialpha[i] * a3;
    out->ecorr_vdw += in->salpha[i] * a3;
  }

  /* GB energy at constant Born radii (agbnp3_cpu_simd_kernels.c:66-151,
     329-460); coincident atoms contribute nothing */
  double eself = 0.0, epair = 0.0;
  for (int i = 0; i < N; i++) {
    eself += df * in->charge[i] * in->charge[i] / br[i];
    for (int j = i + 1; j < N; j++) {
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      double d2 = dx * dx + dy * dy + dz * dz;
      if (!(d2 > 0.0)) continue;
      double qq = in->charge[i] * in->charge[j];
      double bb = br[i] * br[j];
      double et = exp(-0.25 * d2 / bb);
      double f = 1.0 / sqrt(d2 + bb * et);
      double f3 = f * f * f;
      epair += 2.0 * df * qq * f;
      double mw = -2.0 * df * qq * (1.0 - 0.25 * et) * f3;
      gb[j][0] += mw * dx; gb[j][1] += mw * dy; gb[j][2] += mw * dz;
      gb[i][0] -= mw * dx; gb[i][1] -= mw * dy; gb[i][2] -= mw * dz;
      double at = qq * (bb + 0.25 * d2) * et * f3;
      dera[i] += at;
      dera[j] += at;
    }
  }
  out->egb = O_TOKCAL * eself + O_TOKCAL * epair;
  for (int i = 0; i < N; i++) {
    q2ab[i] = (in->charge[i] * in->charge[i] + dera[i] * br[i]) * bder[i];
    abrw[i] = (in->ialpha[i] + in->salpha[i]) * brw[i] * bder[i];
  }

  /* GB and vdW gradients through the Born radii at constant self volumes
     (agbnp3_cpu_simd_kernels.c:681-805) and U_i, V_i
     (agbnp3_cpu_simd_kernels.c:809-904) */
  for (int i = 0; i < NH; i++)
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      double d = sqrt(dx * dx + dy * dy + dz * dz);
      double dq_ji;
      double q_ji = o_q4(&T, rtype[j], rtype[i], d, r[i], &dq_ji); /* j by i */
      deru[i] += q2ab[j] * q_ji;
      derv[i] += abrw[j] * q_ji;
      /* the pair force of j-by-i acts along i-j; the i-by-j half is added
         when the loop visits (j, i) with j heavy */
      double ht = fourpi1 * df * q2ab[j] * dq_ji * sp[i] / d;
      double ut = fourpi1 * abrw[j] * dq_ji * sp[i] / d;
      gb[i][0] += ht * dx; gb[i][1] += ht * dy; gb[i][2] += ht * dz;
      gb[j][0] -= ht * dx; gb[j][1] -= ht * dy; gb[j][2] -= ht * dz;
      gv[i][0] += ut * dx; gv[i][1] += ut * dy; gv[i][2] += ut * dz;
      gv[j][0] -= ut * dx; gv[j][1] -= ut * dy; gv[j][2] -= ut * dz;
    }

  /* water sites (agbnp3.c:1837-2012) and their free volumes, HB energy and
     derivatives (agbnp3_cpu_simd_kernels.c:2637-2954) */
  int ws_cap = 16, nws = 0;
  o_ws *ws = (o_ws *)malloc(sizeof(o_ws) * ws_cap);
  int rc = 0;
  for (int i = 0; i < N; i++) {
    if (in->hbtype[i] == 0) continue;
    o_ws tmp[4];
    memset(tmp, 0, sizeof(tmp));
    int n = o_make_ws(in, i, tmp);
    if (n < 0) {
      rc = -2;
      break;
    }
    if (nws + n > ws_cap) {
      ws_cap = 2 * (nws + n);
      ws = (o_ws *)realloc(ws, sizeof(o_ws) * ws_cap);
    }
    memcpy(ws + nws, tmp, sizeof(o_ws) * n);
    nws += n;
  }
  out->nws = nws;
  out->ehb = 0.0;
  if (rc == 0) {
    const double vw = (4.0 / 3.0) * O_PI * O_HBRAD * O_HBRAD * O_HBRAD;
    const double aw = O_KFC / (O_HBRAD * O_HBRAD);
    /* compat mode: spe index the reference reads in its free-volume loop
       (agbnp3_cpu_simd_kernels.c:2854, read before the assignment at :2859):
       the previously processed overlap's atom within a site, the previous
       site's last parent across sites, and nheavy before the first site.
       Hydrogen indices read 0 (spe is only set for heavy atoms). */
    int prev_atom = NH;
    int *hit = (int *)malloc(sizeof(int) * (NH + 1));
    o_ovl *hov = (o_ovl *)malloc(sizeof(o_ovl) * (NH + 1));
    for (int w = 0; w < nws; w++) {
      o_ws *s = &ws[w];
      o_gauss gw = {aw, O_PFC, {s->pos[0], s->pos[1], s->pos[2]}};
      int nh = 0;
      for (int i = 0; i < NH; i++) {
        double dx = x[i] - s->pos[0], dy = y[i] - s->pos[1], dz = z[i] - s->pos[2];
        double u = (r[i] + O_HBRAD) * 1.6;
        if (dx * dx + dy * dy + dz * dz < u * u) hit[nh++] = i;
      }
      double fv = vw, cut = O_HBSWA0 * vw;
      int nproc = 0;
      for (int q = 0; q < nh; q++) {
        if (!(fv > cut)) continue;
        int i = hit[q];
        o_ovl o;
        o_ogauss(&gw, &atg[i], &o);
        if (!(o.gvolp > 0.0)) continue;
        double spe_used = spe[i];
        if (in->compat) spe_used = prev_atom < NH ? spe[prev_atom] : 0.0;
        fv -= spe_used * o.gvolp;
        prev_atom = i;
        hov[nproc] = o;
        hit[nproc] = i; /* compact processed overlaps (nproc <= q) */
        nproc++;
      }
      double spw = fv / vw, fp;
      double sw = o_poly_switch(spw, O_HBSWA, O_HBSWB, &fp, NULL);
      double dhw = s->khb * fp / vw;
      out->ehb += s->khb * sw;
      if (out->ws_pos && w < out->ws_cap) {
        for (int k = 0; k < 3; k++) out->ws_pos[3 * w + k] = s->pos[k];
        out->ws_sp[w] = spw;
        out->ws_parent0[w] = s->parent[0];
        out->ws_type[w] = s->type;
      }
      double jw[3] = {0, 0, 0};
      for (int q = 0; q < nproc; q++) {
        int i = hit[q];
        o_ovl *o = &hov[q];
        double xi[3] = {x[i], y[i], z[i]};
        double fw = -2.0 * aw * o->gvol * o->fp, fi = -2.0 * ga[i] * o->gvol * o->fp;
        double u = -spe[i] * dhw;
        for (int k = 0; k < 3; k++) {
          gh[i][k] += u * fi * (xi[k] - o->g.c[k]);
          jw[k] += u * fw * (s->pos[k] - o->g.c[k]);
        }
        derh[i] += dhw / vols[i] * o->gvolp;
      }
      for (int p = 0; p < s->nparents; p++) {
        int a = s->parent[p];
        for (int j = 0; j < 3; j++) {
          double t = 0.0;
          for (int k = 0; k < 3; k++) t += jw[k] * s->dpos[p][k][j];
          gh[a][j] += t;
        }
      }
      /* the reference's atom index leaves this site's projection loop at
         its last parent (agbnp3_cpu_simd_kernels.c:2927-2933), which is
         what the next site's first subtraction reads */
      prev_atom = s->parent[s->nparents - 1];
    }
    free(hit);
    free(hov);
  }

  /* U_i, V_i normalisation and the surface-area effective gammas
     (agbnp3_cpu_simd_kernels.c:861-874) */
  for (int i = 0; i < NH; i++) {
    deru[i] /= vols[i];
    derv[i] /= vols[i];
    dervs[i] = fourpi1 * psvol[i] * derv[i];
    derus[i] = df * fourpi1 * psvol[i] * deru[i];
  }

  /* derivatives through the self volumes (agbnp3_cpu_simd_kernels.c:
     1601-1956) and the cavity / surface-area second derivatives
     (agbnp3_cpu_simd_kernels.c:1959-2405), over every kept overlap */
  for (int m = 2; m <= ORC_MAX_ORDER; m++) {
    double sgn = (m % 2) ? 1.0 : -1.0;
    for (int q = 0; q < lev[m].n; q++) {
      o_node *nd = &lev[m].v[q];
      const o_ovl *o = &nd->o;
      double gx[ORC_MAX_ORDER][3], gdr[ORC_MAX_ORDER][3], gdR[ORC_MAX_ORDER];
      double su = 0, sv = 0, sh = 0;
      for (int ii = 0; ii < m; ii++) {
        int k = nd->par[ii];
        gx[ii][0] = x[k];
        gx[ii][1] = y[k];
        gx[ii][2] = z[k];
        su += deru[k];
        sv += derv[k];
        sh += derh[k];
      }
      su *= -df * fourpi1 * vcoef[m];
      sv *= -fourpi1 * vcoef[m];
      sh *= -vcoef[m];
      double inva = 1.0 / o->g.a;
      for (int ii = 0; ii < m; ii++) {
        int k = nd->par[ii];
        double u1 = ga[k] * o->gvol;
        double d2 = 0.0;
        for (int c = 0; c < 3; c++) {
          double ur = -2.0 * u1 * o->fp * (gx[ii][c] - o->g.c[c]);
          gb[k][c] += su * ur;
          gv[k][c] += sv * ur;
          gh[k][c] += sh * ur;
          gdr[ii][c] = -2.0 * u1 * (gx[ii][c] - o->g.c[c]);
          d2 += gdr[ii][c] * gdr[ii][c];
        }
        gdR[ii] = (3.0 * inva * u1 + 0.5 * d2 / u1) / r[k];
      }
      double h3 = o->fpp + o->fp / o->gvol;
      for (int ii = 0; ii < m; ii++) {
        int k = nd->par[ii];
        double u1 = -2.0 * o->fp * (1.0 - ga[k] * inva) / r[k] + h3 * gdR[ii];
        for (int c = 0; c < 3; c++) {
          double ur = u1 * gdr[ii][c];
          gc[k][c] += sgn * gammap[k] * ur;
          gv[k][c] += sgn * dervs[k] * ur;
          gb[k][c] += sgn * derus[k] * ur;
        }
      }
      double h4 = 2.0 * o->fp * inva;
      for (int ii = 0; ii < m; ii++) {
        int k = nd->par[ii];
        for (int jj = 0; jj < m; jj++) {
          if (jj == ii) continue;
          int l = nd->par[jj];
          double u1 = h4 * ga[k] / r[l], u2 = h3 * gdR[jj];
          for (int c = 0; c < 3; c++) {
            double ur = u1 * gdr[jj][c] + u2 * gdr[ii][c];
            gc[k][c] += sgn * gammap[l] * ur;
            gv[k][c] += sgn * dervs[l] * ur;
            gb[k][c] += sgn * derus[l] * ur;
          }
        }
      }
    }
  }

  /* outputs (agbnp3.c:1761-1786) */
  for (int i = 0; i < N; i++) {
    out->sp[i] = i < NH ? sp[i] : 1.0;
    out->br[i] = br[i];
    out->surf_area[i] = i < NH ? surf_f[i] : 0.0;
    for (int c = 0; c < 3; c++) {
      out->dgbdr[3 * i + c] = O_TOKCAL * gb[i][c];
      out->dvwdr[3 * i + c] = gv[i][c];
      out->decav[3 * i + c] = gc[i][c];
      out->dehb[3 * i + c] = gh[i][c];
    }
  }
#define COPY_OUT(name, src) \
  if (out->name) memcpy(out->name, src, sizeof(double) * N)
  COPY_OUT(volumep, volumep);
  COPY_OUT(surf_raw, surf);
  COPY_OUT(spe, spe);
  COPY_OUT(br1, bfil);
  COPY_OUT(dera, dera);
  COPY_OUT(deru, deru);
  COPY_OUT(derv, derv);
  COPY_OUT(derh, derh);
  COPY_OUT(q2ab, q2ab);
  COPY_OUT(abrw, abrw);
  COPY_OUT(psvol, psvol);
  COPY_OUT(gammap, gammap);
  COPY_OUT(derus, derus);
  COPY_OUT(dervs, dervs);
  out->nl_total = nl_n;
  if (out->nl_count) {
    for (int i = 0; i < NH; i++) out->nl_count[i] = nl_off[i + 1] - nl_off[i];
    for (int k = 0; k < nl_n && k < out->nl_cap; k++) out->nl_list[k] = nl[k];
  }
  out->ntypes = nt;
  if (out->tab_y && out->tab_cap >= nt * nt * O_NA) {
    memcpy(out->tab_y, T.y, sizeof(double) * nt * nt * O_NA);
    memcpy(out->tab_y2, T.y2, sizeof(double) * nt * nt * O_NA);
  }
  if (out->rtype) memcpy(out->rtype, rtype, sizeof(int) * N);

  for (int m = 0; m <= ORC_MAX_ORDER; m++) free(lev[m].v);
  free(atg); free(nl); free(nl_off); free(ws); free(T.y); free(T.y2); free(rtype);
  free(vols); free(volumep); free(surf); free(br1); free(sp); free(spe); free(psvol); free(surf_f);
  free(gammap); free(bfil); free(bder); free(br); free(brw); free(dera); free(q2ab); free(abrw);
  free(deru); free(derv); free(derh); free(derus); free(dervs); free(ga);
  free(gb); free(gv); free(gc); free(gh);
  return rc;
}
