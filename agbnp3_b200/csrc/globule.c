/*
 * Seeded synthetic-globule generator for the AGBNP3 benchmarks.
 *
 * Builds a branched self-avoiding heavy-atom walk inside a sphere, decorates
 * it with hydrogens and returns everything agbnp3_new() needs: coordinates
 * (rounded to float, because the engine and the reference both narrow
 * coordinates to float on every call, agbnp3.c:520-525), van der Waals radii,
 * charges, non-polar parameters, HB types and the bond list that forms the
 * NeighList connection table.
 *
 * Walk rules:
 *   - heavy-heavy bonds are 1.53 A long;
 *   - a new heavy atom keeps >= 3.0 A from every heavy atom that is not its
 *     1-2 or 1-3 partner (the bonded parent and the parent's other bonded
 *     neighbours), and >= 2.45 A from its 1-3 partners (bond angles of at
 *     least ~106 degrees);
 *   - the walk is confined to a sphere sized for the requested heavy-atom
 *     density; when the chain tip is trapped the walk branches from another
 *     atom with free valence, and when nothing fits the sphere grows by 1%.
 *     The achieved density is reported back to the caller.
 * Elements: C/N/O/S with probabilities 0.62/0.17/0.19/0.02; maximum heavy
 * valence C 4, N 3, O 2, S 2.  Each heavy atom gets 0-2 hydrogens at 1.0 A
 * (limited by the remaining valence); a terminal oxygen always gets one, so
 * every oxygen has exactly two connections and is typed as a tetrahedral
 * acceptor whose water sites the reference can build (agbnp3.c:1977-2007).
 * Hydrogens bonded to N or O are polar donors.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define HB_INACTIVE 0
#define HB_POLARH 1
#define HB_TETRAHEDRAL 20

typedef struct {
  uint64_t s[4];
} rng_t;

static uint64_t splitmix64(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static void rng_seed(rng_t *r, uint64_t seed) {
  uint64_t x = seed;
  for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* xoshiro256** */
static uint64_t rng_next(rng_t *r) {
  uint64_t *s = r->s;
  uint64_t result = rotl(s[1] * 5, 7) * 9;
  uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}

static double rng_uniform(rng_t *r) { return (rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static double rng_normal(rng_t *r) {
  double u1 = rng_uniform(r), u2 = rng_uniform(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

static void rng_unit_vector(rng_t *r, double v[3]) {
  double z = 2.0 * rng_uniform(r) - 1.0;
  double phi = 2.0 * M_PI * rng_uniform(r);
  double s = sqrt(1.0 - z * z);
  v[0] = s * cos(phi);
  v[1] = s * sin(phi);
  v[2] = z;
}

/* ---- uniform cell grid over a cube, for clash tests ---- */
typedef struct {
  double lo, h;
  int n;
  int *head; /* n^3 */
  int *next; /* per atom */
} grid_t;

static int grid_cell(const grid_t *g, const double p[3], int c[3]) {
  for (int k = 0; k < 3; k++) {
    int v = (int)floor((p[k] - g->lo) / g->h);
    if (v < 0) v = 0;
    if (v >= g->n) v = g->n - 1;
    c[k] = v;
  }
  return (c[2] * g->n + c[1]) * g->n + c[0];
}

static void grid_insert(grid_t *g, const double *pos, int a) {
  int c[3];
  int id = grid_cell(g, pos + 3 * a, c);
  g->next[a] = g->head[id];
  g->head[id] = a;
}

#define MAXB 8
typedef struct {
  int n;
  int nb[MAXB];
} adj_t;

/* true if p is closer than dmin to any heavy atom other than those in
   excl[0..nexcl) */
static int clashes(const grid_t *g, const double *pos, const double p[3], double dmin, const int *excl,
                   int nexcl) {
  int c[3];
  grid_cell(g, p, c);
  double d2min = dmin * dmin;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
        if (x < 0 || y < 0 || z < 0 || x >= g->n || y >= g->n || z >= g->n) continue;
        for (int a = g->head[(z * g->n + y) * g->n + x]; a >= 0; a = g->next[a]) {
          int skip = 0;
          for (int e = 0; e < nexcl; e++)
            if (excl[e] == a) skip = 1;
          if (skip) continue;
          double ux = pos[3 * a] - p[0], uy = pos[3 * a + 1] - p[1], uz = pos[3 * a + 2] - p[2];
          if (ux * ux + uy * uy + uz * uz < d2min) return 1;
        }
      }
  return 0;
}

static int max_valence(int el) { /* 0 C, 1 N, 2 O, 3 S */
  static const int v[4] = {4, 3, 2, 2};
  return v[el];
}

/*
 * Generates one globule.  Arrays are caller-allocated with room for
 * `natoms` atoms and `2*natoms` bonds.  Returns 0 on success.
 *
 *  element[i]: 0 C, 1 N, 2 O, 3 S, 4 H
 *  bonds[2*k], bonds[2*k+1]: bonded pair k (heavy-heavy first, then X-H)
 *  stats[0] = achieved heavy-atom density (1/A^3), stats[1] = sphere radius,
 *  stats[2] = number of branch events, stats[3] = sphere enlargements
 */
int agbnp3_globule_generate(int natoms, uint64_t seed, double density, double noise_sigma,
                            double *x, double *y, double *z, double *radius, double *charge,
                            double *igamma, double *sgamma, double *ialpha, double *salpha,
                            int *hbtype, double *hbcorr, int *element, int *nbonds_out, int *bonds,
                            double *stats) {
  if (natoms < 2) return -1;
  rng_t rng;
  rng_seed(&rng, seed);
  int nheavy = (natoms + 1) / 2;
  int nhyd = natoms - nheavy;

  double R = cbrt(3.0 * nheavy / (4.0 * M_PI * density));
  double *pos = (double *)calloc((size_t)3 * natoms, sizeof(double));
  adj_t *adj = (adj_t *)calloc((size_t)natoms, sizeof(adj_t));
  int *el = element;
  int *hcount = (int *)calloc((size_t)nheavy, sizeof(int));
  int nb = 0;
  int nbranch = 0, nenlarge = 0;

  grid_t g;
  g.h = 3.0;
  double half = 3.0 * R + 10.0; /* room for sphere growth */
  g.lo = -half;
  g.n = (int)ceil(2.0 * half / g.h);
  g.head = (int *)malloc(sizeof(int) * (size_t)g.n * g.n * g.n);
  g.next = (int *)malloc(sizeof(int) * (size_t)natoms);
  if (!pos || !adj || !hcount || !g.head || !g.next) return -2;
  for (long i = 0; i < (long)g.n * g.n * g.n; i++) g.head[i] = -1;

  /* element draw */
  for (int i = 0; i < nheavy; i++) {
    double u = rng_uniform(&rng);
    el[i] = u < 0.62 ? 0 : (u < 0.79 ? 1 : (u < 0.98 ? 2 : 3));
  }

  pos[0] = pos[1] = pos[2] = 0.0;
  grid_insert(&g, pos, 0);
  int tip = 0;
  int excl[MAXB + 1];
  for (int k = 1; k < nheavy; k++) {
    int placed = 0;
    while (!placed) {
      /* grow from the tip first, then branch from random atoms */
      for (int phase = 0; phase < 2 && !placed; phase++) {
        int ntry_parent = phase == 0 ? 1 : 4000;
        for (int tp = 0; tp < ntry_parent && !placed; tp++) {
          int parent = phase == 0 ? tip : (int)(rng_uniform(&rng) * k);
          if (adj[parent].n >= max_valence(el[parent])) continue;
          /* the new atom's valence must allow the bond too */
          int nexcl = 0;
          excl[nexcl++] = parent;
          for (int e = 0; e < adj[parent].n; e++) excl[nexcl++] = adj[parent].nb[e];
          int ndir = phase == 0 ? 60 : 12;
          for (int t = 0; t < ndir; t++) {
            double v[3], p[3];
            rng_unit_vector(&rng, v);
            for (int c = 0; c < 3; c++) p[c] = pos[3 * parent + c] + 1.53 * v[c];
            if (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > R * R) continue;
            if (clashes(&g, pos, p, 3.0, excl, nexcl)) continue;
            /* 1-3 partners: bond angle of at least ~106 degrees */
            int bent = 0;
            for (int e = 1; e < nexcl; e++) {
              const double *q = pos + 3 * excl[e];
              double ux = q[0] - p[0], uy = q[1] - p[1], uz = q[2] - p[2];
              if (ux * ux + uy * uy + uz * uz < 2.45 * 2.45) bent = 1;
            }
            if (bent) continue;
            memcpy(pos + 3 * k, p, sizeof(p));
            grid_insert(&g, pos, k);
            adj[parent].nb[adj[parent].n++] = k;
            adj[k].nb[adj[k].n++] = parent;
            bonds[2 * nb] = parent;
            bonds[2 * nb + 1] = k;
            nb++;
            if (phase == 1) nbranch++;
            tip = k;
            placed = 1;
            break;
          }
        }
      }
      if (!placed) {
        R *= 1.01;
        if (++nenlarge > 2000) {
          free(pos); free(adj); free(hcount); free(g.head); free(g.next);
          return -4;
        }
      }
    }
  }

  /* hydrogens: 0-2 per heavy atom within remaining valence; terminal O gets 1 */
  int hsum = 0;
  for (int i = 0; i < nheavy; i++) {
    int room = max_valence(el[i]) - adj[i].n;
    if (room < 0) room = 0;
    int cap = room < 2 ? room : 2;
    int h = (int)(rng_uniform(&rng) * 3.0);
    if (h > cap) h = cap;
    if (el[i] == 2) h = (adj[i].n == 1) ? 1 : 0;
    hcount[i] = h;
    hsum += h;
  }
  /* adjust to the exact hydrogen total (oxygens keep their count) */
  int guard = 0;
  while (hsum != nhyd && guard < 100000000) {
    guard++;
    int i = (int)(rng_uniform(&rng) * nheavy);
    if (el[i] == 2) continue;
    int room = max_valence(el[i]) - adj[i].n;
    int cap = room < 2 ? room : 2;
    if (hsum < nhyd && hcount[i] < cap) {
      hcount[i]++;
      hsum++;
    } else if (hsum > nhyd && hcount[i] > 0) {
      hcount[i]--;
      hsum--;
    }
  }
  if (hsum != nhyd) {
    /* not enough valence for the requested hydrogen count */
    free(pos); free(adj); free(hcount); free(g.head); free(g.next);
    return -3;
  }

  int ih = nheavy;
  for (int i = 0; i < nheavy; i++) {
    for (int h = 0; h < hcount[i]; h++) {
      double best[3] = {0, 0, 0}, bestd = -1.0;
      for (int t = 0; t < 24; t++) {
        double v[3], p[3];
        rng_unit_vector(&rng, v);
        for (int c = 0; c < 3; c++) p[c] = pos[3 * i + c] + 1.0 * v[c];
        double dmin = 1e30;
        for (int e = 0; e < adj[i].n; e++) {
          int a = adj[i].nb[e];
          double ux = pos[3 * a] - p[0], uy = pos[3 * a + 1] - p[1], uz = pos[3 * a + 2] - p[2];
          double d = ux * ux + uy * uy + uz * uz;
          if (d < dmin) dmin = d;
        }
        if (dmin > bestd) {
          bestd = dmin;
          memcpy(best, p, sizeof(best));
        }
      }
      memcpy(pos + 3 * ih, best, sizeof(best));
      el[ih] = 4;
      adj[i].nb[adj[i].n++] = ih;
      adj[ih].nb[adj[ih].n++] = i;
      bonds[2 * nb] = i;
      bonds[2 * nb + 1] = ih;
      nb++;
      ih++;
    }
  }

  /* parameters */
  static const double rvdw[5] = {1.7, 1.55, 1.52, 1.8, 1.15};
  double qsum = 0.0;
  for (int i = 0; i < natoms; i++) {
    radius[i] = rvdw[el[i]];
    charge[i] = 0.3 * rng_normal(&rng);
    qsum += charge[i];
    igamma[i] = el[i] == 4 ? 0.0 : 0.117;
    sgamma[i] = 0.0;
    salpha[i] = 0.0;
    ialpha[i] = -0.09 + 0.07 * rng_uniform(&rng);
    hbcorr[i] = -1.0 + 0.5 * rng_uniform(&rng);
    hbtype[i] = HB_INACTIVE;
  }
  for (int i = 0; i < natoms; i++) charge[i] -= qsum / natoms;
  for (int i = 0; i < natoms; i++) {
    if (el[i] == 2) hbtype[i] = HB_TETRAHEDRAL;
    if (el[i] == 4) {
      int p = adj[i].nb[0];
      if (el[p] == 1 || el[p] == 2) hbtype[i] = HB_POLARH;
    }
  }

  for (int i = 0; i < natoms; i++) {
    double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    if (noise_sigma > 0.0) {
      px += noise_sigma * rng_normal(&rng);
      py += noise_sigma * rng_normal(&rng);
      pz += noise_sigma * rng_normal(&rng);
    }
    x[i] = (double)(float)px;
    y[i] = (double)(float)py;
    z[i] = (double)(float)pz;
  }
  *nbonds_out = nb;
  if (stats) {
    stats[0] = nheavy / (4.0 / 3.0 * M_PI * R * R * R);
    stats[1] = R;
    stats[2] = nbranch;
    stats[3] = nenlarge;
  }
  free(pos);
  free(adj);
  free(hcount);
  free(g.head);
  free(g.next);
  return 0;
}
